"""The forward splat's fixed-point bound, checked by brute force on the host.

The splat accumulates each tile's detector windows as 32-bit integers at a
per-tile scale S <= 2^30 / (nbound * max|v|), where nbound is the host's bound
on how many voxels of one 64 x 4 x 32 tile can add to one window entry
(tr_geom.h: derive_geometry, fp_section_bound, fp_entry_bound_sep).  Each voxel
adds at most |v| to an entry, so no window entry can overflow as long as the
true count never exceeds nbound.  This test compiles tr_geom.h as host C++,
asks it for nbound on random geometries (general affine projections and
separable ones, tilts to +-75 degrees, in-plane rotations, X tilts) and counts,
for tiles at random sub-pixel offsets, the voxels that actually reach each
entry: entry (q, r) collects the voxels whose detector coordinate (u, v) lies
in [q-1, q+1) x [r-1, r+1) (separable windows: one window row per voxel row,
so the count is per (q, voxel row)).  Runs on the CPU; the count is
independent of the volume and stack sizes, so it covers full-size problems.
"""
import ctypes as C
import math
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

CSRC = Path(__file__).resolve().parents[1] / "autom2_b200" / "csrc"
FX, TY, FTZ = 64, 4, 32  # forward-projection tile (x pairs of 32 lanes, rows, sections)

PROBE = r"""
#include "tr_geom.h"
extern "C" int probe_nbound(const double *c8, int nt, int nx, int ny, int th,
                            float *nbound, int *sep) {
  static trb::TiltGeo g[1024];
  if (nt > 1024) return -1;
  trb::GeomInfo gi;
  int bad = -1;
  const int s = trb::derive_geometry(c8, nt, nx, ny, th, (size_t)1 << 30, g, &gi, &bad);
  *nbound = gi.nbound;
  *sep = gi.sep;
  return s;
}
extern "C" int probe_derive(const double *c8, int nt, int nx, int ny, int th, size_t smem,
                            int *info, int *bad) {
  static trb::TiltGeo g[1024];
  if (nt > 1024) return -1;
  trb::GeomInfo gi{};
  const int s = trb::derive_geometry(c8, nt, nx, ny, th, smem, g, &gi, bad);
  info[0] = gi.fw;
  info[1] = gi.fh;
  info[2] = gi.ffw;
  info[3] = gi.ffh;
  return s;
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory, cuda_include):
    cxx = shutil.which("g++")
    assert cxx, "g++ is needed to compile the geometry header for this test"
    d = tmp_path_factory.mktemp("geomprobe")
    src, so = d / "probe.cpp", d / "probe.so"
    src.write_text(PROBE)
    subprocess.run([cxx, "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{CSRC}",
                    f"-I{cuda_include}", str(src), "-o", str(so)], check=True)
    lib = C.CDLL(str(so))
    lib.probe_nbound.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.POINTER(C.c_float), C.POINTER(C.c_int)]
    lib.probe_nbound.restype = C.c_int
    lib.probe_derive.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int,
                                 C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int)]

    def nbound(c8, nx=1024, ny=1024, th=256):
        c8 = np.ascontiguousarray(c8, np.float64)
        nb, sep = C.c_float(), C.c_int()
        st = lib.probe_nbound(c8.ctypes.data_as(C.POINTER(C.c_double)), len(c8), nx, ny, th,
                              C.byref(nb), C.byref(sep))
        assert st == 0, f"derive_geometry refused the geometry ({st})"
        return float(nb.value), bool(sep.value)

    def derive(c8, nx=1024, ny=1024, th=256, smem=200 * 1024):
        c8 = np.ascontiguousarray(c8, np.float64)
        info, bad = (C.c_int * 4)(), C.c_int()
        st = lib.probe_derive(c8.ctypes.data_as(C.POINTER(C.c_double)), len(c8), nx, ny, th,
                              C.c_size_t(smem), info, C.byref(bad))
        return st, list(info), bad.value
    nbound.derive = derive
    return nbound


def rot(axis, a):
    c, s = math.cos(a), math.sin(a)
    if axis == "x":
        return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    if axis == "y":
        return np.array([[c, 0, -s], [0, 1, 0], [s, 0, c]])
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def general_tilt(rng, theta_deg, psi_sd_deg, alpha_deg):
    """Detector rows of R_z(psi) R_x(alpha) R_y(theta) as [a0..a3, b0..b3]."""
    R = rot("z", math.radians(rng.normal(0, psi_sd_deg))) @ rot("x", math.radians(alpha_deg)) \
        @ rot("y", math.radians(theta_deg))
    a0, b0 = rng.normal(0, 3, size=2)
    return np.array([a0, *R[0], b0, *R[1]])


def max_entry_count(k, sep, rng, offsets=48):
    """Largest number of one tile's voxels that reach one window entry, over
    tiles at random sub-pixel offsets (coordinates in FP64)."""
    a1, a2, a3, b1, b2, b3 = k[1], k[2], k[3], k[5], k[6], k[7]
    x, y, z = np.meshgrid(np.arange(FX), np.arange(TY), np.arange(FTZ), indexing="ij")
    x, y, z = x.ravel(), y.ravel(), z.ravel()
    best = 0
    for _ in range(offsets):
        cu, cv = rng.uniform(-1000, 1000, size=2)
        u = cu + a1 * x + a2 * y + a3 * z
        q0 = np.floor(u).astype(np.int64)
        if sep:  # window rows are voxel rows: the two taps (q0, y), (q0+1, y)
            qs = np.concatenate([q0, q0 + 1]) - q0.min()
            keys = np.concatenate([y, y]) * (qs.max() + 1) + qs
        else:
            v = cv + b1 * x + b2 * y + b3 * z
            r0 = np.floor(v).astype(np.int64)
            # the four taps: (q0, r0), (q0+1, r0), (q0, r0+1), (q0+1, r0+1)
            qq = np.concatenate([q0, q0 + 1, q0, q0 + 1]) - q0.min()
            rr = np.concatenate([r0, r0, r0 + 1, r0 + 1]) - r0.min()
            keys = rr * (qq.max() + 1) + qq
        best = max(best, int(np.bincount(keys).max()))
    return best


@pytest.mark.parametrize("psi_sd,alpha", [(0.5, 0.3), (5.0, 2.0), (30.0, 10.0), (0.0, 0.3)])
def test_general_bound_holds(probe, psi_sd, alpha):
    rng = np.random.default_rng(int(psi_sd * 10 + alpha * 100))
    for theta in np.linspace(-75, 75, 31):
        k = general_tilt(rng, theta, psi_sd, alpha)
        nb, sep = probe(k[None, :])
        assert not sep
        got = max_entry_count(k, False, rng)
        assert got <= nb, f"theta {theta:.1f}: {got} voxels reach one entry, bound {nb}"
        # The bound is per tilt and not loose by more than the lattice-point
        # inequality's perimeter term (cfg1's geometry: 512 against ~200).
        assert nb <= FX * TY * FTZ


def test_cfg1_like_bound_is_512(probe):
    """The cfg1 geometry (61 tilts over +-60 degrees, in-plane rotations of
    0.5 degrees, X tilt 0.3 degrees) gets 16 voxels per section, 512 per
    entry: the bound the splat's fixed-point scale is set from."""
    rng = np.random.default_rng(1)
    k = np.stack([general_tilt(rng, t, 0.5, 0.3) for t in np.linspace(-60, 60, 61)])
    nb, sep = probe(k)
    assert not sep and nb == 512
    assert max(max_entry_count(t, False, rng, offsets=8) for t in k) <= nb


@pytest.mark.parametrize("a1", [1.0, 0.97, 0.75, 0.52, 0.5, 0.34, 0.26, 0.1])
def test_separable_bound_holds(probe, a1):
    rng = np.random.default_rng(int(a1 * 1000))
    for sign in (1, -1):
        k = np.array([rng.normal(0, 3), sign * a1, 0.0, math.sqrt(max(0.0, 1 - a1 * a1)),
                      rng.normal(0, 1), 0.0, 1.0, 0.0])
        nb, sep = probe(k[None, :])
        assert sep
        got = max_entry_count(k, True, rng)
        assert got <= nb, f"a1 {sign * a1}: {got} voxels reach one entry, bound {nb}"


# derive_geometry's status codes (tr_geom.h GeomStatus)
GEOM_OK, GEOM_NONFINITE, GEOM_MAGNITUDE, GEOM_RANGE, GEOM_SMEM, GEOM_WINDOW = range(6)


def test_geometry_refusals_name_the_tilt(probe):
    """Coefficients the kernels cannot stage are refused with the reason,
    and per-tilt failures name the offending tilt (window limits apply to the
    whole series); the context and the no-allocation entry point map these to
    TR_ERR_ARG (non-finite) or TR_ERR_UNSUPPORTED."""
    rng = np.random.default_rng(5)
    good = np.stack([general_tilt(rng, t, 0.5, 0.3) for t in np.linspace(-60, 60, 7)])
    st, info, bad = probe.derive(good)
    assert st == GEOM_OK and bad == -1
    fw, fh, ffw, ffh = info
    assert ffw % 4 == 0 and fw >= 32 and fh >= 5 and ffw >= 64 and ffh >= 5
    cases = [
        (3, 2, np.nan, GEOM_NONFINITE),
        (4, 6, np.inf, GEOM_NONFINITE),
        (2, 1, 2000.0, GEOM_MAGNITUDE),      # a slope above 1024
        (5, 0, 3.0e9, GEOM_RANGE),           # detector columns beyond the int range
        (1, 3, 40.0, GEOM_WINDOW),           # a tile reaching over 511 columns
    ]
    for t, i, v, want in cases:
        k = good.copy()
        k[t, i] = v
        st, _, bad = probe.derive(k)
        assert (st, bad) == (want, -1 if want == GEOM_WINDOW else t), (t, i, v)
    # a window that fits the side limit but not the shared-memory budget
    k = good.copy()
    k[6, 3] = 6.0
    assert probe.derive(k)[0] == GEOM_OK
    st, _, bad = probe.derive(k, smem=4 * 1024)
    assert (st, bad) == (GEOM_SMEM, -1)


def test_separable_windows(probe):
    """Separable geometry (b1 = b3 = 0, b2 = 1) keeps one window row per voxel
    row: four rows whatever the tilt."""
    k = np.array([[0.5, np.cos(a), 0.0, np.sin(a), 0.25, 0.0, 1.0, 0.0]
                  for a in np.radians(np.linspace(-70, 70, 9))])
    st, (fw, fh, ffw, ffh), _ = probe.derive(k)
    assert st == GEOM_OK and fh == 4 and ffh == 4
    span = np.abs(k[:, 1]) * 31 + np.abs(k[:, 3]) * 31
    assert fw == int(np.ceil(span.max())) + 4
