"""Test oracle for the TiltRec reconstruction path.

TEST INFRASTRUCTURE.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this package; it is the checker,
never the product path.

Two oracles live here:

* ``Restatement`` -- our C restatement (``tiltrec_oracle.c``) of the reference
  CPU routines, in float (``orc_*``) and in double (``orc64_*``, the FP64
  oracle).
* ``Reference`` -- the unmodified reference CPU sources
  (``src/TiltRec/src/main/main-mpi.cpp`` / ``main-mpiz.cpp``, ``mrcmx``,
  ``filter``) compiled by ``oracle/Makefile`` into ``oracle/_ref/`` with
  test-only MPI / FFTW / OpenCV C-API shims (exact double-precision DFTs in
  place of cuFFT and OpenCV's).  Present only where it was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
REFERENCE_SOURCES = "/root/reference/src/TiltRec/src"

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build(with_reference: bool | None = None) -> None:
    """Compile the restatement and, where the reference sources exist, the
    reference oracle (``make ref``)."""
    subprocess.run(["make", "-s", "restatement"], cwd=HERE, check=True)
    if with_reference is None:
        with_reference = os.path.isdir(REFERENCE_SOURCES)
    if with_reference:
        subprocess.run(["make", "-s", "ref", "refgpu", f"REF={REFERENCE_SOURCES}"],
                       cwd=HERE, check=True)


def reference_resample_executable() -> str | None:
    """The reference's resample tool (``make ref``: its unmodified sources
    with the test-only OpenCV subset), or None where it was not built."""
    path = os.path.join(REF_DIR, "resample")
    return path if os.path.exists(path) else None


def reference_gpu_executable(layout: int = 0) -> str | None:
    """The reference's own TiltRec-cuda / TiltRecZ-cuda compiled for sm_100a
    (``make refgpu``), or None where they were not built."""
    path = os.path.join(REF_DIR, "TiltRec-cuda" if layout == 0 else "TiltRecZ-cuda")
    return path if os.path.exists(path) else None


class Geom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nt", C.c_int),
                ("th", C.c_int), ("layout", C.c_int), ("z0", C.c_int),
                ("ox", C.c_float), ("oy", C.c_float), ("oz", C.c_float)]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class Restatement:
    """ctypes view of ``liboracle.so``.  Arrays: proj [nt][ny][nx]; volume
    [ny][th][nx] (layout 0, TiltRec) or [th][ny][nx] (layout 1, TiltRecZ);
    coefficients [nt][8] doubles (a0..a3, b0..b3)."""

    def __init__(self, path: str = RESTATEMENT_SO):
        if not os.path.exists(path):
            build(with_reference=False)
        lib = C.CDLL(path)
        self.lib = lib
        lib.orc_coeffs.argtypes = [_f32p, C.c_int, C.c_float, C.c_float,
                                   C.c_float, _f64p]
        lib.orc_filter_rweight.argtypes = [C.c_int, C.c_long, _f32p]
        lib.orc_filter_fbp.argtypes = [C.c_int, C.c_int, C.c_long, _f32p]
        lib.orc_optimal_dft_size.argtypes = [C.c_int]
        lib.orc_resample_bin.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        for pfx, p in (("orc_", _f32p), ("orc64_", _f64p)):
            real = C.c_float if pfx == "orc_" else C.c_double
            g = C.POINTER(Geom)
            getattr(lib, pfx + "backproject").argtypes = [g, _f64p, p, p]
            getattr(lib, pfx + "reproject").argtypes = [g, _f64p, p, p, p]
            getattr(lib, pfx + "update_weights").argtypes = [g, _f64p, p, p, p]
            getattr(lib, pfx + "update_by_projdiff").argtypes = [g, _f64p, p, p, real]
            getattr(lib, pfx + "sirt").argtypes = [g, _f64p, p, p, C.c_int, real]
            getattr(lib, pfx + "sart").argtypes = [g, _f64p, p, p, C.c_int, real]

    @staticmethod
    def geom(nx, ny, nt, th, layout=0, z0=0, origin=None):
        ox, oy, oz = origin if origin is not None else (nx * 0.5, th * 0.5, th * 0.5)
        return Geom(nx, ny, nt, th, layout, z0, ox, oy, oz)

    def coeffs(self, angles, offset=0.0, pitch=0.0, zshift=0.0):
        a = _c(angles, np.float32)
        out = np.zeros((len(a), 8), np.float64)
        self.lib.orc_coeffs(a, len(a), offset, pitch, zshift, out)
        return out

    def filter_rweight(self, proj):
        p = _c(proj, np.float32).copy()
        nx = p.shape[-1]
        self.lib.orc_filter_rweight(nx, p.size // nx, p)
        return p

    def filter_fbp(self, proj, mode=0):
        """FBP row filter (mode 0 Shepp-Logan, 1 Ram-Lak) of a copy of proj."""
        p = _c(proj, np.float32).copy()
        nx = p.shape[-1]
        self.lib.orc_filter_fbp(mode, nx, p.size // nx, p)
        return p

    def resample_bin(self, stack, bin_factor):
        """Area binning of [nt][ny][nx] by an integer factor."""
        p = _c(stack, np.float32)
        nt, ny, nx = p.shape
        out = np.zeros((nt, ny // bin_factor, nx // bin_factor), np.float32)
        self.lib.orc_resample_bin(p, nx, ny, nt, bin_factor, out)
        return out

    def optimal_dft_size(self, n):
        return int(self.lib.orc_optimal_dft_size(n))

    def _pfx(self, fp64):
        return ("orc64_", np.float64) if fp64 else ("orc_", np.float32)

    def backproject(self, g, coeff8, proj, vol, fp64=False):
        pfx, dt = self._pfx(fp64)
        v = _c(vol, dt).copy()
        getattr(self.lib, pfx + "backproject")(C.byref(g), _c(coeff8, np.float64),
                                               _c(proj, dt), v)
        return v

    def reproject(self, g, coeff8_one, vol, fp64=False):
        pfx, dt = self._pfx(fp64)
        val = np.zeros((g.ny, g.nx), dt)
        wt = np.zeros((g.ny, g.nx), dt)
        getattr(self.lib, pfx + "reproject")(C.byref(g), _c(coeff8_one, np.float64),
                                             _c(vol, dt), val, wt)
        return val, wt

    def update_weights(self, g, coeff8_one, diff, valvol, wtvol, fp64=False):
        pfx, dt = self._pfx(fp64)
        vv, wv = _c(valvol, dt).copy(), _c(wtvol, dt).copy()
        getattr(self.lib, pfx + "update_weights")(C.byref(g), _c(coeff8_one, np.float64),
                                                  _c(diff, dt), vv, wv)
        return vv, wv

    def update_by_projdiff(self, g, coeff8_one, diff, vol, gamma, fp64=False):
        pfx, dt = self._pfx(fp64)
        v = _c(vol, dt).copy()
        getattr(self.lib, pfx + "update_by_projdiff")(C.byref(g), _c(coeff8_one, np.float64),
                                                      _c(diff, dt), v, gamma)
        return v

    def sirt(self, g, coeff8, proj, vol, iters, gamma, fp64=False):
        pfx, dt = self._pfx(fp64)
        v = _c(vol, dt).copy()
        getattr(self.lib, pfx + "sirt")(C.byref(g), _c(coeff8, np.float64),
                                        _c(proj, dt), v, iters, gamma)
        return v

    def sart(self, g, coeff8, proj, vol, iters, gamma, fp64=False):
        pfx, dt = self._pfx(fp64)
        v = _c(vol, dt).copy()
        getattr(self.lib, pfx + "sart")(C.byref(g), _c(coeff8, np.float64),
                                        _c(proj, dt), v, iters, gamma)
        return v


def coeff20(coeff8):
    """Expand [nt][8] linear coefficients to the reference's Coeff layout
    (a[10], b[10]) with zero quadratic terms."""
    c8 = np.asarray(coeff8, np.float64).reshape(-1, 8)
    c20 = np.zeros((c8.shape[0], 20), np.float64)
    c20[:, 0:4] = c8[:, 0:4]
    c20[:, 10:14] = c8[:, 4:8]
    return c20


def reference_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f))
               for f in ("libref_y.so", "libref_z.so"))


class Reference:
    """ctypes view of the reference CPU routines built into ``oracle/_ref``
    (see ``oracle/ref_wrap.cpp`` for the entry points)."""

    def __init__(self):
        if not reference_available():
            raise FileNotFoundError("oracle/_ref was not built (make -C oracle ref)")
        y = C.CDLL(os.path.join(REF_DIR, "libref_y.so"))
        z = C.CDLL(os.path.join(REF_DIR, "libref_z.so"))
        self.y, self.z = y, z
        y.ref_coeffs.argtypes = [_f32p, C.c_int, C.c_float, C.c_float, C.c_float, _f64p]
        y.ref_filter_rweight.argtypes = [C.c_int, C.c_int, C.c_int, _f32p]
        y.ref_filter_rweight.restype = C.c_int
        y.ref_filter_fbp.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        y.ref_filter_fbp.restype = C.c_int
        geo = [C.c_int, C.c_int, C.c_int, C.c_int, _f64p, C.c_float, C.c_float, C.c_float]
        y.ref_y_backproject.argtypes = geo + [_f32p, _f32p]
        y.ref_y_sirt.argtypes = geo + [_f32p, _f32p, C.c_int, C.c_float, C.c_int]
        geo1 = [C.c_int, C.c_int, C.c_int, _f64p, C.c_float, C.c_float, C.c_float]
        y.ref_y_reproject.argtypes = geo1 + [_f32p, _f32p, _f32p]
        y.ref_y_update_weights.argtypes = geo1 + [_f32p, _f32p, _f32p]
        y.ref_y_update_by_projdiff.argtypes = geo1 + [_f32p, _f32p, C.c_float]
        y.ref_y_sirt_threaded.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          _f64p, C.c_float, _f32p, C.c_int, C.c_int,
                                          C.c_int, C.c_float]
        y.ref_y_sirt_threaded.restype = C.c_double
        y.ref_y_sirt_zslabs.argtypes = [C.c_int] + geo + [_f32p, _f32p, C.c_int, C.c_float]
        y.ref_y_sirt_zslabs.restype = C.c_double
        z.ref_z_run.argtypes = [C.c_int] + geo + [_f32p, _f32p, C.c_int, C.c_float, C.c_char_p]
        z.ref_z_run.restype = C.c_int
        z.ref_z_admm.argtypes = geo + [_f32p, _f32p, C.c_int, C.c_int, C.c_float, C.c_float,
                                       C.c_char_p]
        z.ref_z_admm.restype = C.c_int

    def coeffs20(self, angles, offset=0.0, pitch=0.0, zshift=0.0):
        a = _c(angles, np.float32)
        out = np.zeros((len(a), 20), np.float64)
        self.y.ref_coeffs(a, len(a), offset, pitch, zshift, out)
        return out

    def filter_rweight(self, proj):
        p = _c(proj, np.float32).copy()
        nt, ny, nx = p.shape
        rc = self.y.ref_filter_rweight(nx, ny, nt, p)
        assert rc == 0
        return p

    def filter_fbp(self, proj, mode=0):
        """The reference's FBP row filter (ApplyFilterInplace mode 0
        Shepp-Logan, 1 Ram-Lak) of a copy of proj [nt][ny][nx], run through
        the OpenCV C-API shim."""
        p = _c(proj, np.float32).copy()
        nt, ny, nx = p.shape
        rc = self.y.ref_filter_fbp(mode, nx, ny, nt, p)
        assert rc == 0, rc
        return p

    def y_backproject(self, nx, ny, nt, th, c20, origin, proj, vol):
        v = _c(vol, np.float32).copy()
        self.y.ref_y_backproject(nx, ny, nt, th, _c(c20, np.float64), *origin,
                                 _c(proj, np.float32).copy(), v)
        return v

    def y_sirt(self, nx, ny, nt, th, c20, origin, proj, vol, iters, gamma, sart=False):
        v = _c(vol, np.float32).copy()
        self.y.ref_y_sirt(nx, ny, nt, th, _c(c20, np.float64), *origin,
                          _c(proj, np.float32).copy(), v, iters, gamma, int(sart))
        return v

    def y_reproject(self, nx, ny, th, c20_one, origin, vol):
        val = np.zeros((ny, nx), np.float32)
        wt = np.zeros((ny, nx), np.float32)
        self.y.ref_y_reproject(nx, ny, th, _c(c20_one, np.float64), *origin,
                               _c(vol, np.float32), val, wt)
        return val, wt

    def y_update_weights(self, nx, ny, th, c20_one, origin, diff, valvol, wtvol):
        vv, wv = _c(valvol, np.float32).copy(), _c(wtvol, np.float32).copy()
        self.y.ref_y_update_weights(nx, ny, th, _c(c20_one, np.float64), *origin,
                                    _c(diff, np.float32).copy(), vv, wv)
        return vv, wv

    def y_update_by_projdiff(self, nx, ny, th, c20_one, origin, diff, vol, gamma):
        v = _c(vol, np.float32).copy()
        self.y.ref_y_update_by_projdiff(nx, ny, th, _c(c20_one, np.float64), *origin,
                                        _c(diff, np.float32).copy(), v, gamma)
        return v

    def y_sirt_threaded(self, nthreads, nx, ny, nt, th, c20, pitch, proj, row0,
                        nrows, iters, gamma):
        return self.y.ref_y_sirt_threaded(nthreads, nx, ny, nt, th, _c(c20, np.float64),
                                          pitch, _c(proj, np.float32), row0, nrows,
                                          iters, gamma)

    def y_sirt_zslabs(self, nthreads, nx, ny, nt, th, c20, origin, proj, vol, iters,
                      gamma):
        """The reference's whole-volume SIRT on host threads over z-slabs
        (exact; see ref_wrap.cpp).  Returns (volume, wall seconds)."""
        v = _c(vol, np.float32).copy()
        t = self.y.ref_y_sirt_zslabs(nthreads, nx, ny, nt, th, _c(c20, np.float64), *origin,
                                     _c(proj, np.float32), v, iters, gamma)
        return v, t

    def z_run(self, mode, nx, ny, nt, th, c20, origin, proj, vol, iters=0, gamma=0.0):
        """mode: 0 BPT, 2 WBP, 3 SIRT, 4 SART (Z layout, vol [th][ny][nx])."""
        v = _c(vol, np.float32).copy()
        with tempfile.TemporaryDirectory() as d:
            rc = self.z.ref_z_run(mode, nx, ny, nt, th, _c(c20, np.float64), *origin,
                                  _c(proj, np.float32), v, iters, gamma, d.encode())
        assert rc == 0, rc
        return v


def _ref_z_admm(self, nx, ny, nt, th, c20, origin, proj, vol, outer, cg, mu, soft):
    """The reference's ADMM (Z layout, vol [th][ny][nx])."""
    v = _c(vol, np.float32).copy()
    with tempfile.TemporaryDirectory() as d:
        rc = self.z.ref_z_admm(nx, ny, nt, th, _c(c20, np.float64), *origin,
                               _c(proj, np.float32), v, outer, cg, mu, soft, d.encode())
    assert rc == 0, rc
    return v


Reference.z_admm = _ref_z_admm


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))
