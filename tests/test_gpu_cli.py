"""The drop-in executables against the reference's own executables (GPU).

The reference TiltRec-mpi / TiltRecZ-mpi are the unmodified reference sources
built into oracle/_ref (one rank).  Both sides read the same MRC stack and
tilt file; the output headers must match field for field (the statistics to
float tolerance) and the volumes to relative L2 1e-5.  TiltRecZ-mpi's BPT and
SIRT abort before writing their output (a double free in the reference), so
those two are checked against the oracle restatement instead.  The reference
FBP filter needs OpenCV, which the oracle build provides as a test-only C-API
shim with exact DFTs."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from autom2_b200 import build
from autom2_b200 import tiltrec as T
from mrc_util import read_mrc, write_angles, write_mrc

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(build.LIB), "..", "bin")
TOL = 1e-5


@pytest.fixture(scope="module")
def case(tmp_path_factory):
    build.build()
    d = tmp_path_factory.mktemp("cli")
    rng = np.random.default_rng(3)
    nx, ny, nt = 64, 40, 13
    ang = np.linspace(-60, 60, nt).astype(np.float32)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    write_mrc(d / "stack.mrc", proj)
    write_angles(d / "a.rawtlt", ang)
    return d, proj, ang


def ours(layout, *args, dialect="cuda"):
    exe = os.path.join(BIN, ("TiltRec-" if layout == 0 else "TiltRecZ-") + dialect)
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    return r


def reference(layout, *args):
    if not O.reference_available():
        pytest.skip("oracle/_ref not built")
    exe = os.path.join(O.REF_DIR, "TiltRec-mpi" if layout == 0 else "TiltRecZ-mpi")
    r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return r


def compare(a_path, b_path, tol=TOL, sections=None):
    ha, ra, da = read_mrc(a_path)
    hb, rb, db = read_mrc(b_path)
    if sections is not None:
        da, db = da[sections], db[sections]
    for f in ("nx", "ny", "nz", "mode", "m", "len", "ang", "map", "next", "creatid", "nlabl"):
        assert np.array_equal(ha[f], hb[f]), f
    # everything outside the statistics is byte-identical
    strip = lambda r: r[:76] + r[88:]  # noqa: E731  (amin/amax/amean at bytes 76..87)
    assert strip(ra) == strip(rb)
    for f in ("amin", "amax", "amean"):
        assert abs(float(ha[f]) - float(hb[f])) <= 1e-4 * max(1.0, abs(float(hb[f]))), f
    assert O.rel_l2(da, db) < tol


@pytest.mark.parametrize("method", ["BPT", "WBP", "SIRT,3,0.5", "SART,1,0.4"])
@pytest.mark.parametrize("geometry", ["0,0,0,12", "1.5,2.0,-1.5,10"])
def test_tiltrec_vs_tiltrec_mpi(case, method, geometry):
    d, proj, ang = case
    a, b = d / f"ours_{method}_{geometry}.mrc", d / f"ref_{method}_{geometry}.mrc"
    common = ["--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
              "--geometry", geometry, "--method", method]
    ours(0, *common, "--output", str(a))
    reference(0, *common, "--output", str(b))
    # With XTILT != 0 a single TiltRec-mpi rank keeps add_right =
    # ceil(|tan(pitch)| * thickness) (main-mpi.cpp:728-740: the first branch
    # resets only add_left), so it reads that many rows past the end of the
    # stack (unread, uninitialised) and reconstructs them into the top
    # sections.  The rows they reach are excluded from the comparison with
    # the reference (two for the one-pass methods; SART's per-tilt updates
    # carry them two rows further: its row 36 still differs from the
    # restatement by 1e-5, row 35 by 5e-7) and compared with the oracle
    # restatement instead, which the whole volume must match.
    pitch = float(geometry.split(",")[1])
    cut = slice(0, proj.shape[1] - (4 if method.startswith("SART") else 2)) if pitch else None
    compare(a, b, sections=cut)
    if pitch:
        _, _, got = read_mrc(a)
        assert O.rel_l2(got, restated(0, proj, ang, geometry, method)) < TOL


def restated(layout, proj, ang, geometry, method):
    """The oracle restatement's reconstruction for a CLI geometry/method."""
    R = O.Restatement()
    nt, ny, nx = proj.shape
    off, pitch, zs, th = (float(v) for v in geometry.split(","))
    th = int(th)
    c8 = R.coeffs(ang, off, pitch, zs)
    org = T.default_origin(layout, nx, ny, th)
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    vshape = (ny, th, nx) if layout == 0 else (th, ny, nx)
    zero = np.zeros(vshape, np.float32)
    parts = method.split(",")
    if parts[0] == "BPT":
        return R.backproject(g, c8, proj, zero)
    if parts[0] == "WBP":
        return R.backproject(g, c8, R.filter_rweight(proj), zero)
    if parts[0] == "FBP":
        return R.backproject(g, c8, R.filter_fbp(proj, 0), zero)
    f = R.sirt if parts[0] == "SIRT" else R.sart
    return f(g, c8, proj, zero, int(parts[1]), float(parts[2]))


def test_initial_volume(case):
    d, proj, ang = case
    th = 8
    init = np.random.default_rng(9).normal(size=(40, th, 64)).astype(np.float32)
    write_mrc(d / "init.mrc", init)
    common = ["--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
              "--geometry", f"0,0,0,{th}", "--method", "SIRT,2,0.5"]
    ours(0, *common, "--output", str(d / "oi.mrc"), "--initial", str(d / "init.mrc"))
    reference(0, *common, "--output", str(d / "ri.mrc"), "--initial", str(d / "init.mrc"))
    compare(d / "oi.mrc", d / "ri.mrc")


@pytest.mark.parametrize("method", ["WBP", "SART,1,0.4"])
def test_tiltrecz_vs_tiltrecz_mpi(case, method):
    d, proj, ang = case
    a, b = d / f"oz_{method}.mrc", d / f"rz_{method}.mrc"
    common = ["--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
              "--geometry", "1.0,0,2.0,12", "--method", method]
    ours(1, *common, "--output", str(a))
    reference(1, *common, "--output", str(b))
    compare(a, b)


@pytest.mark.parametrize("layout", [0, 1])
def test_fbp_vs_reference_mpi(case, restatement, layout):
    """--method FBP against the reference's own TiltRec-mpi / TiltRecZ-mpi
    (whose FBP filter runs through the oracle's OpenCV C-API shim, exact
    DFTs), and against the oracle restatement."""
    d, proj, ang = case
    th = 10
    a, b = d / f"fbp_{layout}.mrc", d / f"rfbp_{layout}.mrc"
    geometry = f"0.5,0,0,{th}"
    common = ["--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
              "--geometry", geometry, "--method", "FBP"]
    ours(layout, *common, "--output", str(a))
    reference(layout, *common, "--output", str(b))
    compare(a, b)
    _, _, got = read_mrc(a)
    assert O.rel_l2(got, restated(layout, proj, ang, geometry, "FBP")) < TOL


@pytest.mark.parametrize("method", ["ADMM,1,1,0.5,0.01", "ADMM,2,1,0.5,0.01"])
def test_tiltrecz_admm_vs_tiltrecz_mpi(case, method):
    """ADMM through the drop-in executable against TiltRecZ-mpi's (bar 1e-4,
    as for the ADMM kernels: its CG amplifies float rounding)."""
    d, proj, ang = case
    a, b = d / f"oz_{method}.mrc", d / f"rz_{method}.mrc"
    common = ["--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
              "--geometry", "0,0,0,10", "--method", method]
    ours(1, *common, "--output", str(a))
    reference(1, *common, "--output", str(b))
    compare(a, b, tol=1e-4)


@pytest.mark.parametrize("method,iters", [("BPT", 0), ("SIRT", 2)])
def test_tiltrecz_vs_oracle(case, restatement, method, iters):
    d, proj, ang = case
    nt, ny, nx = proj.shape
    th = 12
    out = d / f"oz_{method}.mrc"
    m = method if not iters else f"{method},{iters},0.6"
    ours(1, "--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
         "--geometry", f"1.0,0,2.0,{th}", "--method", m, "--output", str(out))
    c8 = restatement.coeffs(ang, 1.0, 0.0, 2.0)
    org = T.default_origin(T.LAYOUT_Z, nx, ny, th)
    g = restatement.geom(nx, ny, nt, th, 1, 0, org)
    zero = np.zeros((th, ny, nx), np.float32)
    want = (restatement.backproject(g, c8, proj, zero) if method == "BPT"
            else restatement.sirt(g, c8, proj, zero, iters, 0.6))
    _, _, got = read_mrc(out)
    assert O.rel_l2(got, want) < TOL


def test_byte_and_short_stacks(case, restatement):
    d, proj, ang = case
    q = np.clip(np.round(proj * 20), -120, 120)
    for mode in (0, 1):
        write_mrc(d / f"stack{mode}.mrc", q, mode=mode, next_bytes=64 if mode else 0)
        common = ["--input", str(d / f"stack{mode}.mrc"), "--tiltfile", str(d / "a.rawtlt"),
                  "--geometry", "0,0,0,8", "--method", "BPT"]
        ours(0, *common, "--output", str(d / f"ob{mode}.mrc"))
        reference(0, *common, "--output", str(d / f"rb{mode}.mrc"))
        compare(d / f"ob{mode}.mrc", d / f"rb{mode}.mrc")


@pytest.mark.parametrize("layout", [0, 1])
def test_f2b_bytes(case, layout):
    """--f2b, mapped on the device and streamed to the file: Y layout in
    64-row slabs with EMA mean/deviation (alpha 0.9, recon_y.cu:164-181), Z
    layout the whole volume with its own statistics (recon_z.cu:164-172);
    z-score clamped to +-10 and mapped to 0..255 (basic.cu:442-475)."""
    d, proj, ang = case
    common = ["--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
              "--geometry", "0,0,0,8", "--method", "BPT"]
    ours(layout, *common, "--output", str(d / f"of{layout}.mrc"))
    ours(layout, *common, "--output", str(d / f"ob{layout}.mrc"), "--f2b")
    _, _, vol = read_mrc(d / f"of{layout}.mrc")
    hb, _, got = read_mrc(d / f"ob{layout}.mrc")
    assert int(hb["mode"]) == 0
    flat = vol.reshape(-1).astype(np.float32)
    slab = 64 * 8 * 64 if layout == 0 else flat.size
    alpha = np.float32(0.9 if layout == 0 else 0.0)
    want = np.zeros(flat.size, np.uint8)
    gm = gs = np.float32(0)
    for s0 in range(0, flat.size, slab):
        c = flat[s0:s0 + slab]
        m = np.float32(c.astype(np.float64).mean())
        sd = np.float32(np.sqrt(np.float32(((c - m) ** 2).astype(np.float64).mean())))
        gm = alpha * gm + (np.float32(1) - alpha) * m
        gs = alpha * gs + (np.float32(1) - alpha) * sd
        n4 = (c.size // 4) * 4
        z = np.clip((c[:n4] - gm) / gs, -10, 10)
        want[s0:s0 + n4] = (((z + 10) / 20) * 255).astype(np.uint8)
    assert np.mean(np.abs(got.reshape(-1).astype(int) - want.astype(int)) <= 1) > 0.999
    # header statistics: the middle section of the byte volume
    mid = got[got.shape[0] // 2].astype(np.float64)
    assert abs(float(hb["amean"]) - mid.mean()) < 1e-3 * max(1.0, mid.mean())


@pytest.mark.parametrize("mode", [2, 1, 0])
def test_resample_executable(case, restatement, tmp_path, mode):
    """The resample drop-in: bytes read unsigned and divided by 255, shorts
    as their value; float output; header the input's with the new sizes."""
    d, proj, ang = case
    rng = np.random.default_rng(mode)
    if mode == 2:
        data = proj
    elif mode == 1:
        data = np.round(proj * 300).astype(np.float32)
    else:
        data = rng.integers(0, 256, size=proj.shape).astype(np.float32)
    src = tmp_path / f"in{mode}.mrc"
    stored = data.astype(np.uint8).view(np.int8) if mode == 0 else data
    write_mrc(src, stored, mode=mode, next_bytes=32 if mode == 1 else 0)
    with open(src, "r+b") as f:  # input statistics the output must carry over
        f.seek(76)
        f.write(np.array([-1.5, 2.5, 0.25], "<f4").tobytes())
    out = tmp_path / f"out{mode}.mrc"
    exe = os.path.join(BIN, "resample")
    r = subprocess.run([exe, "-i", str(src), "-o", str(out), "-b", "3"], capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    hi, _, _ = read_mrc(src)
    ho, _, got = read_mrc(out)
    want = restatement.resample_bin(data / 255.0 if mode == 0 else data, 3)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-6 * max(1.0, np.abs(want).max())
    assert int(ho["mode"]) == 2
    assert [int(v) for v in ho["m"]] == [want.shape[2], want.shape[1], want.shape[0]]
    for f in ("amin", "amax", "amean", "next"):
        assert np.array_equal(ho[f], hi[f]), f
    # The reference's own tool on the same file: the same 1024-byte header
    # (its extended header is uninitialised memory, so only the main header
    # is compared) and the same binned sections.
    ref_exe = O.reference_resample_executable()
    if ref_exe is not None:
        ref_out = tmp_path / f"ref{mode}.mrc"
        r = subprocess.run([ref_exe, "-i", str(src), "-o", str(ref_out), "-b", "3"],
                           capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
        _, rraw, rdata = read_mrc(ref_out)
        _, oraw, _ = read_mrc(out)
        assert oraw == rraw
        assert np.abs(got - rdata).max() <= 1e-6 * max(1.0, np.abs(rdata).max())


@pytest.mark.parametrize("layout,method,geometry", [
    (0, "SIRT,2,0.5", "0,0,0,10"), (0, "WBP", "1.0,0,2.0,12"),
    (1, "WBP", "1.0,0,2.0,12"), (1, "SART,1,0.4", "0,0,0,10")])
def test_mpi_named_executables_vs_reference_mpi(case, layout, method, geometry):
    """TiltRec-mpi / TiltRecZ-mpi, the names the GUI spawns for CPU runs, with
    the mpi option dialect (--initial; --tiltfile long only), against the
    reference's own -mpi executables given the same command line."""
    d, proj, ang = case
    th = int(geometry.split(",")[-1])
    shape = (40, th, 64) if layout == 0 else (th, 40, 64)
    init = np.random.default_rng(5).normal(size=shape).astype(np.float32) * 0.1
    write_mrc(d / f"mi{layout}.mrc", init)
    a, b = d / f"om_{layout}_{method}.mrc", d / f"rm_{layout}_{method}.mrc"
    common = ["--input", str(d / "stack.mrc"), "--tiltfile", str(d / "a.rawtlt"),
              "--geometry", geometry, "--method", method]
    if method.startswith("S"):
        common += ["--initial", str(d / f"mi{layout}.mrc")]
    ours(layout, *common, "--output", str(a), dialect="mpi")
    reference(layout, *common, "--output", str(b))
    compare(a, b)


def test_mpi_dialect_rejects_cuda_only_options(case):
    d, _, _ = case
    exe = os.path.join(BIN, "TiltRec-mpi")
    for extra in (["--f2b"], ["-t", str(d / "a.rawtlt")], ["-a", "y"]):
        r = subprocess.run([exe, "--input", str(d / "stack.mrc"), *extra], capture_output=True,
                           text=True, timeout=60)
        assert r.returncode != 0, extra


@pytest.mark.parametrize("layout", [0, 1])
def test_volume_beyond_the_budget_streams_zslabs(tmp_path, layout):
    """A SIRT volume that does not fit the device budget (TILTREC_HBM_BUDGET)
    is kept in host memory and streamed through the device in autotuned
    z-slabs, as TiltRecZ streams through managed memory: the same file as the
    run without a budget."""
    build.build()
    rng = np.random.default_rng(8 + layout)
    nx, ny, nt, th = 128, 32, 9, 256
    ang = np.linspace(-30, 30, nt).astype(np.float32)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    write_mrc(tmp_path / "s.mrc", proj)
    write_angles(tmp_path / "s.rawtlt", ang)
    common = ["--input", str(tmp_path / "s.mrc"), "--tiltfile", str(tmp_path / "s.rawtlt"),
              "--geometry", f"0,0,0,{th}", "--method", "SIRT,3,0.5"]
    ours(layout, *common, "--output", str(tmp_path / "whole.mrc"))
    # device memory of the two forms, as the library counts it
    c8 = T.geometry_from_angles(ang)
    org = T.default_origin(layout, nx, ny, th)
    vshape = (ny, th, nx) if layout == 0 else (th, ny, nx)
    e = T.Engine(0)
    e.set_problem(nx, ny, nt, th, c8, layout, org)
    e.reconstruct_host("SIRT", proj.copy(), np.zeros(vshape, np.float32), 3, 0.5,
                       zero_start=True)
    whole_bytes = e.scratch_bytes
    e.close()
    e = T.Engine(0)
    e.set_problem(nx, ny, nt, th, c8, layout, org)
    assert e.sirt_host_zslabs(proj.copy(), np.zeros(vshape, np.float32), 3, 0.5, 32) == 32
    slab_bytes = e.scratch_bytes
    e.close()
    assert slab_bytes < whole_bytes
    budget = slab_bytes + (whole_bytes - slab_bytes) // 4
    exe = os.path.join(BIN, "TiltRec-cuda" if layout == 0 else "TiltRecZ-cuda")
    r = subprocess.run([exe, *common, "--output", str(tmp_path / "slabs.mrc")],
                       capture_output=True, text=True, timeout=300,
                       env={**os.environ, "TILTREC_HBM_BUDGET": str(budget)})
    assert r.returncode == 0, r.stderr + r.stdout
    assert "streaming it in z-slabs" in r.stderr
    compare(tmp_path / "slabs.mrc", tmp_path / "whole.mrc", tol=1e-6)
