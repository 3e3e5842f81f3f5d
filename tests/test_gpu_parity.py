"""Parity of the sm_100a kernels, called through the C ABI, with the
reference CPU path (golden fixtures) and the oracle restatement (seeded
random cases).

Tolerance: relative L2 <= 1e-5 against the reference's own float32 CPU path,
the bar the plain FP32 GPU form must meet.  The kernels interpolate with
Q32.32 fixed-point coordinates and sum tilts in registers, so they are not
bit-identical to the reference's per-tilt float updates."""
import zlib

import numpy as np
import pytest
import torch

import oracle as O
from autom2_b200 import tiltrec as T

pytestmark = pytest.mark.gpu
TOL = 1e-5


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _dims(g, name):
    nx, ny, nt, th = (int(v) for v in g[f"{name}/dims"])
    return nx, ny, nt, th, tuple(float(v) for v in g[f"{name}/origin"])


@pytest.mark.parametrize("name", ["ysep", "ygen"])
def test_golden_y_layout(engine, golden, name):
    nx, ny, nt, th, org = _dims(golden, name)
    g = lambda k: golden[f"{name}/{k}"]  # noqa: E731
    engine.set_problem(nx, ny, nt, th, g("coeff8"), T.LAYOUT_Y, org)
    vol = torch.zeros((ny, th, nx), device="cuda")
    engine.backproject(dev(g("proj")), vol)
    assert O.rel_l2(host(vol), g("bpt")) < TOL
    p = dev(g("proj"))
    engine.filter_rweight(p)
    assert O.rel_l2(host(p), g("filtered")) < 2e-6
    vol.zero_()
    engine.backproject(p, vol)
    assert O.rel_l2(host(vol), g("wbp")) < TOL
    vol = dev(g("vol0"))
    engine.sirt(dev(g("proj")), vol, 3, 0.5)
    assert O.rel_l2(host(vol), g("sirt3")) < TOL
    vol = dev(g("vol0"))
    engine.sart(dev(g("proj")), vol, 1, 0.5)
    assert O.rel_l2(host(vol), g("sart1")) < TOL
    val = torch.zeros((nt, ny, nx), device="cuda")
    wt = torch.zeros_like(val)
    engine.forward_project(dev(g("vol0")), val, wt)
    assert O.rel_l2(host(val)[nt // 2], g("fp_val")) < TOL
    assert O.rel_l2(host(wt)[nt // 2], g("fp_wt")) < TOL


def test_golden_z_layout(engine, golden):
    nx, ny, nt, th, org = _dims(golden, "zsep")
    g = lambda k: golden[f"zsep/{k}"]  # noqa: E731
    engine.set_problem(nx, ny, nt, th, g("coeff8"), T.LAYOUT_Z, org)
    vol = torch.zeros((th, ny, nx), device="cuda")
    engine.backproject(dev(g("proj")), vol)
    assert O.rel_l2(host(vol), g("bpt")) < TOL
    vol.zero_()
    engine.wbp(dev(g("proj")), vol)
    assert O.rel_l2(host(vol), g("wbp")) < TOL
    vol = dev(g("vol0"))
    engine.sirt(dev(g("proj")), vol, 2, 0.7)
    assert O.rel_l2(host(vol), g("sirt2")) < TOL


def test_golden_cfg0_scaled(engine, golden):
    nx, ny, nt, th, org = _dims(golden, "cfg0s4")
    g = lambda k: golden[f"cfg0s4/{k}"]  # noqa: E731
    engine.set_problem(nx, ny, nt, th, g("coeff8"), T.LAYOUT_Y, org)
    vol = torch.zeros((ny, th, nx), device="cuda")
    engine.wbp(dev(g("proj")), vol)
    assert O.rel_l2(host(vol), g("wbp")) < TOL
    vol.zero_()
    engine.sirt(dev(g("proj")), vol, 5, 0.5)
    assert O.rel_l2(host(vol), g("sirt5")) < TOL


# ---------------------------------------------------------------- random cases

CASES = {
    # name: (nx, ny, nt, th, amax, offset, pitch, zshift, shift_sigma, rot_deg)
    "sep_shift": (67, 45, 11, 19, 60, 0.0, 0.0, 0.0, 1.0, 0.0),
    "sep_big_shift": (40, 33, 9, 21, 70, 5.0, 0.0, 3.0, 12.0, 0.0),
    "steep": (50, 26, 8, 40, 85, 0.0, 0.0, 0.0, 0.5, 0.0),
    "xtilt": (58, 37, 10, 17, 60, 1.0, 6.0, -2.0, 0.7, 0.0),
    "rotated": (64, 48, 12, 16, 65, 0.0, 0.3, 0.0, 1.0, 3.0),
    "big_rotation": (48, 48, 7, 12, 50, 0.0, 0.0, 0.0, 0.0, 25.0),
}


def _random_case(restatement, name, layout):
    nx, ny, nt, th, amax, off, pitch, zs, sh, rot = CASES[name]
    rng = np.random.default_rng(zlib.crc32(name.encode()) + layout)
    ang = np.sort(rng.uniform(-amax, amax, nt)).astype(np.float32)
    c8 = restatement.coeffs(ang, off, pitch, zs)
    if rot:
        psi = np.deg2rad(rng.normal(0, rot, nt))
        a, b = c8[:, :4].copy(), c8[:, 4:].copy()
        c8[:, :4] = np.cos(psi)[:, None] * a - np.sin(psi)[:, None] * b
        c8[:, 4:] = np.sin(psi)[:, None] * a + np.cos(psi)[:, None] * b
    c8[:, 0] += rng.normal(0, sh, nt)
    c8[:, 4] += rng.normal(0, sh, nt)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    vshape = (ny, th, nx) if layout == 0 else (th, ny, nx)
    vol0 = rng.normal(size=vshape).astype(np.float32)
    org = T.default_origin(layout, nx, ny, th)
    return nx, ny, nt, th, c8, proj, vol0, org


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_random_vs_oracle(engine, restatement, name, layout):
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _random_case(R, name, layout)
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    vol = dev(vol0)
    engine.backproject(dev(proj), vol)
    assert O.rel_l2(host(vol), R.backproject(g, c8, proj, vol0)) < TOL
    val = torch.zeros((nt, ny, nx), device="cuda")
    wt = torch.zeros_like(val)
    engine.forward_project(dev(vol0), val, wt)
    for t in range(nt):
        v, w = R.reproject(g, c8[t], vol0)
        assert O.rel_l2(host(val)[t], v) < TOL, t
        assert O.rel_l2(host(wt)[t], w) < TOL, t
    vol = dev(vol0)
    engine.sirt(dev(proj), vol, 2, 0.6)
    assert O.rel_l2(host(vol), R.sirt(g, c8, proj, vol0, 2, 0.6)) < TOL
    vol = dev(vol0)
    engine.sart(dev(proj), vol, 1, 0.4)
    assert O.rel_l2(host(vol), R.sart(g, c8, proj, vol0, 1, 0.4)) < TOL


def test_exact_integer_geometry(engine, restatement):
    """Tilt 0 with no shift puts every voxel exactly on a detector column
    (dx = 0): the back-projection is the projection row, copied along z.
    The kernels interpolate with one FMA, fma(1+dx, s, b-s), which returns b
    to within one rounding of b-s at dx = 0."""
    nx, ny, nt, th = 33, 9, 1, 5
    c8 = restatement.coeffs(np.zeros(1, np.float32))
    rng = np.random.default_rng(5)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    org = T.default_origin(0, nx, ny, th)
    engine.set_problem(nx, ny, nt, th, c8, 0, org)
    vol = torch.zeros((ny, th, nx), device="cuda")
    engine.backproject(dev(proj), vol)
    out = host(vol)
    want = np.broadcast_to(proj[0][:, None, :], out.shape)
    assert O.rel_l2(out, want) < 1e-6
    assert np.abs(out - want).max() <= 4 * np.finfo(np.float32).eps * np.abs(proj).max()


@pytest.mark.parametrize("layout", [0, 1])
def test_zslabs_add_up(engine, restatement, layout):
    """Back-projecting z-slabs separately equals the whole volume, and the
    forward projections of slabs sum to the whole."""
    nx, ny, nt, th, c8, proj, vol0, org = _random_case(restatement, "rotated", layout)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    full = torch.zeros(vol0.shape, device="cuda")
    engine.backproject(dev(proj), full)
    parts = torch.zeros_like(full)
    for z0, nz in ((0, 5), (5, 7), (12, th - 12)):
        view = parts[:, z0:, :] if layout == 0 else parts[z0:]
        engine.backproject(dev(proj), view, z0, nz)
    assert O.rel_l2(host(parts), host(full)) < 1e-6
    v = dev(vol0)
    whole = torch.zeros((nt, ny, nx), device="cuda")
    engine.forward_project(v, whole)
    summed = torch.zeros_like(whole)
    for z0, nz in ((0, 9), (9, th - 9)):
        view = v[:, z0:, :] if layout == 0 else v[z0:]
        engine.forward_project(view, summed, None, z0, nz)
    # Slabs form different forward-projection tiles, hence different
    # fixed-point scales (see test_cfg1_forward_projection_linear).
    assert O.rel_l2(host(summed), host(whole)) < 2e-5


# FFT sizes M = 16 .. 16384: every first-pass radix (2, 4, 8, none), the
# two-butterfly blocks of M = 16384, and an odd row count (9) so the last
# pair has one row.
@pytest.mark.parametrize("nx", [8, 12, 40, 100, 256, 500, 1024, 4096, 7000])
def test_filter_widths(engine, restatement, nx):
    rng = np.random.default_rng(nx)
    rows = rng.normal(size=(1, 9, nx)).astype(np.float32)
    c8 = restatement.coeffs(np.zeros(1, np.float32))
    engine.set_problem(nx, 9, 1, 4, c8, 0)
    p = dev(rows)
    engine.filter_rweight(p)
    assert O.rel_l2(host(p), restatement.filter_rweight(rows)) < 2e-6


def test_host_buffer_path(engine, golden):
    """tr_reconstruct_host (host in, host out) equals the device path."""
    nx, ny, nt, th, org = _dims(golden, "cfg0s4")
    g = lambda k: golden[f"cfg0s4/{k}"]  # noqa: E731
    engine.set_problem(nx, ny, nt, th, g("coeff8"), T.LAYOUT_Y, org)
    vol = np.zeros((ny, th, nx), np.float32)
    engine.reconstruct_host("WBP", g("proj").copy(), vol)
    assert O.rel_l2(vol, g("wbp")) < TOL
    vol[:] = 0
    engine.reconstruct_host("SIRT", g("proj").copy(), vol, 5, 0.5)
    assert O.rel_l2(vol, g("sirt5")) < TOL
    # Zero start: the host volume is output only (NaNs in it are not read).
    want = vol.copy()
    for method, iters, ref in (("WBP", 0, "wbp"), ("SIRT", 5, "sirt5")):
        vol[:] = np.nan
        engine.reconstruct_host(method, g("proj").copy(), vol, iters, 0.5, zero_start=True)
        assert np.isfinite(vol).all()
        assert O.rel_l2(vol, g(ref)) < TOL
    np.testing.assert_array_equal(vol, want)


def _recon_host(eng, golden, name, method, iters):
    nx, ny, nt, th, org = _dims(golden, name)
    g = lambda k: golden[f"{name}/{k}"]  # noqa: E731
    eng.set_problem(nx, ny, nt, th, g("coeff8"), T.LAYOUT_Y, org)
    vol = np.empty((ny, th, nx), np.float32)
    eng.reconstruct_host(method, g("proj").copy(), vol, iters, 0.5, zero_start=True)
    return vol


@pytest.mark.parametrize("budgeted", [False, True])
def test_scratch_reuse_across_problems(golden, budgeted):
    """A context keeps its scratch buffers across problems.  Alternating SIRT
    on one series with WBP on another reuses them (no growth after the first
    round); under a budget that fits only the SIRT buffers, the buffers idle
    in the current problem make room (WBP's filter spectrum displaces them,
    and SIRT takes the room back).  The volumes match fresh contexts'."""
    jobs = (("cfg0s4", "SIRT", 5), ("ygen", "WBP", 0))
    want = {}
    for name, method, iters in jobs:
        fresh = T.Engine(0)
        want[name] = _recon_host(fresh, golden, name, method, iters)
        fresh.close()
    assert O.rel_l2(want["cfg0s4"], golden["cfg0s4/sirt5"]) < TOL
    assert O.rel_l2(want["ygen"], golden["ygen/wbp"]) < TOL
    eng = T.Engine(0)
    _recon_host(eng, golden, *jobs[0])
    need = eng.scratch_bytes
    eng.close()
    eng = T.Engine(0, hbm_budget=need if budgeted else 0)
    held = []
    for _ in range(2):
        for name, method, iters in jobs + jobs[:1]:
            assert O.rel_l2(_recon_host(eng, golden, name, method, iters), want[name]) < 1e-6
        held.append(eng.scratch_bytes)
    assert held[1] == held[0]
    assert held[0] <= need if budgeted else held[0] > need
    eng.close()


def test_errors_are_reported(engine):
    with pytest.raises(T.TiltRecError):
        engine.set_problem(0, 4, 1, 4, np.zeros((1, 8)))
    engine.set_problem(16, 8, 1, 4, np.array([[0, 1, 0, 0, 0, 0, 1, 0.]]))
    with pytest.raises(T.TiltRecError):
        engine.backproject(torch.zeros(1, device="cuda"), torch.zeros(1, device="cuda"), 3, 5)
    # A tile window wider than the kernels' Q9.23 coordinates address.
    with pytest.raises(T.TiltRecError) as e:
        engine.set_problem(64, 8, 1, 4, np.array([[0, 20, 0, 0, 0, 0, 1, 0.]]))
    assert e.value.status == -7  # TR_ERR_UNSUPPORTED
    small = T.Engine(0, hbm_budget=1024)
    small.set_problem(64, 64, 4, 8, np.tile([[0, 1, 0, 0, 0, 0, 1, 0.]], (4, 1)))
    with pytest.raises(T.TiltRecError) as e:
        small.sirt(torch.zeros((4, 64, 64), device="cuda"),
                   torch.zeros((64, 8, 64), device="cuda"), 1, 0.5)
    assert e.value.status == -3  # TR_ERR_BUDGET
    small.close()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("nx", [64, 300, 1024, 4096])
def test_fbp_filter_widths(engine, restatement, nx, mode):
    """FBP row filters (Shepp-Logan, Ram-Lak) against the oracle's double
    sum; both branches of the reference's mirrored extension (short rows)."""
    rng = np.random.default_rng(nx * 3 + mode)
    rows = rng.normal(size=(2, 5, nx)).astype(np.float32)
    c8 = restatement.coeffs(np.zeros(2, np.float32))
    engine.set_problem(nx, 5, 2, 4, c8, 0)
    p = dev(rows)
    engine.filter_fbp(p, mode)
    want = restatement.filter_fbp(rows, mode)
    got = host(p)
    assert O.rel_l2(got, want) < 1e-6
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()


@pytest.mark.parametrize("mode", [0, 1])
def test_fbp_filter_vs_reference(engine, reference, mode):
    """The FBP row filter against the unmodified reference's
    (ApplyFilterInplace modes 0/1 in oracle/_ref, OpenCV C-API shim with
    exact DFTs), on a stack whose rows take the long mirrored extension."""
    rng = np.random.default_rng(40 + mode)
    nt, ny, nx = 3, 11, 256
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    c8 = T.geometry_from_angles(np.zeros(nt, np.float32))
    engine.set_problem(nx, ny, nt, 4, c8, 0)
    p = dev(proj)
    engine.filter_fbp(p, mode)
    want = reference.filter_fbp(proj, mode)
    got = host(p)
    assert O.rel_l2(got, want) < 1e-6
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()


@pytest.mark.parametrize("layout", [0, 1])
def test_fbp_reconstruction(engine, restatement, layout):
    """--method FBP: Shepp-Logan filter then the back-projection, through the
    host-buffer call, against the oracle."""
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _random_case(R, "xtilt", layout)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    vol = np.zeros(vol0.shape, np.float32)
    engine.reconstruct_host("FBP", proj.copy(), vol)
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    want = R.backproject(g, c8, R.filter_fbp(proj, 0), np.zeros(vol0.shape, np.float32))
    assert O.rel_l2(vol, want) < TOL


@pytest.mark.parametrize("outer,cg", [(1, 1), (2, 1), (3, 1)])
def test_admm_vs_reference(engine, restatement, reference, outer, cg):
    """ADMM against the reference's own ADMM (TiltRecZ-mpi's routine,
    compiled in oracle/_ref), bar 1e-4.  One CG iteration per outer step: the
    reference's CG update p = r + beta p takes beta = +(r.Ap)/(p.Ap), the
    opposite sign of the conjugate direction, so from the second CG iteration
    on it diverges (on this data cg = 3 reaches 9e10 and a 1e-6 change of
    the input changes the result by 100 %; cg = 4 gives NaN).  Both sides run
    that same algorithm; beyond one CG iteration only chaos is compared."""
    nx, ny, nt, th = 48, 20, 9, 10
    rng = np.random.default_rng(outer * 10 + cg)
    ang = np.linspace(-60, 60, nt).astype(np.float32)
    c8 = restatement.coeffs(ang, 0.5, 0.0, 1.0)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    org = T.default_origin(T.LAYOUT_Z, nx, ny, th)
    engine.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Z, org)
    vol = torch.zeros((th, ny, nx), device="cuda")
    engine.admm(dev(proj), vol, outer, cg, 0.5, 0.01)
    want = reference.z_admm(nx, ny, nt, th, O.coeff20(c8), org, proj,
                            np.zeros((th, ny, nx), np.float32), outer, cg, 0.5, 0.01)
    assert np.isfinite(want).all()
    assert O.rel_l2(host(vol), want) < 1e-4


def test_admm_layouts_agree(engine, restatement):
    """The same problem in the Y and Z layouts (same origin) gives the same
    volume, transposed."""
    nx, ny, nt, th = 40, 16, 7, 12
    rng = np.random.default_rng(21)
    c8 = restatement.coeffs(np.linspace(-55, 55, nt).astype(np.float32), 0.0, 2.0, 0.0)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    org = (nx * 0.5, ny * 0.5, th * 0.5)
    engine.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Z, org)
    vz = torch.zeros((th, ny, nx), device="cuda")
    engine.admm(dev(proj), vz, 1, 3, 0.5, 0.01)
    engine.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Y, org)
    vy = torch.zeros((ny, th, nx), device="cuda")
    engine.admm(dev(proj), vy, 1, 3, 0.5, 0.01)
    assert O.rel_l2(host(vy).transpose(1, 0, 2), host(vz)) < 1e-5


@pytest.mark.parametrize("shape,factor", [((3, 64, 96), 2), ((2, 37, 53), 3),
                                          ((1, 1000, 1023), 4), ((2, 40, 40), 1)])
def test_resample_bin(engine, restatement, shape, factor):
    """Device area binning (the resample step) against the oracle."""
    rng = np.random.default_rng(sum(shape) + factor)
    a = rng.normal(size=shape).astype(np.float32)
    got = host(T.resample_bin(dev(a), factor))
    want = restatement.resample_bin(a, factor)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-6 * max(1.0, np.abs(want).max())


def test_bounded_wait_gives_up(engine, golden):
    """A device wait on a barrier nothing completes runs out after its budget
    (50 ms) and reports TR_ERR_TIMEOUT through the sticky word; the context
    is usable afterwards (a reconstruction still matches the fixtures)."""
    import time
    t0 = time.perf_counter()
    assert engine.selftest_wait(50000) == -5  # TR_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    nx, ny, nt, th, org = _dims(golden, "cfg0s4")
    g = lambda k: golden[f"cfg0s4/{k}"]  # noqa: E731
    engine.set_problem(nx, ny, nt, th, g("coeff8"), T.LAYOUT_Y, org)
    vol = torch.zeros((ny, th, nx), device="cuda")
    engine.wbp(dev(g("proj")), vol)
    engine.synchronize()
    assert O.rel_l2(host(vol), g("wbp")) < TOL


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("th,zero_start,iters", [(160, True, 3), (160, False, 2), (40, True, 2),
                                                  (130, False, 1), (128, True, 0)])
def test_host_sirt_with_overlapped_copies(engine, restatement, layout, th, zero_start, iters):
    """tr_reconstruct_host SIRT from page-locked buffers: the stack uploads
    while the weights are computed and the last update runs in z-slabs whose
    sections copy back while the next slab updates.  Same volume as the
    device path (1e-6: the forward projection's float atomic order) and the
    oracle."""
    R = restatement
    rng = np.random.default_rng(th + layout + iters)
    nx, ny, nt = 64, 24, 9
    ang = np.linspace(-60, 60, nt).astype(np.float32)
    c8 = R.coeffs(ang, 0.5, 1.5, 0.0)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    vshape = (ny, th, nx) if layout == 0 else (th, ny, nx)
    vol0 = (np.zeros(vshape, np.float32) if zero_start
            else rng.normal(size=vshape).astype(np.float32) * 0.1)
    org = T.default_origin(layout, nx, ny, th)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    want = dev(vol0)
    engine.sirt(dev(proj), want, iters, 0.5)
    ph = torch.from_numpy(proj).pin_memory()
    vh = torch.from_numpy(np.full(vshape, np.nan, np.float32) if zero_start else vol0.copy())
    vh = vh.pin_memory()
    engine.reconstruct_host("SIRT", ph.numpy(), vh.numpy(), iters, 0.5, zero_start=zero_start)
    got = vh.numpy()
    assert np.isfinite(got).all()
    if iters == 0:  # the starting volume comes back unchanged
        assert np.array_equal(got, host(want))
        return
    assert O.rel_l2(got, host(want)) < 1e-6
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    assert O.rel_l2(got, R.sirt(g, c8, proj, vol0, iters, 0.5)) < 1e-5


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("name", ["xtilt", "rotated", "sep_big_shift"])
def test_deterministic_forward_projection(engine, restatement, name, layout):
    """tr_set_deterministic: the forward projection's flush adds int64 fixed
    point at one launch-wide scale, so repeated SIRT runs are bitwise equal;
    the sums match the default float flush (1e-6) and the oracle (1e-5).  With
    one voxel 1e4 times the rest the launch-wide scale follows that voxel, and
    the deterministic sums still match the float flush's to float precision.
    (The per-tile window scale, common to both flushes, rounds each
    contribution to ~5e-7 of its tile's largest voxel, so both are coarse
    around such a spike; that is the default path's own limit.)"""
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _random_case(R, name, layout)
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    try:
        default = dev(vol0)
        engine.sirt(dev(proj), default, 3, 0.5)
        engine.set_deterministic(True)
        runs = []
        for _ in range(2):
            v = dev(vol0)
            engine.sirt(dev(proj), v, 3, 0.5)
            runs.append(host(v))
        assert np.array_equal(runs[0], runs[1])
        assert O.rel_l2(runs[0], host(default)) < 1e-6
        assert O.rel_l2(runs[0], R.sirt(g, c8, proj, vol0, 3, 0.5)) < 1e-5
        spiky = vol0.copy()
        spiky.reshape(-1)[spiky.size // 3] = 1e4 * np.abs(vol0).max()
        val = torch.zeros((nt, ny, nx), device="cuda")
        engine.forward_project(dev(spiky), val)
        got = host(val)
        engine.set_deterministic(False)
        fval = torch.zeros_like(val)
        engine.forward_project(dev(spiky), fval)
        flt = host(fval)
        # the launch-wide int64 scale adds no error beyond the float flush's
        diff = np.abs(got - flt)
        assert diff.max() <= 1e-6 * np.abs(flt).max()
        assert O.rel_l2(got, flt) < 1e-6
    finally:
        engine.set_deterministic(False)


def test_sirt_gated_fp64_norms(engine, restatement):
    """tr_sirt_gated: the residual norms are FP64 sums of the FP32 residual
    (the first, from a zero volume, is exactly |p| in FP64), decrease, repeat
    exactly, and a relative tolerance stops the loop before an update; with
    no tolerance the volume is tr_sirt's."""
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _random_case(R, "xtilt", 1)
    engine.set_problem(nx, ny, nt, th, c8, 1, org)
    p = dev(proj)
    zero = np.zeros_like(vol0)
    v = dev(zero)
    done, norms = engine.sirt_gated(p, v, 6, 0.5)
    assert done == 6 and len(norms) == 6
    assert abs(norms[0] - np.linalg.norm(proj.astype(np.float64))) <= 1e-13 * norms[0]
    assert np.all(np.diff(norms) < 0)
    w = dev(zero)
    engine.sirt(p, w, 6, 0.5)
    assert O.rel_l2(host(v), host(w)) < 1e-6
    _, again = engine.sirt_gated(p, dev(zero), 6, 0.5)
    assert O.rel_l2(again, norms) < 1e-6
    # stop once an iteration removes less than 30 % of the residual norm
    v = dev(zero)
    done, nr = engine.sirt_gated(p, v, 20, 0.5, rel_tol=0.3)
    assert 0 < done < 20 and len(nr) == done + 1
    assert nr[-2] - nr[-1] < 0.3 * nr[-2]
    assert all(nr[k - 1] - nr[k] >= 0.3 * nr[k - 1] for k in range(1, done))
    w = dev(zero)
    engine.sirt(p, w, done, 0.5)
    assert O.rel_l2(host(v), host(w)) < 1e-6
