"""z-slab SIRT (tr_sirt_zslabs, tr_autotune_zslab): TiltRecZ's split of the
volume along z (TR/main/main-mpiz.cpp:1054-1069) with CuSIRTZ's iteration
(TR/TiltRec_cuda_z/recon_z.cu:85-190), the volume on the device or staged
from host memory slab by slab.

The sweep order (update slab k, then forward-project it into the next
iteration's sums) computes the same sums as the whole-volume SIRT; slab
boundaries are tile boundaries, so only the order of the forward
projection's float atomic adds differs (1e-6 against tr_sirt, 1e-5 against
the oracle)."""
import numpy as np
import pytest
import torch

import oracle as O
from autom2_b200 import tiltrec as T

pytestmark = pytest.mark.gpu


def _case(R, layout, th=80, nx=72, ny=40, nt=11, seed=3):
    rng = np.random.default_rng(seed + layout)
    ang = np.linspace(-60, 60, nt).astype(np.float32)
    c8 = R.coeffs(ang, 0.5, 1.5, 0.0)  # tilt-axis offset and x-tilt: general geometry
    psi = np.deg2rad(rng.normal(0, 0.5, nt))
    a, b = c8[:, :4].copy(), c8[:, 4:].copy()
    c8[:, :4] = np.cos(psi)[:, None] * a - np.sin(psi)[:, None] * b
    c8[:, 4:] = np.sin(psi)[:, None] * a + np.cos(psi)[:, None] * b
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    vshape = (ny, th, nx) if layout == 0 else (th, ny, nx)
    vol0 = rng.normal(size=vshape).astype(np.float32) * 0.1
    org = T.default_origin(layout, nx, ny, th)
    return nx, ny, nt, th, c8, proj, vol0, org


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("where", ["device", "pinned", "numpy"])
@pytest.mark.parametrize("depth", [32, 64, 1000])
def test_zslab_sirt_equals_whole_volume(engine, restatement, layout, where, depth):
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _case(R, layout)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    p = torch.from_numpy(proj).cuda()
    whole = torch.from_numpy(vol0).cuda()
    engine.sirt(p, whole, 3, 0.5)
    if where == "device":
        v = torch.from_numpy(vol0).cuda()
    elif where == "pinned":
        v = torch.from_numpy(vol0).pin_memory()
    else:
        v = vol0.copy()
    engine.sirt_zslabs(p, v, 3, 0.5, depth)
    torch.cuda.synchronize()
    got = v.cpu().numpy() if isinstance(v, torch.Tensor) else v
    assert O.rel_l2(got, whole.cpu().numpy()) < 1e-6
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    assert O.rel_l2(got, R.sirt(g, c8, proj, vol0, 3, 0.5)) < 1e-5


@pytest.mark.parametrize("layout", [0, 1])
def test_zslab_sirt_16bit_storage(engine, restatement, layout):
    """FP16 stack and FP16 residual through the slabs, as tr_sirt_lp."""
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _case(R, layout, seed=11)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    p = torch.from_numpy(proj).cuda()
    q, scale = engine.quantize(p, torch.float16)
    whole = torch.from_numpy(vol0).cuda()
    engine.sirt_lp(q, scale, whole, 3, 0.5, "f16")
    v = torch.from_numpy(vol0).pin_memory()
    engine.sirt_zslabs(q, v, 3, 0.5, 32, scale=scale, resid_dtype="f16")
    assert O.rel_l2(v.numpy(), whole.cpu().numpy()) < 1e-4
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    assert O.rel_l2(v.numpy(), R.sirt(g, c8, proj, vol0, 3, 0.5, fp64=True)) < 1e-3


@pytest.mark.parametrize("where", ["device", "pinned"])
def test_autotune_zslab_picks_a_depth_and_leaves_the_volume(engine, restatement, where):
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _case(R, 1, th=150)
    engine.set_problem(nx, ny, nt, th, c8, 1, org)
    p = torch.from_numpy(proj).cuda()
    v = torch.from_numpy(vol0).cuda() if where == "device" else \
        torch.from_numpy(vol0).pin_memory()
    depth, ms = engine.autotune_zslab(p, v)
    assert depth in (32, 64, 128, 150) and ms > 0
    torch.cuda.synchronize()
    assert torch.equal(v.cpu(), torch.from_numpy(vol0))
    engine.sirt_zslabs(p, v, 2, 0.5, depth)
    torch.cuda.synchronize()
    g = R.geom(nx, ny, nt, th, 1, 0, org)
    assert O.rel_l2(v.cpu().numpy(), R.sirt(g, c8, proj, vol0, 2, 0.5)) < 1e-5


def test_zslab_budget_limits_depth(restatement):
    """Under a budget that holds the 32-section staging but not the
    64-section one, autotuning keeps to the depths that fit."""
    R = restatement
    nx, ny, nt, th, c8, proj, vol0, org = _case(R, 1, th=128, nx=64, ny=64, nt=9)
    section = nx * ny * 4
    p = torch.from_numpy(proj).cuda()
    probe = T.Engine(0)
    try:  # scratch of a 32-section run, measured
        probe.set_problem(nx, ny, nt, th, c8, 1, org)
        probe.sirt_zslabs(p, torch.from_numpy(vol0).pin_memory(), 1, 0.5, 32)
        need32 = probe.scratch_bytes
    finally:
        probe.close()
    e = T.Engine(0, hbm_budget=need32 + 48 * section)  # 64 needs 96 more sections
    try:
        e.set_problem(nx, ny, nt, th, c8, 1, org)
        v = torch.from_numpy(vol0).pin_memory()
        depth, _ = e.autotune_zslab(p, v)
        assert depth == 32
        e.sirt_zslabs(p, v, 2, 0.5, depth)
        g = R.geom(nx, ny, nt, th, 1, 0, org)
        assert O.rel_l2(v.numpy(), R.sirt(g, c8, proj, vol0, 2, 0.5)) < 1e-5
    finally:
        e.close()
