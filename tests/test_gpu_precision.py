"""Mixed precision: 16-bit projection / residual storage (tr_quantize,
tr_backproject_lp, tr_sirt_lp) against the FP64 oracle.

Each reduced-precision result is reported as relative L2 and max-abs error
(the latter relative to the largest reference magnitude) against the
oracle's double-precision reconstruction of the same FP32 series.  Bars:

* the conversion itself is bit-exact against torch's round-to-nearest-even
  conversion of the scaled values, with power-of-two scales;
* back-projecting a 16-bit stack matches the FP64 back-projection of the
  dequantized stack within the plain FP32 bar (1e-5): storage is the only
  approximation;
* SIRT from FP16 projections with an FP32 or FP16 residual stays within
  relative L2 1e-4 of the FP64 SIRT of the unrounded series; a BF16 residual
  (8-bit mantissa, about 2e-3 relative rounding per element) within 2e-4;
  BF16 projections within 2e-3.

Two series: counting-noise projections (small integers, which FP16 and BF16
hold exactly, so only the residual storage rounds) and Gaussian-noise ones
(every projection value rounds)."""
import numpy as np
import pytest
import torch

import oracle as O
from autom2_b200 import synth
from autom2_b200 import tiltrec as T

pytestmark = pytest.mark.gpu
F16, BF16 = torch.float16, torch.bfloat16


def host(t):
    torch.cuda.synchronize()
    return t.float().cpu().numpy() if t.dtype != torch.float32 else t.cpu().numpy()


def errors(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return O.rel_l2(got, ref), float(np.abs(got - ref).max() / np.abs(ref).max())


@pytest.mark.parametrize("dtype", [F16, BF16])
def test_quantize_bit_exact(engine, dtype):
    nt, ny, nx = 7, 33, 70
    rng = np.random.default_rng(3)
    p = rng.normal(size=(nt, ny, nx)) * (10.0 ** np.arange(-3, 4))[:, None, None]
    p[2] = 0.0                      # an all-zero tilt keeps scale 1
    p[4, 0, 0] = 2.0 ** 20          # an exact power of two as the maximum
    p = p.astype(np.float32)
    c8 = np.tile([[0, 1, 0, 0, 0, 0, 1, 0.]], (nt, 1))
    engine.set_problem(nx, ny, nt, 4, c8, T.LAYOUT_Y)
    q, scale = engine.quantize(torch.from_numpy(p).cuda(), dtype)
    s = host(scale)
    assert np.all(s == 2.0 ** np.round(np.log2(s)))
    amax = np.abs(p).reshape(nt, -1).max(1)
    if dtype == F16:
        nz = amax > 0
        assert np.all(amax[nz] / s[nz] > 2.0 ** 13) and np.all(amax[nz] / s[nz] <= 2.0 ** 14)
        assert s[2] == 1.0
    else:
        assert np.all(s == 1.0)
    want = (torch.from_numpy(p) / torch.from_numpy(s)[:, None, None]).to(dtype)
    torch.cuda.synchronize()
    assert torch.equal(q.cpu().view(torch.int16), want.view(torch.int16))


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("nx", [64, 67])   # 16-byte rows (TMA staging) / not
@pytest.mark.parametrize("dtype", [F16, BF16])
def test_backproject_lp_is_storage_only(engine, restatement, layout, nx, dtype):
    R = restatement
    ny, nt, th = 40, 11, 18
    rng = np.random.default_rng(nx + layout)
    ang = np.sort(rng.uniform(-65, 65, nt)).astype(np.float32)
    c8 = R.coeffs(ang, 0.5, 2.0 if layout == 0 else 0.0, 0.0)
    c8[:, 0] += rng.normal(0, 1.0, nt)
    c8[:, 4] += rng.normal(0, 1.0, nt)
    proj = (rng.normal(size=(nt, ny, nx)) * (1 + np.arange(nt))[:, None, None]).astype(np.float32)
    org = T.default_origin(layout, nx, ny, th)
    engine.set_problem(nx, ny, nt, th, c8, layout, org)
    q, scale = engine.quantize(torch.from_numpy(proj).cuda(), dtype)
    deq = host(q) * host(scale)[:, None, None]
    vshape = (ny, th, nx) if layout == 0 else (th, ny, nx)
    vol = torch.zeros(vshape, device="cuda")
    engine.backproject_lp(q, scale, vol)
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    ref_deq = R.backproject(g, c8, deq, np.zeros(vshape), fp64=True)
    assert O.rel_l2(host(vol), ref_deq) < 1e-5
    ref = R.backproject(g, c8, proj, np.zeros(vshape), fp64=True)
    rel, _ = errors(host(vol), ref)
    assert rel < (1e-3 if dtype == F16 else 5e-3)


@pytest.fixture(scope="module", params=["poisson", "gaussian"])
def series(engine, restatement, request):
    """Series at a quarter of cfg1's lengths: 61 tilts, 256^2, Z layout
    volume 256^2 x 64, with Poisson counting noise at a mean of 20 e-/px
    (the mixed-precision configuration's noise model) or cfg1's Gaussian
    noise; and the FP64 oracle SIRT-10 (relaxation 0.5) of it."""
    cfg = synth.config("cfg1", 4)
    c8 = synth.coefficients(cfg)
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    org = T.default_origin(1, nx, ny, th)
    engine.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Z, org)
    proj = synth.project_series(engine, cfg, 1, request.param)
    p = host(proj)
    g = restatement.geom(nx, ny, nt, th, 1, 0, org)
    ref = restatement.sirt(g, c8, p, np.zeros((th, ny, nx)), 10, 0.5, fp64=True)
    return cfg, c8, org, proj, ref, request.param


@pytest.mark.parametrize("pdt,rdt,bar", [
    ("f32", "f32", 1e-5),
    ("f16", "f32", 1e-4),
    ("f16", "f16", 1e-4),
    ("f16", "bf16", 2e-4),
    ("bf16", "bf16", 2e-3),
])
def test_sirt_lp_vs_fp64(engine, series, pdt, rdt, bar, record_property):
    cfg, c8, org, proj, ref, noise = series
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    engine.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Z, org)
    vol = torch.zeros((th, ny, nx), device="cuda")
    if pdt == "f32":
        engine.sirt_lp(proj, None, vol, 10, 0.5, rdt)
    else:
        q, scale = engine.quantize(proj, F16 if pdt == "f16" else BF16)
        engine.sirt_lp(q, scale, vol, 10, 0.5, rdt)
    rel, mx = errors(host(vol), ref)
    record_property("rel_l2_vs_fp64", rel)
    record_property("max_abs_vs_fp64", mx)
    print(f"SIRT-10 proj {pdt} resid {rdt} ({noise} noise): rel-L2 {rel:.3e}, max-abs {mx:.3e} (vs FP64)")
    assert rel < bar


def test_sirt_lp_f32_equals_sirt(engine, series):
    """With FP32 storage tr_sirt_lp computes what tr_sirt computes.  The
    forward projection's global float atomics add tile partial sums in
    arrival order, so two runs agree to float rounding, not bit for bit."""
    cfg, c8, org, proj, _, _ = series
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    engine.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Z, org)
    a = torch.zeros((th, ny, nx), device="cuda")
    b = torch.zeros_like(a)
    engine.sirt(proj, a, 3, 0.5)
    engine.sirt_lp(proj, None, b, 3, 0.5, "f32")
    assert O.rel_l2(host(b), host(a)) < 1e-6


def test_sirt_lp_f16_residual_after_wbp(engine, series, restatement):
    """SIRT from a WBP start (cfg3's WBP-then-SIRT): the residual's range is
    then far from the stack's, and the FP16 residual must take its own
    per-tilt scales to stay finite and within the 1e-4 bar."""
    cfg, c8, org, proj, _, noise = series
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    engine.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Z, org)
    vol = torch.zeros((th, ny, nx), device="cuda")
    f = proj.clone()
    engine.wbp(f, vol)
    q, scale = engine.quantize(proj, F16)
    engine.sirt_lp(q, scale, vol, 3, 0.5, "f16")
    got = host(vol)
    assert np.isfinite(got).all()
    R = restatement
    g = R.geom(nx, ny, nt, th, 1, 0, org)
    p = host(proj)
    ref = R.backproject(g, c8, R.filter_rweight(p), np.zeros((th, ny, nx)), fp64=True)
    ref = R.sirt(g, c8, p, ref, 3, 0.5, fp64=True)
    rel, mx = errors(got, ref)
    print(f"WBP + SIRT-3 proj f16 resid f16 ({noise} noise): rel-L2 {rel:.3e}, max-abs {mx:.3e}")
    assert rel < 1e-4
