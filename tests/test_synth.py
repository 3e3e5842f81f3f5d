"""The seeded synthetic workloads (autom2_b200/synth.py) on the CPU.

The benchmark and the full-size tests stand in for the reference's missing
sample data with generated tilt series.  These checks pin the generated
workloads to their definitions: the sizes and algorithmic work of cfg0-cfg2
(41 x 256^2 WBP into 256^2 x 64: 1.72e8 voxel-tilt updates; 61 x 1024^2
SIRT-30 into 1024^2 x 256: 9.8e11; 61 x 4096^2 SIRT-20 into 4096^2 x 512:
2.10e13), the batched series' and the request stream's distributions, the
geometry perturbations, and that everything is a pure function of its seed.
"""
import numpy as np
import pytest

import oracle as O
from autom2_b200 import synth


def work(cfg):
    """Voxel-tilt updates of one reconstruction: one pass for WBP, two per
    SIRT iteration."""
    passes = 1 if cfg.method == "WBP" else 2 * cfg.iters
    return passes * cfg.ntilt * cfg.nx * cfg.ny * cfg.thickness


@pytest.mark.parametrize("name,shape,ntilt,span,method,iters,vpu", [
    ("cfg0", (256, 256, 64), 41, (-60, 60), "WBP", 0, 1.72e8),
    ("cfg1", (1024, 1024, 256), 61, (-60, 60), "SIRT", 30, 9.8e11),
    ("cfg2", (4096, 4096, 512), 61, (-60, 60), "SIRT", 20, 2.10e13),
])
def test_configurations(name, shape, ntilt, span, method, iters, vpu):
    c = synth.config(name)
    assert (c.nx, c.ny, c.thickness) == shape
    assert c.ntilt == ntilt and (c.angles[0], c.angles[-1]) == span
    assert c.method == method and c.iters == iters
    assert work(c) == pytest.approx(vpu, rel=5e-3)


def test_cfg1_geometry_perturbations():
    """cfg1 adds per-tilt in-plane rotations to the reference geometry (XTILT
    0.3 deg): each tilt's (a, b) rows turn by one angle, so the column norms
    sqrt(a_i^2 + b_i^2) stay those of the reference's coefficients."""
    R = O.Restatement()
    c = synth.config("cfg1")
    base = np.asarray(R.coeffs(c.angles, 0.0, c.xtilt, 0.0), np.float64).reshape(-1, 8)
    got = synth.coefficients(c, base=R.coeffs)
    assert got.shape == (61, 8)
    np.testing.assert_allclose(np.hypot(got[:, 1:4], got[:, 5:8]),
                               np.hypot(base[:, 1:4], base[:, 5:8]), rtol=1e-12, atol=1e-15)
    # the rotation angle of each tilt, from the x column: N(0, 0.5 deg)
    psi = np.degrees(np.arctan2(got[:, 5], got[:, 1]) - np.arctan2(base[:, 5], base[:, 1]))
    assert np.abs(psi).max() < 2.5 and 0.2 < psi.std() < 0.9
    np.testing.assert_array_equal(got, synth.coefficients(c, base=R.coeffs))  # seeded


def test_cfg0_offsets():
    R = O.Restatement()
    c = synth.config("cfg0")
    base = np.asarray(R.coeffs(c.angles, 0.0, 0.0, 0.0), np.float64).reshape(-1, 8)
    got = synth.coefficients(c, base=R.coeffs)
    shift = np.concatenate([got[:, 0] - base[:, 0], got[:, 4] - base[:, 4]])
    assert 0.6 < shift.std() < 1.4  # N(0, 1 px) in x and y
    np.testing.assert_array_equal(got[:, [1, 2, 3, 5, 6, 7]], base[:, [1, 2, 3, 5, 6, 7]])


def test_phantom_is_seeded_and_nonnegative():
    c = synth.config("cfg0", 4)
    a = synth.phantom(c).numpy()
    b = synth.phantom(c).numpy()
    assert a.shape == (c.ny, c.thickness, c.nx)
    np.testing.assert_array_equal(a, b)
    assert a.min() >= 0 and a.max() > 0
    z = synth.phantom(c, layout=1).numpy()  # Z layout is the same volume, sections first
    np.testing.assert_array_equal(z, a.transpose(1, 0, 2))


def test_batch_series_distribution():
    s = synth.batch_series()
    assert len(s) == 64
    assert {c.nx for c in s} <= {512, 1024, 2048} and all(c.nx == c.ny for c in s)
    assert {c.ntilt for c in s} <= {41, 61, 81}
    assert all(64 <= c.thickness < 384 for c in s)
    assert all(60 <= c.angles[-1] <= 70 and c.angles[0] == -c.angles[-1] for c in s)
    assert all(c.iters == 10 and c.gamma == 0.5 for c in s)
    assert [c.nx for c in s] == [c.nx for c in synth.batch_series()]  # seeded


def test_serve_stream_distribution():
    classes, reqs = synth.serve_stream(2000)
    assert len(reqs) == 2000
    t = np.array([r["t"] for r in reqs])
    assert np.all(np.diff(t) > 0)
    assert 3.6 < 1.0 / np.diff(t).mean() < 4.4  # Poisson arrivals at 4 per second
    assert set(classes) <= {(s, n) for s in (512, 1024, 2048) for n in (41, 61, 81)}
    methods = [r["method"] for r in reqs]
    for m in ("WBP", "SIRT-10", "SIRT-30"):
        assert 0.28 < methods.count(m) / len(methods) < 0.39
    assert all(64 <= r["thickness"] < 384 for r in reqs)
    assert reqs == synth.serve_stream(2000)[1]  # seeded
