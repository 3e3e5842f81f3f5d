"""The oracle restatement pinned against the reference (CPU only).

The reference has no tests or golden vectors for TiltRec; the pins are the
reference's own CPU routines compiled from its sources (live, where
oracle/_ref is built) and the fixtures they generated (tests/golden)."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def _case(g, name):
    nx, ny, nt, th = (int(v) for v in g[f"{name}/dims"])
    return nx, ny, nt, th, tuple(float(v) for v in g[f"{name}/origin"])


def test_golden_manifest(golden):
    with open(os.path.join(HERE, "golden", "MANIFEST.json")) as f:
        man = json.load(f)
    assert set(man) == set(golden)
    for k, v in golden.items():
        assert hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest() == man[k], k


@pytest.mark.parametrize("name", ["ysep", "ygen"])
def test_restatement_matches_reference_y(golden, restatement, name):
    R = restatement
    nx, ny, nt, th, org = _case(golden, name)
    c8 = golden[f"{name}/coeff8"]
    proj, vol0 = golden[f"{name}/proj"], golden[f"{name}/vol0"]
    g = R.geom(nx, ny, nt, th, 0, 0, org)
    zero = np.zeros_like(vol0)
    # bit for bit: same float operations in the same order as the reference
    np.testing.assert_array_equal(R.backproject(g, c8, proj, zero), golden[f"{name}/bpt"])
    np.testing.assert_array_equal(R.sirt(g, c8, proj, vol0, 3, 0.5), golden[f"{name}/sirt3"])
    np.testing.assert_array_equal(R.sart(g, c8, proj, vol0, 1, 0.5), golden[f"{name}/sart1"])
    v, w = R.reproject(g, c8[nt // 2], vol0)
    np.testing.assert_array_equal(v, golden[f"{name}/fp_val"])
    np.testing.assert_array_equal(w, golden[f"{name}/fp_wt"])
    # the filter runs its transform in double here, in float in the reference
    f = R.filter_rweight(proj)
    assert O.rel_l2(f, golden[f"{name}/filtered"]) < 2e-7
    assert O.rel_l2(R.backproject(g, c8, f, zero), golden[f"{name}/wbp"]) < 2e-7


def test_restatement_matches_reference_z(golden, restatement):
    R = restatement
    nx, ny, nt, th, org = _case(golden, "zsep")
    c8, proj, vol0 = golden["zsep/coeff8"], golden["zsep/proj"], golden["zsep/vol0"]
    g = R.geom(nx, ny, nt, th, 1, 0, org)
    zero = np.zeros_like(vol0)
    np.testing.assert_array_equal(R.backproject(g, c8, proj, zero), golden["zsep/bpt"])
    np.testing.assert_array_equal(R.sirt(g, c8, proj, vol0, 2, 0.7), golden["zsep/sirt2"])
    wbp = R.backproject(g, c8, R.filter_rweight(proj), zero)
    assert O.rel_l2(wbp, golden["zsep/wbp"]) < 2e-7


def test_restatement_cfg0_scaled(golden, restatement):
    R = restatement
    nx, ny, nt, th, org = _case(golden, "cfg0s4")
    c8, proj = golden["cfg0s4/coeff8"], golden["cfg0s4/proj"]
    g = R.geom(nx, ny, nt, th, 0, 0, org)
    zero = np.zeros((ny, th, nx), np.float32)
    np.testing.assert_array_equal(R.sirt(g, c8, proj, zero, 5, 0.5), golden["cfg0s4/sirt5"])
    wbp = R.backproject(g, c8, R.filter_rweight(proj), zero)
    assert O.rel_l2(wbp, golden["cfg0s4/wbp"]) < 2e-7


def test_geometry_restatement_matches_reference(golden, restatement):
    ang = golden["geom/angles"]
    for par, c20 in zip(golden["geom/params"], golden["geom/coeff20"]):
        c8 = restatement.coeffs(ang, *par)
        np.testing.assert_array_equal(c8, c20[:, [0, 1, 2, 3, 10, 11, 12, 13]])
        assert not np.any(c20[:, 4:10]) and not np.any(c20[:, 14:20])


def test_fp64_oracle_agrees_with_fp32(golden, restatement):
    R = restatement
    nx, ny, nt, th, org = _case(golden, "cfg0s4")
    c8, proj = golden["cfg0s4/coeff8"], golden["cfg0s4/proj"]
    g = R.geom(nx, ny, nt, th, 0, 0, org)
    zero = np.zeros((ny, th, nx), np.float32)
    a = R.sirt(g, c8, proj, zero, 3, 0.5)
    b = R.sirt(g, c8, proj.astype(np.float64), zero.astype(np.float64), 3, 0.5, fp64=True)
    assert O.rel_l2(a, b) < 1e-5


def _filter_numpy(rows):
    """Independent float64 restatement of filter_Rweighting_1D_many
    (filter/filter_prj.cpp:674-736) with numpy's FFT."""
    nx = rows.shape[-1]
    N = nx + nx // 10
    nxp = N - nx + 1
    r = int(np.floor(np.float32(N) * np.float32(0.05)))
    sg = np.float32(N) * np.float32(0.5)
    x = rows.reshape(-1, nx).astype(np.float64)
    j = np.arange(nx, N)
    wa = (j - nx + 1).astype(np.float32) / np.float32(nxp)
    wb = (N - j).astype(np.float32) / np.float32(nxp)
    pad = np.concatenate([x, wa * x[:, :1] + wb * x[:, -1:]], axis=1)
    X = np.fft.rfft(pad, axis=1)
    k = np.arange(X.shape[1])
    W = np.where(k <= r, k, r * np.exp(-((k - r) ** 2).astype(np.float32) / (sg * sg)))
    W = W.astype(np.float64)
    W[0] = 0.2
    y = np.fft.irfft(X * W, n=N, axis=1) * N / nx
    return y[:, :nx].reshape(rows.shape)


@pytest.mark.parametrize("nx", [37, 64, 256, 333])
def test_filter_restatement_vs_numpy(restatement, nx):
    rng = np.random.default_rng(nx)
    rows = rng.normal(size=(5, 7, nx)).astype(np.float32)
    a = restatement.filter_rweight(rows)
    b = _filter_numpy(rows)
    assert O.rel_l2(a, b) < 1e-6


def test_reference_live_random_case(reference, restatement):
    """Fresh seeded inputs through both (where oracle/_ref is built)."""
    rng = np.random.default_rng(99)
    nx, ny, nt, th = 29, 17, 6, 9
    ang = rng.uniform(-80, 80, nt).astype(np.float32)
    c8 = restatement.coeffs(ang, -1.5, 7.0, 2.0)
    c8[:, 0] += rng.normal(0, 3, nt)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    vol = rng.normal(size=(ny, th, nx)).astype(np.float32)
    org = (nx * 0.5, th * 0.5, th * 0.5)
    g = restatement.geom(nx, ny, nt, th, 0, 0, org)
    np.testing.assert_array_equal(
        restatement.backproject(g, c8, proj, vol),
        reference.y_backproject(nx, ny, nt, th, O.coeff20(c8), org, proj, vol))
    np.testing.assert_array_equal(
        restatement.sirt(g, c8, proj, vol, 2, 0.3),
        reference.y_sirt(nx, ny, nt, th, O.coeff20(c8), org, proj, vol, 2, 0.3))


def _fbp_by_dft(row, taps):
    """The reference's FBP row filter step by step with numpy's FFT
    (FileterProjectionSymmetrize, filter_prj.cpp:265-446): edge-padded row,
    mirrored extension to the optimal DFT length, spectrum product with the
    251-tap kernel, scaled inverse, samples [126, 126 + nx)."""
    nx = row.size
    n = nx + 2
    length = len(taps)
    big = n + length - 1
    L = big
    while True:
        r = L
        for q in (2, 3, 5):
            while r % q == 0:
                r //= q
        if r == 1:
            break
        L += 1
    x = np.zeros(L)
    x[1:nx + 1] = row
    x[0], x[n - 1] = row[0], row[-1]
    end = L if n >= L - n else 2 * n
    for i in range(n, end):
        x[i] = x[2 * n - 1 - i]
    f = np.zeros(L)
    f[:length] = taps
    y = np.fft.ifft(np.fft.fft(x) * np.fft.fft(f)).real
    return y[length // 2 + 1: length // 2 + 1 + nx], L


def _taps(mode):
    n = np.arange(-125, 126)
    if mode == 1:
        t = np.where(n == 0, np.pi / 4, np.where(np.abs(n) % 2 == 1, -1.0 / (np.pi * n * n + (n == 0)), 0.0))
        return t.astype(np.float32).astype(np.float64)
    return (-2.0 / (np.pi * (4.0 * n.astype(np.float32).astype(np.float64) ** 2 - 1.0))
            ).astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("nx", [64, 300, 1024])
def test_fbp_filter_restatement_matches_dft_steps(restatement, mode, nx):
    """The restatement's direct sum equals the reference's DFT steps (numpy
    FFT in double) on the same row, for both branches of the mirrored
    extension (short rows mirror only up to twice their length)."""
    rng = np.random.default_rng(nx + mode)
    rows = rng.normal(size=(3, nx)).astype(np.float32)
    got = restatement.filter_fbp(rows, mode)
    for r in range(3):
        want, L = _fbp_by_dft(rows[r].astype(np.float64), _taps(mode))
        assert L == restatement.optimal_dft_size(nx + 2 + 250)
        assert np.abs(got[r] - want).max() <= 1e-5 * np.abs(want).max()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("shape", [(2, 40, 64), (2, 7, 256), (1, 5, 300)])
def test_fbp_filter_restatement_matches_reference(reference, restatement, mode, shape):
    """The restatement's FBP filter equals the unmodified reference's
    (ApplyFilterInplace modes 0/1, FileterProjectionSymmetrize) run in the
    oracle with the OpenCV C-API shim: its image padding, 2-D symmetrisation,
    mirrored extension (both branches: 256- and 300-wide rows take the long
    one), DFT-domain product and crop."""
    rng = np.random.default_rng(sum(shape) + mode)
    proj = rng.normal(size=shape).astype(np.float32)
    want = reference.filter_fbp(proj, mode)
    got = restatement.filter_fbp(proj, mode)
    assert O.rel_l2(got, want) < 1e-6
    assert np.abs(got - want).max() <= 1e-6 * max(1.0, np.abs(want).max())


def test_resample_bin_restatement(restatement):
    """Area binning: a block mean when the factor divides the size; with a
    remainder the cells still tile the image, so the means agree."""
    rng = np.random.default_rng(4)
    a = rng.normal(size=(2, 12, 18)).astype(np.float32)
    got = restatement.resample_bin(a, 3)
    want = a.reshape(2, 4, 3, 6, 3).astype(np.float64).mean(axis=(2, 4))
    assert np.abs(got - want).max() < 1e-6
    b = rng.normal(size=(1, 13, 17)).astype(np.float32)
    for f in (2, 3, 5):
        g = restatement.resample_bin(b, f)
        assert g.shape == (1, 13 // f, 17 // f)
        assert abs(g.mean() - b.astype(np.float64).mean()) < 1e-6


@pytest.mark.parametrize("shape,factor", [((2, 36, 48), 3), ((3, 37, 50), 3), ((1, 64, 40), 4)])
@pytest.mark.parametrize("mode", [2, 1, 0])
def test_resample_restatement_vs_reference_tool(restatement, tmp_path, shape, factor, mode):
    """The reference's own resample tool (its unmodified sources with the
    test-only OpenCV subset, oracle/_ref/resample) against the restatement:
    sections read as float (bytes unsigned / 255, shorts as values), area
    binning, a float output whose header is the input's with the new sizes
    and mode 2 (the tool's closing statistics rewrite never reaches the file,
    so amin / amax / amean stay the input's)."""
    import subprocess
    import sys
    sys.path.insert(0, HERE)
    from mrc_util import read_mrc, write_mrc
    exe = O.reference_resample_executable()
    if exe is None:
        pytest.skip("oracle/_ref/resample is not built here")
    rng = np.random.default_rng(sum(shape) + mode)
    if mode == 2:
        data = rng.normal(size=shape).astype(np.float32)
    elif mode == 1:
        data = np.round(rng.normal(size=shape) * 300).astype(np.float32)
    else:
        data = rng.integers(0, 256, size=shape).astype(np.float32)
    src, out = tmp_path / "in.mrc", tmp_path / "out.mrc"
    write_mrc(src, data.astype(np.uint8).view(np.int8) if mode == 0 else data, mode=mode,
              next_bytes=32 if mode == 1 else 0)
    with open(src, "r+b") as f:
        f.seek(76)
        f.write(np.array([-1.5, 2.5, 0.25], "<f4").tobytes())
    r = subprocess.run([exe, "-i", str(src), "-o", str(out), "-b", str(factor)],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    hi, _, _ = read_mrc(src)
    ho, _, got = read_mrc(out)
    want = restatement.resample_bin(data / 255.0 if mode == 0 else data, factor)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-6 * max(1.0, np.abs(want).max())
    assert int(ho["mode"]) == 2
    assert [int(v) for v in ho["m"]] == [want.shape[2], want.shape[1], want.shape[0]]
    for f in ("amin", "amax", "amean", "next"):
        assert np.array_equal(ho[f], hi[f]), f
