"""Multi-rank reconstruction (autom2_b200.shard) on the CPU: two gloo ranks,
each running the oracle operator on its share, against the oracle's
whole-volume reconstruction.

rows mode (independent rows) has no collective: every rank's band is a
complete problem, so the gathered volume equals the whole one up to the
floating-point rounding of the shifted origin.  zslabs mode sums the slabs'
forward projections in float32 across ranks (a different summation order
than the whole-volume splat), so it matches to float rounding too; the bar
for both is relative L2 1e-6."""
import socket
import zlib

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
from autom2_b200 import shard
from autom2_b200 import tiltrec as T


def test_partition_matches_reference_split():
    # main-mpi.cpp:711-725: the first n % procs ranks take one more row.
    assert [shard.partition(10, 3, r) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    assert [shard.partition(2, 4, r) for r in range(4)] == [(0, 1), (1, 1), (2, 0), (2, 0)]
    for n in (1, 7, 64):
        for procs in (1, 2, 3, 8):
            parts = [shard.partition(n, procs, r) for r in range(procs)]
            assert sum(ln for _, ln in parts) == n
            assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(procs - 1))


def test_plan_follows_geometry(restatement):
    ang = np.linspace(-60, 60, 5).astype(np.float32)
    flat = restatement.coeffs(ang)
    flat[:, 0] += 0.7      # horizontal shifts keep rows independent
    assert shard.rows_independent(flat)
    shifted = flat.copy()
    shifted[:, 4] -= 1.3   # a vertical shift couples neighbouring rows
    assert not shard.rows_independent(shifted)
    assert shard.plan(32, 20, 5, 8, flat, 0, 2, 1).mode == "rows"
    tilted = restatement.coeffs(ang, 0.0, 3.0, 0.0)
    assert not shard.rows_independent(tilted)
    p = shard.plan(32, 20, 5, 8, tilted, 1, 2, 1)
    assert p.mode == "zslabs" and (p.start, p.length) == (4, 4)
    assert p.local_origin() == (16.0, 10.0, 0.0)
    with pytest.raises(ValueError):
        shard.plan(32, 20, 5, 8, tilted, 0, 2, 0, mode="rows")
    q = shard.plan(32, 21, 5, 8, flat, 0, 2, 1)
    assert (q.start, q.length, q.local_origin()) == (11, 10, (16.0, 4.0 - 11, 4.0))
    assert q.local_shape() == (10, 8, 32)


def _cases(R):
    rng = np.random.default_rng(11)
    nx, ny, nt = 24, 15, 7
    ang = np.sort(rng.uniform(-60, 60, nt)).astype(np.float32)
    proj = rng.normal(size=(nt, ny, nx)).astype(np.float32)
    flat = R.coeffs(ang)
    flat[:, 0] += rng.normal(0, 1, nt)
    shifted = flat.copy()
    shifted[:, 4] += rng.normal(0, 1, nt)
    tilted = R.coeffs(ang, 1.0, 4.0, 0.5)
    cases = {}
    for layout in (0, 1):
        for geo, c8 in (("flat", flat), ("shifted", shifted), ("tilted", tilted)):
            for method, it, gm in (("BPT", 0, 0.0), ("WBP", 0, 0.0), ("SIRT", 2, 0.5),
                                   ("SART", 1, 0.4)):
                cases[f"{geo}_{method}_{layout}"] = dict(
                    nx=nx, ny=ny, nt=nt, th=9, coeff8=c8, layout=layout, proj=proj,
                    method=method, iters=it, gamma=gm)
    # More ranks than sections: rank 1 owns none and still joins the sums.
    cases["thin_SIRT_1"] = dict(nx=nx, ny=ny, nt=nt, th=1, coeff8=tilted, layout=1,
                                proj=proj, method="SIRT", iters=2, gamma=0.5)
    cases["forced_zslabs_SIRT_0"] = dict(nx=nx, ny=ny, nt=nt, th=9, coeff8=flat, layout=0,
                                         proj=proj, method="SIRT", iters=2, gamma=0.5,
                                         mode="zslabs")
    return cases


def _whole(R, c):
    nx, ny, nt, th, layout = c["nx"], c["ny"], c["nt"], c["th"], c["layout"]
    org = T.default_origin(layout, nx, ny, th)
    g = R.geom(nx, ny, nt, th, layout, 0, org)
    zero = np.zeros((ny, th, nx) if layout == 0 else (th, ny, nx), np.float32)
    p = c["proj"]
    if c["method"] == "BPT":
        return R.backproject(g, c["coeff8"], p, zero)
    if c["method"] == "WBP":
        return R.backproject(g, c["coeff8"], R.filter_rweight(p), zero)
    f = R.sirt if c["method"] == "SIRT" else R.sart
    return f(g, c["coeff8"], p, zero, c["iters"], c["gamma"])


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(cases, tmp_path, world=2, use_gpu=False, backend="gloo"):
    from shard_ops import run_rank
    mp.start_processes(run_rank,
                       args=(world, free_port(), cases, str(tmp_path), use_gpu, backend),
                       nprocs=world, start_method="spawn", join=True)


def test_two_ranks_match_whole_volume(restatement, tmp_path):
    R = restatement
    cases = _cases(R)
    run_ranks(cases, tmp_path)
    for name, c in cases.items():
        want = _whole(R, c)
        mode = (tmp_path / f"{name}_0.mode").read_text()
        assert mode == c.get("mode", "rows" if name.startswith("flat") else "zslabs"), name
        for rank in range(2):
            got = np.load(tmp_path / f"{name}_{rank}.npy")
            assert got.shape == want.shape, name
            err = O.rel_l2(got, want)
            assert err < 1e-6, (name, rank, err)
    # the seeded cases differ (crc guards against a silently empty dict)
    assert zlib.crc32(",".join(sorted(cases)).encode()) and len(cases) == 26
