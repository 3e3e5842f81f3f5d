"""Test helpers for the multi-rank driver (autom2_b200.shard): the per-rank
operator restated on the CPU by the oracle, and the worker that runs one rank
of a torch.distributed group (gloo) over a list of cases.

The oracle operator is test infrastructure: it lets the N-rank host logic
(partitioning, per-rank origins, the all-reduce between the passes, the
gather) run without a GPU against the oracle's whole-volume reconstruction."""
from __future__ import annotations

import os

import numpy as np
import torch


class OracleOps:
    """The Engine's per-rank methods, computed by the oracle restatement on
    float32 CPU tensors."""

    def __init__(self):
        import oracle
        self.R = oracle.Restatement()

    def set_problem(self, nx, ny, nt, th, coeff8, layout, origin):
        self.g = self.R.geom(nx, ny, nt, th, layout, 0, origin)
        self.c8 = np.asarray(coeff8, np.float64).reshape(nt, 8)

    def backproject(self, proj, vol):
        vol.copy_(torch.from_numpy(self.R.backproject(self.g, self.c8, proj.numpy(), vol.numpy())))

    def filter_rweight(self, proj):
        proj.copy_(torch.from_numpy(self.R.filter_rweight(proj.numpy())))

    def sirt(self, proj, vol, iters, gamma):
        vol.copy_(torch.from_numpy(self.R.sirt(self.g, self.c8, proj.numpy(), vol.numpy(),
                                               iters, gamma)))

    def sart(self, proj, vol, iters, gamma):
        vol.copy_(torch.from_numpy(self.R.sart(self.g, self.c8, proj.numpy(), vol.numpy(),
                                               iters, gamma)))

    def forward_project_tilts(self, vol, t0, n, val, wt=None):
        for i in range(n):
            v, w = self.R.reproject(self.g, self.c8[t0 + i], vol.numpy())
            val[i] += torch.from_numpy(v)
            if wt is not None:
                wt[i] += torch.from_numpy(w)

    def residual(self, proj, val, wt):
        v, w, p = val.numpy(), wt.numpy(), proj.numpy()
        q = np.where(w != 0, v / np.where(w != 0, w, 1), v).astype(np.float32)
        val.copy_(torch.from_numpy(p - q))

    def sirt_update(self, resid, vol, gamma):
        vv = np.zeros(vol.shape, np.float32)
        wv = np.zeros(vol.shape, np.float32)
        for t in range(self.c8.shape[0]):
            vv, wv = self.R.update_weights(self.g, self.c8[t], resid[t].numpy(), vv, wv)
        upd = np.where(wv != 0, vv / np.where(wv != 0, wv, 1) * np.float32(gamma), 0)
        vol += torch.from_numpy(upd.astype(np.float32))

    def sart_update(self, resid_plane, t, vol, gamma):
        r = resid_plane.reshape(resid_plane.shape[-2:]).numpy()
        vol.copy_(torch.from_numpy(self.R.update_by_projdiff(self.g, self.c8[t], r,
                                                             vol.numpy(), gamma)))


def run_rank(rank, world, port, cases, out_dir, use_gpu=False, backend="gloo"):
    """One rank: runs every case through autom2_b200.shard and writes the
    gathered volume of each to out_dir/<case>_<rank>.npy.  backend "nccl"
    (one rank per GPU): the collectives run over NCCL on the CUDA tensors
    themselves (shard.TorchComm); with gloo on a GPU they are staged through
    host memory (HostStagedComm), so ranks can share one GPU."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import torch.distributed as dist

    from autom2_b200 import shard

    if backend == "nccl":
        torch.cuda.set_device(rank)
    dist.init_process_group(backend, init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=120))
    try:
        if use_gpu:
            from autom2_b200.tiltrec import Engine
            ops = Engine(rank if backend == "nccl" else 0)
            comm = shard.TorchComm() if backend == "nccl" else HostStagedComm()
            dev = "cuda"
        else:
            ops = OracleOps()
            comm = shard.TorchComm()
            dev = "cpu"
        for name, c in cases.items():
            proj = torch.from_numpy(c["proj"]).to(dev)
            p = shard.plan(c["nx"], c["ny"], c["nt"], c["th"], c["coeff8"], c["layout"],
                           world, rank, mode=c.get("mode"))
            part = shard.reconstruct(ops, comm, p, proj, c["coeff8"], c["method"],
                                     c.get("iters", 0), c.get("gamma", 0.0))
            full = shard.gather(comm, p, part)
            np.save(os.path.join(out_dir, f"{name}_{rank}.npy"), full.cpu().numpy())
            with open(os.path.join(out_dir, f"{name}_{rank}.mode"), "w") as f:
                f.write(p.mode)
        if use_gpu:
            ops.close()
    finally:
        dist.destroy_process_group()


class HostStagedComm:
    """TorchComm for CUDA tensors over a gloo group: each collective goes
    through host memory (two ranks sharing one GPU in a test)."""

    def __init__(self):
        from autom2_b200 import shard
        self.inner = shard.TorchComm()
        self.rank, self.size = self.inner.rank, self.inner.size

    def all_reduce(self, t):
        torch.cuda.synchronize()
        h = t.cpu()
        self.inner.all_reduce(h)
        t.copy_(h)
        return t

    def all_gather(self, t):
        torch.cuda.synchronize()
        return [x.to(t.device) for x in self.inner.all_gather(t.cpu())]
