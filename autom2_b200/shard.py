"""One reconstruction over several GPUs: one process per GPU, torch.distributed
for the plumbing.

The reference splits a reconstruction across MPI ranks in two ways:

* TiltRec-mpi gives each rank a band of volume rows (Y) plus
  ceil(|tan(pitch)| * thickness) halo rows on each side and reconstructs it
  independently (main/main-mpi.cpp:710-740).  The halo is an approximation
  whenever the geometry couples rows (XTILT, in-plane rotation).
* TiltRecZ-mpi gives each rank a slab of sections (Z) and, in SIRT and SART,
  sums the slabs' forward projections with MPI_Allreduce before the residual
  (main/main-mpiz.cpp:502-601, 1054-1068), which is exact.

Here the plan follows the geometry:

``rows``
    When every tilt maps voxel row Y exactly onto detector row Y (b0 = b1 =
    b3 = 0, b2 = 1: no XTILT, no in-plane rotation, no vertical shift) the
    rows are independent.  Each rank reconstructs its band of rows as a
    problem of its own -- the stack's rows [y0, y1) with the origin's y moved
    by -y0 -- with no halo and no collective.  (A fractional vertical shift
    makes every voxel row splat onto two detector rows, which couples
    neighbouring rows through the SIRT/SART residual.)
``zslabs``
    Otherwise each rank owns sections [z0, z1) of the volume as a problem of
    its own (origin's z moved by -z0).  BPT and WBP need no exchange; SIRT and
    SART all-reduce the forward projections (and, once, the projection
    weights) between the forward and the backward pass, as TiltRecZ-mpi does.

Ranks split rows or sections as the reference does: the first n % procs
ranks take one more (``partition``).

``ops`` is the per-rank reconstruction operator: a
:class:`autom2_b200.tiltrec.Engine` on the rank's GPU (any object with the
same methods works).  ``comm`` sums and gathers tensors across the ranks:
:class:`TorchComm` over a torch.distributed process group (NCCL between
GPUs), or :class:`LocalComm` for one process.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

LAYOUT_Y, LAYOUT_Z = 0, 1


def partition(n: int, procs: int, rank: int) -> tuple[int, int]:
    """(start, length) of rank's share of n rows or sections: the first
    n % procs ranks take n // procs + 1 (main-mpi.cpp:711-725,
    main-mpiz.cpp:1056-1068)."""
    rem = n % procs
    if rank < rem:
        length = n // procs + 1
        return length * rank, length
    length = n // procs
    return length * rank + rem, length


def rows_independent(coeff8) -> bool:
    """True when every tilt maps voxel row Y exactly onto detector row Y."""
    c = np.asarray(coeff8, np.float64).reshape(-1, 8)
    return bool(np.all(c[:, 4] == 0.0) and np.all(c[:, 5] == 0.0) and
                np.all(c[:, 7] == 0.0) and np.all(c[:, 6] == 1.0))


@dataclass
class ShardPlan:
    mode: str                 # "rows" or "zslabs"
    procs: int
    rank: int
    start: int                # first row (rows) or section (zslabs) of this rank
    length: int               # rows or sections of this rank (may be 0)
    nx: int
    ny: int
    nt: int
    th: int
    layout: int
    origin: tuple             # the whole volume's origin

    def local_dims(self):
        """(ny, th) of this rank's problem."""
        if self.mode == "rows":
            return self.length, self.th
        return self.ny, self.length

    def local_origin(self):
        ox, oy, oz = self.origin
        if self.mode == "rows":
            return (ox, oy - self.start, oz)
        return (ox, oy, oz - self.start)

    def local_shape(self):
        ny, th = self.local_dims()
        return (ny, th, self.nx) if self.layout == LAYOUT_Y else (th, ny, self.nx)

    def shard_axis(self) -> int:
        """Axis of the volume array along which the ranks' parts stack."""
        if self.mode == "rows":
            return 0 if self.layout == LAYOUT_Y else 1
        return 1 if self.layout == LAYOUT_Y else 0


def plan(nx, ny, nt, th, coeff8, layout, procs, rank, origin=None, mode=None) -> ShardPlan:
    """The shard plan of one rank (see the module docstring).  mode forces
    "rows" (only valid when the rows are independent) or "zslabs"."""
    if origin is None:
        origin = (nx * 0.5, th * 0.5, th * 0.5) if layout == LAYOUT_Y else \
                 (nx * 0.5, ny * 0.5, th * 0.5)
    indep = rows_independent(coeff8)
    if mode is None:
        mode = "rows" if indep else "zslabs"
    if mode == "rows" and not indep:
        raise ValueError("row sharding needs independent rows (b0 = b1 = b3 = 0, b2 = 1)")
    if mode not in ("rows", "zslabs"):
        raise ValueError(mode)
    start, length = partition(ny if mode == "rows" else th, procs, rank)
    return ShardPlan(mode, procs, rank, start, length, nx, ny, nt, th, layout,
                     tuple(float(v) for v in origin))


class LocalComm:
    """One process: sums and gathers are identities."""
    rank, size = 0, 1

    def all_reduce(self, t):
        return t

    def all_gather(self, t):
        return [t]


class TorchComm:
    """Sums and gathers over a torch.distributed process group (NCCL for CUDA
    tensors across GPUs, gloo for CPU tensors)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def all_reduce(self, t):
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t

    def all_gather(self, t):
        out = [t.new_empty(t.shape) for _ in range(self.size)]
        self.dist.all_gather(out, t.contiguous(), group=self.group)
        return out


def local_stack(p: ShardPlan, proj):
    """This rank's projections: rows [start, start+length) in rows mode, the
    whole stack otherwise."""
    if p.mode == "rows":
        return proj[:, p.start:p.start + p.length].contiguous()
    return proj


def local_initial(p: ShardPlan, vol):
    """This rank's part of a whole starting volume (--initial)."""
    idx = [slice(None)] * 3
    idx[p.shard_axis()] = slice(p.start, p.start + p.length)
    return vol[tuple(idx)].contiguous()


def reconstruct(ops, comm, p: ShardPlan, proj, coeff8, method: str, iters=0, gamma=0.0,
                vol=None):
    """Reconstructs this rank's part; returns it (shape p.local_shape()).

    proj: the whole stack (float32 tensor on the rank's device; WBP filters a
    private copy).  vol: this rank's starting part (zeros if None).  Every
    rank must call this with the same method and sizes: the collectives of
    SIRT and SART run on all ranks, including ranks without sections."""
    import torch
    method = method.upper()
    coeff8 = np.ascontiguousarray(coeff8, np.float64).reshape(p.nt, 8)
    ny_l, th_l = p.local_dims()
    have = p.length > 0
    if vol is None:
        vol = torch.zeros(p.local_shape(), dtype=torch.float32, device=proj.device)
    if have:
        ops.set_problem(p.nx, ny_l, p.nt, th_l, coeff8, p.layout, p.local_origin())
    stack = local_stack(p, proj)

    if p.mode == "rows" or method in ("BPT", "WBP"):
        # No exchange: the rank's part is a complete problem.
        if not have:
            return vol
        if method == "BPT":
            ops.backproject(stack, vol)
        elif method == "WBP":
            f = stack.clone()
            ops.filter_rweight(f)
            ops.backproject(f, vol)
        elif method == "SIRT":
            ops.sirt(stack, vol, iters, gamma)
        elif method == "SART":
            ops.sart(stack, vol, iters, gamma)
        else:
            raise ValueError(method)
        return vol

    # zslabs: sum the slabs' forward projections before each residual.
    nt = p.nt
    val = torch.zeros_like(proj)
    wt = torch.zeros_like(proj)
    if have:
        ops.forward_project_tilts(vol, 0, nt, val, wt)
    comm.all_reduce(wt)
    if method == "SIRT":
        for _ in range(iters):
            val.zero_()
            if have:
                ops.forward_project_tilts(vol, 0, nt, val)
            comm.all_reduce(val)
            if have:
                ops.residual(proj, val, wt)
                ops.sirt_update(val, vol, gamma)
    elif method == "SART":
        for _ in range(iters):
            for t in range(nt):
                v = val[t:t + 1]
                v.zero_()
                if have:
                    ops.forward_project_tilts(vol, t, 1, v)
                comm.all_reduce(v)
                if have:
                    ops.residual(proj[t:t + 1], v, wt[t:t + 1])
                    ops.sart_update(v, t, vol, gamma)
    else:
        raise ValueError(method)
    return vol


def gather(comm, p: ShardPlan, part):
    """The whole volume from every rank's part (on every rank)."""
    import torch
    axis = p.shard_axis()
    full_n = p.ny if p.mode == "rows" else p.th
    most = partition(full_n, p.procs, 0)[1]
    shape = list(part.shape)
    shape[axis] = most
    buf = part.new_zeros(shape)
    idx = [slice(None)] * 3
    idx[axis] = slice(0, part.shape[axis])
    buf[tuple(idx)] = part
    pieces = comm.all_gather(buf)
    out = []
    for r, piece in enumerate(pieces):
        _, length = partition(full_n, p.procs, r)
        idx[axis] = slice(0, length)
        out.append(piece[tuple(idx)])
    return torch.cat(out, dim=axis)
