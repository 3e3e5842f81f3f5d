"""Seeded synthetic tilt series for tests and the benchmark.

The reference's sample data (a GitHub release) is not available, so inputs
are generated: an additive phantom of random ellipsoids plus gold-bead
spheres, voxelised with 2x supersampling, projected with the reference's
forward model (normalised bilinear voxel splat, Reproject val/wt) under each
configuration's geometry, then noised.

Configurations (sizes are nx, ny, tilts, thickness):

* ``cfg0`` -- WBP: 41 tilts -60..60 step 3, 256x256, volume 256x256x64,
  50 ellipsoids + 20 beads, per-tilt x/y offsets N(0, 1 px), XTILT 0,
  Gaussian noise sigma = 0.1 std(projections), seed 0.
* ``cfg1`` -- SIRT-30, gamma 0.5: 61 tilts step 2, 1024x1024, volume
  1024x1024x256, 400 ellipsoids + 80 beads, per-tilt in-plane rotation
  N(0, 0.5 deg), XTILT 0.3 deg, noise 0.3 std, seed 1.
* ``cfg2`` -- SIRT-20 in the Z layout with 16-bit storage: 61 tilts step 2,
  4096x4096, volume 4096x4096x512, 3000 ellipsoids + 300 beads, ideal
  single-axis geometry, Poisson counting noise at a mean of 20 e-/px, seed 2.

Functions take ``scale`` to shrink a configuration (all lengths divided) for
quick tests.  The phantom is built with torch on any device; projecting is
left to the caller (the oracle for fixtures, the engine for full sizes).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Config:
    name: str
    nx: int
    ny: int
    thickness: int
    angles: np.ndarray
    n_ellipsoids: int
    n_beads: int
    seed: int
    xtilt: float = 0.0
    offset_sigma: float = 0.0      # per-tilt x/y shift, pixels
    rotation_sigma: float = 0.0    # per-tilt in-plane rotation, degrees
    noise: float = 0.0             # Gaussian sigma as a fraction of std(proj)
    method: str = "WBP"
    iters: int = 0
    gamma: float = 0.0
    extra: dict = field(default_factory=dict)

    @property
    def ntilt(self) -> int:
        return len(self.angles)


def config(name: str, scale: int = 1) -> Config:
    """The named configuration, optionally with every length divided by
    ``scale`` (object counts scale with the volume)."""
    if name == "cfg0":
        c = Config("cfg0", 256, 256, 64, np.arange(-60, 61, 3, dtype=np.float32),
                   50, 20, 0, offset_sigma=1.0, noise=0.1, method="WBP")
    elif name == "cfg1":
        c = Config("cfg1", 1024, 1024, 256, np.arange(-60, 61, 2, dtype=np.float32),
                   400, 80, 1, xtilt=0.3, rotation_sigma=0.5, noise=0.3,
                   method="SIRT", iters=30, gamma=0.5)
    elif name == "cfg2":
        # Ideal single-axis geometry (no offsets, no XTILT): rows independent.
        c = Config("cfg2", 4096, 4096, 512, np.arange(-60, 61, 2, dtype=np.float32),
                   3000, 300, 2, method="SIRT", iters=20, gamma=0.5)
        c.extra["scale"] = 0.5  # semi-axes U(8, 80) px, bead radius 6 px
        c.extra["noise"] = "poisson"
    else:
        raise KeyError(name)
    if scale > 1:
        s3 = scale ** 3
        c.nx //= scale
        c.ny //= scale
        c.thickness = max(4, c.thickness // scale)
        c.n_ellipsoids = max(3, c.n_ellipsoids // s3 * 4)
        c.n_beads = max(2, c.n_beads // s3 * 4)
        c.extra["scale"] = scale
    return c


def coefficients(cfg: Config, base=None) -> np.ndarray:
    """[ntilt][8] coefficients: the reference geometry for the tilt angles and
    XTILT, then the per-tilt detector shifts (a0, b0) and in-plane rotations
    (rotating (a, b) about the origin) that the configuration adds.

    ``base(angles, offset, pitch, zshift) -> [ntilt][8]`` computes the
    reference geometry; by default the engine's ``tr_geometry_from_angles``.
    The CPU reference arm of the benchmark passes the reference's own
    TranslateAngleToCoefficients / DecorateCoefficients instead, so that it
    never loads the engine."""
    if base is None:
        from .tiltrec import geometry_from_angles as base
    c = np.array(base(cfg.angles, 0.0, cfg.xtilt, 0.0), dtype=np.float64).reshape(-1, 8)
    rng = np.random.default_rng(cfg.seed + 1000)
    nt = cfg.ntilt
    if cfg.rotation_sigma:
        psi = np.deg2rad(rng.normal(0.0, cfg.rotation_sigma, nt))
        a, b = c[:, 0:4].copy(), c[:, 4:8].copy()
        cp, sp = np.cos(psi)[:, None], np.sin(psi)[:, None]
        c[:, 0:4] = cp * a - sp * b
        c[:, 4:8] = sp * a + cp * b
    if cfg.offset_sigma:
        c[:, 0] += rng.normal(0.0, cfg.offset_sigma, nt)
        c[:, 4] += rng.normal(0.0, cfg.offset_sigma, nt)
    return c


def phantom(cfg: Config, layout: int = 0, device="cpu", dtype=None):
    """Additive ellipsoid + bead phantom as a torch tensor, Y layout
    [ny][th][nx] (layout 0) or Z layout [th][ny][nx] (layout 1).
    Objects are voxelised inside their bounding boxes with 2x2x2
    supersampling."""
    import torch
    dtype = dtype or torch.float32
    rng = np.random.default_rng(cfg.seed)
    nx, ny, th = cfg.nx, cfg.ny, cfg.thickness
    scale = cfg.extra.get("scale", 1)
    vol = torch.zeros((ny, th, nx), dtype=torch.float32, device=device)
    objs = []
    for _ in range(cfg.n_ellipsoids):
        ctr = rng.uniform([0, 0, 0], [nx, ny, th])
        axes = rng.uniform(4.0, 40.0, 3) / scale
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        objs.append((ctr, axes, rot, rng.uniform(0.2, 1.0)))
    for _ in range(cfg.n_beads):
        ctr = rng.uniform([0, 0, 0], [nx, ny, th])
        r = max(1.0, 3.0 / scale)
        objs.append((ctr, np.array([r, r, r]), np.eye(3), 5.0))
    off = torch.tensor([0.25, 0.75], device=device)
    for ctr, axes, rot, dens in objs:
        ext = float(np.max(axes)) + 1.0
        lo = np.maximum(np.floor(ctr - ext).astype(int), 0)
        hi = np.minimum(np.ceil(ctr + ext).astype(int) + 1, [nx, ny, th])
        if np.any(hi <= lo):
            continue
        xs = torch.arange(lo[0], hi[0], device=device, dtype=torch.float32)
        ys = torch.arange(lo[1], hi[1], device=device, dtype=torch.float32)
        zs = torch.arange(lo[2], hi[2], device=device, dtype=torch.float32)
        inv = torch.tensor(rot.T / axes[:, None], dtype=torch.float32, device=device)
        occ = torch.zeros((len(ys), len(zs), len(xs)), device=device)
        for dx in off:
            for dy in off:
                for dz in off:
                    px = xs + dx - float(ctr[0])
                    py = ys + dy - float(ctr[1])
                    pz = zs + dz - float(ctr[2])
                    Y, Z, X = torch.meshgrid(py, pz, px, indexing="ij")
                    pts = torch.stack([X, Y, Z], dim=-1) @ inv.T
                    occ += (pts.pow(2).sum(-1) <= 1.0).float()
        vol[lo[1]:hi[1], lo[2]:hi[2], lo[0]:hi[0]] += float(dens) * occ / 8.0
    if layout == 1:
        vol = vol.permute(1, 0, 2).contiguous()
    return vol.to(dtype)


def add_noise(proj, cfg: Config, seed_offset: int = 7):
    """Gaussian noise with sigma = cfg.noise * std(proj) (seeded, numpy)."""
    p = np.asarray(proj, np.float32)
    rng = np.random.default_rng(cfg.seed + seed_offset)
    sigma = cfg.noise * float(p.std())
    return (p + rng.normal(0.0, sigma, p.shape)).astype(np.float32)


def project_series(engine, cfg: Config, layout: int = 0, noise: str = "gaussian",
                   mean_counts: float = 20.0):
    """Tilt series of ``cfg``'s phantom on the device, projected with the
    engine's forward model (val/wt where wt != 0) under the problem already
    set on ``engine``; returns a contiguous float32 CUDA tensor [nt][ny][nx].

    noise: ``"gaussian"`` adds sigma = cfg.noise * std; ``"poisson"`` maps the
    projections linearly onto [0, 2 * mean_counts] and draws counting noise
    (electrons per pixel); ``"none"`` leaves them clean.  Seeded from
    cfg.seed."""
    import torch
    nx, ny, nt = cfg.nx, cfg.ny, cfg.ntilt
    ph = phantom(cfg, layout, device="cuda")
    val = torch.zeros((nt, ny, nx), device="cuda")
    wt = torch.zeros_like(val)
    engine.forward_project(ph, val, wt)
    proj = torch.where(wt != 0, val / torch.where(wt != 0, wt, 1), 0)
    del ph, val, wt
    g = torch.Generator(device="cuda").manual_seed(cfg.seed + 7)
    if noise == "gaussian":
        proj += cfg.noise * proj.std() * torch.randn(proj.shape, device="cuda", generator=g)
    elif noise == "poisson":
        lo, hi = proj.min(), proj.max()
        proj = (proj - lo) * (2.0 * mean_counts / torch.clamp(hi - lo, min=1e-30))
        proj = torch.poisson(proj, generator=g)
    elif noise != "none":
        raise ValueError(noise)
    torch.cuda.synchronize()
    return proj.contiguous()


def serve_stream(n: int, rate: float = 4.0, seed: int = 7):
    """The serving configuration's request stream (seeded): Poisson arrivals
    at ``rate`` per second; each request draws its series from the batched
    configuration's distribution (projection size from {512^2, 1024^2,
    2048^2}, tilt count from {41, 61, 81}, thickness U(64, 384)) and asks WBP,
    SIRT-10 or SIRT-30 (uniform).  Returns (classes, requests): one phantom
    series Config per (size, tilts) class, angles over +-U(60, 70) degrees,
    whose projections every request of that class reconstructs at its own
    thickness; requests are dicts (t, cls, thickness, method, iters)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    classes = {}
    reqs = []
    for k in range(n):
        size = int(rng.choice([512, 1024, 2048]))
        nt = int(rng.choice([41, 61, 81]))
        th = int(rng.uniform(64, 384))
        m = int(rng.integers(3))
        key = (size, nt)
        if key not in classes:
            amax = float(rng.uniform(60.0, 70.0))
            c = Config(f"serve{size}x{nt}", size, size, 256 * size // 2048,
                       np.linspace(-amax, amax, nt).astype(np.float32), 50, 20,
                       seed * 1000 + len(classes), offset_sigma=1.0, noise=0.1)
            c.extra["scale"] = 256.0 / size
            classes[key] = c
        reqs.append(dict(t=float(t[k]), cls=key, thickness=th,
                         method=["WBP", "SIRT-10", "SIRT-30"][m], iters=[0, 10, 30][m]))
    return classes, reqs


def batch_series(n: int = 64, seed: int = 3) -> list[Config]:
    """The batched configuration's tilt series (seeded): projection size
    drawn from {512^2, 1024^2, 2048^2}, tilt count from {41, 61, 81} over
    +-U(60, 70) degrees, thickness U(64, 384) voxels; cfg0's ellipsoid and
    bead phantom (50 + 20 objects, per-tilt offsets N(0, 1 px), noise 0.1 std)
    with lengths scaled to the projection size.  Each series is WBP followed
    by SIRT-10 (relaxation 0.5) from the WBP result."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = int(rng.choice([512, 1024, 2048]))
        nt = int(rng.choice([41, 61, 81]))
        amax = float(rng.uniform(60.0, 70.0))
        th = int(rng.uniform(64, 384))
        c = Config(f"batch{i}", size, size, th,
                   np.linspace(-amax, amax, nt).astype(np.float32), 50, 20,
                   seed * 1000 + i, offset_sigma=1.0, noise=0.1, method="WBP+SIRT",
                   iters=10, gamma=0.5)
        c.extra["scale"] = 256.0 / size
        out.append(c)
    return out
