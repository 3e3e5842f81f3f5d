"""Benchmark: plain FP32 SIRT-30 (relaxation 0.5) on the 1024^2 x 61-tilt
tilt series, volume 1024 x 1024 x 256 (the SIRT configuration), through the
TiltRec B200 engine's C ABI.

One step = one complete reconstruction: upload of the series' geometry
(which also recomputes its projection and voxel weights), a zeroed volume and
30 SIRT iterations (forward splat, residual, back-projection and update).
Metric: voxel-projection updates per second (VPU/s; each SIRT iteration
counts 2 x tilts x voxels).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent reconstruction per GPU (one process per GPU under
torchrun; the path needs no exchange between series), scaling "weak".

--impl reference times the reference's own CPU implementation of the path
(the compiled reference sources in oracle/_ref, else the oracle restatement)
on the host's cores, on a bounded row sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "voxel-proj updates/s"
UNIT = "VPU/s"
WORKLOAD = "SIRT-30 FP32, 61 tilts 1024x1024, volume 1024x1024x256 (cfg1)"


def coeff_separable(c8) -> bool:
    """The engine's separable test: b1 = b3 = 0 and b2 = 1 for every tilt."""
    c = np.asarray(c8, np.float64).reshape(-1, 8)
    return bool(np.all(c[:, 5] == 0) and np.all(c[:, 7] == 0) and np.all(c[:, 6] == 1))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes per full cfg1 launch of the dominant kernels, from one ncu
# capture each (dram__bytes_read.sum + dram__bytes_write.sum of the cfg1
# geometry at half the lengths: stack 61 x 512^2, volume 512^2 x 128), scaled
# by component to the full launch: voxel-side bytes x 8, detector-side bytes
# x 4.  fp_kernel: 134.2 MB volume read x 8 + (66.6 MB read + 64.8 MB
# written) x 4; bp_tma_kernel (SIRT): (134.2 MB volume read + 110.9 MB
# written) x 8 + 229.2 MB detector-side reads x 4.  Captured with
#   ncu --set full --clock-control none -k regex:<kernel> -s <n> -c 1 \
#       python bench.py --kernels --scale 2 --iters 2
# (fp_kernel: -s 4, the first timed iteration's; bp_tma_kernel: -s 1).
TRAFFIC_BYTES_PER_LAUNCH = {"fp_kernel": 1.5992e9, "bp_kernel": 2.8776e9}


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed
    region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                smax = float(p[1])
            except ValueError:
                continue
            for n, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_series(eng, torch, cfg, coeff):
    """Synthetic cfg1 tilt series on the device: ellipsoid + bead phantom,
    projected with the engine's forward model (val/wt), plus Gaussian noise
    of 0.3 x std.  Input generation only; it is outside the timed region."""
    from autom2_b200 import synth
    return synth.project_series(eng, cfg, 0, "gaussian")


def cpu_baseline(cfg, coeff, proj_np, target_s: float = 12.0):
    """The reference SIRT on a bounded row sample, all host threads.  Each
    thread owns an even share of the sampled rows plus the reference's XTILT
    halo (ceil(|tan(pitch)| * th) rows per side, as a TiltRec-mpi rank does);
    every row a thread reconstructs counts as work."""
    import math

    import oracle
    nthreads = os.cpu_count() or 1
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    halo = math.ceil(abs(math.tan(math.radians(cfg.xtilt))) * th)

    def rows_done(r0, rows):
        base, rem = divmod(rows, nthreads)
        total = 0
        for r in range(nthreads):
            s = r0 + r * base + min(r, rem)
            e = s + base + (1 if r < rem else 0)
            if e > s:
                total += (e - s) + min(halo, s) + min(halo, ny - e)
        return total

    if oracle.reference_available():
        ref = oracle.Reference()
        c20 = oracle.coeff20(coeff)
        kind = "reference"

        def run(rows):
            r0 = ny // 2 - rows // 2
            t = ref.y_sirt_threaded(nthreads, nx, ny, nt, th, c20, cfg.xtilt, proj_np,
                                    r0, rows, 1, cfg.gamma)
            return t, rows_done(r0, rows)
    else:
        R = oracle.Restatement()
        kind = "port"

        def run(rows):
            r0 = ny // 2 - rows // 2
            o = (nx * 0.5, th * 0.5 - r0, th * 0.5)
            g = R.geom(nx, rows, nt, th, 0, 0, o)
            t0 = time.perf_counter()
            R.sirt(g, coeff, proj_np[:, r0:r0 + rows].copy(),
                   np.zeros((rows, th, nx), np.float32), 1, cfg.gamma)
            return time.perf_counter() - t0, rows
    rows = nthreads
    t, done = run(rows)
    per_row = t / max(1.0, done / nthreads)          # seconds per row per thread
    want = max(1, int(target_s / per_row) - 2 * halo)  # rows per thread
    rows = min(ny - 2 * halo, want * nthreads)
    if rows > nthreads:
        t, done = run(rows)
    vpu = 2.0 * nt * done * th * nx
    return {"value": vpu / t, "unit": UNIT, "cores": nthreads, "kind": kind,
            "sample": f"1 SIRT iteration of the cfg1 series on {rows} of {ny} rows "
                      f"({done} rows incl. XTILT halos, {nthreads} threads), {t:.1f} s"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    import oracle
    from autom2_b200 import synth
    cfg = synth.config("cfg1")
    # The geometry comes from the reference's own TranslateAngleToCoefficients
    # and DecorateCoefficients (oracle/_ref), else the oracle restatement of
    # them: this arm never loads the engine library.
    if oracle.reference_available():
        ref = oracle.Reference()

        def base(a, o, p, z):
            c20 = ref.coeffs20(a, o, p, z)
            return np.concatenate([c20[:, 0:4], c20[:, 10:14]], axis=1)
    else:
        base = oracle.Restatement().coeffs
    coeff = synth.coefficients(cfg, base=base)
    rng = np.random.default_rng(1)
    # The CPU arm reconstructs row samples of the same series shape; the
    # input values do not change its timing.
    proj = rng.normal(size=(cfg.ntilt, cfg.ny, cfg.nx)).astype(np.float32)
    vals = []
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(cfg, coeff, proj, target_s=6.0 if i < args.warmup else 10.0)
        if i >= args.warmup:
            vals.append(b)
    value = statistics.median(v["value"] for v in vals)
    cb = dict(vals[-1])
    cb["value"] = value
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample": cb["sample"]},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from autom2_b200 import build, synth
    from autom2_b200 import tiltrec as T

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    build.build_lib()
    cfg = synth.config("cfg1")
    coeff = synth.coefficients(cfg)
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    eng = T.Engine(dev)
    eng.set_problem(nx, ny, nt, th, coeff, T.LAYOUT_Y)
    proj = make_series(eng, torch, cfg, coeff)
    vol = torch.zeros((ny, th, nx), device="cuda")
    vpu_step = 2.0 * cfg.iters * nt * nx * ny * th
    stream = torch.cuda.current_stream()

    def step():
        eng.update_geometry(coeff)
        vol.zero_()
        eng.sirt(proj, vol, cfg.iters, cfg.gamma)

    def barrier():
        if ws > 1:
            dist.barrier()

    # L2 (126 MB) holds a small part of the 1 GB volume and 256 MB stack
    # that every pass streams, so no extra flush is needed between steps.
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    if ws > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = ws * vpu_step / (ms / 1e3)

    # Roofline of the dominant kernel (back-projection with SIRT update).
    # Algorithmic bytes per launch: residual stack (nt*ny*nx*4, staged once
    # per tile window from L2) + voxel weights read (4 B/voxel) + volume
    # read and write (8 B/voxel).
    hbm, peak_kind = peaks()
    val = torch.zeros((nt, ny, nx), device="cuda")
    nvox = nx * ny * th
    bp_bytes = nt * ny * nx * 4 + nvox * 12
    fp_bytes = nvox * 4 + nt * ny * nx * 4
    reps = 5
    eng.sirt(proj, vol, 1, cfg.gamma)  # weights ready, resid in scratch
    torch.cuda.synchronize()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record(stream)
    for _ in range(reps):
        eng.backproject(proj, vol)
    b1.record(stream)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(reps):
        eng.forward_project(vol, val)
    f1.record(stream)
    torch.cuda.synchronize()
    bp_ms = b0.elapsed_time(b1) / reps
    fp_ms = f0.elapsed_time(f1) / reps
    # bytes for the timed normalised back-projection: stack + volume RMW
    bpn_bytes = nt * ny * nx * 4 + nvox * 8
    dominant = "fp_kernel" if fp_ms > bp_ms else "bp_kernel"
    kms, kbytes = (fp_ms, fp_bytes) if fp_ms > bp_ms else (bp_ms, bpn_bytes)
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = TRAFFIC_BYTES_PER_LAUNCH.get(dominant)
    vpu_kernel = nt * nvox
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "kernel": dominant,
                "peak_source": peak_kind,
                "kernel_ms": kms, "kernel_vpu_per_s": vpu_kernel / (kms / 1e3),
                "fp_ms": fp_ms, "bp_ms": bp_ms,
                "note": "back-projection and forward splat are FP32-issue and "
                        "shared-memory bound (no tensor-core form); HBM fraction "
                        "reported as asked"}

    # End to end through the C ABI with host buffers, as the drop-in CLI
    # runs it: geometry, H2D of the stack, 30 iterations from a zero volume
    # (the reference's default start), D2H of the volume.
    proj_h = proj.cpu().pin_memory()
    vol_h = torch.empty((ny, th, nx)).pin_memory()
    proj_np, vol_np = proj_h.numpy(), vol_h.numpy()
    e2e_steps = max(1, min(args.steps, 3))
    eng.update_geometry(coeff)
    eng.reconstruct_host("SIRT", proj_np, vol_np, cfg.iters, cfg.gamma, zero_start=True)  # warm
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.update_geometry(coeff)
        eng.reconstruct_host("SIRT", proj_np, vol_np, cfg.iters, cfg.gamma, zero_start=True)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    if ws > 1:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": ws * vpu_step / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": int(proj_np.nbytes),
           "d2h_bytes_per_step": int(vol_np.nbytes), "ms_per_step": e2e_s * 1e3}

    # The same step with 16-bit storage: FP16 projections (per-tilt
    # power-of-two scales) and an FP16 residual, FP32 volume and sums.
    q, qscale = eng.quantize(proj, torch.float16)
    torch.cuda.synchronize()
    l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lp_steps = max(1, min(args.steps, 2))
    l0.record(stream)
    for _ in range(lp_steps):
        eng.update_geometry(coeff)
        vol.zero_()
        eng.sirt_lp(q, qscale, vol, cfg.iters, cfg.gamma, "f16")
    l1.record(stream)
    torch.cuda.synchronize()
    lp_ms = l0.elapsed_time(l1) / lp_steps
    del q, qscale
    # The same step with deterministic forward projections (int64 sums).
    eng.set_deterministic(True)
    eng.update_geometry(coeff)
    vol.zero_()
    eng.sirt(proj, vol, 1, cfg.gamma)  # scratch, weights
    torch.cuda.synchronize()
    d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d0.record(stream)
    for _ in range(lp_steps):
        eng.update_geometry(coeff)
        vol.zero_()
        eng.sirt(proj, vol, cfg.iters, cfg.gamma)
    d1.record(stream)
    torch.cuda.synchronize()
    det_ms = d0.elapsed_time(d1) / lp_steps
    eng.set_deterministic(False)
    variants = {"sirt_f16_storage": {
        "ms_per_step": lp_ms, "value": ws * vpu_step / (lp_ms / 1e3), "unit": UNIT,
        "storage": "projections and residual FP16 (per-tilt scale), volume FP32",
        "bytes_saved_per_iter": int(2 * nt * ny * nx * 2)},
        "sirt_deterministic": {
        "ms_per_step": det_ms, "value": ws * vpu_step / (det_ms / 1e3), "unit": UNIT,
        "forward_projection": "int64 fixed-point sums, bitwise repeatable"}}

    line = None
    if rank == 0:
        cb = cpu_baseline(cfg, coeff, proj.cpu().numpy()) if ws == 1 else None
        # weights: splat of ones, tile classification, border-tile weight pass
        # (+ per-row weights for separable geometry); then (fp, resid, bp) per
        # iteration
        launches_per_step = 3 + int(coeff_separable(coeff)) + 3 * cfg.iters
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": WORKLOAD, "method": "SIRT", "iters": cfg.iters,
                           "gamma": cfg.gamma, "tilts": nt, "proj": [ny, nx],
                           "volume": [nx, ny, th], "layout": "Y",
                           "l2": "inputs larger than L2 (1.07 GB volume, 256 MB stack)",
                           "parallelism": f"replicas x{ws}"},
                "roofline": roofline, "cpu_baseline": cb, "e2e": e2e,
                "gpu_launches": launches_per_step * args.steps,
                "clocks": clk.summary(), "variants": variants}
        print(json.dumps(line), flush=True)
    eng.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line


def run_kernels(args):
    """Profiling case: the cfg1 series with every length divided by --scale,
    then --iters SIRT iterations (forward splat, residual, back-projection
    with update per iteration) after the weight passes.  Prints timings
    only; not a bench line."""
    import torch

    from autom2_b200 import build, synth
    from autom2_b200 import tiltrec as T
    build.build_lib()
    cfg = synth.config("cfg1", args.scale)
    coeff = synth.coefficients(cfg)
    if args.separable:  # ideal single-axis geometry: the separable kernels
        coeff = T.geometry_from_angles(cfg.angles)
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    eng = T.Engine(0)
    eng.set_problem(nx, ny, nt, th, coeff, T.LAYOUT_Y)
    proj = make_series(eng, torch, cfg, coeff)
    vol = torch.zeros((ny, th, nx), device="cuda")
    eng.sirt(proj, vol, 1, cfg.gamma)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    eng.sirt(proj, vol, args.iters, cfg.gamma)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(1, args.iters)
    # One R-weighting filter of the stack (the WBP filter) after the SIRT
    # iterations, on a copy.
    filt = proj.clone()
    eng.filter_rweight(filt)  # builds the kernel spectrum
    filt.copy_(proj)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    eng.filter_rweight(filt)
    f1.record()
    torch.cuda.synchronize()
    print(json.dumps({"case": f"cfg1/{args.scale}" + (" separable" if args.separable else ""),
                      "proj": [nt, ny, nx],
                      "volume": [nx, ny, th], "iters": args.iters,
                      "ms_per_iter": ms, "rweight_ms": f0.elapsed_time(f1)}), flush=True)
    eng.close()


def run_cfg0(args):
    """WBP configuration (41 tilts, 256^2, volume 256x256x64): device-resident
    filter + back-projection timed with CUDA events, the host-buffer call
    end to end, and the reference's own CPU filter + BackProject (oracle/_ref,
    one thread) on the same input, with the parity of the two volumes."""
    import torch

    import oracle
    from autom2_b200 import build, synth
    from autom2_b200 import tiltrec as T
    build.build_lib()
    torch.cuda.set_device(0)
    cfg = synth.config("cfg0")
    c8 = synth.coefficients(cfg)
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    eng = T.Engine(0)
    eng.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Y)
    proj = synth.project_series(eng, cfg, 0, "gaussian")
    vol = torch.zeros((ny, th, nx), device="cuda")
    work = proj.clone()
    reps = 200
    for _ in range(5):
        work.copy_(proj)
        eng.wbp(work, vol)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record()
    for _ in range(reps):
        work.copy_(proj)
    c1.record()
    e0.record()
    for _ in range(reps):
        work.copy_(proj)
        eng.wbp(work, vol)
    e1.record()
    torch.cuda.synchronize()
    ms = (e0.elapsed_time(e1) - c0.elapsed_time(c1)) / reps
    vpu = nt * nx * ny * th
    # Host buffers (pinned) through the C ABI; the library filters its device
    # copy of the stack, so the host stack is reused unchanged.
    proj_h = proj.cpu().pin_memory()
    vol_h = torch.empty((ny, th, nx)).pin_memory()
    pn, vn = proj_h.numpy(), vol_h.numpy()
    eng.reconstruct_host("WBP", pn, vn, zero_start=True)
    t0 = time.perf_counter()
    for _ in range(20):
        eng.reconstruct_host("WBP", pn, vn, zero_start=True)
    e2e_ms = (time.perf_counter() - t0) / 20 * 1e3
    ours = vn.copy()
    ref = {"available": oracle.reference_available()}
    if ref["available"]:
        R = oracle.Reference()
        c20 = oracle.coeff20(c8)
        p_np = proj.cpu().numpy()
        t0 = time.perf_counter()
        f = R.filter_rweight(p_np)
        rv = R.y_backproject(nx, ny, nt, th, c20, (nx * 0.5, th * 0.5, th * 0.5), f,
                             np.zeros((ny, th, nx), np.float32))
        ref_s = time.perf_counter() - t0
        ref.update({"value": vpu / ref_s, "seconds": ref_s, "cores": 1,
                    "kind": "reference", "rel_l2_ours_vs_reference": oracle.rel_l2(ours, rv)})
    eng.close()
    print(json.dumps({"workload": "cfg0", "metric": "voxel-proj updates/s", "unit": "VPU/s",
                      "value": vpu / (ms / 1e3), "ms_per_reconstruction": ms,
                      "e2e": {"value": vpu / (e2e_ms / 1e3), "ms": e2e_ms,
                              "h2d_bytes": int(pn.nbytes),
                              "d2h_bytes": int(vn.nbytes)},
                      "cpu_reference": ref, "dtype": "f32", "data": "synthetic",
                      "config": {"method": "WBP", "tilts": nt, "proj": [ny, nx],
                                 "volume": [nx, ny, th], "layout": "Y"}}), flush=True)


def run_cfg2(args):
    """Mixed-precision configuration: SIRT-20 in the Z layout, 61 tilts of
    4096^2, volume 4096x4096x512 (34 GB), counting noise; FP16 projections and
    residuals with FP32 volume and sums, beside the plain FP32 form on the same
    GPU.  Error against the FP64 oracle on a band of rows (the ideal geometry
    makes rows independent, so the band is an exact sub-problem)."""
    import torch

    import oracle
    from autom2_b200 import build, synth
    from autom2_b200 import tiltrec as T
    build.build_lib()
    torch.cuda.set_device(0)
    cfg = synth.config("cfg2")
    c8 = synth.coefficients(cfg)
    nx, ny, nt, th = cfg.nx, cfg.ny, cfg.ntilt, cfg.thickness
    org = T.default_origin(T.LAYOUT_Z, nx, ny, th)
    eng = T.Engine(0)
    eng.set_problem(nx, ny, nt, th, c8, T.LAYOUT_Z, org)
    t0 = time.perf_counter()
    proj = synth.project_series(eng, cfg, T.LAYOUT_Z, "poisson")
    gen_s = time.perf_counter() - t0
    vol = torch.zeros((th, ny, nx), device="cuda")
    iters = args.iters if args.iters != 2 else cfg.iters
    vpu = 2.0 * iters * nt * nx * ny * th

    def timed(fn):
        vol.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    eng.sirt(proj, vol, 1, cfg.gamma)  # weights, warm
    t_f32 = timed(lambda: eng.sirt(proj, vol, iters, cfg.gamma))
    band = 4
    r0 = ny // 2 - band // 2
    f32_band = vol[:, r0:r0 + band].cpu().numpy()
    q, scale = eng.quantize(proj, torch.float16)
    t_lp = timed(lambda: eng.sirt_lp(q, scale, vol, iters, cfg.gamma, "f16"))
    lp_band = vol[:, r0:r0 + band].cpu().numpy()
    p_band = proj[:, r0:r0 + band].cpu().numpy()
    # The same FP16 SIRT through z-slabs: the volume host-resident (page-locked)
    # and streamed through three device slabs at the autotuned depth, then the
    # device-resident volume swept slab by slab at that depth.
    del vol
    torch.cuda.empty_cache()
    hvol = torch.zeros((th, ny, nx), pin_memory=True)
    depth, sweep_ms = eng.autotune_zslab(q, hvol, scale, "f16")
    hvol.zero_()
    t0 = time.perf_counter()
    eng.sirt_zslabs(q, hvol, iters, cfg.gamma, depth, scale, "f16")
    t_host = time.perf_counter() - t0
    host_band = hvol[:, r0:r0 + band].numpy().copy()
    del hvol
    dvol = torch.zeros((th, ny, nx), device="cuda")
    vol = dvol
    t_dev = timed(lambda: eng.sirt_zslabs(q, dvol, iters, cfg.gamma, depth, scale, "f16"))
    dev_band = dvol[:, r0:r0 + band].cpu().numpy()
    del dvol, vol
    eng.close()
    R = oracle.Restatement()
    g = R.geom(nx, band, nt, th, T.LAYOUT_Z, 0, (org[0], org[1] - r0, org[2]))
    t0 = time.perf_counter()
    ref = R.sirt(g, c8, p_band, np.zeros((th, band, nx)), iters, cfg.gamma, fp64=True)
    oracle_s = time.perf_counter() - t0

    def err(a):
        a64 = np.asarray(a, np.float64)
        return {"rel_l2": oracle.rel_l2(a64, ref),
                "max_abs_rel": float(np.abs(a64 - ref).max() / np.abs(ref).max())}

    print(json.dumps({"workload": "cfg2", "metric": "voxel-proj updates/s", "unit": "VPU/s",
                      "value": vpu / t_lp, "seconds": t_lp,
                      "dtype": "f16 storage (projections, residual), f32 volume and sums",
                      "vs_fp64_oracle": err(lp_band),
                      "plain_f32": {"value": vpu / t_f32, "seconds": t_f32,
                                    "vs_fp64_oracle": err(f32_band)},
                      "zslab": {"depth": depth, "autotune_sweep_ms": sweep_ms,
                                "host_resident": {"value": vpu / t_host, "seconds": t_host,
                                                  "vs_fp64_oracle": err(host_band)},
                                "device_resident": {"value": vpu / t_dev, "seconds": t_dev,
                                                    "vs_fp64_oracle": err(dev_band)}},
                      "oracle": {"rows": [r0, r0 + band], "seconds": oracle_s},
                      "generation_s": gen_s, "data": "synthetic",
                      "config": {"method": f"SIRT-{iters}", "tilts": nt, "proj": [ny, nx],
                                 "volume": [nx, ny, th], "layout": "Z",
                                 "noise": "Poisson, mean 20 e-/px"}}), flush=True)


class OutputPool:
    """Reusable output volumes per projection size (the batch and serving
    runs keep only this many results alive at once)."""

    def __init__(self, make, sizes_counts):
        import threading as th
        self.cv = th.Condition()
        self.free = {k: [make(k) for _ in range(n)] for k, n in sizes_counts.items()}

    def take(self, key):
        with self.cv:
            self.cv.wait_for(lambda: bool(self.free[key]))
            return self.free[key].pop()

    def give(self, key, buf):
        with self.cv:
            self.free[key].append(buf)
            self.cv.notify_all()


def job_vpu(c, wbp, iters):
    """Voxel-projection updates of one job: WBP one pass, SIRT two per
    iteration."""
    return (int(wbp) + 2 * iters) * c.ntilt * c.nx * c.ny * c.thickness


def run_batch(args):
    """Batched configuration: 64 uneven tilt series, WBP then SIRT-10 each,
    run (1) one at a time through the engine in FP32 (the plain GPU form) and
    (2) all together through the scheduler (persistent graph-replayed steps,
    16-bit storage).  Inputs are device-resident; one JSON line."""
    import torch

    from autom2_b200 import build, synth
    from autom2_b200 import tiltrec as T
    build.build_lib()
    torch.cuda.set_device(0)
    specs = synth.batch_series(args.jobs or 64, seed=3)
    eng = T.Engine(0)
    series = []
    for c in specs:
        c8 = synth.coefficients(c)
        eng.set_problem(c.nx, c.ny, c.ntilt, c.thickness, c8, T.LAYOUT_Y)
        series.append((c, c8, synth.project_series(eng, c, 0, "gaussian")))
    total_vpu = sum(job_vpu(c, True, c.iters) for c, _, _ in series)
    cmp_idx = [i for i, (c, _, _) in enumerate(series) if c.nx <= 1024][:4]

    def vol_for(buf, c):
        return buf[: c.ny * c.thickness * c.nx].view(c.ny, c.thickness, c.nx)

    # (1) plain FP32, one series at a time
    maxv = max(c.nx * c.ny * c.thickness for c, _, _ in series)
    buf = torch.empty(maxv, device="cuda")
    plain_ref = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i, (c, c8, proj) in enumerate(series):
        eng.set_problem(c.nx, c.ny, c.ntilt, c.thickness, c8, T.LAYOUT_Y)
        v = vol_for(buf, c)
        v.zero_()
        f = proj.clone()
        eng.wbp(f, v)
        del f
        eng.sirt(proj, v, c.iters, c.gamma)
        if i in cmp_idx:
            plain_ref[i] = v.clone()
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    del buf
    eng.close()

    # (2) the scheduler, all jobs submitted at once
    counts = {512: 8, 1024: 6, 2048: 4}
    pool = OutputPool(lambda n: torch.empty(n * n * 384, device="cuda"), counts)
    free, _ = torch.cuda.mem_get_info()
    budget = int(free - 8e9)
    S = T.Scheduler(0, hbm_budget=budget, proj_dtype=args.storage, resid_dtype=args.storage)
    probe_i = next(i for i, (c, _, _) in enumerate(series) if c.nx == 1024)
    c, c8, proj = series[probe_i]
    pv = torch.zeros((c.ny, c.thickness, c.nx), device="cuda")
    tuned = S.autotune(S.job(proj, pv, c8, T.LAYOUT_Y, sirt_iters=2, gamma=c.gamma))
    del pv
    import threading as th

    def run_sched():
        results = {}
        lat = [0.0] * len(series)

        def waiter(i, jid, key, b):
            try:
                lat[i] = S.wait(jid)
                if i in cmp_idx:
                    results[i] = vol_for(b, series[i][0]).clone()
            finally:
                pool.give(key, b)

        threads = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i, (c, c8, proj) in enumerate(series):
            b = pool.take(c.nx)
            v = vol_for(b, c)
            jid = S.submit(S.job(proj, v, c8, T.LAYOUT_Y, wbp=True, sirt_iters=c.iters,
                                 gamma=c.gamma))
            t = th.Thread(target=waiter, args=(i, jid, c.nx, b))
            t.start()
            threads.append(t)
        for t in threads:
            t.join()
        torch.cuda.synchronize()
        span = time.perf_counter() - t0
        errs = []
        for i in cmp_idx:
            a, r = results[i].double(), plain_ref[i].double()
            errs.append(float((a - r).norm() / r.norm()))
        return span, lat, errs

    t_batch, lat, errs = run_sched()
    info = S.stats()
    S.set_policy("srpt")
    t_srpt, lat_srpt, errs_srpt = run_sched()
    S.close()
    # The same policy with FP32 storage (the plain form's): the scheduler's own
    # cost, without the 16-bit conversions.
    S = T.Scheduler(0, hbm_budget=budget, proj_dtype="f32", resid_dtype="f32")
    S.set_policy("srpt")
    t_srpt32, lat_srpt32, errs_srpt32 = run_sched()
    S.close()
    line = {"workload": "batch", "metric": "voxel-proj updates/s", "unit": "VPU/s",
            "value": total_vpu / t_batch, "n_gpus": 1, "higher_is_better": True,
            "jobs": len(series), "recon_per_hour": len(series) / t_batch * 3600,
            "seconds": t_batch, "dtype": f"{args.storage} storage, f32 accumulate",
            "plain": {"value": total_vpu / t_plain, "seconds": t_plain,
                      "recon_per_hour": len(series) / t_plain * 3600, "dtype": "f32",
                      "form": "one series at a time, engine tr_wbp + tr_sirt"},
            "speedup_vs_plain": t_plain / t_batch,
            "rel_l2_vs_plain_f32": {"max": max(errs), "jobs": cmp_idx},
            "p50_latency_s": statistics.median(lat), "autotune": {"smem_bp": tuned[0],
                                                                   "ctas_per_sm": tuned[1]},
            "srpt": {"value": total_vpu / t_srpt, "seconds": t_srpt,
                     "recon_per_hour": len(series) / t_srpt * 3600,
                     "speedup_vs_plain": t_plain / t_srpt,
                     "p50_latency_s": statistics.median(lat_srpt),
                     "mean_latency_s": float(np.mean(lat_srpt)),
                     "rel_l2_vs_plain_f32_max": max(errs_srpt),
                     "form": "the same scheduler, shortest remaining work first, per-job "
                             "kernels"},
            "srpt_f32_storage": {"value": total_vpu / t_srpt32, "seconds": t_srpt32,
                                 "recon_per_hour": len(series) / t_srpt32 * 3600,
                                 "speedup_vs_plain": t_plain / t_srpt32,
                                 "p50_latency_s": statistics.median(lat_srpt32),
                                 "rel_l2_vs_plain_f32_max": max(errs_srpt32)},
            "scheduler": info, "data": "synthetic",
            "config": {"series": "64 seeded: N in {512,1024,2048}, T in {41,61,81} over "
                                 "+-U(60,70) deg, th U(64,384); WBP then SIRT-10 (0.5)",
                       "budget_bytes": budget}}
    print(json.dumps(line), flush=True)


def run_serve(args):
    """Serving configuration: a seeded Poisson stream (rate --rate, default 4
    per second; seed 7) of --jobs requests (default 200: a prefix of the
    2000-request stream), each drawn from the batched configuration's series
    distribution and asking WBP, SIRT-10 or SIRT-30; host buffers in, host
    volume out, 150 GB HBM budget.  Forms, each fed the same arrivals:
      * plain: one request at a time in arrival order through
        tr_reconstruct_host (FP32), a FIFO single server;
      * the scheduler (16-bit storage) under each step policy, fed by a
        front end that keeps --inflight requests submitted (the shortest
        pending one next under SRPT, the oldest under the batched policy):
        pure shortest remaining work, the same aged (work divided by
        1 + wait / --aging, in the front end and the scheduler), batched.
    Latency runs from arrival to the volume in host memory.  Each request's
    middle volume row from the scheduler is compared with the plain FP32
    result (relative L2)."""
    import threading as th

    import torch

    from autom2_b200 import build, synth
    from autom2_b200 import tiltrec as T
    build.build_lib()
    torch.cuda.set_device(0)
    n = args.jobs or 200
    rate = args.rate or 4.0
    classes, reqs = synth.serve_stream(n, rate, seed=7)
    eng = T.Engine(0)
    series = {}
    t0 = time.perf_counter()
    for key, c in classes.items():
        c8 = synth.coefficients(c)
        eng.set_problem(c.nx, c.ny, c.ntilt, c.thickness, c8, T.LAYOUT_Y)
        p = synth.project_series(eng, c, 0, "gaussian").cpu().pin_memory()
        series[key] = (c, c8, p)
    gen_s = time.perf_counter() - t0
    K = args.inflight
    sizes = sorted({key[0] for key in classes})
    bufs = {s: [torch.empty(s * s * 384).pin_memory() for _ in range(K)] for s in sizes}

    def work(k):
        r = reqs[k]
        c = series[r["cls"]][0]
        return (int(r["iters"] == 0) + 2 * r["iters"]) * c.ntilt * c.nx * c.ny * r["thickness"]

    mean_vpu = float(np.mean([work(k) for k in range(n)]))

    def out_view(buf, c, thk):
        return buf[: c.ny * thk * c.nx].view(c.ny, thk, c.nx)

    def serve(run_one, order, limit):
        """Feeds arrivals to `run_one(k, buf, finish)` with at most `limit`
        in flight; returns latencies, makespan, middle rows."""
        lock = th.Condition()
        pending, done_at, rows = [], [0.0] * n, [None] * n
        state = {"inflight": 0, "next": 0}
        free = {s: list(bufs[s]) for s in sizes}
        start = time.perf_counter()

        def finish(k, buf):
            c = series[reqs[k]["cls"]][0]
            done_at[k] = time.perf_counter() - start
            rows[k] = out_view(buf, c, reqs[k]["thickness"])[c.ny // 2].numpy().copy()
            with lock:
                free[c.nx].append(buf)
                state["inflight"] -= 1
                lock.notify_all()

        threads = []
        for _ in range(n):
            with lock:
                while True:
                    now = time.perf_counter() - start
                    while state["next"] < n and reqs[state["next"]]["t"] <= now:
                        pending.append(state["next"])
                        state["next"] += 1
                    if pending and state["inflight"] < limit:
                        break
                    wait = 0.05
                    if state["next"] < n:
                        wait = min(wait, max(0.0, reqs[state["next"]]["t"] - now))
                    lock.wait(timeout=wait)
                if order == "fifo" or order == "batched":
                    k = pending[0]
                else:  # shortest work first, aged for "srpt_aged"
                    age = args.aging if order == "srpt_aged" else 0.0
                    now = time.perf_counter() - start
                    k = min(pending, key=lambda q: work(q) / (
                        1.0 + (now - reqs[q]["t"]) / age if age > 0 else 1.0))
                pending.remove(k)
                state["inflight"] += 1
                buf = free[series[reqs[k]["cls"]][0].nx].pop()
            t = run_one(k, buf, finish)
            if t is not None:
                threads.append(t)
        for t in threads:
            t.join()
        lat = [done_at[k] - reqs[k]["t"] for k in range(n)]
        return lat, max(done_at), rows

    # plain: FIFO single server, one request at a time
    def plain_one(k, buf, finish):
        r = reqs[k]
        c, c8, p = series[r["cls"]]
        eng.set_problem(c.nx, c.ny, c.ntilt, r["thickness"], c8, T.LAYOUT_Y)
        v = out_view(buf, c, r["thickness"])
        eng.reconstruct_host("WBP" if r["iters"] == 0 else "SIRT", p.numpy(), v.numpy(),
                             r["iters"], 0.5, zero_start=True)
        finish(k, buf)
        return None

    lat_p, span_p, rows_p = serve(plain_one, "fifo", 1)
    eng.close()
    free_b, _ = torch.cuda.mem_get_info()
    budget = min(int(args.budget_gb * 1e9), int(free_b - 8e9))
    forms = {}
    for form in ("srpt", "srpt_aged", "batched"):
        S = T.Scheduler(0, hbm_budget=budget, proj_dtype=args.storage, resid_dtype=args.storage)
        S.set_policy("batched" if form == "batched" else "srpt")
        if form == "srpt_aged":
            S.set_aging(args.aging)

        def sched_one(k, buf, finish, S=S):
            r = reqs[k]
            c, c8, p = series[r["cls"]]
            v = out_view(buf, c, r["thickness"])
            jid = S.submit(S.job(p.numpy(), v.numpy(), c8, T.LAYOUT_Y, wbp=r["iters"] == 0,
                                 sirt_iters=r["iters"], gamma=0.5))

            def waiter():
                try:
                    S.wait(jid)
                finally:  # a failed job still releases its slot (and is reported)
                    finish(k, buf)
            t = th.Thread(target=waiter)
            t.start()
            return t

        lat, span, rows = serve(sched_one, form, K)
        info = S.stats()
        S.close()
        errs = [oracle_free_rel_l2(a, b) for a, b in zip(rows, rows_p)]
        forms[form] = {"value": n / span * 3600, "makespan_s": span,
                         "p50_latency_s": pct(lat, 50), "p99_latency_s": pct(lat, 99),
                         "mean_latency_s": float(np.mean(lat)),
                         "rel_l2_vs_plain_f32_middle_row": {"max": max(errs),
                                                            "median": pct(errs, 50)},
                         "scheduler": info}
    best = forms["srpt"]
    line = {"workload": "serve", "metric": "reconstructions/hour", "unit": "recon/h",
            "value": best["value"], "higher_is_better": True, "n_gpus": 1,
            "jobs": n, "arrival_rate_per_s": rate, "offered_vpu_per_s": mean_vpu * rate,
            "p50_latency_s": best["p50_latency_s"], "p99_latency_s": best["p99_latency_s"],
            "makespan_s": best["makespan_s"],
            "dtype": f"{args.storage} storage, f32 accumulate",
            "speedup_vs_plain": span_p / best["makespan_s"],
            "p50_latency_ratio_plain_over_srpt": pct(lat_p, 50) / best["p50_latency_s"],
            "plain": {"value": n / span_p * 3600, "p50_latency_s": pct(lat_p, 50),
                      "p99_latency_s": pct(lat_p, 99), "mean_latency_s": float(np.mean(lat_p)),
                      "makespan_s": span_p,
                      "form": "FIFO, one request at a time through tr_reconstruct_host, f32"},
            "scheduler_forms": forms, "generation_s": gen_s, "data": "synthetic",
            "config": {"stream": f"Poisson {rate}/s, seed 7, first {n} of the 2000-request "
                                 "stream", "series": "N in {512,1024,2048}, T in {41,61,81} "
                                 "over +-U(60,70) deg, th U(64,384)",
                       "methods": "uniform WBP / SIRT-10 / SIRT-30 (0.5)",
                       "host_buffers": "pinned", "budget_bytes": budget,
                       "inflight": K, "error": "rel-L2 of each request's middle row vs the "
                       "plain FP32 result (an FP64 oracle is out of reach at these sizes)"}}
    print(json.dumps(line), flush=True)


def pct(x, q):
    return float(np.percentile(np.asarray(x), q))


def oracle_free_rel_l2(a, b):
    a64, b64 = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a64 - b64) / max(np.linalg.norm(b64), 1e-300))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--kernels", action="store_true",
                    help="profiling case only (see run_kernels)")
    ap.add_argument("--scale", type=int, default=2)
    ap.add_argument("--iters", type=int, default=2)
    ap.add_argument("--separable", action="store_true",
                    help="profiling case: ideal single-axis geometry")
    ap.add_argument("--workload", default="sirt",
                    choices=["sirt", "cfg0", "cfg2", "batch", "serve"],
                    help="sirt: the headline SIRT-30 line; batch / serve: the batched "
                         "and serving configurations (one JSON line each)")
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--rate", type=float, default=0.0,
                    help="serve: arrivals per second (default 4)")
    ap.add_argument("--inflight", type=int, default=4,
                    help="serve: requests the front end keeps submitted")
    ap.add_argument("--aging", type=float, default=5.0,
                    help="serve: aging time (s) of the aged shortest-work-first form")
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--storage", default="f16", choices=["f32", "f16", "bf16"])
    args = ap.parse_args()
    if args.workload == "cfg0":
        run_cfg0(args)
    elif args.workload == "cfg2":
        run_cfg2(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.kernels:
        run_kernels(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
