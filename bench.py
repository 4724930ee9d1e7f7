"""Benchmark: X-ray band map (0.5-7 keV) of 4,194,304 synthetic gas cells, 1024^2
pixels along z through 6 Mpc, adaptive RKF4(5) at relative tolerance 1e-3.

One step = the whole band-map job: per-cell X-ray flux, particle-grid build and
the adaptive line-of-sight projection of 1,048,576 rays. Metric: Mrays/s.

  value  -- inputs resident in HBM, device time of the step (CUDA events on the
            library's stream), L2 flushed (256 MiB write) before every step.
  e2e    -- the same call through the public C ABI with pinned host buffers:
            H2D of the cells and D2H of the image inside the timed region.

python bench.py [--gpus N --steps K --warmup W] [--impl reference]
N > 1 (torchrun): every rank renders its own replica of the job (the path is
independent per image); value = all rays / max over ranks of the step time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mrays/s (X-ray map, 1e-3 tol)"
NX = NY = 1024
BOX = 6000.0
Z_START = 0.0      # camera plane along z (0: the face of the cube)
DEPTH = BOX        # integration depth
REL_TOL = 1e-3
E_MIN, E_MAX, NUM_SAMPLES = 0.5, 7.0, 100
REDSHIFT, DL = 0.2, 978500.0
WORKLOAD = "xray_band_map_4M_cells_1024sq_rtol1e-3"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


TUNING_FILE = os.path.join(ROOT, "illcrawl_b200", "data", "render_tuning.json")


def tune_schedule(ctx, cam, args, gpu_name):
    """z window of the adaptive render: --z-window if given, else the cached
    autotuner result for this workload and GPU, else run the autotuner (a
    sample of tile rows per candidate, outside the timed region) and cache."""
    import illcrawl_b200 as ilc
    if args.z_window is not None:
        ctx.set_z_window(args.z_window)
        return {"z_window": args.z_window, "source": "command line"}
    key = f"{gpu_name}|xray_band_map_4M_cells_{NX}sq_rtol1e-3|z0={Z_START}|depth={DEPTH}"
    cache = json.load(open(TUNING_FILE)) if os.path.exists(TUNING_FILE) else {}
    if key in cache:
        ctx.set_z_window(cache[key]["z_window"])
        return dict(cache[key], source="cache")
    best, times = ctx.autotune_z_window(cam, DEPTH, REL_TOL, 0.0, ilc.CONTROLLER_FP64,
                                        sample_stride=max(1, NY // 64))
    cache[key] = {"z_window": best, "kernel_ms": times}
    try:
        json.dump(cache, open(TUNING_FILE, "w"), indent=1, sort_keys=True)
    except OSError:
        pass
    return dict(cache[key], source="autotuner")


def make_inputs():
    from illcrawl_b200 import synthetic
    cells = synthetic.xray_cells()
    xyz4 = cells.xyzq(np.zeros(cells.n, np.float32))
    return cells, xyz4


def camera_args():
    return ((BOX / 2, BOX / 2, Z_START), (0.0, 0.0, 1.0), 0.0, BOX * NX / 1024, NX, NY)


def algorithmic_bytes(st, n_cells, n_rays):
    # cell range + float4 per candidate, RKF state per step, output per ray,
    # per-cell value once + Gaunt table.
    return (8 * st["cells_visited"] + 16 * st["candidates"] + 24 * st["steps"] + 4 * n_rays
            + 16 * n_cells + 47304)


def cpu_baseline(cells, nthreads, sample_rays=2048, seed=1):
    """The oracle on the host cores: emissivity + grid over all cells, render of
    a random pixel sample; extrapolated to the full image."""
    import oracle
    import illcrawl_b200 as ilc
    table = ilc.load_gaunt_table()
    t0 = time.perf_counter()
    q = oracle.xray_band(table, cells.rho, cells.u, cells.xe, REDSHIFT, DL, E_MIN, E_MAX,
                         NUM_SAMPLES, nthreads=nthreads)
    g = oracle.Grid(cells.xyzq(q))
    t_fixed = time.perf_counter() - t0
    pix = np.random.default_rng(seed).choice(NX * NY, sample_rays, replace=False)
    t0 = time.perf_counter()
    g.render(oracle.camera(*camera_args()), DEPTH, 0.0, REL_TOL, mode=1, pix=pix,
             nthreads=nthreads)
    t_render = time.perf_counter() - t0
    t_full = t_fixed + t_render * (NX * NY) / sample_rays
    return NX * NY / t_full / 1e6, t_fixed, t_render


def run_reference(args, rank, world):
    """--impl reference: the oracle (CPU restatement of the reference path, the
    reference itself being OpenCL+Boost+MPI+HDF5 that cannot be built here) on
    all host cores, rank 0 only."""
    if rank != 0:
        return
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    cells, _ = make_inputs()
    sample = 256
    vals = []
    for i in range(args.warmup + args.steps):
        v, tf, tr = cpu_baseline(cells, cores, sample_rays=sample, seed=100 + i)
        if i >= args.warmup:
            vals.append(v)
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": NX * NY / (v * 1e6) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded NFW + uniform gas cells)",
            "config": {"workload": f"xray_band_map_4M_cells_{NX}sq_rtol1e-3", "cells": 4194304, "image": [NX, NY],
                       "rel_tol": REL_TOL},
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "port",
                             "sample": f"per step: per-cell X-ray flux + grid build over all "
                                       f"4,194,304 cells, render of {sample} random rays of the "
                                       f"1024^2 image, extrapolated to 1,048,576 rays"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch
    import illcrawl_b200 as ilc
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    cells, xyz4 = make_inputs()
    n = cells.n
    ctx = ilc.Context(local_rank)
    ctx.load_gaunt()
    if args.z_window is not None:
        ctx.set_z_window(args.z_window)
    cam = ilc.camera(*camera_args())
    scaling = ilc.LosScaling(1.0, 1.0, ilc.DA_PIXEL_AREA)
    dev = torch.device("cuda", local_rank)
    d_cells = torch.from_numpy(xyz4).to(dev)
    d_rho, d_u, d_xe = (torch.from_numpy(a).to(dev) for a in (cells.rho, cells.u, cells.xe))
    d_img = torch.empty((NY, NX), dtype=torch.float32, device=dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)

    def step():
        return ctx.project_xray_flux(d_cells, d_rho, d_u, d_xe, cam, DEPTH, rel_tol=REL_TOL,
                                     controller=ilc.CONTROLLER_FP64, e_min=E_MIN, e_max=E_MAX,
                                     num_samples=NUM_SAMPLES, scaling=scaling, image=d_img)

    for i in range(max(args.warmup, 1)):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        step()
        if i == 0:
            tuned = tune_schedule(ctx, cam, args, torch.cuda.get_device_name(dev))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    total_ms, last_stats = 0.0, None
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            flush.fill_(float(_))
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _, last_stats = step()
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    launches = ctx.kernel_launches - launches0
    if dist:
        dist.barrier()
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    rays = NX * NY * world
    value = rays / (ms_per_step * 1e-3) / 1e6

    # e2e: host (pinned) buffers through the public API
    h_cells = torch.from_numpy(xyz4).pin_memory()
    h_rho, h_u, h_xe = (torch.from_numpy(a).pin_memory() for a in (cells.rho, cells.u, cells.xe))
    h_img = torch.empty((NY, NX), dtype=torch.float32).pin_memory()

    def e2e_step():
        return ctx.project_xray_flux(h_cells.numpy(), h_rho.numpy(), h_u.numpy(),
                                     h_xe.numpy(), cam, DEPTH, rel_tol=REL_TOL,
                                     controller=ilc.CONTROLLER_FP64, e_min=E_MIN, e_max=E_MAX,
                                     num_samples=NUM_SAMPLES, scaling=scaling,
                                     image=h_img.numpy())

    e2e_value = None
    if not args.no_e2e:
        e2e_step()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e2e_steps = max(1, min(args.steps, 2))
        e2e_s = 0.0
        for _ in range(e2e_steps):
            flush.fill_(2.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            e2e_s += time.perf_counter() - t0
        e2e_s /= e2e_steps
        if dist:
            t = torch.tensor([e2e_s], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e_value = rays / e2e_s / 1e6

    if rank != 0:
        ctx.close()
        return
    hbm, peak_kind = peaks()
    kbytes = algorithmic_bytes(last_stats, n, NX * NY)
    achieved = kbytes / (last_stats["kernel_ms"] * 1e-3) / 1e9
    cores = os.cpu_count() or 1
    cpu_v = None if args.no_cpu else cpu_baseline(cells, cores)[0]
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded NFW + uniform gas cells, numpy PCG64 seed 20171)",
        "config": {"workload": f"xray_band_map_4M_cells_{NX}sq_rtol1e-3", "cells": n, "image": [NX, NY], "z_range_kpc": DEPTH, "camera_z": Z_START,
                   "rel_tol": REL_TOL, "controller": "fp64", "band_keV": [E_MIN, E_MAX],
                   "parallelism": f"replicas x{world}", "schedule": tuned,
                   "l2": "flushed by a 256 MiB write before every step"},
        "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": int(28 * n),
                "d2h_bytes_per_step": int(4 * NX * NY)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "peak_kind": peak_kind, "kernel": "render_kernel",
                     "kernel_ms": last_stats["kernel_ms"], "algorithmic_bytes": kbytes},
        "cpu_baseline": {"value": cpu_v, "unit": "Mrays/s", "cores": cores, "kind": "port",
                         "sample": "per-cell X-ray flux + grid build over all 4,194,304 cells "
                                   "and 2048 random rays of the 1024^2 image, extrapolated"},
        "clocks": clk.summary(),
        "gpu_launches": launches,
        "render_stats": last_stats,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--image", type=int, default=1024,
                    help="image side in pixels (1024 = the benchmark; smaller only for profiling)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiling)")
    ap.add_argument("--z-window", type=float, default=None,
                    help="z window of the adaptive schedule in kpc (default: the tuned value)")
    ap.add_argument("--z-start", type=float, default=0.0,
                    help="camera plane position along z (profiling cases only)")
    ap.add_argument("--z-range", type=float, default=None,
                    help="integration depth in kpc (default: the 6 Mpc box; profiling only)")
    args = ap.parse_args()
    global NX, NY, Z_START, DEPTH
    NX = NY = args.image
    Z_START = args.z_start
    DEPTH = BOX if args.z_range is None else args.z_range
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    from illcrawl_b200 import build
    build.build()
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
