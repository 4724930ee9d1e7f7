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
REF_SAMPLE = 256    # oracle rays per reference-arm step


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
    """Schedule of the render kernel (orders work only, never changes a
    result). Persistent engine: tile shape, blocks per SM and z window from
    the cache for this GPU and workload, else defaults; --autotune re-runs the
    autotuner on the same camera at half resolution (8,192 tiles) and caches
    the winner. Grid engine: z window and occupancy, likewise."""
    import illcrawl_b200 as ilc
    cache = json.load(open(TUNING_FILE)) if os.path.exists(TUNING_FILE) else {}
    base = f"{gpu_name}|xray_band_map_4M_cells_{NX}sq_rtol1e-3|z0={Z_START}|depth={DEPTH}"
    if args.engine == "grid":
        ctx.set_render_engine(ilc.ENGINE_GRID)
        if args.z_window is not None:
            ctx.set_z_window(args.z_window)
            return {"engine": "grid", "z_window": args.z_window, "source": "command line"}
        key = base
        if key in cache and not args.autotune:
            ctx.set_z_window(cache[key]["z_window"])
            ctx.set_render_occupancy(cache[key]["occupancy"])
            return dict(cache[key], engine="grid", source="cache")
        bw, bo, times = ctx.autotune_render(cam, DEPTH, REL_TOL, 0.0, ilc.CONTROLLER_FP64,
                                            sample_stride=max(1, NY // 64))
        cache[key] = {"z_window": bw, "occupancy": bo,
                      "kernel_ms": {f"w{w}_o{o}": t for (w, o), t in times.items()}}
        src = "autotuner"
    else:
        ctx.set_render_engine(ilc.ENGINE_PERSISTENT)
        key = base + "|persistent"
        if args.z_window is not None or args.tile_w is not None or args.occupancy is not None:
            tw = 4 if args.tile_w is None else args.tile_w
            zw = 80.0 if args.z_window is None else args.z_window
            oc = 4 if args.occupancy is None else args.occupancy
            ctx.set_batch_schedule(tw, oc, zw, True)
            return {"engine": "persistent", "tile_w": tw, "occupancy": oc,
                    "z_window": zw, "source": "command line"}
        if key in cache and not args.autotune:
            e = cache[key]
            ctx.set_batch_schedule(e["tile_w"], e["occupancy"], e["z_window"], True)
            return dict(e, engine="persistent", source="cache")
        if not args.autotune:
            ctx.set_batch_schedule(8, 4, 40.0, True)
            return {"engine": "persistent", "tile_w": 8, "occupancy": 4, "z_window": 40.0,
                    "source": "default"}
        half = ilc.camera(*camera_args()[:4], NX // 2, NY // 2)
        q = ctx.tuning_values
        bt, bo, bw, times = ctx.autotune_batched(q, [ilc.job(half, z_range=DEPTH)], REL_TOL, 0.0,
                                                 tile_ws=(0, 4, 8), occupancies=(4, 5),
                                                 windows=(20.0, 80.0))
        cache[key] = {"tile_w": bt, "occupancy": bo, "z_window": bw,
                      "kernel_ms": {f"t{t}_o{o}_w{w}": v for (t, o, w), v in times.items()}}
        src = "autotuner"
    try:
        json.dump(cache, open(TUNING_FILE, "w"), indent=1, sort_keys=True)
    except OSError:
        pass
    return dict(cache[key], engine=args.engine, source=src)


def measured_traffic(args):
    """DRAM bytes (read + write) of one render launch of this workload, from
    the committed ncu capture of the same bench command (profiles/); None for
    other workloads or engines."""
    p = os.path.join(ROOT, "profiles", "batched_kernel_xray_band_map_1024sq_traffic.json")
    if args.engine != "persistent" or NX != 1024 or Z_START != 0.0 or DEPTH != BOX:
        return None
    try:
        return int(json.load(open(p))["dram_bytes_per_launch"])
    except (OSError, ValueError, KeyError):
        return None


def max_over_ranks(value, device):
    """The slowest rank's time (every rank takes this collective in the same
    order). Replicas share nothing else: no data-path collective."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, seconds_per_rank, device):
    """Whole-job throughput of N replicas: all ranks' units / the slowest
    rank's time."""
    import torch.distributed as dist
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    return units_per_rank * world / max_over_ranks(seconds_per_rank, device)


def make_inputs():
    from illcrawl_b200 import synthetic
    cells = synthetic.xray_cells()
    xyz4 = cells.xyzq(np.zeros(cells.n, np.float32))
    return cells, xyz4


def camera_args():
    return ((BOX / 2, BOX / 2, Z_START), (0.0, 0.0, 1.0), 0.0, BOX * NX / 1024, NX, NY)


def workload_config(world):
    """The config object both arms print (same keys, same values)."""
    return {"workload": f"xray_band_map_4M_cells_{NX}sq_rtol1e-3", "cells": 4194304,
            "image": [NX, NY], "z_range_kpc": DEPTH, "camera_z": Z_START, "rel_tol": REL_TOL,
            "controller": "fp64", "band_keV": [E_MIN, E_MAX],
            "parallelism": f"replicas x{world}",
            "l2": "flushed by a 256 MiB write before every step"}


SAMPLE_SEED = 20171


def sample_pixels(n=256, seed=SAMPLE_SEED):
    """The accuracy sample: the same 256 seeded rays as baseline/bytes_cfg1.json."""
    return np.sort(np.random.default_rng(seed).choice(NX * NY, n, replace=False))


def rel_stats(a, ref):
    ref = np.asarray(ref, np.float64)
    r = np.abs(np.asarray(a, np.float64) - ref) / np.abs(ref)
    return {"median": float(np.median(r)), "p90": float(np.quantile(r, 0.9)),
            "p99": float(np.quantile(r, 0.99)), "max": float(r.max())}


def algorithmic_bytes(st, n_cells, n_rays):
    # cell range + float4 per candidate, RKF state per step, output per ray,
    # per-cell value once + Gaunt table.
    return (8 * st["cells_visited"] + 16 * st["candidates"] + 24 * st["steps"] + 4 * n_rays
            + 16 * n_cells + 47304)


def oracle_setup(cells, nthreads):
    """The oracle's per-cell band flux and grid over all cells (timed)."""
    import oracle
    import illcrawl_b200 as ilc
    table = ilc.load_gaunt_table()
    t0 = time.perf_counter()
    q = oracle.xray_band(table, cells.rho, cells.u, cells.xe, REDSHIFT, DL, E_MIN, E_MAX,
                         NUM_SAMPLES, nthreads=nthreads)
    g = oracle.Grid(cells.xyzq(q))
    return g, time.perf_counter() - t0


def oracle_render_rate(g, nthreads, sample_rays, seed):
    """The oracle renders sample_rays random rays of the map; returns seconds."""
    import oracle
    pix = np.random.default_rng(seed).choice(NX * NY, sample_rays, replace=False)
    t0 = time.perf_counter()
    g.render(oracle.camera(*camera_args()), DEPTH, 0.0, REL_TOL, mode=1, pix=pix,
             nthreads=nthreads)
    return time.perf_counter() - t0


def cpu_baseline(cells, nthreads, sample_rays=2048, seed=1):
    """The oracle on the host cores: band flux + grid over all cells, then a
    render of sample_rays random rays. Returns (Mrays/s of the render, the
    grid/flux seconds, the render seconds, the oracle grid)."""
    g, t_fixed = oracle_setup(cells, nthreads)
    t_render = oracle_render_rate(g, nthreads, sample_rays, seed)
    return sample_rays / t_render / 1e6, t_fixed, t_render, g


def spectrum_jobs(ilc, div, seed=20172):
    """The batched uneven workload: 48 seeded cameras around the halo, sides
    drawn from {256, 512, 768, 1024} (divided by div for a bounded sample),
    circular apertures of radius U(0.5, 3) Mpc, every ray over its chord of
    the r = 3 Mpc sphere, widened to at least 0.6 Mpc (a 10x spread)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centre = np.full(3, BOX / 2)
    jobs = []
    for _ in range(48):
        v = rng.normal(size=3)
        look = v / np.linalg.norm(v)
        side = int(rng.choice([256, 512, 768, 1024])) // div
        cam = ilc.camera(tuple(centre - 3500.0 * look), tuple(look),
                         float(rng.uniform(0.0, 2.0 * np.pi)), BOX, side, side)
        jobs.append(ilc.job(cam, aperture_radius=float(rng.uniform(500.0, 3000.0)),
                            sphere_center=tuple(centre), sphere_radius=3000.0,
                            min_chord=600.0))
    return jobs


def spectral_table(ctx, d_rho, d_u, d_xe):
    """Cell-major table of 128 log-spaced bins over 0.3-10 keV
    (xray_spectral_flux per bin)."""
    edges = np.geomspace(0.3, 10.0, 129)
    e = edges[:-1].astype(np.float32)
    w = np.diff(edges).astype(np.float32)
    return ctx.xray_spectrum(d_rho, d_u, d_xe, e, w)


def rays_of(jobs):
    tot = 0
    for j in jobs:
        n = j.camera.num_pix_x
        c = (np.arange(n) + 0.5 - 0.5 * n) * (BOX / n)
        tot += int(np.sum(c[:, None] ** 2 + c[None, :] ** 2 <= j.aperture_radius ** 2))
    return tot


def timed_batched(ctx, torch, vals, jobs):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, st = ctx.render_batched(vals, jobs)
    torch.cuda.synchronize()
    return time.perf_counter() - t0, st


SPECTRAL_SUBSET = (0, 8, 16, 24)   # sides 512, 256, 512, 1024 at full size


def spectral_schedule(ctx, ilc, tab, gpu_name, args):
    """Schedule of the 128-channel batched kernel: from the cache for this GPU,
    else the autotuner on the full-size subset's cameras at a quarter of their
    sides (every candidate renders all 128 bins), cached."""
    cache = json.load(open(TUNING_FILE)) if os.path.exists(TUNING_FILE) else {}
    key = f"{gpu_name}|xray_spectrum_128bins_4M_cells|batched"
    if key in cache and not args.autotune:
        e = cache[key]
        ctx.set_batch_schedule(e["tile_w"], e["occupancy"], e["z_window"], True)
        return dict(e, source="cache")
    small = spectrum_jobs(ilc, 4)
    tune_jobs = [small[i] for i in SPECTRAL_SUBSET]
    bt, bo, bw, times = ctx.autotune_batched(tab, tune_jobs, REL_TOL, 0.0, tile_ws=(0, 4, 8),
                                             occupancies=(0, 4), windows=(40.0, 160.0))
    cache[key] = {"tile_w": bt, "occupancy": bo, "z_window": bw,
                  "kernel_ms": {f"t{t}_o{o}_w{w}": v for (t, o, w), v in times.items()}}
    try:
        json.dump(cache, open(TUNING_FILE, "w"), indent=1, sort_keys=True)
    except OSError:
        pass
    return dict(cache[key], source="autotuner")


def batched_leg(ctx, ilc, torch, d_rho, d_u, d_xe, args, band_schedule, gpu_name):
    """The batched uneven spectral workload (48 seeded cameras, sides from
    {256, 512, 768, 1024}, circular apertures of 0.5-3 Mpc, rays over their
    chord of the 3 Mpc sphere, 128 log-spaced bins over 0.3-10 keV).

    * all_48: every camera in one launch, sides divided by --batched-div (all
      48 cameras at full size are ~8 M rays x 128 bins, beyond a bench run);
    * full_size: cameras 0, 8, 16 and 24 at their full sides (256-1024^2):
      one batched launch for all 4 cameras x 128 bins against the plain path,
      one launch per (camera, bin) image as the reference renders a spectrum
      (spectrum.cpp:89-109), timed on --plain-bins bins per camera and scaled
      to 128 bins."""
    tab = spectral_table(ctx, d_rho, d_u, d_xe)
    sched = spectral_schedule(ctx, ilc, tab, gpu_name, args)
    ctx.render_batched(tab, [ilc.job(ilc.camera((0, 0, 0), (0, 0, 1), 0, 1, 1, 1),
                                     z_range=1.0)])  # allocation warm-up
    out = {"workload": "48 cameras, sides {256..1024}, apertures 0.5-3 Mpc, chords of the "
                       "3 Mpc sphere, 128 bins 0.3-10 keV, rtol 1e-3, FP64 controller",
           "bins": 128, "schedule": sched}
    if args.batched_div > 0:
        jobs = spectrum_jobs(ilc, args.batched_div)
        t_all, st_all = timed_batched(ctx, torch, tab, jobs)
        r_all = rays_of(jobs)
        out["all_48"] = {"sides": f"/{args.batched_div}", "rays": r_all, "seconds": t_all,
                         "kernel_s": st_all["kernel_ms"] * 1e-3,
                         "mrays_per_s": r_all / t_all / 1e6, "stats": st_all}
    full = spectrum_jobs(ilc, 1)
    sub = [full[i] for i in SPECTRAL_SUBSET]
    t_b, st_b = timed_batched(ctx, torch, tab, sub)
    # plain arm: the single-image kernel with the band map's schedule
    ctx.set_batch_schedule(band_schedule["tile_w"], band_schedule["occupancy"],
                           band_schedule["z_window"], True)
    nb = max(1, min(args.plain_bins, 128))
    bins = [int(round((k + 0.5) * 128 / nb)) for k in range(nb)]
    t_plain, k_plain, per = 0.0, 0.0, []
    for ci, j in enumerate(sub):
        for b in bins:
            vb = tab[:, b].contiguous()
            t, sj = timed_batched(ctx, torch, vb, [j])
            t_plain += t
            k_plain += sj["kernel_ms"] * 1e-3
            per.append({"camera": SPECTRAL_SUBSET[ci], "bin": b, "seconds": t})
    scale = 128.0 / nb
    r_sub = rays_of(sub)
    out["full_size"] = {
        "cameras": list(SPECTRAL_SUBSET),
        "sides": [j.camera.num_pix_x for j in sub], "rays": r_sub,
        "batched_s": t_b, "batched_kernel_s": st_b["kernel_ms"] * 1e-3,
        "batched_mrays_per_s": r_sub / t_b / 1e6,
        "batched_mray_bins_per_s": r_sub * 128 / t_b / 1e6, "batched_stats": st_b,
        "plain_bins_timed_per_camera": bins, "plain_launches_timed": len(per),
        "plain_s_128_bins": t_plain * scale, "plain_kernel_s_128_bins": k_plain * scale,
        "plain_launches": per,
        "batched_over_plain": t_plain * scale / t_b}
    return out


def accuracy_leg(img, g):
    """Error of the benchmark's map on the 256 sampled rays (outside the timed
    region): bit equality with the oracle (fp32, FP64 controller), relative
    error against the FP64 oracle at the same tolerance and against a
    converged FP64 render (rtol 1e-5), and the FP64 oracle's own error at the
    benchmark tolerance against the converged render."""
    import oracle
    ocam = oracle.camera(*camera_args())
    pix = sample_pixels()
    got = np.asarray(img, np.float32).ravel()[pix]
    out, *_ = g.render(ocam, DEPTH, 0.0, REL_TOL, mode=1, pix=pix)
    scale = np.float32(oracle.los_scale(ocam, DEPTH, 1.0, 1.0, 0))
    want = (out * scale).astype(np.float32)
    same = int(np.sum(got.view(np.uint32) == want.view(np.uint32)))
    raw = got.astype(np.float64) / float(scale)
    o64, *_ = g.render(ocam, DEPTH, 0.0, REL_TOL, mode=2, pix=pix)
    conv, *_ = g.render(ocam, DEPTH, 0.0, 1e-5, mode=2, pix=pix)
    return {"sample": f"256 seeded rays (numpy default_rng({SAMPLE_SEED}))",
            "bit_exact_vs_oracle": same, "rays": len(pix),
            "vs_fp64_oracle_same_tol": rel_stats(raw, o64),
            "vs_fp64_converged_rtol1e-5": rel_stats(raw, conv),
            "fp64_oracle_same_tol_vs_converged": rel_stats(o64, conv)}, conv


def tolerance_leg(step_at, conv):
    """The same map at tighter relative tolerances (outside the timed region):
    kernel time and the sampled pixels' error against the converged FP64
    render, i.e. what a per-pixel error bound of 1e-3 costs. step_at(rtol)
    renders the map and returns (device image, stats)."""
    import oracle
    ocam = oracle.camera(*camera_args())
    scale = float(np.float32(oracle.los_scale(ocam, DEPTH, 1.0, 1.0, 0)))
    out = {}
    for rtol in (5e-4, 2.5e-4):
        img, st = step_at(rtol)
        got = img.cpu().numpy().ravel()[sample_pixels()].astype(np.float64) / scale
        out[f"rtol{rtol:g}"] = {"kernel_ms": st["kernel_ms"], "steps": st["steps"],
                                "vs_fp64_converged_rtol1e-5": rel_stats(got, conv)}
    return out


def fixed_leg(ctx, ilc, torch, cam, flush, g):
    """The band map with a fixed 2048-step sequence (h = 6000/2048 kpc, every
    step accepted), device-timed, and its error on the sample against the
    FP64 replay of the same sequence."""
    import oracle
    for _ in range(2):
        flush.fill_(3.0)
        torch.cuda.synchronize()
        img, st = ctx.render_fixed(cam, DEPTH, 2048, device_output=True)
    got = img.cpu().numpy().ravel()[sample_pixels()]
    ocam = oracle.camera(*camera_args())
    o32, _ = g.render_fixed(ocam, DEPTH, 2048, precision=0, pix=sample_pixels())
    o64, _ = g.render_fixed(ocam, DEPTH, 2048, precision=1, pix=sample_pixels())
    return {"steps_per_ray": 2048, "kernel_ms": st["kernel_ms"],
            "mrays_per_s": NX * NY / (st["kernel_ms"] * 1e-3) / 1e6,
            "bit_exact_vs_oracle": int(np.sum(got.view(np.uint32) == o32.view(np.uint32))),
            "vs_fp64_replay": rel_stats(got, o64)}


def query_leg(ctx, ilc, torch):
    """The nn8 query workload of the projected-density cells (262,144 seeded
    cells, NFW r_s 300 kpc in a 3 Mpc cube, q = rho): 2^20 uniform random
    queries in the cube, device-resident, through ilc_nn8_query with the
    one-thread-per-query walk and with the warp-per-query walk (cells and
    candidates 32 at a time, hits by ballot). Device time of the query call
    (CUDA events on the library's stream), best of 5 after 2 warm-ups; the two
    engines' values compared bit for bit."""
    from illcrawl_b200 import synthetic
    dev = torch.device("cuda", torch.cuda.current_device())
    cells = synthetic.plain_density_cells()
    ctx.setup_particles(torch.from_numpy(cells.xyzq(cells.rho)).to(dev))
    rng = np.random.default_rng(20170)
    q = np.zeros((1 << 20, 4), np.float32)
    q[:, :3] = (rng.random((1 << 20, 3)) * cells.box).astype(np.float32)
    dq = torch.from_numpy(q).to(dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    out = {"workload": "2^20 uniform nn8 queries, 262,144 NFW cells in a 3 Mpc cube"}
    vals = {}
    for name, eng in (("thread", ilc.QUERY_THREAD), ("warp", ilc.QUERY_WARP)):
        ctx.set_query_engine(eng)
        times = []
        for i in range(7):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            v = ctx.nn8_query(dq)
            e1.record(stream)
            e1.synchronize()
            if i >= 2:
                times.append(e0.elapsed_time(e1))
        vals[name] = v.cpu().numpy()
        out[name] = {"ms": min(times), "mqueries_per_s": (1 << 20) / min(times) * 1e3 / 1e6}
    ctx.set_query_engine(ilc.QUERY_THREAD)
    out["bit_identical"] = bool(np.array_equal(vals["thread"].view(np.uint32),
                                               vals["warp"].view(np.uint32)))
    return out


def bytes_provenance(stats):
    """The oracle-counted bytes of the 256 sampled rays (baseline/bytes_cfg1.json,
    made by baseline/make_bytes.py; the GPU tests check the kernel's per-ray
    counters against it) beside the kernel's own count over the whole image."""
    p = os.path.join(ROOT, "baseline", "bytes_cfg1.json")
    if NX != 1024 or Z_START != 0.0 or DEPTH != BOX or not os.path.exists(p):
        return None
    d = json.load(open(p))
    gpu_per_ray = (8 * stats["cells_visited"] + 16 * stats["candidates"] + 24 * stats["steps"]
                   + 4 * NX * NY) / (NX * NY)
    return {"file": "baseline/bytes_cfg1.json", "oracle_rays": len(d["rays"]),
            "oracle_mean_bytes_per_ray": d["mean_bytes_per_ray"],
            "kernel_mean_bytes_per_ray_whole_image": gpu_per_ray}


def adjoint_leg(ctx, ilc, cells, args):
    """Adjoint cost on the 512^2 band map: loss sum (log I - log I_t)^2 with
    I_t rendered from the same cells with log T + a seeded Gaussian random
    field (sigma 0.1, correlation length 200 kpc); gradient with respect to
    per-cell log rho and log T. adjoint/forward = adjoint kernel time over the
    forward render time of the same call."""
    from illcrawl_b200 import synthetic
    side = 512
    cam = ilc.camera((BOX / 2, BOX / 2, Z_START), (0.0, 0.0, 1.0), 0.0, BOX, side, side)
    field = synthetic.gaussian_random_field_at(cells.pos, BOX, 0.1, 200.0, 256, 20174)
    u_t = synthetic.perturbed_internal_energy(cells, field)
    xyz4 = cells.xyzq(np.zeros(cells.n, np.float32))
    target, _ = ctx.project_xray_flux(xyz4, cells.rho, u_t, cells.xe, cam, DEPTH,
                                      rel_tol=REL_TOL, e_min=E_MIN, e_max=E_MAX,
                                      num_samples=NUM_SAMPLES)
    out = {"workload": "512^2 band map, 4,194,304 cells, target log T + GRF(0.1, 200 kpc)"}
    # the fastest forward of the same map: the persistent work-queue kernel
    _, fst = ctx.project_xray_flux(xyz4, cells.rho, cells.u, cells.xe, cam, DEPTH,
                                   rel_tol=REL_TOL, e_min=E_MIN, e_max=E_MAX,
                                   num_samples=NUM_SAMPLES)
    out["forward_persistent_ms"] = fst["kernel_ms"]
    for name, mode in (("checkpoint", ilc._lib.ADJOINT_CHECKPOINT),
                       ("recompute", ilc._lib.ADJOINT_RECOMPUTE)):
        _, _, _, st = ctx.adjoint_xray_flux(xyz4, cells.rho, cells.u, cells.xe, cam, DEPTH,
                                            target, mode=mode, rel_tol=REL_TOL,
                                            e_min=E_MIN, e_max=E_MAX, num_samples=NUM_SAMPLES)
        out[name] = {"forward_ms": st["forward_ms"], "adjoint_ms": st["adjoint_ms"],
                     "quantity_ms": st["quantity_ms"],
                     "adjoint_over_forward": st["adjoint_ms"] / st["forward_ms"],
                     "adjoint_over_persistent_forward": st["adjoint_ms"] / fst["kernel_ms"],
                     "loss": st["loss"]}
    return out


def run_reference(args, rank, world):
    """--impl reference: the oracle (CPU restatement of the reference path, the
    reference itself being OpenCL+Boost+MPI+HDF5 that cannot be built here) on
    all host cores, rank 0 only. The per-cell band flux and the grid are built
    once (timed, reported); every step then renders REF_SAMPLE random rays of
    the map, so steps and ms_per_step describe the work done, and value is
    the render rate (the grid and flux are ~0.1 % of a full image's oracle
    time, reported apart). The full-image time it implies is a separate field."""
    if rank != 0:
        return
    import oracle
    oracle.build()
    cores = os.cpu_count() or 1
    cells, _ = make_inputs()
    g, t_fixed = oracle_setup(cells, cores)
    times = []
    for i in range(args.warmup + args.steps):
        t = oracle_render_rate(g, cores, REF_SAMPLE, seed=100 + i)
        if i >= args.warmup:
            times.append(t)
    t_step = float(np.mean(times))
    v = REF_SAMPLE / t_step / 1e6
    full_s = t_fixed + t_step * (NX * NY) / REF_SAMPLE
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mrays/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded NFW + uniform gas cells, numpy PCG64 seed 20171)",
            "config": workload_config(world),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "port",
                             "sample": f"per step: the oracle renders {REF_SAMPLE} random rays "
                                       f"of the 1024^2 map (adaptive, FP64 controller) on "
                                       f"{cores} threads; the per-cell flux and the grid over "
                                       f"all 4,194,304 cells are built once before the steps"},
            "grid_and_flux_s": t_fixed,
            "full_image_estimate": {"seconds": full_s, "mrays_per_s": NX * NY / full_s / 1e6,
                                    "how": "grid and flux once + the mean step time x "
                                           f"{NX * NY // REF_SAMPLE} (not rendered)"},
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

    tuned = None
    ctx.set_render_engine(ilc.ENGINE_PERSISTENT if args.engine == "persistent"
                          else ilc.ENGINE_GRID)
    for i in range(max(args.warmup, 1)):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        step()
        if i == 0:  # the schedule only orders work: tuned after the first step
            if args.autotune and args.engine == "persistent":
                ctx.tuning_values = ctx.xray_flux(d_rho, d_u, d_xe, REDSHIFT, DL, E_MIN, E_MAX,
                                                  NUM_SAMPLES)
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
    total_ms = max_over_ranks(total_ms, dev)
    ms_per_step = total_ms / args.steps
    rays = NX * NY * world
    value = replica_value(NX * NY, ms_per_step * 1e-3, dev) / 1e6

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
        e2e_steps = 1
        e2e_s = 0.0
        for _ in range(e2e_steps):
            flush.fill_(2.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            e2e_s += time.perf_counter() - t0
        e2e_s /= e2e_steps
        e2e_value = replica_value(NX * NY, e2e_s, dev) / 1e6

    extra = {}
    gpu_name = torch.cuda.get_device_name(dev)
    cores = os.cpu_count() or 1
    g_oracle, cpu_v, cpu_info = None, None, None
    if world == 1 and not args.no_cpu:
        # the oracle's grid serves the CPU baseline and the accuracy checks
        cpu_v, t_fixed, t_render, g_oracle = cpu_baseline(cells, cores)
        cpu_info = {"grid_and_flux_s": t_fixed, "render_s": t_render}
    if g_oracle is not None and not args.no_accuracy:
        extra["accuracy"], conv = accuracy_leg(d_img.cpu().numpy(), g_oracle)
        extra["tighter_tolerance"] = tolerance_leg(
            lambda rt: ctx.project_xray_flux(d_cells, d_rho, d_u, d_xe, cam, DEPTH, rel_tol=rt,
                                             controller=ilc.CONTROLLER_FP64, e_min=E_MIN,
                                             e_max=E_MAX, num_samples=NUM_SAMPLES,
                                             scaling=scaling), conv)
        extra["fixed_2048"] = fixed_leg(ctx, ilc, torch, cam, flush, g_oracle)
    band_sched = tuned if tuned and "tile_w" in tuned else {"tile_w": 4, "occupancy": 4,
                                                             "z_window": 80.0}
    if world == 1 and not args.no_batched:
        extra["batched"] = batched_leg(ctx, ilc, torch, d_rho, d_u, d_xe, args, band_sched,
                                       gpu_name)
    if world == 1 and not args.no_adjoint:
        extra["adjoint"] = adjoint_leg(ctx, ilc, cells, args)
    if world == 1 and not args.no_queries:
        extra["nn8_queries"] = query_leg(ctx, ilc, torch)
    del g_oracle
    if rank != 0:
        ctx.close()
        return
    hbm, peak_kind = peaks()
    kbytes = algorithmic_bytes(last_stats, n, NX * NY)
    achieved = kbytes / (last_stats["kernel_ms"] * 1e-3) / 1e9
    traffic = measured_traffic(args)
    line = {
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded NFW + uniform gas cells, numpy PCG64 seed 20171)",
        "config": workload_config(world),
        "schedule": tuned,
        "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": int(28 * n),
                "d2h_bytes_per_step": int(4 * NX * NY)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "traffic_over_algorithmic": None if traffic is None else traffic / kbytes,
                     "peak_kind": peak_kind,
                     "kernel": "batched_kernel" if args.engine == "persistent" else "render_kernel",
                     "kernel_ms": last_stats["kernel_ms"], "algorithmic_bytes": kbytes,
                     "bytes_source": bytes_provenance(last_stats),
                     "note": "algorithmic bytes of the survey's byte model (every candidate of "
                             "every visited cell, per query); the kernel reads far fewer DRAM "
                             "bytes (traffic) because the grid stays in L2 and one load serves "
                             "4 points: the walk is latency-bound, not DRAM-bound"},
        "cpu_baseline": {"value": cpu_v, "unit": "Mrays/s", "cores": cores, "kind": "port",
                         "sample": "the oracle renders 2048 random rays of the 1024^2 map "
                                   "(adaptive, FP64 controller) after building the per-cell "
                                   "flux and the grid over all 4,194,304 cells",
                         "timings": cpu_info},
        "clocks": clk.summary(),
        "gpu_launches": launches,
        "render_stats": last_stats,
    }
    line.update(extra)
    print(json.dumps(line), flush=True)
    ctx.close()


def run_scale(args):
    """--config 4: the scale workload on one GPU. 67,108,864 seeded cells in an
    8 Mpc cube (two NFW halos, 3:1, 1.5 Mpc apart, 10 % background):

    * per-cell band flux + grid build, device-timed; the grid checked against
      the oracle's (cell ranges, sorted->original map and sorted particles, bit
      for bit);
    * the 2048^2 0.5-7 keV band map along z through the 8 Mpc box (adaptive,
      rtol 1e-3, FP64 controller), device-timed, with the clocks sampled;
    * its adjoint with per-ray step checkpoints, in bands of pixel rows that
      fit a 64 GiB checkpoint budget, against a target that is the map times
      a seeded per-pixel lognormal (sigma 0.1);
    * a 64-bin spectrum (log bins 0.3-10 keV) over a 512^2 aperture (4 Mpc
      camera, circular aperture of radius 2 Mpc through the whole box) in one
      batched launch."""
    import torch
    import oracle
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    box, side = 8000.0, 2048
    t0 = time.perf_counter()
    cells = synthetic.scale_cells()
    t_gen = time.perf_counter() - t0
    n = cells.n
    ctx = ilc.Context(0)
    ctx.load_gaunt()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    d_rho, d_u, d_xe = (torch.from_numpy(a).to(dev) for a in (cells.rho, cells.u, cells.xe))
    d_cells = torch.from_numpy(cells.xyzq(np.zeros(n, np.float32))).to(dev)
    out = {"workload": "scale: 67,108,864 cells, 8 Mpc cube, two NFW halos 3:1 + 10 % "
                       "background", "cells": n, "generate_s": t_gen}

    def dev_time(fn):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1)

    # per-cell flux + grid
    for _ in range(2):
        q, ms_q = dev_time(lambda: ctx.xray_flux(d_rho, d_u, d_xe, REDSHIFT, DL, E_MIN, E_MAX,
                                                 NUM_SAMPLES))
        xyzq = torch.cat([d_cells[:, :3], q[:, None]], dim=1).contiguous()
        _, ms_g = dev_time(lambda: ctx.setup_particles(xyzq))
    d = ctx.grid_describe()
    gc, gs2u, gsrt = ctx.grid_export()
    t0 = time.perf_counter()
    og = oracle.Grid(xyzq.cpu().numpy())
    oc, os2u, osrt, _ = og.export()
    grid_ok = (np.array_equal(d["min_corner"], og.min_corner) and
               np.array_equal(d["cell_sizes"], og.cell_sizes) and np.array_equal(gc, oc) and
               np.array_equal(gs2u, os2u) and
               np.array_equal(gsrt.view(np.uint32), osrt.view(np.uint32)))
    t_og = time.perf_counter() - t0
    del og, oc, os2u, osrt, gc, gs2u, gsrt
    out["flux_ms"], out["grid_ms"] = ms_q, ms_g
    out["grid"] = {"num_cells": [int(v) for v in d["num_cells"]],
                   "bit_exact_vs_oracle": bool(grid_ok), "oracle_build_s": t_og}
    # 2048^2 band map
    cam = ilc.camera((box / 2, box / 2, 0.0), (0.0, 0.0, 1.0), 0.0, box, side, side)
    d_img = torch.empty((side, side), dtype=torch.float32, device=dev)

    def band_map():
        return ctx.project_xray_flux(d_cells, d_rho, d_u, d_xe, cam, box, rel_tol=REL_TOL,
                                     controller=ilc.CONTROLLER_FP64, e_min=E_MIN, e_max=E_MAX,
                                     num_samples=NUM_SAMPLES, image=d_img)
    band_map()  # warm-up (allocations, graph)
    with ClockSampler(0) as clk:
        (_, st), ms = dev_time(band_map)
    out["band_map"] = {"image": [side, side], "z_range_kpc": box, "ms": ms,
                       "kernel_ms": st["kernel_ms"], "mrays_per_s": side * side / ms * 1e3 / 1e6,
                       "stats": st, "clocks": clk.summary()}
    # adjoint, step checkpoints in row bands
    img = d_img.cpu().numpy()
    rng = np.random.default_rng(20174)
    target = (img * np.exp(0.1 * rng.standard_normal(img.shape))).astype(np.float32)
    ctx.set_checkpoint_budget(64 << 30)
    xyz0 = cells.xyzq(np.zeros(n, np.float32))
    with ClockSampler(0) as clk:
        _, g_r, g_t, ast = ctx.adjoint_xray_flux(xyz0, cells.rho, cells.u, cells.xe, cam, box,
                                                 target, mode=ilc._lib.ADJOINT_CHECKPOINT,
                                                 rel_tol=REL_TOL, e_min=E_MIN, e_max=E_MAX,
                                                 num_samples=NUM_SAMPLES)
    cap = int(np.ceil(box / 0.2)) + 2
    rows = min(side, max(8, (64 << 30) // (side * cap * 4) // 8 * 8))
    out["adjoint"] = {"mode": "checkpoint", "checkpoint_budget_bytes": 64 << 30,
                      "band_rows": rows, "bands": -(-side // rows),
                      "forward_ms": ast["forward_ms"], "adjoint_ms": ast["adjoint_ms"],
                      "quantity_ms": ast["quantity_ms"],
                      "adjoint_over_forward": ast["adjoint_ms"] / ast["forward_ms"],
                      "loss": ast["loss"], "finite": bool(np.all(np.isfinite(g_r)) and
                                                          np.all(np.isfinite(g_t))),
                      "clocks": clk.summary()}
    del g_r, g_t
    # 64-bin spectrum over a 512^2 aperture
    edges = np.geomspace(0.3, 10.0, 65)
    e = edges[:-1].astype(np.float32)
    w = np.diff(edges).astype(np.float32)
    tab, ms_t = dev_time(lambda: ctx.xray_spectrum(d_rho, d_u, d_xe, e, w))
    ctx.setup_particles(xyzq)
    scam = ilc.camera((box / 2, box / 2, 0.0), (0.0, 0.0, 1.0), 0.0, 4000.0, 512, 512)
    job = [ilc.job(scam, z_range=box, aperture_radius=2000.0)]
    ctx.render_batched(tab, job)  # warm-up: channel table sort, graph
    (imgs, sst), ms_s = dev_time(lambda: ctx.render_batched(tab, job))
    c = (np.arange(512) + 0.5 - 256) * (4000.0 / 512)
    rays = int(np.sum(c[:, None] ** 2 + c[None, :] ** 2 <= 2000.0 ** 2))
    out["spectrum"] = {"bins": 64, "image": [512, 512], "aperture_kpc": 2000.0, "rays": rays,
                       "table_ms": ms_t, "ms": ms_s, "kernel_ms": sst["kernel_ms"],
                       "mrays_per_s": rays / ms_s * 1e3 / 1e6,
                       "mray_bins_per_s": rays * 64 / ms_s * 1e3 / 1e6, "stats": sst}
    line = {"config": 4, "impl": "ours", "n_gpus": 1, "dtype": "f32",
            "data": "synthetic (seeded, numpy PCG64 seed 20174)"}
    line.update(out)
    print(json.dumps(line), flush=True)
    ctx.close()


def run_spectrum_probe(args):
    """--spectrum-probe: one small 128-channel batched render (camera 16 of the
    spectral workload, a 512^2 view with a 1.2 Mpc aperture, at half its side:
    8,328 rays), three launches, for profiling the multi-channel kernel."""
    import torch
    import illcrawl_b200 as ilc
    cells, xyz4 = make_inputs()
    ctx = ilc.Context(0)
    ctx.load_gaunt()
    dev = torch.device("cuda", 0)
    d_rho, d_u, d_xe = (torch.from_numpy(a).to(dev) for a in (cells.rho, cells.u, cells.xe))
    q = ctx.xray_flux(d_rho, d_u, d_xe, REDSHIFT, DL, E_MIN, E_MAX, NUM_SAMPLES)
    d_cells = torch.from_numpy(xyz4).to(dev)
    ctx.setup_particles(torch.cat([d_cells[:, :3], q[:, None]], dim=1).contiguous())
    tab = spectral_table(ctx, d_rho, d_u, d_xe)
    spectral_schedule(ctx, ilc, tab, torch.cuda.get_device_name(dev), args)
    job = [spectrum_jobs(ilc, 2)[16]]
    out = []
    for _ in range(3):
        _, st = ctx.render_batched(tab, job)
        out.append(st["kernel_ms"])
    print(json.dumps({"spectrum_probe": {"rays": rays_of(job), "bins": 128,
                                         "kernel_ms": out, "stats": st}}), flush=True)
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
    ap.add_argument("--occupancy", type=int, default=None, choices=[0, 3, 4, 5],
                    help="blocks per SM of the persistent schedule (default: the tuned value)")
    ap.add_argument("--tile-w", type=int, default=None,
                    help="work-item width of the persistent schedule (default: the tuned value)")
    ap.add_argument("--engine", default="persistent", choices=["persistent", "grid"],
                    help="render kernel: persistent work queue (default) or one block per tile")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-vs-plain spectral leg")
    ap.add_argument("--batched-div", type=int, default=8,
                    help="the all-48-camera batched run uses sides divided by this "
                         "(0: skip it); the batched-vs-plain comparison is at full size")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the accuracy and fixed-step legs (they need the CPU oracle)")
    ap.add_argument("--plain-bins", type=int, default=2,
                    help="bins timed per camera in the plain per-(camera, bin) arm of the "
                         "full-size spectral comparison, scaled to 128")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint-cost leg")
    ap.add_argument("--no-queries", action="store_true",
                    help="skip the 2^20-query nn8 leg (thread vs warp engine)")
    ap.add_argument("--autotune", action="store_true",
                    help="re-run the schedule autotuner and update the cache")
    ap.add_argument("--z-start", type=float, default=0.0,
                    help="camera plane position along z (profiling cases only)")
    ap.add_argument("--z-range", type=float, default=None,
                    help="integration depth in kpc (default: the 6 Mpc box; profiling only)")
    ap.add_argument("--spectrum-probe", action="store_true",
                    help="profiling only: three small 128-channel batched launches")
    ap.add_argument("--config", type=int, default=1, choices=[1, 4],
                    help="1: the band-map benchmark (default); 4: the 67 M-cell scale "
                         "workload, one GPU, one pass of each of its parts")
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
    if args.spectrum_probe:
        run_spectrum_probe(args)
        return
    if args.config == 4:
        if world > 1:
            raise SystemExit("--config 4 runs on one GPU")
        run_scale(args)
        return
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
