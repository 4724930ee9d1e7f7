"""Multi-process forms of the nn8 consumers, as the reference's distributed_*
classes run them over MPI: the work split by uniform_work_partitioner
(uniform_work_partitioner.cpp:33-64) over the ranks of a torch.distributed
process group (one process per GPU), and one reduce where the reference has
one (distributed_mc_radial_profile's shell sums, profile.cpp:310-318).

The band map and spectra have no exchange step: their ranks are independent
replicas (or take disjoint cameras with :func:`own_jobs`). Every function
takes the group's collectives in the same order on every rank.
"""
import numpy as np

from . import DV_VOLUME, mc_profile_points, mc_profile_shells


def uniform_work_partitioner(num_jobs, rank, world):
    """(own_begin, own_end) of uniform_work_partitioner::run (uniform_work_
    partitioner.cpp:33-64): rank p starts at floor(num_jobs / world * p) in
    double; the last rank ends at num_jobs."""
    if world < 1 or not 0 <= rank < world or num_jobs < 0:
        raise ValueError("rank must lie in [0, world) and num_jobs be >= 0")
    per = float(num_jobs) / float(world)
    begins, cur = [], 0
    for proc in range(world):
        begins.append(cur)
        cur = int(per * float(proc + 1))
    end = num_jobs if rank == world - 1 else begins[rank + 1]
    return begins[rank], end


def _rank_world(group):
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def own_jobs(jobs, group=None):
    """This rank's share of a list of frames / cameras (distributed_animation,
    animation.cpp:85-100), for one ilc_render_batched call per rank."""
    rank, world = _rank_world(group)
    b, e = uniform_work_partitioner(len(jobs), rank, world)
    return list(jobs[b:e]), (b, e)


def distributed_volumetric_tomography(ctx, cam, dV, z_range, group=None):
    """distributed_volumetric_tomography::create_tomographic_cube
    (volumetric_tomography.cpp:116-137): z_range / pixel size slices (at
    least one), this rank's share of them. Returns (local cube, (begin, end))."""
    rank, world = _rank_world(group)
    total = int(z_range / (cam.screen_width / cam.num_pix_x))
    if total == 0:
        total = 1
    b, e = uniform_work_partitioner(total, rank, world)
    return ctx.volumetric_tomography(cam, dV, b, e - b), (b, e)


def _shell_volumes(max_radius, num_radii):
    """Shell volumes of profile.cpp:320-355, in the same double arithmetic."""
    r = lambda i: i * (max_radius / num_radii)
    out = np.zeros(num_radii)
    for i in range(num_radii):
        a = 0.0 if i == 0 else 0.5 * (r(i - 1) + r(i))
        b = 0.5 * (r(i + 1) + r(i))
        out[i] = 4. / 3 * np.pi * (b * b * b - a * a * a)
    return out


def distributed_mc_radial_profile(ctx, center, max_radius, num_radii, sample_density, seed=0,
                                  dV_mode=DV_VOLUME, volume_conversion=1.0, root=0, group=None,
                                  evaluate=None, batch=1 << 22):
    """distributed_mc_radial_profile::operator() (profile.cpp:47-74, 130-234):
    this rank's share of the global sample sequence (uniform_work_partitioner
    over all samples), the nn8 value at each (``evaluate(points)``; default
    the particles of ``ctx``), per-shell sums in double, one reduce (sum) to
    ``root`` and the volume factor there (apply_volume_factor, profile.cpp:
    236-256). Returns the profile on root and None on the other ranks."""
    import torch
    import torch.distributed as dist
    rank, world = _rank_world(group)
    if evaluate is None:
        evaluate = lambda pts: ctx.nn8_query(pts)
    _, counts = mc_profile_shells(max_radius, num_radii, sample_density)
    prefix = np.concatenate([[0], np.cumsum(counts.astype(np.int64))])
    b, e = uniform_work_partitioner(int(prefix[-1]), rank, world)
    sums = np.zeros(num_radii, np.float64)
    for g0 in range(b, e, batch):
        n = min(batch, e - g0)
        pts = mc_profile_points(center, max_radius, num_radii, sample_density, seed, g0, n)
        vals = np.asarray(evaluate(pts), np.float32)
        shells = np.searchsorted(prefix, g0 + np.arange(n), side="right") - 1
        np.add.at(sums, shells, vals.astype(np.float64))
    if world > 1:
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.tensor(sums, dtype=torch.float64, device=dev)
        dist.reduce(t, dst=root, op=dist.ReduceOp.SUM, group=group)
        sums = t.cpu().numpy()
    if rank != root:
        return None
    vol = _shell_volumes(max_radius, num_radii)
    dv = vol / counts.astype(np.float64)
    conv = float(volume_conversion)
    eff = dv * conv if dV_mode == DV_VOLUME else (dv * conv) / (vol * conv)
    return sums * eff
