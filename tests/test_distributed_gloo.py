"""The multi-process consumers (illcrawl_b200.distributed) with world size 2
over gloo on the CPU: the reference's uniform_work_partitioner split, a
distributed Monte-Carlo profile whose reduced shell sums equal the
single-process oracle profile, and the tomography / frame splits tiling
their ranges."""
import os
import sys

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _partition_ref(n, rank, world):
    per = n / world
    begins = [0] + [int(per * (p + 1)) for p in range(world - 1)]
    return begins[rank], (n if rank == world - 1 else begins[rank + 1])


@pytest.mark.parametrize("n", [0, 1, 7, 100, 1001, 4_832_035, 2 ** 40 + 3])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partitioner_tiles_the_jobs(n, world):
    sys.path.insert(0, ROOT)
    from illcrawl_b200.distributed import uniform_work_partitioner
    prev = 0
    for r in range(world):
        b, e = uniform_work_partitioner(n, r, world)
        assert (b, e) == _partition_ref(n, r, world)
        assert b == prev and e >= b
        prev = e
    assert prev == n


class _FakeTomography:
    """Stands in for a context: a cube of the asked-for slice count, filled
    with the index of its first slice."""

    def volumetric_tomography(self, cam, dV, initial_z_step, num_steps):
        return np.zeros((num_steps, cam.num_pix_y, cam.num_pix_x), np.float32) + initial_z_step


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import oracle
        import illcrawl_b200 as ilc
        from illcrawl_b200 import distributed, synthetic
        c = synthetic.small_cells(20_000, seed=71)
        g = oracle.Grid(c.xyzq(c.rho))
        ev = lambda pts: g.nn8(pts, slots=False)[0]
        center = (505.0, 495.0, 500.0)
        prof = distributed.distributed_mc_radial_profile(
            None, center, 450.0, 10, 3e-4, seed=13, dV_mode=ilc.DV_MEAN, root=1, evaluate=ev,
            batch=5000)
        cam = ilc.camera((500, 500, 0), (0, 0, 1), 0.0, 1000.0, 4, 3)
        cube, rng = distributed.distributed_volumetric_tomography(_FakeTomography(), cam, 1.0,
                                                                  1000.0)
        frames, frng = distributed.own_jobs(list(range(11)))
        q.put((rank, None if prof is None else prof.tolist(), rng, cube.shape[0],
               float(cube.min()) if cube.size else None, frng, frames))
    finally:
        dist.destroy_process_group()


def test_distributed_profile_and_splits(oracle_mod, cuda_lib):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 31500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
    assert all(p.exitcode == 0 for p in procs)
    res = dict((r[0], r[1:]) for r in (q.get(timeout=5) for _ in range(2)))
    # the profile arrives on root 1 only and equals the single-process oracle
    assert res[0][0] is None and res[1][0] is not None
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(20_000, seed=71)
    g = oracle_mod.Grid(c.xyzq(c.rho))
    want = oracle_mod.mc_radial_profile(g, (505.0, 495.0, 500.0), 450.0, 10, 3e-4, seed=13,
                                        dV_mode=1)
    assert np.allclose(np.array(res[1][0]), want, rtol=1e-12, atol=0.0)
    # tomography: 4 slices (z range 1000 / pixel size 250), rank 0 [0, 2), rank 1 [2, 4)
    assert res[0][1] == (0, 2) and res[1][1] == (2, 4)
    assert res[0][2] == 2 and res[1][2] == 2 and res[1][3] == 2.0
    # frames: 11 split 5 / 6
    assert res[0][4] == (0, 5) and res[1][4] == (5, 11)
    assert res[0][5] + res[1][5] == list(range(11))


def test_single_process_profile_needs_no_group(oracle_mod, cuda_lib):
    sys.path.insert(0, ROOT)
    from illcrawl_b200 import distributed, synthetic
    c = synthetic.small_cells(5_000, seed=72)
    g = oracle_mod.Grid(c.xyzq(c.rho))
    prof = distributed.distributed_mc_radial_profile(
        None, (500.0, 500.0, 500.0), 300.0, 6, 1e-4, seed=2, volume_conversion=2.0,
        evaluate=lambda p: g.nn8(p, slots=False)[0], batch=777)
    want = oracle_mod.mc_radial_profile(g, (500.0, 500.0, 500.0), 300.0, 6, 1e-4, seed=2,
                                        volume_conversion=2.0)
    assert np.allclose(prof, want, rtol=1e-12, atol=0.0)
