"""Multi-GPU is replicas only: every rank renders its own copy of the job and
the benchmark reduces only the timing (max over ranks). This checks that
reduction with world_size 2 over gloo on the CPU."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        secs = [2.0, 3.5][rank]                # rank 1 is the slowest replica
        slow = bench.max_over_ranks(secs, "cpu")
        val = bench.replica_value(1000, secs, "cpu")
        q.put((rank, slow, val))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, slow, val in res:
        assert slow == pytest.approx(3.5)
        assert val == pytest.approx(2 * 1000 / 3.5)


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(1.25, "cpu") == 1.25
    assert bench.replica_value(10, 2.0, "cpu") == 5.0
