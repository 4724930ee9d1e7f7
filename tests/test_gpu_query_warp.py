"""The warp-cooperative nn8 query (ILC_QUERY_WARP: one warp per query, cells
and candidates 32 at a time, hits inserted in candidate order) against the
oracle and against the one-thread walk: neighbour indices, distances, values
and the search counters bit for bit, on the 2^20-query density workload, on
edge queries (outside the grid, on particles, NaN) and through the block
merge of the reference's blocksize < N mode."""
import time

import numpy as np
import pytest

from conftest import random_queries
from test_gpu_parity import same_bits

pytestmark = pytest.mark.gpu


@pytest.fixture
def warp_engine(ctx):
    import illcrawl_b200 as ilc
    ctx.set_query_engine(ilc.QUERY_WARP)
    yield ctx
    ctx.set_query_engine(ilc.QUERY_THREAD)


def _timed_query(ctx, q):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = ctx.nn8_query(q, slots=True)
    torch.cuda.synchronize()
    return r, time.perf_counter() - t0


def test_warp_query_density_workload_bit_exact(ctx, oracle_mod):
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    c = synthetic.plain_density_cells()
    pts = c.xyzq(c.rho)
    ctx.setup_particles(pts)
    q = random_queries(1 << 20, 0.0, c.box, seed=515151)
    import torch
    dq = torch.from_numpy(q).cuda()
    ctx.set_query_engine(ilc.QUERY_THREAD)
    (tv, ti, td), _ = _timed_query(ctx, dq)
    tt = min(_timed_query(ctx, dq)[1] for _ in range(3))
    ctx.set_query_engine(ilc.QUERY_WARP)
    try:
        (wv, wi, wd), _ = _timed_query(ctx, dq)
        tw = min(_timed_query(ctx, dq)[1] for _ in range(3))
    finally:
        ctx.set_query_engine(ilc.QUERY_THREAD)
    print("2^20 queries: thread walk %.3f ms, warp walk %.3f ms" % (tt * 1e3, tw * 1e3))
    g = oracle_mod.Grid(pts)
    oval, oidx, od8, ost = g.nn8(q)
    for v, i, d in ((tv, ti, td), (wv, wi, wd)):
        v, i, d = (a.cpu().numpy() if hasattr(a, "cpu") else a for a in (v, i, d))
        assert np.array_equal(i, oidx)
        assert same_bits(d, od8)
        assert same_bits(v, oval)


def test_warp_query_counters_equal_thread_walk(ctx, oracle_mod):
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(60_000, seed=17)
    pts = c.xyzq(c.rho)
    ctx.setup_particles(pts)
    q = random_queries(50_000, -100.0, 1100.0, seed=3)
    st = []
    for eng in (ilc.QUERY_THREAD, ilc.QUERY_WARP):
        ctx.set_query_engine(eng)
        ctx.nn8_query(q, slots=True)
        st.append(ctx.last_query_stats())
    ctx.set_query_engine(ilc.QUERY_THREAD)
    _, _, _, ost = oracle_mod.Grid(pts).nn8(q)
    assert st[0] == st[1] == (int(ost[0]), int(ost[1]))


def test_warp_query_edge_queries(warp_engine, oracle_mod):
    from illcrawl_b200 import synthetic
    ctx = warp_engine
    c = synthetic.small_cells(20_000, seed=5)
    pts = c.xyzq(c.rho)
    ctx.setup_particles(pts)
    g = oracle_mod.Grid(pts)
    q = random_queries(4096, -3000.0, 4000.0, seed=1)
    q[:8, :3] = pts[:8, :3]
    q[8, :3] = np.nan
    q[9, :3] = [1e30, -1e30, 0]
    val, idx, d8 = ctx.nn8_query(q, slots=True)
    oval, oidx, od8, _ = g.nn8(q)
    assert np.array_equal(idx, oidx)
    assert same_bits(d8, od8)
    assert same_bits(val, oval)


def test_warp_query_dense_and_tiny_grids(warp_engine, oracle_mod):
    """Cells with hundreds of particles (candidate rounds spanning cells) and
    grids of fewer than 8 particles (empty slots)."""
    ctx = warp_engine
    rng = np.random.default_rng(9)
    dense = np.repeat(rng.random((40, 4)).astype(np.float32) * 10, 60, axis=0)
    dense[:, :3] += rng.normal(0, 0.01, (dense.shape[0], 3)).astype(np.float32)
    for p in (dense, rng.random((5, 4)).astype(np.float32)):
        ctx.setup_particles(p)
        q = random_queries(3000, -1.0, 11.0, seed=4)
        val, idx, d8 = ctx.nn8_query(q, slots=True)
        oval, oidx, od8, _ = oracle_mod.Grid(p).nn8(q)
        assert np.array_equal(idx, oidx)
        assert same_bits(d8, od8)
        assert same_bits(val, oval)


def test_warp_query_merge_two_blocks(warp_engine, oracle_mod):
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    ctx = warp_engine
    c = synthetic.small_cells(30_000, seed=8)
    pts = c.xyzq(c.rho)
    q = random_queries(2000, 200.0, 800.0, seed=2)
    be = ilc.Nn8Backend(ctx)
    be.setup_evaluation_points(q)
    be.setup_particles(pts[:15_000])
    be.run()
    first = be.retrieve_results().copy()
    be.setup_particles(pts[15_000:])
    be.run()
    merged = be.retrieve_results()
    o1, lists = oracle_mod.nn8_lists(oracle_mod.Grid(pts[:15_000]), q)
    o2, lists = oracle_mod.nn8_lists(oracle_mod.Grid(pts[15_000:]), q, merge=True, lists=lists)
    assert same_bits(first, o1)
    assert same_bits(merged, o2)
