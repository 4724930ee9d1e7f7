"""GPU cell ingestion (ilc_ingest_cells) against the oracle: periodic
correction, cutout and compaction bit-exact in content and order, on a
periodic box with a cutout that straddles the period, and the kept cells
building the same grid as the oracle's."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cells(seed, n, box):
    rng = np.random.default_rng(seed)
    xyz = (rng.random((n, 3)) * box).astype(np.float32)
    q = rng.lognormal(0.0, 1.0, n).astype(np.float32)
    return xyz, q


@pytest.mark.parametrize("n", [1, 300, 257 * 255, 2_000_003])
def test_ingest_bit_exact(ctx, oracle_mod, n):
    box = 75000.0
    xyz, q = _cells(n, n, box)
    # a cutout across the periodic boundary, plus cells exactly on its faces
    center, extent, period = (74000.0, 500.0, 37000.0), (9000.0, 9000.0, 60000.0), (box,) * 3
    if n >= 8:
        xyz[:4] = [[69500.0, 500.0, 37000.0], [78500.0 - box, 500.0, 37000.0],
                   [74000.0, -4000.0, 37000.0], [74000.0, 5000.0 + 1e-3, 37000.0]]
    out, idx = ctx.ingest_cells(xyz, q, center, extent, period, border=100.0)
    oout, oidx = oracle_mod.ingest_cells(xyz, q, center, extent, period, border=100.0)
    assert np.array_equal(idx, oidx)
    assert np.array_equal(out.view(np.uint32), oout.view(np.uint32))


def test_ingest_feeds_the_grid(ctx, oracle_mod):
    box = 10000.0
    xyz, q = _cells(7, 400_000, box)
    args = ((9500.0, 9500.0, 5000.0), (3000.0, 3000.0, 8000.0), (box,) * 3)
    out, idx = ctx.ingest_cells(xyz, q, *args)
    oout, _ = oracle_mod.ingest_cells(xyz, q, *args)
    assert len(out) > 1000
    ctx.setup_particles(out)
    cells, s2u, srt = ctx.grid_export()
    ocells, os2u, osrt, _ = oracle_mod.Grid(oout).export()
    assert np.array_equal(cells, ocells) and np.array_equal(s2u, os2u)
    assert np.array_equal(srt.view(np.uint32), osrt.view(np.uint32))


def test_ingest_without_values_and_empty_result(ctx, oracle_mod):
    xyz, _ = _cells(3, 1000, 100.0)
    out, idx = ctx.ingest_cells(xyz, None, (5000.0, 0, 0), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    assert len(out) == 0
    out, idx = ctx.ingest_cells(xyz, None, (50.0, 50.0, 50.0), (40.0, 40.0, 40.0), (0.0, 0.0, 0.0))
    oout, oidx = oracle_mod.ingest_cells(xyz, None, (50.0, 50.0, 50.0), (40.0, 40.0, 40.0),
                                         (0.0, 0.0, 0.0))
    assert np.array_equal(idx, oidx) and np.all(out[:, 3] == 0.0)
