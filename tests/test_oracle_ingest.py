"""Cell ingestion in the oracle (periodic correction + volume cutout + order-
preserving compaction of reconstructing_data_crawler::run), on hand-placed
cells."""
import numpy as np


def test_periodic_correction_and_cutout_by_hand(oracle_mod):
    center, extent, period = (100.0, 100.0, 100.0), (40.0, 40.0, 40.0), (1000.0, 1000.0, 1000.0)
    xyz = np.array([
        [100.0, 100.0, 100.0],     # centre: kept
        [1090.0, 100.0, 100.0],    # one period above: wraps to 90, kept
        [-910.0, 100.0, 100.0],    # one period below: wraps to 90, kept
        [80.0, 120.0, 100.0],      # exactly on the box faces: kept (<= and >=)
        [79.9, 100.0, 100.0],      # just outside: dropped
        [1170.0, 100.0, 100.0],    # wraps to 170: inside the 100 kpc border, outside the box
        [500.0, 100.0, 100.0],     # far: no wrap, dropped
        [100.0, 1110.0, 85.0],     # y wraps to 110: kept
    ], np.float32)
    q = np.arange(8, dtype=np.float32) + 0.5
    out, idx = oracle_mod.ingest_cells(xyz, q, center, extent, period, border=100.0)
    assert idx.tolist() == [0, 1, 2, 3, 7]
    assert np.allclose(out[:, :3], [[100, 100, 100], [90, 100, 100], [90, 100, 100],
                                    [80, 120, 100], [100, 110, 85]])
    assert np.array_equal(out[:, 3], q[idx])


def test_border_limits_the_wrap(oracle_mod):
    # a wrapped image outside the border-widened box is not taken
    xyz = np.array([[1300.0, 100.0, 100.0]], np.float32)
    out, idx = oracle_mod.ingest_cells(xyz, None, (100, 100, 100), (40, 40, 40), (1000, 1000, 1000),
                                       border=100.0)
    assert len(idx) == 0
    out, idx = oracle_mod.ingest_cells(xyz, None, (100, 100, 100), (40, 40, 40), (1000, 1000, 1000),
                                       border=300.0)
    assert len(idx) == 0   # wraps to 300, inside the widened box but outside the cutout
