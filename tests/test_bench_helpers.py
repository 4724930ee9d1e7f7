"""Host-side helpers of bench.py (CPU): the uneven spectral workload is
seeded and bounded, and the recorded DRAM traffic is used only for the
workload it was measured on."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_spectrum_jobs_are_seeded_and_bounded():
    sys.path.insert(0, ROOT)
    import bench
    import illcrawl_b200 as ilc
    a = bench.spectrum_jobs(ilc, 8)
    b = bench.spectrum_jobs(ilc, 8)
    assert len(a) == 48
    for x, y in zip(a, b):
        assert tuple(x.camera.look_at) == tuple(y.camera.look_at)
        assert x.camera.num_pix_x in (32, 64, 96, 128)
        assert 500.0 <= x.aperture_radius <= 3000.0
        assert x.sphere_radius == 3000.0 and x.min_chord == 600.0


def test_measured_traffic_only_for_its_workload():
    sys.path.insert(0, ROOT)
    import argparse
    import bench
    args = argparse.Namespace(engine="persistent")
    bench.NX, bench.Z_START, bench.DEPTH = 1024, 0.0, bench.BOX
    assert bench.measured_traffic(args) > 0
    bench.NX = 256
    assert bench.measured_traffic(args) is None
    bench.NX = 1024
    assert bench.measured_traffic(argparse.Namespace(engine="grid")) is None
