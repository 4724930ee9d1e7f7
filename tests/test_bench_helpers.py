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


def test_both_arms_print_the_same_config():
    sys.path.insert(0, ROOT)
    import bench
    bench.NX = bench.NY = 1024
    bench.Z_START, bench.DEPTH = 0.0, bench.BOX
    a, b = bench.workload_config(1), bench.workload_config(1)
    assert a == b and a["cells"] == 4194304 and a["image"] == [1024, 1024]
    assert a["rel_tol"] == 1e-3 and a["controller"] == "fp64"


def test_accuracy_sample_is_the_bytes_file_sample():
    sys.path.insert(0, ROOT)
    import json
    import numpy as np
    import bench
    bench.NX = bench.NY = 1024
    d = json.load(open(os.path.join(ROOT, "baseline", "bytes_cfg1.json")))
    assert np.array_equal(bench.sample_pixels(), [r["pixel"] for r in d["rays"]])
    for r in d["rays"]:
        assert r["bytes"] == 8 * r["cells_visited"] + 16 * r["candidates"] + 24 * r["steps"] + 4
    assert abs(d["mean_bytes_per_ray"] - np.mean([r["bytes"] for r in d["rays"]])) < 1e-6


def test_reference_arm_reports_the_work_it_did(capsys):
    """Every step renders REF_SAMPLE rays on the oracle; ms_per_step is that
    step's time and value the rate of those rays."""
    sys.path.insert(0, ROOT)
    import argparse
    import json
    import bench
    bench.NX = bench.NY = 1024
    bench.Z_START, bench.DEPTH = 0.0, bench.BOX
    old = bench.REF_SAMPLE
    bench.REF_SAMPLE = 8
    try:
        bench.run_reference(argparse.Namespace(steps=2, warmup=0), 0, 1)
    finally:
        bench.REF_SAMPLE = old
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["steps"] == 2
    assert abs(line["value"] - 8 / (line["ms_per_step"] * 1e-3) / 1e6) < 1e-12
    assert line["config"] == bench.workload_config(1)
    assert line["full_image_estimate"]["seconds"] > line["ms_per_step"] * 1e-3
