"""Counts the algorithmic bytes of the X-ray band-map workload on the oracle.

The workload: 4,194,304 seeded gas cells (illcrawl_b200.synthetic.xray_cells),
0.5-7 keV band flux, 1024^2 pixels along z through the 6 Mpc box, adaptive
RKF4(5) at relative tolerance 1e-3 with the FP64 step controller. For 256
seeded pixels the oracle's search counters give, per ray, the RKF steps, the
grid cells visited and the candidate particles tested, summed over the 4
integrand points of every step (volumetric_nn8_reconstruction.cl:157-203
visits a cell and tests every particle in it). Per ray:

    bytes = 8 * cells + 16 * candidates + 24 * steps + 4

(an int2 cell range per visited cell, a float4 per candidate, the ray state
per step, the output pixel); per image add 16 * N + 47,304 (each cell's value
once, the Gaunt table). Writes baseline/bytes_cfg1.json; the GPU kernel's own
counters for the same rays are checked against it by the GPU tests.

    python baseline/make_bytes.py
"""
import concurrent.futures
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

SIDE, BOX, REL_TOL = 1024, 6000.0, 1e-3
SAMPLE, SAMPLE_SEED = 256, 20171


def sample_pixels():
    return np.sort(np.random.default_rng(SAMPLE_SEED).choice(SIDE * SIDE, SAMPLE, replace=False))


def ray_bytes(cells, cands, steps):
    return 8 * cells + 16 * cands + 24 * steps + 4


def main():
    import oracle
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    oracle.build()
    c = synthetic.xray_cells()
    q = oracle.xray_band(ilc.load_gaunt_table(), c.rho, c.u, c.xe, 0.2, 978500.0, 0.5, 7.0, 100)
    g = oracle.Grid(c.xyzq(q))
    cam = oracle.camera((BOX / 2, BOX / 2, 0.0), (0.0, 0.0, 1.0), 0.0, BOX, SIDE, SIDE)
    pix = sample_pixels()

    def one(p):
        _, steps, acc, st, rc = g.render(cam, BOX, 0.0, REL_TOL, mode=1, pix=np.array([p]),
                                         nthreads=1)
        assert rc == 0
        return int(steps[0]), int(acc[0]), int(st[0]), int(st[1])

    with concurrent.futures.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        rows = list(ex.map(one, pix))
    rays = []
    for p, (steps, acc, cells, cands) in zip(pix, rows):
        rays.append({"pixel": int(p), "steps": steps, "accepted": acc, "cells_visited": cells,
                     "candidates": cands, "bytes": ray_bytes(cells, cands, steps)})
    per_ray = float(np.mean([r["bytes"] for r in rays]))
    out = {"workload": "xray_band_map_4M_cells_1024sq_rtol1e-3",
           "cells": int(c.n), "image": [SIDE, SIDE], "rel_tol": REL_TOL, "controller": "fp64",
           "formula": "per ray 8*cells_visited + 16*candidates + 24*steps + 4; "
                      "per image + 16*cells + 47304",
           "sample": {"pixels": SAMPLE, "seed": SAMPLE_SEED,
                      "rule": "numpy default_rng(seed).choice(1024*1024, 256, replace=False), sorted"},
           "per_image_bytes": 16 * int(c.n) + 47304,
           "mean_bytes_per_ray": per_ray,
           "rays": rays}
    with open(os.path.join(HERE, "bytes_cfg1.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("mean bytes per ray %.4g over %d rays" % (per_ray, len(rays)))


if __name__ == "__main__":
    main()
