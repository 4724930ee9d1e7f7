"""Parity at the benchmark's own workload: the 0.5-7 keV X-ray band map of the
4,194,304 seeded gas cells (synthetic.xray_cells), 1024^2 pixels along z
through the 6 Mpc box, adaptive RKF4(5) at relative tolerance 1e-3 with the
FP64 step controller, and the same map with a fixed 2048-step sequence.

* per-cell band flux and the particle grid (cell ranges, sorted particles,
  sorted->original map) bit-exact against the oracle at full size;
* the map through ilc_project_xray_flux (the benchmark's call): 256 seeded
  pixels bit-exact against the oracle, and their error against the FP64
  oracle at the same tolerance and against a converged FP64 render
  (rtol 1e-5);
* the same map at rtol 5e-4: the sampled pixels bit-exact against the oracle
  and every one within 1e-3 of the converged FP64 render;
* per-ray work counters (steps, cells visited, candidates tested) of the same
  256 rays equal the oracle's counts committed in baseline/bytes_cfg1.json,
  from which the benchmark's algorithmic bytes follow; the one-block-per-tile
  kernel's full image equals the persistent kernel's bit for bit;
* the fixed 2048-step map: the sampled pixels bit-exact against the oracle and
  within 1e-5 of the FP64 replay of the same sequence.
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT
from test_gpu_parity import same_bits

pytestmark = pytest.mark.gpu

SIDE, BOX, REL_TOL = 1024, 6000.0, 1e-3
Z, DL, EMIN, EMAX, NS = 0.2, 978500.0, 0.5, 7.0, 100
CAM = ((BOX / 2, BOX / 2, 0.0), (0.0, 0.0, 1.0), 0.0, BOX, SIDE, SIDE)


def sample_pixels():
    """The 256 rays of baseline/bytes_cfg1.json (the benchmark's accuracy sample)."""
    return np.sort(np.random.default_rng(20171).choice(SIDE * SIDE, 256, replace=False))


def rel_stats(a, ref):
    ref = np.asarray(ref, np.float64)
    r = np.abs(np.asarray(a, np.float64) - ref) / np.abs(ref)
    return {"median": float(np.median(r)), "p90": float(np.quantile(r, 0.9)),
            "p99": float(np.quantile(r, 0.99)), "max": float(r.max())}


@pytest.fixture(scope="module")
def band(ctx, oracle_mod, gaunt_table):
    from illcrawl_b200 import synthetic
    cells = synthetic.xray_cells()
    ctx.load_gaunt()
    q = ctx.xray_flux(cells.rho, cells.u, cells.xe, Z, DL, EMIN, EMAX, NS)
    oq = oracle_mod.xray_band(gaunt_table, cells.rho, cells.u, cells.xe, Z, DL, EMIN, EMAX, NS)
    g = oracle_mod.Grid(cells.xyzq(oq))
    return cells, q, oq, g


@pytest.fixture(scope="module")
def band_map(ctx, band):
    """The benchmark's call: raw cells in, scaled map out (device tensors)."""
    import torch
    import illcrawl_b200 as ilc
    cells = band[0]
    dev = torch.device("cuda", 0)
    d_cells = torch.from_numpy(cells.xyzq(np.zeros(cells.n, np.float32))).to(dev)
    d_rho, d_u, d_xe = (torch.from_numpy(a).to(dev) for a in (cells.rho, cells.u, cells.xe))
    ctx.set_render_engine(ilc.ENGINE_PERSISTENT)
    img, st = ctx.project_xray_flux(d_cells, d_rho, d_u, d_xe, ilc.camera(*CAM), BOX,
                                    rel_tol=REL_TOL, controller=ilc.CONTROLLER_FP64,
                                    e_min=EMIN, e_max=EMAX, num_samples=NS,
                                    scaling=ilc.LosScaling(1.0, 1.0, ilc.DA_PIXEL_AREA))
    return img.cpu().numpy(), st


@pytest.fixture(scope="module")
def converged(band, oracle_mod):
    """The 256 sampled pixels rendered by the FP64 oracle at rtol 1e-5 (unscaled)."""
    g = band[3]
    conv, *_ = g.render(oracle_mod.camera(*CAM), BOX, 0.0, 1e-5, mode=2, pix=sample_pixels())
    return np.asarray(conv, np.float64)


def test_band_map_cells_and_grid_bit_exact(ctx, band):
    cells, q, oq, g = band
    assert same_bits(q, oq)
    ctx.setup_particles(cells.xyzq(q))
    d = ctx.grid_describe()
    assert np.array_equal(d["min_corner"], g.min_corner)
    assert np.array_equal(d["cell_sizes"], g.cell_sizes)
    assert np.array_equal(d["num_cells"], g.num_cells)
    rc, rs2u, rsrt = ctx.grid_export()
    oc, os2u, osrt, _ = g.export()
    assert np.array_equal(rs2u, os2u)
    assert np.array_equal(rc, oc)
    assert np.array_equal(rsrt.view(np.uint32), osrt.view(np.uint32))


def test_band_map_sampled_pixels_bit_exact_and_error_vs_fp64(band, band_map, oracle_mod,
                                                             converged):
    cells, q, oq, g = band
    img, st = band_map
    ocam = oracle_mod.camera(*CAM)
    pix = sample_pixels()
    out, steps, acc, ost, rc = g.render(ocam, BOX, 0.0, REL_TOL, mode=1, pix=pix)
    assert rc == 0
    scale = oracle_mod.los_scale(ocam, BOX, 1.0, 1.0, 0)
    got = img.ravel()[pix]
    assert same_bits(got, (out * scale).astype(np.float32))
    raw = got.astype(np.float64) / float(scale)
    o64, *_ = g.render(ocam, BOX, 0.0, REL_TOL, mode=2, pix=pix)
    conv = converged
    e_same = rel_stats(raw, o64)
    e_conv = rel_stats(raw, conv)
    e_o64 = rel_stats(o64, conv)
    print("vs FP64 oracle at rtol 1e-3:", e_same)
    print("vs converged FP64 (rtol 1e-5):", e_conv)
    print("FP64 oracle at rtol 1e-3 vs converged:", e_o64)
    # The adaptive method's own error at rtol 1e-3: the FP64 oracle is off the
    # converged integral by up to ~2e-3 on this sample as well. The fp32 map
    # is as close to the converged integral as the FP64 oracle is.
    assert e_same["median"] < 1e-3 and e_same["p90"] < 2 * REL_TOL
    assert e_conv["median"] < 1e-3 and e_conv["p90"] < 2 * REL_TOL
    assert e_conv["max"] < 1.5 * max(e_o64["max"], REL_TOL)
    assert e_same["max"] < 5 * REL_TOL


def test_band_map_per_pixel_error_below_1e3_at_rtol_5e4(ctx, band, oracle_mod, converged):
    """A per-pixel error bound of 1e-3 against the converged integral needs a
    tighter tolerance than 1e-3 (the adaptive method's own error at 1e-3 is up
    to ~2e-3, for the FP64 oracle too): at rtol 5e-4 the map's sampled pixels
    are bit-exact against the oracle and every one is within 1e-3 of the
    converged FP64 render."""
    import torch
    import illcrawl_b200 as ilc
    cells, q, oq, g = band
    dev = torch.device("cuda", 0)
    d_cells = torch.from_numpy(cells.xyzq(np.zeros(cells.n, np.float32))).to(dev)
    d_rho, d_u, d_xe = (torch.from_numpy(a).to(dev) for a in (cells.rho, cells.u, cells.xe))
    img, st = ctx.project_xray_flux(d_cells, d_rho, d_u, d_xe, ilc.camera(*CAM), BOX,
                                    rel_tol=5e-4, controller=ilc.CONTROLLER_FP64,
                                    e_min=EMIN, e_max=EMAX, num_samples=NS,
                                    scaling=ilc.LosScaling(1.0, 1.0, ilc.DA_PIXEL_AREA))
    ocam = oracle_mod.camera(*CAM)
    pix = sample_pixels()
    out, *_ = g.render(ocam, BOX, 0.0, 5e-4, mode=1, pix=pix)
    scale = oracle_mod.los_scale(ocam, BOX, 1.0, 1.0, 0)
    got = img.cpu().numpy().ravel()[pix]
    assert same_bits(got, (out * scale).astype(np.float32))
    e = rel_stats(got.astype(np.float64) / float(scale), converged)
    print("rtol 5e-4 vs converged FP64:", e)
    assert e["max"] < 1e-3


def test_band_map_ray_counters_match_oracle_bytes(ctx, band, band_map):
    import illcrawl_b200 as ilc
    cells, q, oq, g = band
    img, st = band_map
    ctx.setup_particles(cells.xyzq(q))
    simg, rs, sst = ctx.render_ray_stats(ilc.camera(*CAM), BOX, REL_TOL, 0.0,
                                         ilc.CONTROLLER_FP64,
                                         scaling=ilc.LosScaling(1.0, 1.0, ilc.DA_PIXEL_AREA))
    # the one-block-per-tile kernel and the persistent kernel: same map
    assert same_bits(simg, img)
    assert sst["steps"] == st["steps"] and sst["cells_visited"] == st["cells_visited"]
    assert sst["candidates"] == st["candidates"]
    assert int(rs[:, 0].sum()) == st["steps"] and int(rs[:, 2].sum()) == st["cells_visited"]
    ref = json.load(open(os.path.join(ROOT, "baseline", "bytes_cfg1.json")))
    pix = np.array([r["pixel"] for r in ref["rays"]])
    assert np.array_equal(pix, sample_pixels())
    for r in ref["rays"]:
        s = rs[r["pixel"]]
        assert (int(s[0]), int(s[1]), int(s[2]), int(s[3])) == (
            r["steps"], r["accepted"], r["cells_visited"], r["candidates"]), r["pixel"]
        assert 8 * int(s[2]) + 16 * int(s[3]) + 24 * int(s[0]) + 4 == r["bytes"]


def test_band_map_fixed_2048_steps(ctx, band, oracle_mod):
    import illcrawl_b200 as ilc
    cells, q, oq, g = band
    ctx.setup_particles(cells.xyzq(q))
    img, st = ctx.render_fixed(ilc.camera(*CAM), BOX, 2048)
    assert st["steps"] == 2048 * SIDE * SIDE
    ocam = oracle_mod.camera(*CAM)
    pix = sample_pixels()
    out, _ = g.render_fixed(ocam, BOX, 2048, precision=0, pix=pix)
    got = img.ravel()[pix]
    assert same_bits(got, out)
    o64, _ = g.render_fixed(ocam, BOX, 2048, precision=1, pix=pix)
    e = rel_stats(got, o64)
    print("fixed 2048 steps, fp32 vs FP64 replay:", e)
    assert e["max"] < 1e-5
