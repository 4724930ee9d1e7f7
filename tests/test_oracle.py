"""CPU checks of the oracle against the reference's own data and hand-computed
known answers (the reference ships no tests or golden vectors of its own)."""
import hashlib
import math
import os

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden_spiral():
    rows = [l.split() for l in open(os.path.join(GOLDEN, "spiral_table.txt"))
            if not l.startswith("#")]
    return np.array(rows, np.int8).reshape(8, 125, 3)


def test_spiral_table_matches_reference_fixture(oracle_mod):
    assert np.array_equal(oracle_mod.spiral_table(), golden_spiral())


def test_spiral_table_matches_reference_source_when_present(oracle_mod):
    src = os.environ.get("ILLCRAWL_REFERENCE")
    ref = os.path.join(src, "particle_grid_iteration_order.cl") if src else ""
    if not ref or not os.path.exists(ref):
        pytest.skip("reference sources not present (set ILLCRAWL_REFERENCE to a checkout)")
    import re
    ents = re.findall(r"\(char4\)\(\s*(-?\d+),\s*(-?\d+),\s*(-?\d+),", open(ref).read())
    t = np.array(ents, np.int8).reshape(8, 125, 3)
    assert np.array_equal(oracle_mod.spiral_table(), t)


def test_vendored_gaunt_table_is_the_reference_file(gaunt_table):
    sha, rows, cols = open(os.path.join(GOLDEN, "gaunt_factor.sha256")).read().split()
    raw = open(os.path.join(ROOT, "illcrawl_b200", "data", "gaunt_factor.dat"), "rb").read()
    assert hashlib.sha256(raw).hexdigest() == sha
    assert gaunt_table.shape == (int(rows), int(cols)) == (146, 81)
    assert np.array_equal(gaunt_table, np.loadtxt(os.path.join(ROOT, "illcrawl_b200", "data",
                                                               "gaunt_factor.dat"), np.float32))


def test_gaunt_lookup_half_texel_blend(oracle_mod, gaunt_table):
    t = gaunt_table
    # Evaluating exactly at table node (i, j) samples texel coordinate (i, j);
    # OpenCL texel centres are at i + 0.5, so the result is the average of
    # nodes i-1, i (and j-1, j).
    for i, j in [(10, 20), (40, 73), (1, 1), (79, 144)]:
        lg, lu = -6.0 + 0.2 * i, -16.0 + 0.2 * j
        got = oracle_mod.gaunt_lookup(t, np.float32(lg), np.float32(lu))
        want = 0.25 * (t[j - 1, i - 1] + t[j - 1, i] + t[j, i - 1] + t[j, i])
        assert got == pytest.approx(want, rel=2e-5)
    # At texel centres (node + half spacing) the sample is the node itself.
    for i, j in [(10, 20), (40, 73)]:
        lg, lu = -6.0 + 0.2 * (i + 0.5), -16.0 + 0.2 * (j + 0.5)
        assert oracle_mod.gaunt_lookup(t, np.float32(lg), np.float32(lu)) == \
            pytest.approx(t[j, i], rel=2e-5)
    # Far outside the table: CLK_ADDRESS_CLAMP border = 0.
    assert oracle_mod.gaunt_lookup(t, np.float32(-9.0), np.float32(0.0)) == 0.0
    assert oracle_mod.gaunt_lookup(t, np.float32(0.0), np.float32(20.0)) == 0.0
    # Half a texel outside the first node: blend towards the zero border.
    got = oracle_mod.gaunt_lookup(t, np.float32(-6.0), np.float32(-16.0 + 0.2 * 10.5))
    assert got == pytest.approx(0.5 * t[10, 0], rel=2e-5)


def test_own_log_exp_accuracy(oracle_mod):
    rng = np.random.default_rng(0)
    xs = np.concatenate([10.0 ** rng.uniform(-30, 30, 4000), [1.0, 2.0, 0.5, 1e-40, 3e38]])
    for x in xs.astype(np.float32):
        got = np.float64(oracle_mod.logf(x))
        want = math.log(float(x))
        ulp = np.spacing(np.float32(want)) if want != 0 else 1e-45
        assert abs(got - want) <= 4 * abs(ulp) + 1e-7 * (want == 0), (x, got, want)
    for x in np.concatenate([rng.uniform(-100, 88, 4000), [0.0, -1e-8, 1e-8]]).astype(np.float32):
        got = np.float64(oracle_mod.expf(x))
        want = math.exp(float(x))
        assert abs(got - want) <= 4 * np.spacing(np.float32(want)) + 1e-45, (x, got, want)
    assert oracle_mod.logf(0.0) == -np.inf and np.isnan(oracle_mod.logf(-1.0))
    assert oracle_mod.expf(-200.0) == 0.0 and oracle_mod.expf(100.0) == np.inf


def test_camera_plane_known_answer(oracle_mod):
    cam = oracle_mod.camera((3000, 3000, 0), (0, 0, 1), 0.0, 6000, 1024, 1024)
    p = oracle_mod.camera_setup(cam)
    # look = z, so the basis starts from y: b0 = y x z = x, b1 = z x x = y
    assert np.array_equal(p[:12], np.float32([0, 0, 1, 1, 0, 0, 0, 1, 0, 0, 0, 0]))
    assert p[12] == np.float32(6000 / 1024)
    cam = oracle_mod.camera((0, 0, 0), (1, 0, 0), math.pi / 2, 10, 10, 10)
    p = oracle_mod.camera_setup(cam)
    b0, b1 = p[3:6], p[6:9]
    assert abs(float(np.dot(b0, [1, 0, 0]))) < 1e-6 and abs(float(np.dot(b1, [1, 0, 0]))) < 1e-6
    assert abs(float(np.dot(b0, b1))) < 1e-6


def test_grid_known_answer(oracle_mod):
    # 8 particles on the corners of a unit cube plus one inside.
    pts = np.array([[x, y, z, 1.0] for x in (0, 1) for y in (0, 1) for z in (0, 1)] +
                   [[0.5, 0.5, 0.5, 2.0]], np.float32)
    g = oracle_mod.Grid(pts)
    # bbox [-0.1, 1.1]^3, V = 1.2^3, cell width cbrt(8/9 * V) = 1.2 * (8/9)^(1/3)
    w = math.cbrt(8.0 / 9.0 * (1.2 ** 3))
    assert g.cell_sizes[0] == np.float32(w)
    assert list(g.num_cells) == [math.ceil(1.2 / w)] * 3
    cells, s2u, srt, keys = g.export()
    assert np.all(np.diff(keys.astype(np.int64)) >= 0)
    assert np.array_equal(srt, pts[s2u])
    assert cells[:, 1].max() == 9


def test_nn8_lattice_known_answer(oracle_mod):
    # A 6^3 lattice of spacing 1 with q = x index; the query at a lattice point
    # has itself at distance 0 -> weight inf -> result NaN (inf/inf), as the
    # reference's finalize; a query at a cube centre has 8 neighbours at
    # sqrt(3)/2 with equal weights -> mean of their q.
    g1 = np.arange(6, dtype=np.float32)
    X, Y, Z = np.meshgrid(g1, g1, g1, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel(), X.ravel()], 1).astype(np.float32)
    g = oracle_mod.Grid(pts)
    q = np.array([[2.5, 2.5, 2.5, 0], [1.5, 3.5, 2.5, 0]], np.float32)
    val, idx, d8, _ = g.nn8(q)
    assert val[0] == pytest.approx(2.5, rel=1e-6) and val[1] == pytest.approx(1.5, rel=1e-6)
    assert np.allclose(d8, math.sqrt(3) / 2, rtol=1e-6)
    assert sorted(pts[idx[0], 0].tolist()) == [2, 2, 2, 2, 3, 3, 3, 3]


def test_rkf_known_answers(oracle_mod):
    # Constant field: every particle carries q = c, so the integrand is c
    # everywhere. With the reference's delta4 weights (2197/4101 instead of
    # 2197/4104, integration.cl:66) a step adds h*c*S, S = sum of the weights
    # = 1.000392...; the first step has k1 = 0 (the reference's initial
    # evaluation, integration.cpp:211) and adds h*c*(S - 25/216).
    rng = np.random.default_rng(1)
    pts = np.zeros((4000, 4), np.float32)
    pts[:, :3] = rng.random((4000, 3)) * 100
    pts[:, 3] = 2.0
    g = oracle_mod.Grid(pts)
    cam = oracle_mod.camera((50, 50, 0), (0, 0, 1), 0, 20, 4, 4)
    out, st = g.render_fixed(cam, 100.0, 10)
    S = 25 / 216 + 1408 / 2565 + 2197 / 4101 - 1 / 5
    assert S == pytest.approx(1.000392, abs=1e-6)
    want = 2.0 * 10.0 * (10 * S - 25 / 216)
    assert np.allclose(out, want, rtol=2e-6)
    # Adaptive: with a constant integrand delta4 == delta5 only if the weights
    # sum equal; the 2197/4101 quirk makes them differ slightly, the integral
    # must still be within 1e-3 of c*L.
    out, steps, acc, st, rc = g.render(cam, 100.0, 0.0, 1e-3, mode=0)
    assert rc == 0 and np.all(np.abs(out - 200.0) < 0.2 + 200.0 * 1e-3 * 2)
