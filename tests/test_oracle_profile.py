"""Monte-Carlo radial profiles (distributed_mc_radial_profile, profile.cpp:
26-355) on the CPU: the shell layout and sample counts of the library's host
code and of the oracle against a plain Python restatement, the oracle's
sampler against a numpy restatement bit for bit, the sampler's statistics,
and the profile of a constant field."""
import math

import numpy as np
import pytest

M1, M2, M3 = np.uint64(0x9e3779b97f4a7c15), np.uint64(0xbf58476d1ce4e5b9), np.uint64(0x94d049bb133111eb)


def _shells_py(R, N, density):
    """profile.cpp:93-128 and 320-355 in Python floats (IEEE doubles)."""
    radius = lambda i: i * (R / N)
    rmin = [0.0 if i == 0 else 0.5 * (radius(i - 1) + radius(i)) for i in range(N)]
    rmax = [0.5 * (radius(i + 1) + radius(i)) for i in range(N)]
    vol = [4. / 3 * math.pi * (b * b * b - a * a * a) for a, b in zip(rmin, rmax)]
    expected = 0.0
    for v in vol:
        expected += v * density
    sq = 0.0
    for v in vol:
        sq += v * v
    norm = expected / sq
    counts = [max(1, int(norm * (v * v))) for v in vol]
    return [radius(i) for i in range(N)], counts, rmin, rmax


def _mix(z):
    with np.errstate(over="ignore"):
        z = z + M1
        z = (z ^ (z >> np.uint64(30))) * M2
        z = (z ^ (z >> np.uint64(27))) * M3
    return z ^ (z >> np.uint64(31))


def _draw(seed, k, j):
    with np.errstate(over="ignore"):
        h = _mix(_mix(np.uint64(seed) ^ _mix(k)) + np.uint64(j))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _cbrt_newton(u):
    m, e = np.frexp(u)
    r = np.mod(e, 3)
    m = np.ldexp(m, r)
    e = e - r
    y = np.ones_like(u)
    for _ in range(8):
        y = (2.0 * y + m / (y * y)) / 3.0
    return np.where(u > 0, np.ldexp(y, e // 3), 0.0)


def _points_np(seed, center, R, N, density):
    """random.cpp:28-86 with the hashed draws, vectorised over samples."""
    _, counts, rmin, rmax = _shells_py(R, N, density)
    shell = np.repeat(np.arange(N), counts)
    k = np.arange(shell.size, dtype=np.uint64)
    x1 = np.zeros(k.size); x2 = np.zeros(k.size); r = np.zeros(k.size)
    done = np.zeros(k.size, bool)
    for a in range(64):
        t1 = -1.0 + (1.0 - -1.0) * _draw(seed, k, 2 * a)
        t2 = -1.0 + (1.0 - -1.0) * _draw(seed, k, 2 * a + 1)
        rr = t1 * t1 + t2 * t2
        take = ~done & (rr <= 1.0)
        x1[take], x2[take], r[take] = t1[take], t2[take], rr[take]
        done |= take
    s = np.sqrt(1.0 - r)
    p = np.stack([2 * x1 * s, 2 * x2 * s, 1 - 2 * r], 1)
    lo = np.array(rmin)[shell] * np.array(rmin)[shell] * np.array(rmin)[shell]
    hi = np.array(rmax)[shell] * np.array(rmax)[shell] * np.array(rmax)[shell]
    u = lo + (hi - lo) * _draw(seed, k, 128)
    rad = _cbrt_newton(u)
    return (rad[:, None] * p + np.asarray(center)[None, :]).astype(np.float32), shell


@pytest.mark.parametrize("R,N,density", [(3000.0, 30, 1e-6), (500.0, 1, 1e-3), (1.0, 64, 7.0),
                                         (400.0, 17, 0.01)])
def test_shells_match_python_restatement(oracle_mod, cuda_lib, R, N, density):
    import illcrawl_b200 as ilc
    radii, counts, _, _ = _shells_py(R, N, density)
    r1, c1 = ilc.mc_profile_shells(R, N, density)
    r2, c2 = oracle_mod.mc_profile_shells(R, N, density)
    assert np.array_equal(r1, np.array(radii)) and np.array_equal(r2, np.array(radii))
    assert c1.tolist() == counts and c2.tolist() == counts
    assert min(counts) >= 1


def test_shells_reject_bad_arguments(oracle_mod, cuda_lib):
    import illcrawl_b200 as ilc
    for args in ((0.0, 10, 1.0), (10.0, 0, 1.0), (10.0, 10, 0.0), (float("nan"), 3, 1.0),
                 (1e6, 10, 1e9), (10.0, (1 << 20) + 1, 1.0)):
        with pytest.raises(ilc.IlcError):
            ilc.mc_profile_shells(*args)
        with pytest.raises(ValueError):
            oracle_mod.mc_profile_shells(*args)


def test_cube_root_within_an_ulp():
    rng = np.random.default_rng(3)
    u = np.concatenate([rng.uniform(0, 1, 5000) * 10.0 ** rng.integers(-30, 30, 5000),
                        np.array([1.0, 8.0, 27.0, 1e-300, 1e300, 0.5, 2.0])])
    got = _cbrt_newton(u)
    want = np.cbrt(u)
    ulp = np.abs(got - want) / np.spacing(want)
    assert ulp.max() <= 1.0, ulp.max()
    assert got[-7] == 1.0 and got[-6] == 2.0 and got[-5] == 3.0


def test_oracle_samples_match_numpy_restatement(oracle_mod):
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(20_000, seed=61)
    g = oracle_mod.Grid(c.xyzq(c.rho))
    center = (500.0, 500.0, 500.0)
    prof, pts, vals = oracle_mod.mc_radial_profile(g, center, 400.0, 12, 1e-4, seed=99,
                                                   samples=True)
    want, shell = _points_np(99, center, 400.0, 12, 1e-4)
    assert np.array_equal(pts[:, :3].view(np.uint32), want.view(np.uint32))
    assert np.all(pts[:, 3] == 0)
    # values are the oracle's own nn8 at those points
    assert np.array_equal(vals.view(np.uint32), g.nn8(pts, slots=False)[0].view(np.uint32))
    # per-shell double sums in sample order, times dV = V / n
    _, counts, rmin, rmax = _shells_py(400.0, 12, 1e-4)
    first = np.concatenate([[0], np.cumsum(counts)])
    for s in range(12):
        acc = 0.0
        for v in vals[first[s]:first[s + 1]]:
            acc += float(v)
        vol = 4. / 3 * math.pi * (rmax[s] ** 3 - rmin[s] ** 3)
        assert prof[s] == pytest.approx(acc * vol / counts[s], rel=1e-13)


def test_sampler_statistics():
    """Uniform in volume within the shell and isotropic."""
    center = (0.0, 0.0, 0.0)
    pts, shell = _points_np(5, center, 100.0, 4, 0.05)
    _, counts, rmin, rmax = _shells_py(100.0, 4, 0.05)
    s = 3
    sel = pts[shell == s].astype(np.float64)
    assert sel.shape[0] == counts[s] and counts[s] > 20_000
    r = np.linalg.norm(sel, axis=1)
    assert np.all(r >= rmin[s] * (1 - 1e-6)) and np.all(r <= rmax[s] * (1 + 1e-6))
    t = (r ** 3 - rmin[s] ** 3) / (rmax[s] ** 3 - rmin[s] ** 3)
    assert abs(t.mean() - 0.5) < 0.01 and abs(t.var() - 1 / 12) < 0.005
    d = sel / r[:, None]
    assert np.all(np.abs(d.mean(0)) < 0.02)
    assert np.all(np.abs((d * d).mean(0) - 1 / 3) < 0.01)


@pytest.mark.parametrize("mode", [0, 1])
def test_constant_field_profile(oracle_mod, mode):
    """q = 2.5 everywhere: the mean profile is 2.5 and the volume profile
    2.5 * V_shell * conv, up to nn8's weighted mean rounding."""
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(10_000, seed=62)
    g = oracle_mod.Grid(c.xyzq(np.full(c.n, 2.5, np.float32)))
    prof = oracle_mod.mc_radial_profile(g, (500.0, 500.0, 500.0), 300.0, 10, 1e-3, seed=1,
                                        dV_mode=mode, volume_conversion=0.125)
    _, _, rmin, rmax = _shells_py(300.0, 10, 1e-3)
    vol = np.array([4. / 3 * math.pi * (b ** 3 - a ** 3) for a, b in zip(rmin, rmax)])
    want = np.full(10, 2.5) if mode == 1 else 2.5 * vol * 0.125
    assert np.allclose(prof, want, rtol=1e-6)


@pytest.mark.parametrize("seed,R,N,density,first,count", [(99, 400.0, 12, 1e-4, 0, None),
                                                          (3, 1000.0, 8, 1e-5, 5000, 20000),
                                                          (2 ** 63 + 5, 50.0, 3, 0.2, 17, 1)])
def test_library_sampler_matches_oracle(oracle_mod, cuda_lib, seed, R, N, density, first, count):
    """The library's sampler source (host build of the code the device runs:
    shell search, hashed draws, Marsaglia point, Newton cube root) makes the
    oracle's sample points bit for bit."""
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(2_000, seed=66)
    g = oracle_mod.Grid(c.xyzq(c.rho))
    center = (480.5, 510.25, 499.0)
    _, opts, _ = oracle_mod.mc_radial_profile(g, center, R, N, density, seed=seed, samples=True)
    total = opts.shape[0]
    n = total - first if count is None else count
    pts = ilc.mc_profile_points(center, R, N, density, seed=seed, first=first, count=n)
    assert pts.shape == (n, 4)
    assert np.array_equal(pts.view(np.uint32), opts[first:first + n].view(np.uint32))


def test_library_sampler_rejects_out_of_range(cuda_lib):
    import illcrawl_b200 as ilc
    total = int(ilc.mc_profile_shells(100.0, 4, 0.01)[1].sum())
    with pytest.raises(ilc.IlcError):
        ilc.mc_profile_points((0, 0, 0), 100.0, 4, 0.01, first=total - 1, count=2)
    assert ilc.mc_profile_points((0, 0, 0), 100.0, 4, 0.01, first=total, count=0).shape == (0, 4)
