"""The seeded synthetic gas cells that stand in for simulation data: the
shapes and distributions the workloads are specified with (NFW halos with
radii by the inverse CDF of M(<r), truncation, a 10 % uniform background,
the halos' mass ratio, the density and temperature laws, u from T through
the reference's get_temperature), and reproducibility from the seed."""
import numpy as np

from illcrawl_b200 import synthetic


def _nfw_cdf(r, r_s, r_max):
    m = lambda x: np.log1p(x) - x / (1.0 + x)  # noqa: E731
    return m(r / r_s) / m(r_max / r_s)


def test_same_seed_same_cells_other_seed_other_cells():
    a = synthetic.small_cells(5000, seed=4)
    b = synthetic.small_cells(5000, seed=4)
    c = synthetic.small_cells(5000, seed=5)
    for x, y in ((a.pos, b.pos), (a.rho, b.rho), (a.u, b.u)):
        assert np.array_equal(x, y)
    assert not np.array_equal(a.pos, c.pos)


def test_band_map_cells_follow_their_specification():
    """4,194,304-cell workload at a smaller count: NFW r_s 400 kpc truncated at
    3 Mpc around the centre of a 6 Mpc cube, 10 % uniform background."""
    n = 200_000
    box = 6000.0
    halo = synthetic.Halo((box / 2,) * 3, 400.0, 3000.0)
    c = synthetic.generate(n, box, [halo], seed=20171)
    assert c.n == n and c.pos.dtype == np.float32
    n_bg = int(round(0.1 * n))
    nfw, bg = c.pos[: n - n_bg].astype(np.float64), c.pos[n - n_bg:].astype(np.float64)
    r = np.linalg.norm(nfw - box / 2, axis=1)
    assert r.max() <= 3000.0 * (1 + 1e-6)
    # radii follow M(<r) / M(r_max): Kolmogorov-Smirnov distance of the sample
    rs = np.sort(r)
    ks = np.max(np.abs(_nfw_cdf(rs, 400.0, 3000.0) - np.arange(1, rs.size + 1) / rs.size))
    assert ks < 0.01
    # isotropic directions: the mean unit vector is near zero
    u = (nfw - box / 2) / r[:, None]
    assert np.all(np.abs(u.mean(axis=0)) < 0.01)
    # the background fills the cube uniformly
    assert bg.min() >= 0.0 and bg.max() <= box
    assert np.all(np.abs(bg.mean(axis=0) - box / 2) < 0.01 * box)


def test_density_and_temperature_laws():
    n = 200_000
    halo = synthetic.Halo((500.0, 500.0, 500.0), 100.0, 500.0)
    c = synthetic.generate(n, 1000.0, [halo], seed=9, background=0.0)
    r = np.linalg.norm(c.pos.astype(np.float64) - 500.0, axis=1)
    x = np.maximum(r / 100.0, 1e-3)
    # log-normal scatter around the NFW density: sigma 0.3, median at the profile
    lr = np.log(c.rho.astype(np.float64) / (synthetic.RHO_S / (x * (1 + x) ** 2)))
    assert abs(np.median(lr)) < 0.01 and abs(lr.std() - 0.3) < 0.01
    # temperature 5e7 K (1 + r/r_s)^-1/2 with log-normal scatter 0.2
    lt = np.log(c.temperature.astype(np.float64) / (synthetic.T0 * (1 + r / 100.0) ** -0.5))
    assert abs(np.median(lt)) < 0.01 and abs(lt.std() - 0.2) < 0.01
    assert np.all(c.xe == np.float32(1.16))


def test_internal_energy_inverts_the_reference_temperature():
    """T = (gamma - 1) mu u 121.1475502 with mu = 4 / (1 + 3 X_H + 4 X_H x_e)
    (quantities.cl:48-61), in float64."""
    T = np.geomspace(1e5, 1e9, 50)
    xe = np.full(50, 1.16)
    u = synthetic.internal_energy_from_temperature(T, xe)
    mu = 4.0 / (1.0 + 3.0 * synthetic.X_H + 4.0 * synthetic.X_H * xe)
    assert np.allclose((5.0 / 3.0 - 1.0) * mu * u * 121.1475502, T, rtol=1e-12)


def test_scale_workload_halos_have_mass_ratio_3_to_1():
    """The scale workload's two halos (r_s 450 and 300 kpc, 1.5 Mpc apart,
    3:1) and background, at a smaller count."""
    box = 8000.0
    c = box / 2
    halos = [synthetic.Halo((c - 750.0, c, c), 450.0, 3000.0, 3.0),
             synthetic.Halo((c + 750.0, c, c), 300.0, 3000.0, 1.0)]
    n = 400_000
    cells = synthetic.generate(n, box, halos, seed=20174)
    n_nfw = n - int(round(0.1 * n))
    k0 = int(np.floor(3.0 / 4.0 * n_nfw))
    k0 += n_nfw - k0 - int(np.floor(1.0 / 4.0 * n_nfw))
    first = cells.pos[:k0].astype(np.float64)
    second = cells.pos[k0:n_nfw].astype(np.float64)
    assert abs(first.shape[0] / second.shape[0] - 3.0) < 1e-3
    assert np.linalg.norm(first - (c - 750.0, c, c), axis=1).max() <= 3000.0 * (1 + 1e-6)
    assert np.linalg.norm(second - (c + 750.0, c, c), axis=1).max() <= 3000.0 * (1 + 1e-6)
