"""Oracle restatement of the Chandra count-rate and photon-flux quantities
(quantities.cl:432-675) on the CPU.

* the 1D ARF lookup follows the OpenCL linear sampler (texel centres at
  i + 0.5, border 0), checked against a float32 numpy restatement through the
  spectral count rate, bit for bit;
* the total count rate is the channel count rates summed in channel order,
  bit for bit;
* the fp32 quantities agree with the FP64 oracle, and the FP64 photon flux
  with a Python emulation of the reference's energy integration.
"""
import numpy as np
import pytest

from conftest import reference_arf

Z, DL = 0.2, 978500.0
X0, DX = 0.105322271585, 0.010644


def _cells(n, seed):
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(n, seed=seed)
    return c.rho, c.u, c.xe


def _arf_np(arf, x):
    """evaluate_tabulated_function in float32 numpy (independent of the C
    restatement): u = (x - x0) / dx, blend of texels floor(u - 0.5) and the
    next with weight frac(u - 0.5), zero outside the table."""
    f = np.float32
    u = (f(x) - f(X0)) / f(DX)
    us = u - f(0.5)
    fu = np.floor(us)
    i0 = int(fu)
    a = us - fu
    t0 = f(arf[i0]) if 0 <= i0 < arf.size else f(0)
    t1 = f(arf[i0 + 1]) if 0 <= i0 + 1 < arf.size else f(0)
    return (f(1) - a) * t0 + a * t1


@pytest.fixture(scope="module", params=["reference", "synthetic"])
def arf(request):
    """The reference's own ARF (golden fixture from chandra.cpp) and a seeded
    stand-in on the same energy grid."""
    if request.param == "reference":
        table, x0, dx = reference_arf()
        assert (x0, dx) == (X0, DX)
        return table
    from illcrawl_b200 import synthetic
    return synthetic.synthetic_arf()


@pytest.mark.parametrize("E", [X0, X0 + 0.3 * DX, 0.5, 1.3, 2.1, 7.9, X0 + 1023.6 * DX,
                               X0 + 1024.4 * DX, X0 + 1030 * DX, X0 - 0.4 * DX, 0.01])
def test_spectral_count_rate_is_emission_over_energy_times_arf(oracle_mod, gaunt_table, arf, E):
    rho, u, xe = _cells(300, 41)
    f = np.float32
    dE = f(0.05)
    got = oracle_mod.chandra_spectral_count_rate(gaunt_table, arf, X0, DX, rho, u, xe, Z, DL,
                                                 f(E), dE)
    em = oracle_mod.xray_bin(gaunt_table, rho, u, xe, Z, DL, f(E), dE)
    ez = (f(1) + f(Z)) * f(E)
    want = em / ez * (_arf_np(arf, E) * f(1e-4))
    assert np.array_equal(got.view(np.uint32), want.astype(np.float32).view(np.uint32))
    if E > X0 + 1025 * DX or E < X0 - DX:
        assert np.all(got == 0)


def test_total_count_rate_is_channel_sum(oracle_mod, gaunt_table, arf):
    rho, u, xe = _cells(200, 42)
    f = np.float32
    total = oracle_mod.chandra_count_rate(gaunt_table, arf, X0, DX, rho, u, xe, Z, DL)
    acc = np.zeros(rho.size, np.float32)
    for k in range(arf.size):
        e = f(X0) + f(k) * f(DX)
        acc = acc + oracle_mod.chandra_spectral_count_rate(gaunt_table, arf, X0, DX, rho, u, xe,
                                                           Z, DL, e, f(DX))
    assert np.array_equal(total.view(np.uint32), acc.view(np.uint32))
    assert np.all(total > 0)


def test_count_rate_fp32_vs_fp64(oracle_mod, gaunt_table, arf):
    rho, u, xe = _cells(400, 43)
    a = oracle_mod.chandra_count_rate(gaunt_table, arf, X0, DX, rho, u, xe, Z, DL)
    b = oracle_mod.chandra_count_rate(gaunt_table, arf, X0, DX, rho, u, xe, Z, DL, precision=1)
    rel = np.abs(a.astype(np.float64) - b) / b
    assert rel.max() < 1e-4, rel.max()


def _spectral_integral(oracle_mod, gaunt_table, rho, u, xe, e_min, e_max, rel_tol, photon):
    """integrate_spectral_flux (quantities.cl:156-239) emulated in float64
    Python on top of the FP64 emission: rkf_advance (integration.cl:47-132)
    with (absolute, relative) tolerance (rel_tol, 1), epsilon 0 and step
    bounds [1e-3, 100]; PHOTON_FLUX divides every sample by its energy."""
    def f(e):
        v = float(oracle_mod.xray_bin(gaunt_table, rho, u, xe, 0.0, DL, e, 1.0, precision=1)[0])
        return v / e if photon else v
    acc, pos, end = 0.0, e_min, e_max
    h = (end - pos) * rel_tol
    k1 = f(pos)
    steps = 0
    while pos < end:
        p = [pos + 3 / 8 * h, pos + 12 / 13 * h, pos + h, pos + 0.5 * h]
        v = [f(x) for x in p]
        d4 = (25 / 216 * k1 + 1408 / 2565 * v[0] + 2197 / 4101 * v[1] - 1 / 5 * v[2]) * h
        d5 = (16 / 135 * k1 + 6656 / 12825 * v[0] + 28561 / 56430 * v[1] - 9 / 50 * v[2]
              + 2 / 55 * v[3]) * h
        old = pos
        pos += h
        s = 2.0
        if d4 != d5:
            tol = max(rel_tol, abs(acc / pos))
            s = (tol * h / (2 * abs(d5 - d4))) ** 0.25
        nh = min(max(s * h, 1e-3), 100.0)
        if nh / h < 0.95:
            pos = old
        else:
            acc += d4
            k1 = v[2]
            steps += 1
        h = nh
        if pos + h >= end:
            h = end - pos
    return acc, steps


def test_photon_flux_vs_fp64_and_emulation(oracle_mod, gaunt_table):
    rho, u, xe = _cells(200, 44)
    pf = oracle_mod.xray_photon_flux(gaunt_table, rho, u, xe, Z, DL, 0.1, 10.0, 100)
    pd = oracle_mod.xray_photon_flux(gaunt_table, rho, u, xe, Z, DL, 0.1, 10.0, 100, precision=1)
    rel = np.abs(pf.astype(np.float64) - pd) / pd
    assert np.median(rel) < 1e-5 and rel.max() < 1e-3, (np.median(rel), rel.max())
    # The reference's absolute tolerance (1 / num_samples) dwarfs emissions of
    # ~1e-9, so after the first step (range / num_samples) the controller
    # jumps to the largest step: the band integral is a few RKF panels.
    for i in range(0, 200, 40):
        want, steps = _spectral_integral(oracle_mod, gaunt_table, rho[i:i + 1], u[i:i + 1],
                                         xe[i:i + 1], (1 + Z) * 0.1, (1 + Z) * 10.0, 0.01, True)
        assert steps <= 4
        # float32 emission samples move the error estimate, hence the steps,
        # by ~1e-6; a different integration would differ by tens of percent
        assert abs(pd[i] - want * 1e-4) <= 1e-4 * want * 1e-4, (i, pd[i], want * 1e-4)


def test_photon_flux_is_flux_over_energy(oracle_mod, gaunt_table):
    """photons * mean energy = energy flux: their ratio lies in the band."""
    rho, u, xe = _cells(200, 45)
    pf = oracle_mod.xray_photon_flux(gaunt_table, rho, u, xe, Z, DL, 0.5, 7.0, 100, precision=1)
    ef = oracle_mod.xray_band(gaunt_table, rho, u, xe, Z, DL, 0.5, 7.0, 100, precision=1)
    mean_e = ef.astype(np.float64) * 1e-4 / pf   # keV per photon at the source
    assert np.all(mean_e > (1 + Z) * 0.5) and np.all(mean_e < (1 + Z) * 7.0)


def test_reference_arf_fixture():
    """The fixture holds chandra.cpp's table as the compiler makes it: 1024
    float32 entries from x_min 0.105322271585 keV in steps of 0.010644 keV,
    the first of them the literals 7.977484415e-07f and 3.577559582e-08f."""
    table, x0, dx = reference_arf()
    assert table.dtype == np.float32 and table.shape == (1024,)
    assert (x0, dx) == (0.105322271585, 0.010644)
    assert table[0] == np.float32(7.977484415e-07) and table[1] == np.float32(3.577559582e-08)
    assert np.all(np.isfinite(table)) and np.all(table > 0)
    assert 400.0 < table.max() < 450.0   # peak effective area in cm^2
