"""GPU parity of the Chandra count-rate and photon-flux quantities
(quantities.cl:432-675) through the C ABI against the oracle, bit for bit,
and of maps and spectra rendered from them:

* xray_photon_flux, chandra_xray_total_count_rate, chandra_xray_spectral_count_rate
  per cell, including channels outside the ARF (rate 0);
* the cell-major Chandra spectrum table equals the per-channel quantity;
* an adaptive count-rate map and a batched Chandra spectrum (the frames of
  chandra_spectrum_quantity_generator) equal the oracle's renders;
* a Chandra quantity before ilc_arf_load fails with ILC_ERR_NO_ARF_TABLE.
"""
import numpy as np
import pytest

from conftest import reference_arf

from test_gpu_parity import same_bits

pytestmark = pytest.mark.gpu

Z, DL = 0.2, 978500.0
X0, DX = 0.105322271585, 0.010644


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


def test_chandra_needs_arf(cuda_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(100, seed=50)
    with ilc.Context(0) as fresh:
        fresh.load_gaunt()
        with pytest.raises(ilc.IlcError, match="ARF"):
            fresh.chandra_count_rate(c.rho, c.u, c.xe)
        with pytest.raises(ilc.IlcError):
            fresh.load_arf(np.ones(4, np.float32), X0, 0.0)       # dx must be > 0
        with pytest.raises(ilc.IlcError):
            fresh.load_arf(np.ones(70_000, np.float32), X0, DX)   # more than 65536 samples


def test_photon_flux_bit_exact(ctx, oracle_mod, gaunt_table):
    from illcrawl_b200 import synthetic
    c = synthetic.xray_cells(n=100_000, seed=98)
    ctx.load_gaunt()
    for lo, hi, ns in ((0.1, 10.0, 100), (0.5, 7.0, 37)):
        q = ctx.xray_photon_flux(c.rho, c.u, c.xe, Z, DL, lo, hi, ns)
        oq = oracle_mod.xray_photon_flux(gaunt_table, c.rho, c.u, c.xe, Z, DL, lo, hi, ns)
        assert same_bits(q, oq)


def test_chandra_count_rates_bit_exact(ctx, oracle_mod, gaunt_table, arf):
    from illcrawl_b200 import synthetic
    c = synthetic.xray_cells(n=20_000, seed=97)
    ctx.load_gaunt()
    ctx.load_arf(arf, X0, DX)
    tot = ctx.chandra_count_rate(c.rho, c.u, c.xe, Z, DL)
    otot = oracle_mod.chandra_count_rate(gaunt_table, arf, X0, DX, c.rho, c.u, c.xe, Z, DL)
    assert same_bits(tot, otot)
    # cold, thin background cells underflow to 0 in fp32, as in the oracle
    assert np.all(tot >= 0) and np.count_nonzero(tot) > tot.size // 2
    # channels inside, on the edges of and outside the table
    for e in (X0, 0.4, 1.3, 2.1, X0 + 1023.7 * DX, X0 + 1030 * DX, 0.01):
        r = ctx.chandra_spectral_count_rate(c.rho, c.u, c.xe, e, DX, Z, DL)
        o = oracle_mod.chandra_spectral_count_rate(gaunt_table, arf, X0, DX, c.rho, c.u, c.xe,
                                                   Z, DL, e, DX)
        assert same_bits(r, o), e
    # cell-major spectrum table == the per-channel quantity
    e, w = synthetic.chandra_spectrum_channels(16)
    tab = ctx.chandra_spectrum(c.rho, c.u, c.xe, e, w, Z, DL)
    for b in range(16):
        o = oracle_mod.chandra_spectral_count_rate(gaunt_table, arf, X0, DX, c.rho, c.u, c.xe,
                                                   Z, DL, e[b], w[b])
        assert same_bits(tab[:, b], o), b


def test_chandra_count_rate_map_and_spectrum_render(ctx, oracle_mod, gaunt_table, arf):
    """A count-rate map (the reference's default quantity) by the adaptive
    render, and a 12-channel Chandra spectrum by the batched render, each
    bit-exact against the oracle's render of the oracle's per-cell values."""
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(30_000, seed=51)
    ctx.load_gaunt()
    ctx.load_arf(arf, X0, DX)
    q = oracle_mod.chandra_count_rate(gaunt_table, arf, X0, DX, c.rho, c.u, c.xe, Z, DL)
    assert same_bits(ctx.chandra_count_rate(c.rho, c.u, c.xe, Z, DL), q)
    pts = c.xyzq(q)
    ctx.setup_particles(pts)
    g = oracle_mod.Grid(pts)
    args = ((500, 500, 0), (0, 0, 1), 0.3, 900.0, 20, 18)
    img, st = ctx.render_adaptive(ilc.camera(*args), 1000.0, 1e-3, 0.0, ilc.CONTROLLER_FP64)
    out, steps, acc, ost, rc = g.render(oracle_mod.camera(*args), 1000.0, 0.0, 1e-3, mode=1)
    assert rc == 0
    assert same_bits(img, out)
    assert st["steps"] == steps.sum()

    e, w = synthetic.chandra_spectrum_channels(12)
    tab = ctx.chandra_spectrum(c.rho, c.u, c.xe, e, w, Z, DL)
    pts0 = c.xyzq(np.zeros(c.n, np.float32))
    ctx.setup_particles(pts0)
    g0 = oracle_mod.Grid(pts0)
    cam = ((500, 500, -100), (0, 0, 1), 0.3, 900.0, 10, 9)
    jobs = [ilc.job(ilc.camera(*cam), aperture_radius=350.0, sphere_center=(500, 500, 500),
                    sphere_radius=400.0, min_chord=80.0)]
    ojobs = [oracle_mod.job(oracle_mod.camera(*cam), aperture_radius=350.0,
                            sphere_center=(500, 500, 500), sphere_radius=400.0, min_chord=80.0)]
    got, _ = ctx.render_batched(tab, jobs)
    want, _, rc = oracle_mod.render_batched(g0, tab, ojobs, 0.0, 1e-3)
    assert rc == 0
    assert same_bits(got, want)
    assert np.count_nonzero(want) > 0
