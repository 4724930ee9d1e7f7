"""GPU parity of the Monte-Carlo radial profile (ilc_mc_radial_profile,
distributed_mc_radial_profile of profile.cpp:26-355) against the oracle:

* every sample point and nn8 value bit for bit (same hashed draws, same
  double sampler, same nn8);
* the profile within 1e-12 relative: the device sums each shell in 8192-sample
  segments, the oracle in sample order;
* a profile of 4.8 M samples crosses the 4 M-sample device batch;
* no particles / bad arguments fail with their status.
"""
import numpy as np
import pytest

from test_gpu_parity import same_bits

pytestmark = pytest.mark.gpu


def _cells(n, seed):
    from illcrawl_b200 import synthetic
    return synthetic.small_cells(n, seed=seed)


@pytest.mark.parametrize("mode", [0, 1])
def test_profile_samples_bit_exact(ctx, oracle_mod, mode):
    import illcrawl_b200 as ilc
    c = _cells(30_000, 63)
    pts = c.xyzq(c.rho)
    ctx.setup_particles(pts)
    g = oracle_mod.Grid(pts)
    center = (500.0, 480.0, 510.0)
    dv = ilc.DV_VOLUME if mode == 0 else ilc.DV_MEAN
    prof, sp, sv = ctx.mc_radial_profile(center, 420.0, 16, 2e-4, seed=7, dV_mode=dv,
                                         volume_conversion=0.5, samples=True)
    oprof, osp, osv = oracle_mod.mc_radial_profile(g, center, 420.0, 16, 2e-4, seed=7,
                                                   dV_mode=mode, volume_conversion=0.5,
                                                   samples=True)
    assert sp.shape == osp.shape and sp.shape[0] == 56425
    assert same_bits(sp, osp)
    assert same_bits(sv, osv)
    assert np.allclose(prof, oprof, rtol=1e-12, atol=0.0)
    assert np.all(prof > 0)
    # the profile without sample outputs is the same computation
    assert np.array_equal(ctx.mc_radial_profile(center, 420.0, 16, 2e-4, seed=7, dV_mode=dv,
                                                volume_conversion=0.5), prof)


def test_profile_across_device_batches(ctx, oracle_mod):
    c = _cells(60_000, 64)
    pts = c.xyzq(c.rho)
    ctx.setup_particles(pts)
    g = oracle_mod.Grid(pts)
    center = (500.0, 500.0, 500.0)
    prof, _, sv = ctx.mc_radial_profile(center, 1000.0, 8, 1.4e-3, seed=11, samples=True)
    oprof, _, osv = oracle_mod.mc_radial_profile(g, center, 1000.0, 8, 1.4e-3, seed=11,
                                                 samples=True)
    assert sv.shape[0] == 4_832_035 > (1 << 22)
    assert same_bits(sv, osv)
    assert np.allclose(prof, oprof, rtol=1e-12, atol=0.0)


def test_profile_errors(cuda_lib):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import illcrawl_b200 as ilc
    with ilc.Context(0) as fresh:
        with pytest.raises(ilc.IlcError, match="NO_PARTICLES"):
            fresh.mc_radial_profile((0.0, 0.0, 0.0), 10.0, 4, 1.0)
        c = _cells(2_000, 65)
        fresh.setup_particles(c.xyzq(c.rho))
        with pytest.raises(ilc.IlcError, match="INVALID_ARGUMENT"):
            fresh.mc_radial_profile((500.0, 500.0, 500.0), 10.0, 4, 1.0, dV_mode=2)
        with pytest.raises(ilc.IlcError, match="INVALID_ARGUMENT"):
            fresh.mc_radial_profile((500.0, 500.0, 500.0), -1.0, 4, 1.0)
