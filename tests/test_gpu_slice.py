"""GPU volumetric slices and tomography against the oracle: the nn8
reconstruction on a camera plane, bit-exact for one sample per pixel;
jittered extra samples reproducible for a seed and close to the single-sample
slice on average."""
import numpy as np
import pytest

from test_gpu_parity import same_bits

pytestmark = pytest.mark.gpu


def test_slice_bit_exact(ctx, oracle_mod):
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(40_000, seed=51)
    pts = c.xyzq(c.rho)
    ctx.setup_particles(pts)
    g = oracle_mod.Grid(pts)
    look = np.array([0.2, -0.4, 0.894427191])
    look /= np.linalg.norm(look)
    args = (tuple(np.array([500.0, 480.0, 510.0]) - 10 * look), tuple(look), 0.3, 700.0, 37, 29)
    dV = (700.0 / 37) ** 3
    img = ctx.volumetric_slice(ilc.camera(*args), dV)
    want = oracle_mod.volumetric_slice(g, oracle_mod.camera(*args), dV)
    assert same_bits(img, want)
    a = ctx.volumetric_slice(ilc.camera(*args), dV, additional_samples=3, seed=9)
    b = ctx.volumetric_slice(ilc.camera(*args), dV, additional_samples=3, seed=9)
    assert same_bits(a, b)
    ok = want > 0
    assert np.median(np.abs(a[ok] - want[ok]) / want[ok]) < 0.5


def test_tomography_bit_exact(ctx, oracle_mod):
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(30_000, seed=52)
    pts = c.xyzq(c.rho)
    ctx.setup_particles(pts)
    g = oracle_mod.Grid(pts)
    look = np.array([0.3, 0.1, -0.948683298])
    look /= np.linalg.norm(look)
    pos = np.array([520.0, 470.0, 800.0])
    width, nx, ny = 500.0, 19, 23
    dV = 2.5
    cube = ctx.volumetric_tomography(ilc.camera(tuple(pos), tuple(look), 1.1, width, nx, ny), dV,
                                     initial_z_step=3, num_steps=5)
    ps = width / nx
    for z in range(5):
        t = float(3 + z) * ps                 # the camera moved along look_at, in double
        pz = tuple(pos[j] + t * look[j] for j in range(3))
        want = oracle_mod.volumetric_slice(g, oracle_mod.camera(pz, tuple(look), 1.1, width, nx,
                                                                ny), dV)
        assert same_bits(cube[z], want)
