"""The oracle's batched render definition (CPU): it reduces to the plain
render for one channel without mask or chord, identical channels give
identical images, chords and masks follow their geometric definition, and
jointly stepped channels stay within 2x the RKF tolerance of each channel
rendered on its own in double."""
import numpy as np


def _grid(oracle_mod, n=12_000, seed=41):
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(n, seed=seed)
    pts = c.xyzq(c.rho)
    return c, pts, oracle_mod.Grid(pts)


def test_single_channel_equals_plain_render(oracle_mod):
    c, pts, g = _grid(oracle_mod)
    cam = oracle_mod.camera((500, 500, 0), (0, 0, 1), 0.0, 1000.0, 11, 9)
    out, steps, acc, st, rc = g.render(cam, 1000.0, 0.0, 1e-3, mode=1)
    bo, bst, brc = oracle_mod.render_batched(g, pts[:, 3].copy(),
                                             [oracle_mod.job(cam, z_range=1000.0)])
    assert rc == 0 and brc == 0
    assert np.array_equal(out.view(np.uint32), bo.view(np.uint32))
    assert bst[0] == steps.sum() and bst[1] == acc.sum()
    assert bst[2] == st[0] and bst[3] == st[1]


def test_identical_channels_identical_images(oracle_mod):
    c, pts, g = _grid(oracle_mod)
    cam = oracle_mod.camera((500, 500, 0), (0.3, 0.2, 0.932737905), 0.4, 900.0, 8, 7)
    v = np.stack([c.rho] * 4, 1)
    out, _, rc = oracle_mod.render_batched(g, v, [oracle_mod.job(cam, z_range=900.0)])
    out = out.reshape(4, -1)
    assert rc == 0
    for k in range(1, 4):
        assert np.array_equal(out[0].view(np.uint32), out[k].view(np.uint32))


def test_chord_and_mask_geometry(oracle_mod):
    look = np.array([0.48, -0.6, 0.64])
    look /= np.linalg.norm(look)
    centre = np.array([500.0, 480.0, 510.0])
    cam = oracle_mod.camera(tuple(centre - 700 * look), tuple(look), 1.1, 800.0, 40, 30)
    jb = oracle_mod.job(cam, aperture_radius=300.0, sphere_center=tuple(centre),
                        sphere_radius=350.0, min_chord=70.0)
    d = oracle_mod.camera_setup(cam).astype(np.float64)  # look, b0, b1, min corner, ps
    ps = 800.0 / 40
    n_masked = 0
    for ix in range(0, 40, 3):
        for iy in range(0, 30, 4):
            masked, o, ln = oracle_mod.ray_span(jb, ix, iy)
            dx, dy = (ix + 0.5 - 20) * ps, (iy + 0.5 - 15) * ps
            assert masked == (dx * dx + dy * dy > 300.0 ** 2)
            n_masked += masked
            pix = d[9:12] + ix * ps * d[3:6] + iy * ps * d[6:9]
            w = centre - pix
            t = w @ look
            b2 = w @ w - t * t
            half = max(np.sqrt(max(350.0 ** 2 - b2, 0.0)), 35.0)
            z0, z1 = max(t - half, 0.0), t + half
            assert abs(ln - (z1 - z0)) < 1e-2
            assert np.allclose(o, pix + z0 * look, atol=5e-2)
    assert 0 < n_masked


def test_joint_steps_within_tolerance_of_fp64_per_channel(oracle_mod):
    c, pts, g = _grid(oracle_mod, n=8_000, seed=43)
    rng = np.random.default_rng(2)
    V = 6
    v = (c.rho[:, None] * (c.u[:, None] / c.u.mean()) ** rng.uniform(-1, 1, size=(1, V)))
    v = v.astype(np.float32)
    cam = oracle_mod.camera((500, 500, -100), (0, 0, 1), 0.0, 800.0, 10, 10)
    jb = oracle_mod.job(cam, sphere_center=(500, 500, 500), sphere_radius=400.0, min_chord=80.0)
    rays = [(0, p) for p in range(0, 100, 3)]
    got, st, rc = oracle_mod.render_batched(g, v, [jb], 0.0, 1e-3, rays=rays)
    ref, _, rc2 = oracle_mod.render_batched(g, v, [jb], 0.0, 1e-3, rays=rays, precision=1)
    assert rc == 0 and rc2 == 0
    ok = ref > 0
    rel = np.abs(got[ok] - ref[ok]) / ref[ok]
    # the same bar as the plain adaptive render: 2x rtol for the bulk (the
    # RKF controls the local error per step, not the per-pixel total)
    assert np.median(rel) < 2e-3 and np.quantile(rel, 0.9) < 2e-3 and rel.max() < 1e-2


def test_empty_chords_and_full_masks_give_zero(oracle_mod):
    c, pts, g = _grid(oracle_mod, n=5_000, seed=44)
    # camera looking away from the sphere: every chord starts behind the plane
    cam = oracle_mod.camera((500, 500, 2000), (0, 0, 1), 0.0, 400.0, 6, 5)
    jb = oracle_mod.job(cam, sphere_center=(500, 500, 500), sphere_radius=300.0, min_chord=0.0)
    out, st, rc = oracle_mod.render_batched(g, c.rho, [jb])
    assert rc == 0 and np.all(out == 0.0) and st[0] == 0
    # an aperture smaller than half a pixel masks every pixel
    cam2 = oracle_mod.camera((500, 500, 0), (0, 0, 1), 0.0, 400.0, 6, 6)
    jb2 = oracle_mod.job(cam2, z_range=1000.0, aperture_radius=1e-3)
    out, st, rc = oracle_mod.render_batched(g, np.stack([c.rho] * 3, 1), [jb2])
    assert rc == 0 and np.all(out == 0.0) and st[0] == 0


def test_scale_multiplies_every_channel(oracle_mod):
    c, pts, g = _grid(oracle_mod, n=5_000, seed=45)
    cam = oracle_mod.camera((500, 500, 0), (0, 0, 1), 0.0, 600.0, 5, 4)
    v = np.stack([c.rho, 2 * c.rho], 1).astype(np.float32)
    a, _, _ = oracle_mod.render_batched(g, v, [oracle_mod.job(cam, z_range=1000.0, scale=1.0)])
    b, _, _ = oracle_mod.render_batched(g, v, [oracle_mod.job(cam, z_range=1000.0, scale=0.25)])
    assert np.array_equal(b, (a * np.float32(0.25)).astype(np.float32))
