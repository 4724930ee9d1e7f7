"""CPU checks of the oracle adjoint: the gradient of
L = sum_pixels (log I - log I_target)^2 with respect to per-cell log density
and log temperature, with the step sequence frozen from the forward pass and
the neighbour choice fixed, against central finite differences (h = 1e-3) of
the same frozen-sequence function in double precision."""
import numpy as np

H = 1e-3
Z, DL, EMIN, EMAX, NS = 0.2, 978500.0, 0.5, 7.0, 100


def _problem(oracle_mod, gaunt_table):
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(3000, seed=31, box=300.0, r_s=40.0)
    cam = oracle_mod.camera((150, 150, 0), (0, 0, 1), 0.0, 120.0, 10, 10)
    q = oracle_mod.xray_band(gaunt_table, c.rho, c.u, c.xe, Z, DL, EMIN, EMAX, NS, precision=1)
    g = oracle_mod.Grid(c.xyzq(q))
    _, hs, n, rc = g.render_record(cam, 300.0, 0.0, 1e-3, mode=1, cap=8192)
    assert rc == 0
    return c, cam, q, g, hs, n


def _loss(oracle_mod, gaunt_table, c, cam, hs, n, rho, u, target):
    q = oracle_mod.xray_band(gaunt_table, rho, u, c.xe, Z, DL, EMIN, EMAX, NS, precision=1)
    g = oracle_mod.Grid(c.xyzq(q))
    I = g.render_replay(cam, hs, n, precision=1).astype(np.float64)
    return float(np.sum((np.log(I) - np.log(target)) ** 2))


def test_band_flux_dlnT_matches_finite_differences(oracle_mod, gaunt_table):
    from illcrawl_b200 import synthetic
    c = synthetic.small_cells(64, seed=4, box=300.0, r_s=40.0)
    q, dq, _ = oracle_mod.xray_band_grad(gaunt_table, c.rho, c.u, c.xe, Z, DL, EMIN, EMAX, NS,
                                         precision=1)
    h = 1e-4  # small step: fewer stencils straddle a texel edge of the Gaunt table
    up = oracle_mod.xray_band(gaunt_table, c.rho, (c.u * np.exp(h)).astype(np.float32), c.xe,
                              Z, DL, EMIN, EMAX, NS, precision=1).astype(np.float64)
    dn = oracle_mod.xray_band(gaunt_table, c.rho, (c.u * np.exp(-h)).astype(np.float32), c.xe,
                              Z, DL, EMIN, EMAX, NS, precision=1).astype(np.float64)
    # u is rounded to float32, so use the exact ln-ratio of the perturbed inputs
    lr = np.log((c.u * np.exp(h)).astype(np.float32).astype(np.float64)) - \
        np.log((c.u * np.exp(-h)).astype(np.float32).astype(np.float64))
    fd = (up - dn) / lr
    ok = np.abs(q) > 0
    rel = np.abs(dq[ok] - fd[ok]) / np.maximum(np.abs(fd[ok]), 1e-30)
    # The Gaunt factor is a bilinear table: where the +-h stencil straddles a
    # texel edge the difference quotient averages two slopes, so a few cells
    # deviate at the 1e-3 level; at h = 1e-4 the float32 rounding of q limits
    # the difference quotient to ~5e-4.
    assert np.median(rel) < 5e-4 and rel.max() < 2e-3


def test_oracle_adjoint_matches_central_differences(oracle_mod, gaunt_table):
    c, cam, q, g, hs, n = _problem(oracle_mod, gaunt_table)
    I = g.render_replay(cam, hs, n, precision=1).astype(np.float64)
    rng = np.random.default_rng(5)
    target = I * np.exp(0.2 * rng.normal(size=I.shape))
    gI = 2.0 * (np.log(I) - np.log(target)) / I
    grad_q = oracle_mod.adjoint(g, cam, hs, n, gI, precision=1)
    _, dq, dqr = oracle_mod.xray_band_grad(gaunt_table, c.rho, c.u, c.xe, Z, DL, EMIN, EMAX, NS,
                                           precision=1)
    g_lnrho = grad_q * dqr
    g_lnT = grad_q * dq
    # cells with the largest gradients plus random ones
    pick = list(np.argsort(-np.abs(g_lnrho))[:5]) + list(rng.choice(c.n, 3, replace=False))
    for p in pick:
        for which in ("rho", "T"):
            rho_p, rho_m = c.rho.copy(), c.rho.copy()
            u_p, u_m = c.u.copy(), c.u.copy()
            if which == "rho":
                rho_p[p] = np.float32(c.rho[p] * np.exp(H))
                rho_m[p] = np.float32(c.rho[p] * np.exp(-H))
                lr = np.log(np.float64(rho_p[p])) - np.log(np.float64(rho_m[p]))
                an = g_lnrho[p]
            else:
                u_p[p] = np.float32(c.u[p] * np.exp(H))
                u_m[p] = np.float32(c.u[p] * np.exp(-H))
                lr = np.log(np.float64(u_p[p])) - np.log(np.float64(u_m[p]))
                an = g_lnT[p]
            fd = (_loss(oracle_mod, gaunt_table, c, cam, hs, n, rho_p, u_p, target) -
                  _loss(oracle_mod, gaunt_table, c, cam, hs, n, rho_m, u_m, target)) / lr
            scale = max(abs(fd), abs(an), 1e-12 * np.abs(g_lnrho).max())
            assert abs(an - fd) <= 1e-3 * scale + 1e-9 * np.abs(g_lnrho).max(), (p, which, an, fd)
