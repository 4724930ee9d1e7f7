"""The adjoint at the benchmark's adjoint workload: the 512^2 X-ray band map of
the 4,194,304 seeded cells, loss L = sum over pixels (log I - log I_t)^2 with
I_t rendered from the same cells with log T + a seeded Gaussian random field
(sigma 0.1, correlation length 200 kpc), gradient with respect to per-cell
ln rho and ln T (8.4 M parameters), the step sequence frozen from the forward
pass.

The C ABI's adjoint is wrapped in a torch.autograd.Function here, in the test
harness only, and checked
* against central finite differences (h = 1e-3 in ln rho and ln T) of the
  same frozen-sequence loss on 64 seeded cells, evaluated by the GPU frozen
  replay with the step increments summed in double;
* against the FP64 oracle's gradient on a subset of rays;
* checkpoint against recompute mode.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BOX, SIDE, REL_TOL = 6000.0, 512, 1e-3
Z, DL, EMIN, EMAX, NS = 0.2, 978500.0, 0.5, 7.0, 100
CAM = ((BOX / 2, BOX / 2, 0.0), (0.0, 0.0, 1.0), 0.0, BOX, SIDE, SIDE)
H = 1e-3
CAP = 24576   # recorded steps per ray (the longest rays of this map take ~19,000)


@pytest.fixture(scope="module")
def problem(ctx):
    import illcrawl_b200 as ilc
    from illcrawl_b200 import synthetic
    cells = synthetic.xray_cells()
    field = synthetic.gaussian_random_field_at(cells.pos, BOX, 0.1, 200.0, 256, 20174)
    u_t = synthetic.perturbed_internal_energy(cells, field)
    ctx.load_gaunt()
    xyz0 = cells.xyzq(np.zeros(cells.n, np.float32))
    target, _ = ctx.project_xray_flux(xyz0, cells.rho, u_t, cells.xe, ilc.camera(*CAM), BOX,
                                      rel_tol=REL_TOL, e_min=EMIN, e_max=EMAX, num_samples=NS)
    return cells, xyz0, target


def make_loss_function(ctx, cells, xyz0, target, mode):
    """L(ln rho, ln u) through ilc_adjoint_xray_flux; ln T = ln u + const at
    fixed x_e, so dL/dln u is the adjoint's dL/dln T."""
    import torch
    import illcrawl_b200 as ilc

    class XrayBandLoss(torch.autograd.Function):
        @staticmethod
        def forward(fctx, ln_rho, ln_u):
            rho = torch.exp(ln_rho).to(torch.float32).cpu().numpy()
            u = torch.exp(ln_u).to(torch.float32).cpu().numpy()
            img, g_r, g_t, st = ctx.adjoint_xray_flux(xyz0, rho, u, cells.xe, ilc.camera(*CAM),
                                                      BOX, target, mode=mode, rel_tol=REL_TOL,
                                                      e_min=EMIN, e_max=EMAX, num_samples=NS)
            fctx.save_for_backward(torch.from_numpy(g_r), torch.from_numpy(g_t))
            fctx.stats = st
            XrayBandLoss.last = (img, st)
            return torch.tensor(st["loss"], dtype=torch.float64)

        @staticmethod
        def backward(fctx, grad_out):
            g_r, g_t = fctx.saved_tensors
            return grad_out * g_r.double(), grad_out * g_t.double()

    return XrayBandLoss


@pytest.fixture(scope="module")
def gradients(ctx, problem):
    """Checkpoint-mode gradient through autograd."""
    import torch
    cells, xyz0, target = problem
    F = make_loss_function(ctx, cells, xyz0, target, 0)
    ln_rho = torch.from_numpy(np.log(cells.rho.astype(np.float64))).requires_grad_()
    ln_u = torch.from_numpy(np.log(cells.u.astype(np.float64))).requires_grad_()
    loss = F.apply(ln_rho, ln_u)
    loss.backward()
    img, st = F.last
    return ln_rho.grad.numpy().copy(), ln_u.grad.numpy().copy(), img, st


def test_autograd_wrapper_and_cost(ctx, problem, gradients):
    """The autograd gradient is the C ABI's, recompute mode agrees with
    checkpoint mode, and one adjoint pass costs at most 3 forward passes."""
    import torch
    cells, xyz0, target = problem
    g_r, g_t, img, st = gradients
    assert np.all(np.isfinite(g_r)) and np.all(np.isfinite(g_t))
    assert np.count_nonzero(g_r) > cells.n // 100
    F1 = make_loss_function(ctx, cells, xyz0, target, 1)
    a = torch.from_numpy(np.log(cells.rho.astype(np.float64))).requires_grad_()
    b = torch.from_numpy(np.log(cells.u.astype(np.float64))).requires_grad_()
    F1.apply(a, b).backward()
    r1, t1 = a.grad.numpy(), b.grad.numpy()
    assert np.linalg.norm(g_r - r1) / np.linalg.norm(g_r) < 1e-5
    assert np.linalg.norm(g_t - t1) / np.linalg.norm(g_t) < 1e-5
    _, st1 = F1.last
    for s in (st, st1):
        ratio = s["adjoint_ms"] / s["forward_ms"]
        print("adjoint / forward:", ratio, s)
        assert ratio <= 3.0


def _record(ctx, cam):
    """The forward pass's accepted step sizes, recorded on the device."""
    import torch
    import illcrawl_b200 as ilc
    rays = SIDE * SIDE
    hs = torch.empty((rays, CAP), dtype=torch.float32, device="cuda:0")
    n = torch.empty(rays, dtype=torch.int32, device="cuda:0")
    img = np.zeros((SIDE, SIDE), np.float32)
    st = ilc.RenderStats()
    ctx.check(ctx.L.ilc_render_record(ctx.h, ctypes.byref(cam), BOX,
                                      ilc.Tolerance(0.0, REL_TOL), ilc.CONTROLLER_FP64,
                                      ctypes.c_void_p(hs.data_ptr()),
                                      ctypes.c_void_p(n.data_ptr()), CAP, 1,
                                      img.ctypes.data_as(ctypes.c_void_p), 0, ctypes.byref(st)))
    return hs, n, img


def _replay64(ctx, cam, hs, n):
    import illcrawl_b200 as ilc
    out = np.zeros((SIDE, SIDE), np.float64)
    st = ilc.RenderStats()
    ctx.check(ctx.L.ilc_render_frozen_f64(ctx.h, ctypes.byref(cam), BOX,
                                          ctypes.c_void_p(hs.data_ptr()),
                                          ctypes.c_void_p(n.data_ptr()), CAP, 1, None,
                                          out.ctypes.data_as(ctypes.c_void_p), 0,
                                          ctypes.byref(st)))
    return out


def _pixel_cells(ctx, cam, axis):
    """Grid cell index of every pixel's ray along x (axis 0) or y (axis 1):
    the ray of a view along z keeps its x and y."""
    import illcrawl_b200 as ilc
    d = ctx.grid_describe()
    plane = ilc.camera_plane(cam)   # look(3), b0(3), b1(3), min corner(3), pixel size
    f = np.float32
    i = np.arange(SIDE, dtype=np.float32)
    t = i * f(plane[12])
    # pixel corner coordinate along the axis; the other term is 0 for this view
    base = f(plane[9 + axis]) + t * f(plane[3 + 3 * axis + axis])
    return np.floor((base - d["min_corner"][axis]) / d["cell_sizes"][axis]).astype(np.int64)


def test_adjoint_matches_central_differences_on_64_cells(ctx, problem, gradients, oracle_mod,
                                                         gaunt_table):
    """Central differences (h = 1e-3) of the frozen-sequence loss for 64
    seeded cells, each perturbation of all 64 cells in one replay: a cell can
    only change rays whose walks reach its grid cell, i.e. rays within 2 grid
    cells of it in x and y (the spiral order spans offsets -2..2), so cells
    whose windows of +-3 grid cells do not overlap are separated by summing
    the per-pixel loss change over each window."""
    import illcrawl_b200 as ilc
    cells, xyz0, target = problem
    g_r, g_t, img, st = gradients
    cam = ilc.camera(*CAM)
    q = ctx.xray_flux(cells.rho, cells.u, cells.xe, Z, DL, EMIN, EMAX, NS)
    ctx.setup_particles(cells.xyzq(q))
    hs, n, rimg = _record(ctx, cam)
    assert np.array_equal(rimg.view(np.uint32), img.view(np.uint32))
    d = ctx.grid_describe()
    cell_of = np.floor((cells.pos - d["min_corner"]) / d["cell_sizes"]).astype(np.int64)
    px_cx, px_cy = _pixel_cells(ctx, cam, 0), _pixel_cells(ctx, cam, 1)
    # 64 seeded cells among those with a gradient of at least 1e-3 of the largest
    big = np.nonzero((np.abs(g_r) > 1e-3 * np.abs(g_r).max()) &
                     (np.abs(g_t) > 1e-3 * np.abs(g_t).max()))[0]
    rng = np.random.default_rng(20173)
    chosen, taken = [], []
    for p in rng.permutation(big):
        c = cell_of[p]
        if all(max(abs(c[0] - o[0]), abs(c[1] - o[1])) > 6 for o in taken):
            chosen.append(p)
            taken.append(c)
        if len(chosen) == 64:
            break
    assert len(chosen) == 64
    chosen = np.array(chosen)
    win = []
    for p in chosen:
        c = cell_of[p]
        mx = np.abs(px_cx - c[0]) <= 3
        my = np.abs(px_cy - c[1]) <= 3
        win.append(np.outer(my, mx))   # (y, x)
    tgt = target.astype(np.float64)

    def window_losses(I):
        with np.errstate(divide="ignore", invalid="ignore"):
            term = np.where((I > 0) & (tgt > 0), (np.log(I) - np.log(tgt)) ** 2, 0.0)
        return np.array([term[w].sum() for w in win])

    scale = 1.0   # the adjoint's loss uses the unscaled map (no scaling given)
    fd = {}
    for which in ("rho", "T"):
        res = []
        for sgn in (1.0, -1.0):
            rho, u = cells.rho.copy(), cells.u.copy()
            if which == "rho":
                rho[chosen] = (cells.rho[chosen] * np.exp(sgn * H)).astype(np.float32)
            else:
                u[chosen] = (cells.u[chosen] * np.exp(sgn * H)).astype(np.float32)
            qs = ctx.xray_flux(rho, u, cells.xe, Z, DL, EMIN, EMAX, NS)
            ctx.setup_particles(cells.xyzq(qs))
            res.append((window_losses(_replay64(ctx, cam, hs, n) * scale),
                        rho[chosen].astype(np.float64), u[chosen].astype(np.float64)))
        (lp, rp, up), (lm, rm, um) = res
        lr = np.log(rp) - np.log(rm) if which == "rho" else np.log(up) - np.log(um)
        fd[which] = (lp - lm) / lr
    ctx.setup_particles(cells.xyzq(q))
    # q is proportional to rho^2 (the energy integration's steps do not depend
    # on the scale), but its T dependence runs through the bilinear Gaunt
    # table: a cell whose +-h stencil straddles a texel edge has a difference
    # quotient that averages two slopes. Such cells are found per cell, on q
    # itself, and left out of the T comparison.
    oracle, tab = oracle_mod, gaunt_table
    r_, u_, x_ = cells.rho[chosen], cells.u[chosen], cells.xe[chosen]
    _, dq, _ = oracle.xray_band_grad(tab, r_, u_, x_, Z, DL, EMIN, EMAX, NS, precision=1)
    up = (u_ * np.exp(H)).astype(np.float32)
    dn = (u_ * np.exp(-H)).astype(np.float32)
    qp = oracle.xray_band(tab, r_, up, x_, Z, DL, EMIN, EMAX, NS, precision=1)
    qm = oracle.xray_band(tab, r_, dn, x_, Z, DL, EMIN, EMAX, NS, precision=1)
    lr = np.log(up.astype(np.float64)) - np.log(dn.astype(np.float64))
    dq_fd = (qp.astype(np.float64) - qm.astype(np.float64)) / lr
    smooth = np.abs(dq_fd - dq) <= 1e-4 * np.abs(dq)
    print("cells whose q is smooth in T over the stencil:", int(smooth.sum()), "of 64")
    assert smooth.sum() >= 48
    worst = 0.0
    for which, an_all, keep in (("rho", g_r, np.ones(64, bool)), ("T", g_t, smooth)):
        an = an_all[chosen].astype(np.float64)[keep]
        f = fd[which][keep]
        err = np.abs(an - f) / np.maximum(np.abs(f), 1e-6 * np.abs(an_all).max())
        print(which, "FD vs adjoint on", int(keep.sum()), "cells: median", np.median(err),
              "max", err.max())
        worst = max(worst, err.max())
    assert worst < 1e-3


def test_adjoint_matches_oracle_gradients_on_a_ray_subset(ctx, problem, oracle_mod, gaunt_table):
    """The target equals the forward map except on 24 seeded rays, so only
    those rays seed the adjoint. Their gradient against the oracle's adjoint
    of the same rays and recorded steps: the fp32 oracle (same arithmetic as
    the kernels, other summation order) to 1e-4, and the FP64 oracle within
    the deviation the fp32 oracle itself has from it. That deviation comes
    from the fp32 ray positions: z summed in fp32 over ~14,000 steps, as the
    reference's integrator sums it, places the evaluation points up to ~1 kpc
    off the FP64 positions, which moves weight between neighbouring cells."""
    import illcrawl_b200 as ilc
    cells, xyz0, target = problem
    cam = ilc.camera(*CAM)
    img, _, _, _ = ctx.adjoint_xray_flux(xyz0, cells.rho, cells.u, cells.xe, cam, BOX, target,
                                         mode=1, rel_tol=REL_TOL, e_min=EMIN, e_max=EMAX,
                                         num_samples=NS)
    rng = np.random.default_rng(77)
    flat = img.ravel()
    pix = np.sort(rng.choice(np.nonzero(flat > np.quantile(flat, 0.5))[0], 24, replace=False))
    t2 = flat.copy()
    t2[pix] = target.ravel()[pix]
    t2 = t2.reshape(SIDE, SIDE)
    img2, g_r, g_t, st = ctx.adjoint_xray_flux(xyz0, cells.rho, cells.u, cells.xe, cam, BOX, t2,
                                               mode=0, rel_tol=REL_TOL, e_min=EMIN, e_max=EMAX,
                                               num_samples=NS)
    assert np.array_equal(img2.view(np.uint32), img.view(np.uint32))
    q32 = oracle_mod.xray_band(gaunt_table, cells.rho, cells.u, cells.xe, Z, DL, EMIN, EMAX, NS)
    g = oracle_mod.Grid(cells.xyzq(q32))
    ocam = oracle_mod.camera(*CAM)
    I, hs, nacc, rc = g.render_record(ocam, BOX, 0.0, REL_TOL, mode=1, pix=pix, cap=CAP)
    assert rc == 0
    assert np.array_equal(I.view(np.uint32), flat[pix].view(np.uint32))
    Id = I.astype(np.float64)
    gI = 2.0 * (np.log(Id) - np.log(t2.ravel()[pix].astype(np.float64))) / Id
    grad64 = np.asarray(oracle_mod.adjoint(g, ocam, hs, nacc, gI, pix=pix, precision=1))
    grad32 = np.asarray(oracle_mod.adjoint(g, ocam, hs, nacc, gI, pix=pix, precision=0),
                        np.float64)
    for prec in (0, 1):
        _, dqT, dqR = oracle_mod.xray_band_grad(gaunt_table, cells.rho, cells.u, cells.xe, Z,
                                                DL, EMIN, EMAX, NS, precision=prec)
        for name, dq, got in (("rho", dqR, g_r), ("T", dqT, g_t)):
            got = got.astype(np.float64)
            if prec == 0:
                want = grad32 * dq
                big = np.abs(want) > 1e-2 * np.abs(want).max()
                rel = np.abs(got[big] - want[big]) / np.abs(want[big])
                print(name, "vs fp32 oracle on 24 rays: max", rel.max())
                assert rel.max() < 1e-4
            else:
                want = grad64 * dq
                o32 = grad32 * dq
                err = np.linalg.norm(got - want) / np.linalg.norm(want)
                err32 = np.linalg.norm(o32 - want) / np.linalg.norm(want)
                big = np.abs(want) > 1e-2 * np.abs(want).max()
                rel = np.abs(got[big] - want[big]) / np.abs(want[big])
                rel32 = np.abs(o32[big] - want[big]) / np.abs(want[big])
                print(name, "vs FP64 oracle on 24 rays: norm", err, "q0.99",
                      np.quantile(rel, 0.99), "max", rel.max(), "| fp32 oracle vs FP64: norm",
                      err32, "q0.99", np.quantile(rel32, 0.99))
                assert err < 1.05 * err32 + 1e-5
                assert np.quantile(rel, 0.99) < 1.05 * np.quantile(rel32, 0.99) + 1e-4
                assert err < 1e-2
