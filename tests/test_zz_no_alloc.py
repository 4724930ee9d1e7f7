"""The allocation-free grid build (ilc_grid_build_noalloc) gives the same grid
as the regular entry point (ilc_nn8_setup_particles + ilc_grid_export).

It serves callers that cannot allocate device memory where they need a grid
(fixed-budget real-time loops, hosts whose allocator owns the device memory):
the test owns every device buffer and the entry point only uses its fixed
internal scratch array. Two calls in a row check that the shared scratch left
by one call does not leak into the next, and a build of exactly
ILC_NOALLOC_MAX_PARTICLES particles fills every region of the scratch array.
This file is collected last, so a run that stops at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc_build(lib, torch, pts):
    import illcrawl_b200 as ilc
    dev = torch.device("cuda", 0)
    n = pts.shape[0]
    d_in = torch.from_numpy(pts).to(dev)
    d_sorted = torch.empty((n, 4), dtype=torch.float32, device=dev)
    d_s2u = torch.empty(n, dtype=torch.int32, device=dev)
    desc = ilc._lib.GridDesc()
    cap = max(64, n)  # first call: a guess; the descriptor reports what is needed
    for _ in range(2):
        d_cells = torch.empty((cap, 2), dtype=torch.int32, device=dev)
        st = lib.ilc_grid_build_noalloc(
            ctypes.c_void_p(d_in.data_ptr()), n, ctypes.c_void_p(d_sorted.data_ptr()),
            ctypes.c_void_p(d_cells.data_ptr()), cap, ctypes.c_void_p(d_s2u.data_ptr()),
            ctypes.byref(desc), None)
        if st == 0:
            break
        assert st == 1 and desc.total_cells > cap  # too small: size from the descriptor
        cap = int(desc.total_cells)
    assert st == 0
    total = int(desc.total_cells)
    return (np.array(desc.min_corner, np.float32), np.array(desc.cell_sizes, np.float32),
            np.array(desc.num_cells, np.int32), d_cells[:total].cpu().numpy(),
            d_s2u.cpu().numpy().view(np.uint32), d_sorted.cpu().numpy())


def test_noalloc_grid_matches_regular_entry_point_twice(ctx):
    import torch
    from illcrawl_b200 import synthetic
    lib = ctx.L
    for seed, n in ((61, 200_000), (62, 50_000)):   # two calls in a row, different sizes
        c = synthetic.small_cells(n, seed=seed)
        pts = c.xyzq(c.rho)
        mn, cs, nc, cells, s2u, srt = _noalloc_build(lib, torch, pts)
        ctx.setup_particles(pts)
        d = ctx.grid_describe()
        rcells, rs2u, rsrt = ctx.grid_export()
        assert np.array_equal(mn, d["min_corner"]) and np.array_equal(cs, d["cell_sizes"])
        assert np.array_equal(nc, d["num_cells"])
        assert np.array_equal(cells, rcells)
        assert np.array_equal(s2u, rs2u)
        assert np.array_equal(srt.view(np.uint32), rsrt.view(np.uint32))


def test_noalloc_grid_at_its_maximum_size(ctx):
    """n = ILC_NOALLOC_MAX_PARTICLES: all 512 sort tiles and the whole key,
    value and histogram regions of the scratch array are in use."""
    import torch
    from illcrawl_b200 import synthetic
    lib = ctx.L
    n = 1 << 20
    c = synthetic.small_cells(n, seed=63)
    pts = c.xyzq(c.rho)
    mn, cs, nc, cells, s2u, srt = _noalloc_build(lib, torch, pts)
    ctx.setup_particles(pts)
    d = ctx.grid_describe()
    rcells, rs2u, rsrt = ctx.grid_export()
    assert np.array_equal(mn, d["min_corner"]) and np.array_equal(cs, d["cell_sizes"])
    assert np.array_equal(nc, d["num_cells"])
    assert np.array_equal(cells, rcells)
    assert np.array_equal(s2u, rs2u)
    assert np.array_equal(srt.view(np.uint32), rsrt.view(np.uint32))


def test_noalloc_rejects_more_than_its_maximum(ctx):
    import torch
    import illcrawl_b200 as ilc
    lib = ctx.L
    n = (1 << 20) + 1
    d = torch.zeros((8, 4), dtype=torch.float32, device="cuda:0")
    desc = ilc._lib.GridDesc()
    st = lib.ilc_grid_build_noalloc(ctypes.c_void_p(d.data_ptr()), n,
                                    ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(d.data_ptr()),
                                    8, ctypes.c_void_p(d.data_ptr()), ctypes.byref(desc), None)
    assert st == 1


def test_noalloc_rejects_a_grid_beyond_2_32_cells(ctx):
    """Particles 1e30 apart along x: the cells per axis do not fit an int32;
    the call reports ILC_ERR_GRID_TOO_LARGE before it writes any output."""
    import torch
    import illcrawl_b200 as ilc
    lib = ctx.L
    pts = torch.tensor([[0, 0, 0, 1], [1e30, 0, 0, 1], [5e29, 0, 0, 1]], dtype=torch.float32,
                       device="cuda:0")
    out = torch.zeros((8, 4), dtype=torch.float32, device="cuda:0")
    desc = ilc._lib.GridDesc()
    st = lib.ilc_grid_build_noalloc(ctypes.c_void_p(pts.data_ptr()), 3,
                                    ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                    8, ctypes.c_void_p(out.data_ptr()), ctypes.byref(desc), None)
    assert st == 8  # ILC_ERR_GRID_TOO_LARGE
    assert torch.count_nonzero(out).item() == 0
