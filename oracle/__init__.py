"""ctypes bindings to the CPU oracle (``oracle/libilc_oracle.so``).

Test infrastructure only: imported by ``tests/``, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` / ``--impl reference`` legs of ``bench.py``, where
it is the checker and the timed CPU restatement. The product package
``illcrawl_b200`` never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libilc_oracle.so")
_lib = None


class OracleCamera(ctypes.Structure):
    _fields_ = [("position", ctypes.c_double * 3), ("look_at", ctypes.c_double * 3),
                ("roll", ctypes.c_double), ("screen_width", ctypes.c_double),
                ("nx", ctypes.c_int32), ("ny", ctypes.c_int32)]


def build():
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    P = ctypes.c_void_p
    i64, i32, f32, f64 = ctypes.c_int64, ctypes.c_int32, ctypes.c_float, ctypes.c_double
    L.orc_spiral_table.argtypes = [P]
    L.orc_logf.argtypes = [f32]; L.orc_logf.restype = f32
    L.orc_expf.argtypes = [f32]; L.orc_expf.restype = f32
    L.orc_grid_build.argtypes = [P, i64, P]; L.orc_grid_build.restype = P
    L.orc_grid_free.argtypes = [P]
    L.orc_grid_info.argtypes = [P, P, P, P, P]
    L.orc_grid_export.argtypes = [P, P, P, P, P]
    L.orc_nn8_query.argtypes = [P, P, i64, ctypes.c_int, P, P, P, P, ctypes.c_int]
    L.orc_camera_setup.argtypes = [P, P]
    L.orc_render.argtypes = [P, P, f64, f64, f64, ctypes.c_int, i64, P, i64, P, P, P, P,
                             ctypes.c_int]
    L.orc_render_fixed.argtypes = [P, P, f64, i64, ctypes.c_int, P, i64, P, P, ctypes.c_int]
    L.orc_render_record.argtypes = [P, P, f64, f64, f64, ctypes.c_int, i64, P, i64, P, P, i64,
                                    P, ctypes.c_int]
    L.orc_render_replay.argtypes = [P, P, P, i64, P, i64, P, ctypes.c_int, P, P, ctypes.c_int]
    L.orc_los_scale.argtypes = [P, f64, f64, f64, ctypes.c_int]; L.orc_los_scale.restype = f32
    L.orc_gaunt_lookup.argtypes = [P, ctypes.c_int, ctypes.c_int, f32, f32]
    L.orc_gaunt_lookup.restype = f32
    L.orc_temperature.argtypes = [P, P, i64, P]
    L.orc_xray_band.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, i64, f32, f32, f32, f32,
                                ctypes.c_int, ctypes.c_int, P, ctypes.c_int]
    L.orc_xray_bin.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, i64, f32, f32, f32, f32,
                               ctypes.c_int, P, ctypes.c_int]
    L.orc_xray_photon_flux.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, i64, f32, f32,
                                       f32, f32, ctypes.c_int, ctypes.c_int, P, ctypes.c_int]
    L.orc_chandra_count_rate.argtypes = [P, ctypes.c_int, ctypes.c_int, P, ctypes.c_int, f32,
                                         f32, P, P, P, i64, f32, f32, ctypes.c_int, P,
                                         ctypes.c_int]
    L.orc_chandra_spectral_count_rate.argtypes = [P, ctypes.c_int, ctypes.c_int, P,
                                                  ctypes.c_int, f32, f32, P, P, P, i64, f32,
                                                  f32, f32, f32, ctypes.c_int, P, ctypes.c_int]


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def camera(position, look_at, roll, screen_width, nx, ny):
    c = OracleCamera()
    c.position[:] = [float(v) for v in position]
    c.look_at[:] = [float(v) for v in look_at]
    c.roll, c.screen_width, c.nx, c.ny = float(roll), float(screen_width), int(nx), int(ny)
    return c


def spiral_table():
    out = np.zeros((8, 125, 3), np.int8)
    lib().orc_spiral_table(_p(out))
    return out


def logf(x):
    return np.float32(lib().orc_logf(float(x)))


def expf(x):
    return np.float32(lib().orc_expf(float(x)))


class Grid:
    """Grid built by the oracle from float4 (x, y, z, q) particles."""

    def __init__(self, xyzq):
        self.xyzq = np.ascontiguousarray(xyzq, np.float32).reshape(-1, 4)
        st = ctypes.c_int32(0)
        self.h = lib().orc_grid_build(_p(self.xyzq), self.xyzq.shape[0], ctypes.byref(st))
        if not self.h:
            raise ValueError(f"oracle grid build failed (status {st.value})")
        mn = np.zeros(3, np.float32); cs = np.zeros(3, np.float32)
        n3 = np.zeros(3, np.int32); tot = np.zeros(1, np.uint64)
        lib().orc_grid_info(self.h, _p(mn), _p(cs), _p(n3), _p(tot))
        self.min_corner, self.cell_sizes, self.num_cells = mn, cs, n3
        self.total_cells = int(tot[0])

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_grid_free(self.h)
            self.h = None

    def export(self):
        n = self.xyzq.shape[0]
        cells = np.zeros((self.total_cells, 2), np.int32)
        s2u = np.zeros(n, np.uint32)
        srt = np.zeros((n, 4), np.float32)
        keys = np.zeros(n, np.uint64)
        lib().orc_grid_export(self.h, _p(cells), _p(s2u), _p(srt), _p(keys))
        return cells, s2u, srt, keys

    def nn8(self, pts, precision=0, nthreads=0, slots=True):
        pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 4)
        n = pts.shape[0]
        out = np.zeros(n, np.float32)
        idx = np.zeros((n, 8), np.int32) if slots else None
        d8 = np.zeros((n, 8), np.float32) if slots else None
        st = np.zeros(2, np.uint64)
        lib().orc_nn8_query(self.h, _p(pts), n, precision, _p(out), _p(idx), _p(d8), _p(st),
                            nthreads)
        return out, idx, d8, st

    def render(self, cam, z_range, atol, rtol, mode=0, pix=None, max_steps=1 << 22, nthreads=0):
        npix = cam.nx * cam.ny if pix is None else len(pix)
        pixa = None if pix is None else np.ascontiguousarray(pix, np.int64)
        out = np.zeros(npix, np.float32)
        steps = np.zeros(npix, np.int32); acc = np.zeros(npix, np.int32)
        st = np.zeros(2, np.uint64)
        rc = lib().orc_render(self.h, ctypes.byref(cam), z_range, atol, rtol, mode, max_steps,
                              _p(pixa), npix, _p(out), _p(steps), _p(acc), _p(st), nthreads)
        return out, steps, acc, st, rc

    def render_fixed(self, cam, z_range, n_steps, precision=0, pix=None, nthreads=0):
        npix = cam.nx * cam.ny if pix is None else len(pix)
        pixa = None if pix is None else np.ascontiguousarray(pix, np.int64)
        out = np.zeros(npix, np.float32)
        st = np.zeros(2, np.uint64)
        lib().orc_render_fixed(self.h, ctypes.byref(cam), z_range, n_steps, precision,
                               _p(pixa), npix, _p(out), _p(st), nthreads)
        return out, st

    def render_record(self, cam, z_range, atol, rtol, mode=0, pix=None, cap=4096,
                      max_steps=1 << 22, nthreads=0):
        npix = cam.nx * cam.ny if pix is None else len(pix)
        pixa = None if pix is None else np.ascontiguousarray(pix, np.int64)
        out = np.zeros(npix, np.float32)
        hs = np.zeros((npix, cap), np.float32)
        n = np.zeros(npix, np.int32)
        rc = lib().orc_render_record(self.h, ctypes.byref(cam), z_range, atol, rtol, mode,
                                     max_steps, _p(pixa), npix, _p(out), _p(hs), cap, _p(n),
                                     nthreads)
        return out, hs, n, rc

    def render_replay(self, cam, hs, n, pix=None, precision=0, nthreads=0):
        hs = np.ascontiguousarray(hs, np.float32)
        npix = hs.shape[0]
        pixa = None if pix is None else np.ascontiguousarray(pix, np.int64)
        n = np.ascontiguousarray(n, np.int32)
        out = np.zeros(npix, np.float32)
        out_d = np.zeros(npix, np.float64) if precision == 1 else None
        lib().orc_render_replay(self.h, ctypes.byref(cam), _p(pixa), npix, _p(hs), hs.shape[1],
                                _p(n), precision, _p(out), _p(out_d), nthreads)
        return out if out_d is None else out_d


def camera_setup(cam):
    out = np.zeros(13, np.float32)
    lib().orc_camera_setup(ctypes.byref(cam), _p(out))
    return out


def los_scale(cam, z_range, length_conv=1.0, area_conv=1.0, dA_mode=0):
    return np.float32(lib().orc_los_scale(ctypes.byref(cam), z_range, length_conv, area_conv,
                                          dA_mode))


def gaunt_lookup(table, lg, lu):
    t = np.ascontiguousarray(table, np.float32)
    return np.float32(lib().orc_gaunt_lookup(_p(t), t.shape[1], t.shape[0], float(lg), float(lu)))


def temperature(u, xe):
    u = np.ascontiguousarray(u, np.float32); xe = np.ascontiguousarray(xe, np.float32)
    out = np.zeros_like(u)
    lib().orc_temperature(_p(u), _p(xe), u.size, _p(out))
    return out


def xray_band(table, rho, u, xe, z, dL, Emin, Emax, num_samples, precision=0, nthreads=0):
    t = np.ascontiguousarray(table, np.float32)
    rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
    out = np.zeros_like(rho)
    lib().orc_xray_band(_p(t), t.shape[1], t.shape[0], _p(rho), _p(u), _p(xe), rho.size, z, dL,
                        Emin, Emax, num_samples, precision, _p(out), nthreads)
    return out


def xray_bin(table, rho, u, xe, z, dL, E, dE, precision=0, nthreads=0):
    t = np.ascontiguousarray(table, np.float32)
    rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
    out = np.zeros_like(rho)
    lib().orc_xray_bin(_p(t), t.shape[1], t.shape[0], _p(rho), _p(u), _p(xe), rho.size, z, dL,
                       E, dE, precision, _p(out), nthreads)
    return out


def xray_photon_flux(table, rho, u, xe, z, dL, Emin, Emax, num_samples, precision=0,
                     nthreads=0):
    """xray_photon_flux (quantities.cl:640-675) per cell [photons/s/kpc^3/cm^2]."""
    t = np.ascontiguousarray(table, np.float32)
    rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
    out = np.zeros_like(rho)
    lib().orc_xray_photon_flux(_p(t), t.shape[1], t.shape[0], _p(rho), _p(u), _p(xe), rho.size,
                               z, dL, Emin, Emax, num_samples, precision, _p(out), nthreads)
    return out


def chandra_count_rate(table, arf, arf_x0, arf_dx, rho, u, xe, z, dL, precision=0, nthreads=0):
    """chandra_xray_total_count_rate (quantities.cl:510-557) per cell: the
    count rates of all ARF channels x0 + k dx (width dx) summed in order."""
    t = np.ascontiguousarray(table, np.float32)
    a = np.ascontiguousarray(arf, np.float32)
    rho, u, xe = (np.ascontiguousarray(v, np.float32) for v in (rho, u, xe))
    out = np.zeros_like(rho)
    lib().orc_chandra_count_rate(_p(t), t.shape[1], t.shape[0], _p(a), a.size, arf_x0, arf_dx,
                                 _p(rho), _p(u), _p(xe), rho.size, z, dL, precision, _p(out),
                                 nthreads)
    return out


def chandra_spectral_count_rate(table, arf, arf_x0, arf_dx, rho, u, xe, z, dL, E, dE,
                                precision=0, nthreads=0):
    """chandra_xray_spectral_count_rate (quantities.cl:584-622) per cell for
    the channel (E, dE)."""
    t = np.ascontiguousarray(table, np.float32)
    a = np.ascontiguousarray(arf, np.float32)
    rho, u, xe = (np.ascontiguousarray(v, np.float32) for v in (rho, u, xe))
    out = np.zeros_like(rho)
    lib().orc_chandra_spectral_count_rate(_p(t), t.shape[1], t.shape[0], _p(a), a.size, arf_x0,
                                          arf_dx, _p(rho), _p(u), _p(xe), rho.size, z, dL, E, dE,
                                          precision, _p(out), nthreads)
    return out


def _declare_lists(L):
    P = ctypes.c_void_p
    L.orc_nn8_query_lists.argtypes = [P, P, ctypes.c_int64, ctypes.c_int, P, P, P, P,
                                      ctypes.c_int]


def nn8_lists(grid, pts, merge=False, lists=None, nthreads=0):
    """nn8 with explicit running lists (d, v, original id), as the reference's
    multi-block merge. Returns (values, (list_d, list_v, list_id))."""
    L = lib()
    if not getattr(L, "_lists_declared", False):
        _declare_lists(L)
        L._lists_declared = True
    pts = np.ascontiguousarray(pts, np.float32).reshape(-1, 4)
    n = pts.shape[0]
    if lists is None:
        lists = (np.zeros((n, 8), np.float32), np.zeros((n, 8), np.float32),
                 np.zeros((n, 8), np.int32))
    ld, lv, li = (np.ascontiguousarray(a) for a in lists)
    out = np.zeros(n, np.float32)
    L.orc_nn8_query_lists(grid.h, _p(pts), n, int(merge), _p(ld), _p(lv), _p(li), _p(out),
                          nthreads)
    return out, (ld, lv, li)


def _declare_adjoint(L):
    P, i64 = ctypes.c_void_p, ctypes.c_int64
    L.orc_xray_band_grad.argtypes = [P, ctypes.c_int, ctypes.c_int, P, P, P, i64, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                     ctypes.c_int, P, P, P, ctypes.c_int]
    L.orc_adjoint.argtypes = [P, P, P, i64, P, i64, P, P, ctypes.c_int, P, ctypes.c_int]


def _adj_lib():
    L = lib()
    if not getattr(L, "_adj_declared", False):
        _declare_adjoint(L)
        L._adj_declared = True
    return L


def xray_band_grad(table, rho, u, xe, z, dL, Emin, Emax, num_samples, precision=0, nthreads=0):
    """Per-cell band flux q, dq/dlnT and dq/dlnrho (exact derivatives of the
    adaptive energy integration)."""
    t = np.ascontiguousarray(table, np.float32)
    rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
    q = np.zeros_like(rho)
    dq = np.zeros(rho.shape, np.float64)
    dqr = np.zeros(rho.shape, np.float64)
    _adj_lib().orc_xray_band_grad(_p(t), t.shape[1], t.shape[0], _p(rho), _p(u), _p(xe),
                                  rho.size, z, dL, Emin, Emax, num_samples, precision, _p(q),
                                  _p(dq), _p(dqr), nthreads)
    return q, dq, dqr


def adjoint(grid, cam, hs, n, gI, pix=None, precision=1, nthreads=0):
    """sum_k gI[k] * dI_k/dq over frozen step sequences; float64 array in the
    original particle order."""
    hs = np.ascontiguousarray(hs, np.float32)
    n = np.ascontiguousarray(n, np.int32)
    gI = np.ascontiguousarray(gI, np.float64)
    pixa = None if pix is None else np.ascontiguousarray(pix, np.int64)
    grad = np.zeros(grid.xyzq.shape[0], np.float64)
    _adj_lib().orc_adjoint(grid.h, ctypes.byref(cam), _p(pixa), hs.shape[0], _p(hs), hs.shape[1],
                           _p(n), _p(gI), precision, _p(grad), nthreads)
    return grad


# ---- batched render (jobs = cameras with masks and chords, V channels) ----
class OracleJob(ctypes.Structure):
    _fields_ = [("camera", OracleCamera), ("z_range", ctypes.c_double),
                ("aperture_radius", ctypes.c_double), ("sphere_center", ctypes.c_double * 3),
                ("sphere_radius", ctypes.c_double), ("min_chord", ctypes.c_double),
                ("scale", ctypes.c_float), ("pad", ctypes.c_int32),
                ("out_offset", ctypes.c_uint64)]


def _declare_batched(L):
    P, i64 = ctypes.c_void_p, ctypes.c_int64
    L.orc_render_batched.argtypes = [P, P, ctypes.c_int32, P, ctypes.c_int32, ctypes.c_double,
                                     ctypes.c_double, i64, P, i64, ctypes.c_int, P, P,
                                     ctypes.c_int]
    L.orc_ray_span.argtypes = [P, ctypes.c_int32, ctypes.c_int32, P, P, P]


def job(cam, z_range=0.0, aperture_radius=0.0, sphere_center=(0.0, 0.0, 0.0),
        sphere_radius=0.0, min_chord=0.0, scale=1.0, out_offset=0):
    return OracleJob(cam, z_range, aperture_radius, (ctypes.c_double * 3)(*sphere_center),
                     sphere_radius, min_chord, scale, 0, out_offset)


def jobs_array(jobs):
    arr = (OracleJob * len(jobs))()
    for i, j in enumerate(jobs):
        arr[i] = j
    return arr


def render_batched(grid, values, jobs, atol=0.0, rtol=1e-3, rays=None, precision=0,
                   max_steps=1 << 22, nthreads=0):
    """values: (n,) or (n, V) per-cell channels in original order. rays: None
    (whole images at the job offsets; returns the flat image buffer) or an
    (m, 2) array of (job, pixel) pairs (returns m x V). Returns (out, stats4, rc)."""
    L = lib()
    if not hasattr(L, "_batched_declared"):
        _declare_batched(L)
        L._batched_declared = True
    vals = np.ascontiguousarray(values, np.float32)
    V = 1 if vals.ndim == 1 else vals.shape[1]
    arr = jobs_array(jobs)
    if rays is None:
        total = max(int(j.out_offset) + V * j.camera.nx * j.camera.ny for j in jobs)
        out = np.zeros(total, np.float32)
        ra, nr = None, 0
    else:
        ra = np.ascontiguousarray(rays, np.int64).reshape(-1, 2)
        nr = ra.shape[0]
        out = np.zeros((nr, V), np.float32)
    st = np.zeros(4, np.uint64)
    rc = L.orc_render_batched(grid.h, _p(vals), V, ctypes.byref(arr), len(jobs), atol, rtol,
                              max_steps, _p(ra), nr, precision, _p(out), _p(st), nthreads)
    return out, st, rc


def ray_span(jb, ix, iy):
    L = lib()
    if not hasattr(L, "_batched_declared"):
        _declare_batched(L)
        L._batched_declared = True
    m = ctypes.c_int32(0)
    o = np.zeros(3, np.float32)
    ln = ctypes.c_float(0.0)
    L.orc_ray_span(ctypes.byref(jb), ix, iy, ctypes.byref(m), _p(o), ctypes.byref(ln))
    return bool(m.value), o, ln.value


def ingest_cells(xyz, q, center, extent, periodic, border=100.0):
    """Periodic correction + cutout + compaction of the crawler's row loop:
    (xyzq (m, 4), input indices (m,))."""
    L = lib()
    if not hasattr(L, "_ingest_declared"):
        P = ctypes.c_void_p
        L.orc_ingest_cells.argtypes = [P, P, ctypes.c_int64, P, P, P, ctypes.c_double, P, P]
        L.orc_ingest_cells.restype = ctypes.c_int64
        L._ingest_declared = True
    xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
    n = xyz.shape[0]
    qa = None if q is None else np.ascontiguousarray(q, np.float32)
    out = np.zeros((n, 4), np.float32)
    idx = np.zeros(n, np.uint32)
    c3 = lambda v: np.ascontiguousarray(v, np.float64)
    ce, ex, pe = c3(center), c3(extent), c3(periodic)
    k = L.orc_ingest_cells(_p(xyz), _p(qa), n, _p(ce), _p(ex), _p(pe), float(border), _p(out),
                           _p(idx))
    return out[:k], idx[:k]


def volumetric_slice(grid, cam, dV=1.0, nthreads=0):
    L = lib()
    if not hasattr(L, "_slice_declared"):
        P = ctypes.c_void_p
        L.orc_volumetric_slice.argtypes = [P, P, ctypes.c_double, P, ctypes.c_int]
        L._slice_declared = True
    out = np.zeros(cam.nx * cam.ny, np.float32)
    L.orc_volumetric_slice(grid.h, ctypes.byref(cam), float(dV), _p(out), nthreads)
    return out.reshape(cam.ny, cam.nx)


def _declare_profile(L):
    P, f64 = ctypes.c_void_p, ctypes.c_double
    L.orc_mc_profile_shells.argtypes = [f64, ctypes.c_int, f64, P, P]
    L.orc_mc_radial_profile.argtypes = [P, P, f64, ctypes.c_int, f64, ctypes.c_uint64,
                                        ctypes.c_int, f64, P, P, P, ctypes.c_int]


def _profile_lib():
    L = lib()
    if not getattr(L, "_profile_declared", False):
        _declare_profile(L)
        L._profile_declared = True
    return L


def mc_profile_shells(max_radius, num_radii, sample_density):
    """Shell radii and sample counts of distributed_mc_radial_profile
    (profile.cpp:93-128, 320-355)."""
    radii = np.zeros(num_radii, np.float64)
    counts = np.zeros(num_radii, np.uint64)
    rc = _profile_lib().orc_mc_profile_shells(float(max_radius), int(num_radii),
                                              float(sample_density), _p(radii), _p(counts))
    if rc:
        raise ValueError("invalid profile shells")
    return radii, counts


def mc_radial_profile(grid, center, max_radius, num_radii, sample_density, seed=0, dV_mode=0,
                      volume_conversion=1.0, samples=False, nthreads=0):
    """The oracle's Monte-Carlo radial profile of the grid's q around center:
    the profile, and with samples=True every sample point (total, 4) and
    nn8 value (total,) in sample order."""
    L = _profile_lib()
    total = int(mc_profile_shells(max_radius, num_radii, sample_density)[1].sum())
    c = np.ascontiguousarray(center, np.float64)
    prof = np.zeros(num_radii, np.float64)
    pts = np.zeros((total, 4), np.float32) if samples else None
    vals = np.zeros(total, np.float32) if samples else None
    rc = L.orc_mc_radial_profile(grid.h, _p(c), float(max_radius), int(num_radii),
                                 float(sample_density), int(seed), int(dV_mode),
                                 float(volume_conversion), _p(prof), _p(pts), _p(vals), nthreads)
    if rc:
        raise ValueError("invalid profile arguments")
    return (prof, pts, vals) if samples else prof
