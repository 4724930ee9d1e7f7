"""illcrawl_b200 -- B200 (sm_100a) backend for illcrawl's volumetric projection path.

Python-side view of the C ABI (``include/ilc.h``), used by the tests and the
benchmark. Names follow the reference's interfaces:

* :class:`Nn8Backend` -- ``reconstruction_backend`` / ``reconstruction_backends::nn8``
  (reconstruction_backend.hpp:35-58, volumetric_reconstruction_backend_nn8.hpp:36-82)
* :func:`create_projection` -- ``volumetric_integration::create_projection``
  (volumetric_integration.cpp:32-88)
* :func:`xray_flux`, :func:`xray_spectral_flux`, :func:`xray_photon_flux`,
  :func:`chandra_count_rate`, :func:`chandra_spectral_count_rate`,
  :func:`mean_temperature` -- the quantity kernels of quantities.cl
* :func:`load_gaunt_table` -- ``util::data_table_loader`` on gaunt_factor.dat
  (data_table_loader.hpp:39-97)
* :meth:`Context.volumetric_slice`, :meth:`Context.volumetric_tomography`,
  :meth:`Context.mc_radial_profile` -- the other nn8 consumers
  (volumetric_slice.cpp, volumetric_tomography.cpp, profile.cpp);
  :mod:`illcrawl_b200.distributed` splits them over processes as the
  reference's distributed_* classes do

All compute runs in ``libilcuda.so``; nothing here falls back to the CPU.
"""
import ctypes
import os

import numpy as np

from . import _lib
QUERY_THREAD, QUERY_WARP = 0, 1

from ._lib import (CONTROLLER_FP64, CONTROLLER_REF32, DA_INVERSE_RANGE, DA_PIXEL_AREA, DA_UNIT,
                   DV_MEAN, DV_VOLUME, ENGINE_GRID, ENGINE_PERSISTENT, Camera, IlcError, Job,
                   LosScaling, RenderStats, Tolerance)

DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
GAUNT_FILE = os.path.join(DATA_DIR, "gaunt_factor.dat")

# Reference defaults (illcrawl_app.hpp:140-143, 197-199)
REDSHIFT = 0.2
LUMINOSITY_DISTANCE = 978500.0


def _ptr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):  # torch tensor on the device
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def _is_dev(a):
    return 1 if hasattr(a, "data_ptr") and getattr(a, "is_cuda", False) else 0


def load_gaunt_table(path=GAUNT_FILE):
    """Parses a whitespace table, skipping lines that start with '#', as
    util::data_table_loader does (data_table_loader.hpp:39-97). Returns a
    (rows, columns) float32 array: rows = log(u), columns = log(gamma^2)."""
    rows = []
    width = None
    with open(path) as f:
        for line in f:
            if line.startswith("#") or len(line.rstrip("\n")) == 0:
                continue
            vals = line.split()
            if width is None:
                width = len(vals)
            elif len(vals) != width:
                raise ValueError(f"invalid row in {path}: expected {width} entries")
            rows.append([np.float32(v) for v in vals])
    return np.asarray(rows, np.float32)


def camera(position, look_at, roll, screen_width, num_pix_x, num_pix_y):
    c = Camera()
    c.position[:] = [float(v) for v in position]
    c.look_at[:] = [float(v) for v in look_at]
    c.roll, c.screen_width = float(roll), float(screen_width)
    c.num_pix_x, c.num_pix_y = int(num_pix_x), int(num_pix_y)
    return c


def job(cam, z_range=0.0, aperture_radius=0.0, sphere_center=(0.0, 0.0, 0.0),
        sphere_radius=0.0, min_chord=0.0, scale=1.0, out_offset=0):
    """One camera of a batched render (ilc_job)."""
    return Job(cam, z_range, aperture_radius, (ctypes.c_double * 3)(*sphere_center),
               sphere_radius, min_chord, scale, 0, out_offset)


def pack_jobs(jobs, n_channels):
    """Assigns consecutive output blocks (V x ny x nx each) to the jobs in
    order; returns (ctypes array, total elements)."""
    arr = (Job * len(jobs))()
    off = 0
    for i, j in enumerate(jobs):
        j.out_offset = off
        arr[i] = j
        off += n_channels * j.camera.num_pix_x * j.camera.num_pix_y
    return arr, off


def write_fits(path, data, cards=()):
    """FITS image / cube of float32 data (ilc_fits_write_image). data: (ny, nx)
    or (nz, ny, nx). cards: (key, value[, comment]) with float, int, bool or
    str values, appended as the reference appends its settings."""
    a = np.ascontiguousarray(data, np.float32)
    if a.ndim not in (2, 3):
        raise ValueError("2 or 3 dimensions")
    naxes = np.ascontiguousarray(a.shape[::-1], np.int64)
    arr = (_lib.FitsCard * max(1, len(cards)))()
    keep = []
    for i, c in enumerate(cards):
        key, val = c[0], c[1]
        com = c[2] if len(c) > 2 else None
        k = _lib.FitsCard()
        k.key = key.encode()
        keep.append(k.key)
        if isinstance(val, bool):
            k.type, k.integer = 3, int(val)
        elif isinstance(val, (int, np.integer)):
            k.type, k.integer = 1, int(val)
        elif isinstance(val, (float, np.floating)):
            k.type, k.number = 0, float(val)
        else:
            k.type, k.text = 2, str(val).encode()
        k.comment = None if com is None else com.encode()
        arr[i] = k
    L = _lib.load()
    st = L.ilc_fits_write_image(str(path).encode(), _ptr(a), a.ndim, _ptr(naxes), arr,
                                len(cards))
    if st:
        raise IlcError(st, f"could not write {path}")


def mc_profile_shells(max_radius, num_radii, sample_density):
    """Shell radii and per-shell sample counts of a Monte-Carlo radial profile
    (ilc_mc_profile_shells; host only)."""
    radii = np.zeros(num_radii, np.float64)
    counts = np.zeros(num_radii, np.uint64)
    st = _lib.load().ilc_mc_profile_shells(float(max_radius), int(num_radii),
                                            float(sample_density), _ptr(radii), _ptr(counts))
    if st != _lib.ILC_OK:
        raise IlcError(st, "invalid profile shells (radius, 1..2^20 radii, density, at most "
                           "2^40 samples)")
    return radii, counts


def mc_profile_points(center, max_radius, num_radii, sample_density, seed=0, first=0,
                      count=None):
    """Sample points first .. first + count - 1 of a Monte-Carlo radial profile
    (ilc_mc_profile_points; host only), (count, 4) float32 with w = 0."""
    if count is None:
        count = int(mc_profile_shells(max_radius, num_radii, sample_density)[1].sum()) - first
    c = np.ascontiguousarray(center, np.float64)
    out = np.zeros((count, 4), np.float32)
    st = _lib.load().ilc_mc_profile_points(_ptr(c), float(max_radius), int(num_radii),
                                            float(sample_density), int(seed), int(first),
                                            int(count), _ptr(out))
    if st != _lib.ILC_OK:
        raise IlcError(st, "invalid profile sample range or shells")
    return out


def camera_plane(cam):
    out = np.zeros(13, np.float32)
    st = _lib.load().ilc_camera_plane(ctypes.byref(cam), _ptr(out))
    if st:
        raise IlcError(st, "invalid camera")
    return out


def los_scale(cam, z_range, length_conversion=1.0, area_conversion=1.0, dA_mode=DA_PIXEL_AREA):
    s = LosScaling(length_conversion, area_conversion, dA_mode)
    return np.float32(_lib.load().ilc_los_scale(ctypes.byref(cam), z_range, ctypes.byref(s)))


class Context:
    """One device context (stream, grid, Gaunt table, scratch) -- ilc_ctx."""

    def __init__(self, device=0):
        self.L = _lib.load()
        self.h = self.L.ilc_create(int(device))
        if not self.h:
            raise RuntimeError(f"ilc_create({device}) failed: no usable CUDA device")
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.L.ilc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def check(self, st):
        if st != _lib.ILC_OK:
            raise IlcError(st, self.L.ilc_last_error(self.h).decode())

    @property
    def stream(self):
        return self.L.ilc_get_stream(self.h)

    def set_step_limit(self, n):
        self.check(self.L.ilc_set_step_limit(self.h, int(n)))

    def set_z_window(self, kpc):
        self.check(self.L.ilc_set_z_window(self.h, float(kpc)))

    def set_render_engine(self, engine):
        self.check(self.L.ilc_set_render_engine(self.h, int(engine)))

    def set_render_occupancy(self, blocks_per_sm):
        self.check(self.L.ilc_set_render_occupancy(self.h, int(blocks_per_sm)))

    def autotune_render(self, cam, z_range, rel_tol=1e-3, abs_tol=0.0,
                        controller=CONTROLLER_FP64, windows=(0, 5, 10, 20, 40, 80),
                        occupancies=(0, 4, 5), sample_stride=16):
        """Times the adaptive render on a sample of tile rows for each
        (z window, occupancy) pair, sets the fastest on the context; returns
        (best window, best occupancy, {(window, occupancy): ms})."""
        win = np.ascontiguousarray(windows, np.float32)
        occ = np.ascontiguousarray(occupancies, np.int32)
        times = np.zeros(len(win) * len(occ), np.float32)
        bw, bo = ctypes.c_float(0.0), ctypes.c_int32(0)
        self.check(self.L.ilc_autotune_render(self.h, ctypes.byref(cam), float(z_range),
                                              Tolerance(abs_tol, rel_tol), controller,
                                              _ptr(win), len(win), _ptr(occ), len(occ),
                                              int(sample_stride), ctypes.byref(bw),
                                              ctypes.byref(bo), _ptr(times)))
        tt = {(float(w), int(o)): float(times[i * len(occ) + j])
              for i, w in enumerate(win) for j, o in enumerate(occ)}
        return float(bw.value), int(bo.value), tt

    # ---- grid / nn8
    def setup_particles(self, xyzq):
        if not _is_dev(xyzq):
            xyzq = np.ascontiguousarray(xyzq, np.float32).reshape(-1, 4)
        n = xyzq.shape[0]
        self.check(self.L.ilc_nn8_setup_particles(self.h, _ptr(xyzq), n, _is_dev(xyzq)))

    def grid_describe(self):
        d = _lib.GridDesc()
        self.check(self.L.ilc_grid_describe(self.h, ctypes.byref(d)))
        return {"min_corner": np.array(d.min_corner, np.float32),
                "cell_sizes": np.array(d.cell_sizes, np.float32),
                "num_cells": np.array(d.num_cells, np.int32),
                "total_cells": int(d.total_cells), "num_particles": int(d.num_particles)}

    def grid_export(self):
        d = self.grid_describe()
        n = d["num_particles"]
        cells = np.zeros((d["total_cells"], 2), np.int32)
        s2u = np.zeros(n, np.uint32)
        srt = np.zeros((n, 4), np.float32)
        self.check(self.L.ilc_grid_export(self.h, _ptr(cells), _ptr(s2u), _ptr(srt), 0))
        return cells, s2u, srt

    def nn8_query(self, points, merge_previous=False, slots=False):
        dev = _is_dev(points)
        if not dev:
            points = np.ascontiguousarray(points, np.float32).reshape(-1, 4)
        n = points.shape[0]
        if dev:
            import torch
            out = torch.empty(n, dtype=torch.float32, device=points.device)
            idx = torch.empty((n, 8), dtype=torch.int32, device=points.device) if slots else None
            d8 = torch.empty((n, 8), dtype=torch.float32, device=points.device) if slots else None
        else:
            out = np.zeros(n, np.float32)
            idx = np.zeros((n, 8), np.int32) if slots else None
            d8 = np.zeros((n, 8), np.float32) if slots else None
        self.check(self.L.ilc_nn8_query(self.h, _ptr(points), n, int(merge_previous), _ptr(out),
                                        _ptr(idx), _ptr(d8), dev))
        return (out, idx, d8) if slots else out

    # ---- quantities
    def load_gaunt(self, table=None, x0=-6.0, y0=-16.0, dx=0.2, dy=0.2):
        t = load_gaunt_table() if table is None else np.ascontiguousarray(table, np.float32)
        self.check(self.L.ilc_gaunt_load(self.h, _ptr(t), t.shape[1], t.shape[0], x0, y0, dx, dy))
        return t

    def _q3(self, rho, u, xe):
        dev = _is_dev(u)
        if not dev:
            rho = None if rho is None else np.ascontiguousarray(rho, np.float32)
            u = np.ascontiguousarray(u, np.float32)
            xe = np.ascontiguousarray(xe, np.float32)
        n = u.shape[0]
        if dev:
            import torch
            out = torch.empty(n, dtype=torch.float32, device=u.device)
        else:
            out = np.zeros(n, np.float32)
        return rho, u, xe, n, out, dev

    def xray_flux(self, rho, u, xe, redshift=REDSHIFT, luminosity_distance=LUMINOSITY_DISTANCE,
                  e_min=0.1, e_max=10.0, num_samples=100):
        rho, u, xe, n, out, dev = self._q3(rho, u, xe)
        self.check(self.L.ilc_quantity_xray_flux(self.h, _ptr(rho), _ptr(u), _ptr(xe), n,
                                                 redshift, luminosity_distance, e_min, e_max,
                                                 num_samples, _ptr(out), dev))
        return out

    def xray_spectral_flux(self, rho, u, xe, energy, energy_bin_width, redshift=REDSHIFT,
                           luminosity_distance=LUMINOSITY_DISTANCE):
        rho, u, xe, n, out, dev = self._q3(rho, u, xe)
        self.check(self.L.ilc_quantity_xray_spectral_flux(self.h, _ptr(rho), _ptr(u), _ptr(xe),
                                                          n, redshift, luminosity_distance,
                                                          energy, energy_bin_width, _ptr(out),
                                                          dev))
        return out

    def xray_spectrum(self, rho, u, xe, energies, widths, redshift=REDSHIFT,
                      luminosity_distance=LUMINOSITY_DISTANCE):
        """Per-cell flux in every bin, cell-major (n, n_bins)."""
        dev = _is_dev(u)
        if not dev:
            rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
        e = np.ascontiguousarray(energies, np.float32)
        w = np.ascontiguousarray(widths, np.float32)
        n, nb = u.shape[0], e.shape[0]
        if dev:
            import torch
            out = torch.empty((n, nb), dtype=torch.float32, device=u.device)
        else:
            out = np.zeros((n, nb), np.float32)
        self.check(self.L.ilc_quantity_xray_spectrum(self.h, _ptr(rho), _ptr(u), _ptr(xe), n,
                                                     redshift, luminosity_distance, _ptr(e),
                                                     _ptr(w), nb, _ptr(out), dev))
        return out

    def xray_photon_flux(self, rho, u, xe, redshift=REDSHIFT,
                         luminosity_distance=LUMINOSITY_DISTANCE, e_min=0.1, e_max=10.0,
                         num_samples=100):
        """xray_photon_flux per cell [photons/s/kpc^3/cm^2] (the reference's
        defaults for the quantity: 0.1-10 keV, 100 samples)."""
        rho, u, xe, n, out, dev = self._q3(rho, u, xe)
        self.check(self.L.ilc_quantity_xray_photon_flux(self.h, _ptr(rho), _ptr(u), _ptr(xe), n,
                                                        redshift, luminosity_distance, e_min,
                                                        e_max, num_samples, _ptr(out), dev))
        return out

    def load_arf(self, table, x_min, dx):
        """Chandra ARF [cm^2]: len(table) samples from x_min [keV] in steps of
        dx (the caller supplies the table; chandra::arf, chandra.cpp)."""
        t = np.ascontiguousarray(table, np.float32).ravel()
        self.check(self.L.ilc_arf_load(self.h, _ptr(t), t.size, x_min, dx))
        return t

    def chandra_count_rate(self, rho, u, xe, redshift=REDSHIFT,
                           luminosity_distance=LUMINOSITY_DISTANCE):
        """Per-cell count rate over every ARF channel [counts/s/kpc^3]."""
        rho, u, xe, n, out, dev = self._q3(rho, u, xe)
        self.check(self.L.ilc_quantity_chandra_count_rate(self.h, _ptr(rho), _ptr(u), _ptr(xe),
                                                          n, redshift, luminosity_distance,
                                                          _ptr(out), dev))
        return out

    def chandra_spectral_count_rate(self, rho, u, xe, energy, energy_bin_width,
                                    redshift=REDSHIFT, luminosity_distance=LUMINOSITY_DISTANCE):
        """Per-cell count rate in the channel (energy, energy_bin_width)."""
        rho, u, xe, n, out, dev = self._q3(rho, u, xe)
        self.check(self.L.ilc_quantity_chandra_spectral_count_rate(
            self.h, _ptr(rho), _ptr(u), _ptr(xe), n, redshift, luminosity_distance, energy,
            energy_bin_width, _ptr(out), dev))
        return out

    def chandra_spectrum(self, rho, u, xe, energies, widths, redshift=REDSHIFT,
                         luminosity_distance=LUMINOSITY_DISTANCE):
        """Per-cell count rate in every channel, cell-major (n, n_bins)."""
        dev = _is_dev(u)
        if not dev:
            rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
        e = np.ascontiguousarray(energies, np.float32)
        w = np.ascontiguousarray(widths, np.float32)
        n, nb = u.shape[0], e.shape[0]
        if dev:
            import torch
            out = torch.empty((n, nb), dtype=torch.float32, device=u.device)
        else:
            out = np.zeros((n, nb), np.float32)
        self.check(self.L.ilc_quantity_chandra_spectrum(self.h, _ptr(rho), _ptr(u), _ptr(xe), n,
                                                        redshift, luminosity_distance, _ptr(e),
                                                        _ptr(w), nb, _ptr(out), dev))
        return out

    def mean_temperature(self, u, xe):
        _, u, xe, n, out, dev = self._q3(None, u, xe)
        self.check(self.L.ilc_quantity_temperature(self.h, _ptr(u), _ptr(xe), n, _ptr(out), dev))
        return out

    # ---- line of sight integration
    def _image(self, cam, like_device):
        if like_device:
            import torch
            return torch.empty((cam.num_pix_y, cam.num_pix_x), dtype=torch.float32,
                               device=f"cuda:{self.device}")
        return np.zeros((cam.num_pix_y, cam.num_pix_x), np.float32)

    def render_adaptive(self, cam, z_range, rel_tol=1e-3, abs_tol=0.0,
                        controller=CONTROLLER_FP64, scaling=None, device_output=False):
        img = self._image(cam, device_output)
        st = RenderStats()
        sc = None if scaling is None else ctypes.byref(scaling)
        self.check(self.L.ilc_render_adaptive(self.h, ctypes.byref(cam), float(z_range),
                                              Tolerance(abs_tol, rel_tol), controller, sc,
                                              _ptr(img), 1 if device_output else 0,
                                              ctypes.byref(st)))
        return img, st.as_dict()

    def project_xray_flux(self, cells, rho, u, xe, cam, z_range, rel_tol=1e-3, abs_tol=0.0,
                          controller=CONTROLLER_FP64, redshift=REDSHIFT,
                          luminosity_distance=LUMINOSITY_DISTANCE, e_min=0.5, e_max=7.0,
                          num_samples=100, scaling=None, image=None):
        """X-ray band map from raw cells in one call (ilc_project_xray_flux).
        Inputs are all host arrays or all device tensors; the image follows."""
        dev = _is_dev(u)
        if not dev:
            cells = np.ascontiguousarray(cells, np.float32).reshape(-1, 4)
            rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
        if image is None:
            image = self._image(cam, dev)
        st = RenderStats()
        sc = None if scaling is None else ctypes.byref(scaling)
        self.check(self.L.ilc_project_xray_flux(
            self.h, _ptr(cells), _ptr(rho), _ptr(u), _ptr(xe), int(u.shape[0]), redshift,
            luminosity_distance, e_min, e_max, num_samples, ctypes.byref(cam), float(z_range),
            Tolerance(abs_tol, rel_tol), controller, sc, _ptr(image), dev, ctypes.byref(st)))
        return image, st.as_dict()

    def adjoint_xray_flux(self, cells, rho, u, xe, cam, z_range, target, mode=0, rel_tol=1e-3,
                          abs_tol=0.0, controller=CONTROLLER_FP64, redshift=REDSHIFT,
                          luminosity_distance=LUMINOSITY_DISTANCE, e_min=0.5, e_max=7.0,
                          num_samples=100, scaling=None):
        """Band map + gradient of sum (log I - log target)^2 with respect to
        per-cell ln rho and ln T (ilc_adjoint_xray_flux). Host arrays in,
        host arrays out. mode: 0 checkpoint, 1 recompute."""
        cells = np.ascontiguousarray(cells, np.float32).reshape(-1, 4)
        rho, u, xe = (np.ascontiguousarray(a, np.float32) for a in (rho, u, xe))
        target = np.ascontiguousarray(target, np.float32)
        n = u.shape[0]
        img = np.zeros((cam.num_pix_y, cam.num_pix_x), np.float32)
        g_r = np.zeros(n, np.float32)
        g_t = np.zeros(n, np.float32)
        st = _lib.AdjointStats()
        sc = None if scaling is None else ctypes.byref(scaling)
        self.check(self.L.ilc_adjoint_xray_flux(
            self.h, _ptr(cells), _ptr(rho), _ptr(u), _ptr(xe), n, redshift, luminosity_distance,
            e_min, e_max, num_samples, ctypes.byref(cam), float(z_range),
            Tolerance(abs_tol, rel_tol), controller, sc, _ptr(target), int(mode), _ptr(img),
            _ptr(g_r), _ptr(g_t), 0, ctypes.byref(st)))
        return img, g_r, g_t, st.as_dict()

    # ---- volumetric slice
    def volumetric_slice(self, cam, dV=1.0, additional_samples=0, seed=0):
        img = self._image(cam, False)
        self.check(self.L.ilc_volumetric_slice(self.h, ctypes.byref(cam), float(dV),
                                               int(additional_samples), int(seed), _ptr(img), 0))
        return img

    def volumetric_tomography(self, cam, dV=1.0, initial_z_step=0, num_steps=1):
        cube = np.zeros((num_steps, cam.num_pix_y, cam.num_pix_x), np.float32)
        self.check(self.L.ilc_volumetric_tomography(self.h, ctypes.byref(cam), float(dV),
                                                    int(initial_z_step), int(num_steps),
                                                    _ptr(cube), 0))
        return cube

    # ---- Monte-Carlo radial profiles
    def mc_radial_profile(self, center, max_radius, num_radii, sample_density, seed=0,
                          dV_mode=DV_VOLUME, volume_conversion=1.0, samples=False):
        """distributed_mc_radial_profile of the particles' q around center
        (ilc_mc_radial_profile): the profile (num_radii doubles), and with
        samples=True also every sample point (total, 4) and value (total,)."""
        c = np.ascontiguousarray(center, np.float64)
        prof = np.zeros(num_radii, np.float64)
        pts = vals = None
        if samples:
            total = int(mc_profile_shells(max_radius, num_radii, sample_density)[1].sum())
            pts = np.zeros((total, 4), np.float32)
            vals = np.zeros(total, np.float32)
        self.check(self.L.ilc_mc_radial_profile(self.h, _ptr(c), float(max_radius), int(num_radii),
                                                float(sample_density), int(seed), int(dV_mode),
                                                float(volume_conversion), _ptr(prof), _ptr(pts),
                                                _ptr(vals)))
        return (prof, pts, vals) if samples else prof

    # ---- cell ingestion
    def ingest_cells(self, xyz, q, center, extent, periodic, border=100.0):
        """Periodic correction + cutout + compaction (ilc_ingest_cells). Host
        arrays in, host arrays out: (xyzq (m, 4), input indices (m,))."""
        xyz = np.ascontiguousarray(xyz, np.float32).reshape(-1, 3)
        n = xyz.shape[0]
        qa = None if q is None else np.ascontiguousarray(q, np.float32)
        out = np.zeros((n, 4), np.float32)
        idx = np.zeros(n, np.uint32)
        m = ctypes.c_uint64(0)
        c3 = lambda v: (ctypes.c_double * 3)(*[float(x) for x in v])
        self.check(self.L.ilc_ingest_cells(self.h, _ptr(xyz), _ptr(qa), n, c3(center), c3(extent),
                                           c3(periodic), float(border), _ptr(out), _ptr(idx),
                                           ctypes.byref(m), 0))
        k = int(m.value)
        return out[:k], idx[:k]

    # ---- batched render
    def last_query_stats(self):
        """(cells visited, candidates tested) of the last nn8_query."""
        a, b = ctypes.c_uint64(0), ctypes.c_uint64(0)
        self.check(self.L.ilc_nn8_query_stats(self.h, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def set_query_engine(self, engine):
        """QUERY_THREAD (0, default) or QUERY_WARP (1) for nn8 queries."""
        self.check(self.L.ilc_set_query_engine(self.h, int(engine)))

    def set_checkpoint_budget(self, nbytes):
        """Device bytes the checkpoint adjoint may hold for step checkpoints."""
        self.check(self.L.ilc_set_checkpoint_budget(self.h, int(nbytes)))

    def set_batch_schedule(self, tile_w=8, blocks_per_sm=4, z_window=40.0, cost_order=True):
        self.check(self.L.ilc_set_batch_schedule(self.h, int(tile_w), int(blocks_per_sm),
                                                 float(z_window), 1 if cost_order else 0))

    def render_batched(self, values, jobs, rel_tol=1e-3, abs_tol=0.0, images=None):
        """values: (n,) or (n, V) per-cell channels (original particle order;
        host array or device tensor). jobs: list of ilc_job (their out_offset
        is assigned here, consecutively). Returns (flat images, stats); job
        k's block is images[off_k : off_k + V*ny*nx] as (V, ny, nx)."""
        dev = _is_dev(values)
        if not dev:
            values = np.ascontiguousarray(values, np.float32)
        V = 1 if values.ndim == 1 else int(values.shape[1])
        arr, total = pack_jobs(jobs, V)
        if images is None:
            if dev:
                import torch
                images = torch.zeros(total, dtype=torch.float32, device=values.device)
            else:
                images = np.zeros(total, np.float32)
        st = RenderStats()
        self.check(self.L.ilc_render_batched(self.h, _ptr(values), V, dev, arr, len(jobs),
                                             Tolerance(abs_tol, rel_tol), _ptr(images), total,
                                             _is_dev(images), ctypes.byref(st)))
        return images, st.as_dict()

    def autotune_batched(self, values, jobs, rel_tol=1e-3, abs_tol=0.0,
                         tile_ws=(0, 4, 8, 16, 32), occupancies=(0, 4, 5), windows=(0.0, 40.0)):
        """Times every (tile_w, occupancy, z_window) on the jobs, sets the
        fastest; returns (tile_w, occupancy, window, {(t, o, w): ms})."""
        dev = _is_dev(values)
        if not dev:
            values = np.ascontiguousarray(values, np.float32)
        V = 1 if values.ndim == 1 else int(values.shape[1])
        arr, _ = pack_jobs(jobs, V)
        tw = np.ascontiguousarray(tile_ws, np.int32)
        oc = np.ascontiguousarray(occupancies, np.int32)
        wn = np.ascontiguousarray(windows, np.float32)
        times = np.zeros(len(tw) * len(oc) * len(wn), np.float32)
        bt, bo, bw = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_float(0.0)
        self.check(self.L.ilc_autotune_batched(self.h, _ptr(values), V, dev, arr, len(jobs),
                                               Tolerance(abs_tol, rel_tol), _ptr(tw), len(tw),
                                               _ptr(oc), len(oc), _ptr(wn), len(wn),
                                               ctypes.byref(bt), ctypes.byref(bo),
                                               ctypes.byref(bw), _ptr(times)))
        tt = {}
        for i, t in enumerate(tw):
            for j, o in enumerate(oc):
                for q, w in enumerate(wn):
                    tt[(int(t), int(o), float(w))] = float(times[(i * len(oc) + j) * len(wn) + q])
        return int(bt.value), int(bo.value), float(bw.value), tt

    @property
    def kernel_launches(self):
        return int(self.L.ilc_kernel_launches(self.h))

    def render_record(self, cam, z_range, capacity, rel_tol=1e-3, abs_tol=0.0,
                      controller=CONTROLLER_FP64):
        """Adaptive render plus every ray's accepted step sizes:
        (image, step_sizes (rays, capacity), n_steps (rays,), stats)."""
        img = self._image(cam, False)
        rays = cam.num_pix_x * cam.num_pix_y
        hs = np.zeros((rays, capacity), np.float32)
        n = np.zeros(rays, np.int32)
        st = RenderStats()
        self.check(self.L.ilc_render_record(self.h, ctypes.byref(cam), float(z_range),
                                            Tolerance(abs_tol, rel_tol), controller, _ptr(hs),
                                            _ptr(n), capacity, 0, _ptr(img), 0,
                                            ctypes.byref(st)))
        return img, hs, n, st.as_dict()

    def render_ray_stats(self, cam, z_range, rel_tol=1e-3, abs_tol=0.0,
                         controller=CONTROLLER_FP64, scaling=None):
        """Adaptive render plus each ray's work counters (ilc_render_ray_stats):
        (image, counters (rays, 4) uint64 = steps, accepted, cells visited,
        candidates tested, stats)."""
        img = self._image(cam, False)
        rays = cam.num_pix_x * cam.num_pix_y
        rs = np.zeros((rays, 4), np.uint64)
        st = RenderStats()
        sc = None if scaling is None else ctypes.byref(scaling)
        self.check(self.L.ilc_render_ray_stats(self.h, ctypes.byref(cam), float(z_range),
                                               Tolerance(abs_tol, rel_tol), controller, sc,
                                               _ptr(img), _ptr(rs), 0, ctypes.byref(st)))
        return img, rs, st.as_dict()

    def render_frozen(self, cam, z_range, step_sizes, n_steps, scaling=None):
        """Replays per-ray step sequences (rays x capacity), all accepted."""
        hs = np.ascontiguousarray(step_sizes, np.float32)
        n = np.ascontiguousarray(n_steps, np.int32)
        img = self._image(cam, False)
        st = RenderStats()
        sc = None if scaling is None else ctypes.byref(scaling)
        self.check(self.L.ilc_render_frozen(self.h, ctypes.byref(cam), float(z_range), _ptr(hs),
                                            _ptr(n), hs.shape[1], 0, sc, _ptr(img), 0,
                                            ctypes.byref(st)))
        return img, st.as_dict()

    def render_fixed(self, cam, z_range, num_steps, scaling=None, device_output=False):
        img = self._image(cam, device_output)
        st = RenderStats()
        sc = None if scaling is None else ctypes.byref(scaling)
        self.check(self.L.ilc_render_fixed(self.h, ctypes.byref(cam), float(z_range),
                                           int(num_steps), sc, _ptr(img),
                                           1 if device_output else 0, ctypes.byref(st)))
        return img, st.as_dict()


class Nn8Backend:
    """The reconstruction_backend interface (reconstruction_backend.hpp:35-58)
    over the CUDA context; selectable as ``--reconstructor.voronoi nn8_cuda``."""

    def __init__(self, ctx):
        self.ctx = ctx
        self._points = None
        self._first = True
        self._result = None
        self._blocksize = 0

    def get_required_additional_datasets(self):
        return []

    def get_backend_name(self):
        return "volumetric/nn8_cuda"

    def init_backend(self, blocksize):
        self._blocksize = int(blocksize)

    def setup_particles(self, particles, additional_datasets=()):
        self.ctx.setup_particles(particles)

    def setup_evaluation_points(self, points, num_points=None):
        pts = points if num_points is None else points[:num_points]
        self._points = pts
        self._first = True
        self._result = None

    def run(self):
        if self._points is None:
            raise IlcError(1, "run() before setup_evaluation_points()")
        self._result = self.ctx.nn8_query(self._points, merge_previous=not self._first)
        self._first = False

    def retrieve_results(self):
        return self._result


def create_projection(ctx, cam, z_range, rel_tol=1e-2, abs_tol=0.0, dA_mode=DA_PIXEL_AREA,
                      length_conversion=1.0, area_conversion=1.0, controller=CONTROLLER_FP64):
    """volumetric_integration::create_projection: adaptive line-of-sight image,
    scaled by length_conversion * dA_eff (volumetric_integration.cpp:74-87)."""
    s = LosScaling(length_conversion, area_conversion, dA_mode)
    return ctx.render_adaptive(cam, z_range, rel_tol, abs_tol, controller, scaling=s)
