"""Seeded synthetic gas cells standing in for an Illustris snapshot cutout.

No simulation data is available, so every workload draws its cells from this
generator: numpy ``Generator(PCG64(seed))``, sampled in float64 and cast to
float32. Units are kpc and M_sun/kpc^3 (unit converter a = h = 1).

* 90 % of the cells follow NFW profiles: radius by inverting
  M(<r) ~ ln(1+x) - x/(1+x), x = r/r_s, truncated at r_max, isotropic
  directions; the remaining 10 % are uniform in the cube.
* density  rho = rho_s / (x (1+x)^2) * LogNormal(0, 0.3), rho_s = 1.8e5
* temperature T = 5e7 K * (1 + r/r_s)^-1/2 * LogNormal(0, 0.2)
* electron abundance x_e = 1.16 (n_e/n_H)
* specific internal energy u is T inverted through the reference's
  get_temperature (quantities.cl:48-61), because the X-ray kernels take
  (rho, u, x_e) as their inputs.

Metallicity (0.3 solar), cell volume and smoothing length are not generated:
the reference's X-ray formula and the nn8 reconstruction do not read them
(quantities.cl:112-133, volumetric_reconstruction_backend_nn8.cpp:32-35).
"""
from dataclasses import dataclass, field

import numpy as np

RHO_S = 1.8e5
T0 = 5.0e7
X_H = 0.76


@dataclass
class Halo:
    center: tuple       # kpc
    r_s: float          # kpc
    r_max: float        # kpc, truncation radius
    weight: float = 1.0  # share of the NFW cells


@dataclass
class CellSet:
    pos: np.ndarray          # (N, 3) float32, kpc
    rho: np.ndarray          # (N,) float32, M_sun/kpc^3
    u: np.ndarray            # (N,) float32, (km/s)^2
    xe: np.ndarray           # (N,) float32
    temperature: np.ndarray  # (N,) float32, K (float64 target cast to float32)
    box: float               # cube side, kpc; the cube is [0, box]^3
    halos: list = field(default_factory=list)

    @property
    def n(self):
        return self.pos.shape[0]

    def xyzq(self, q):
        """float4 (x, y, z, q) particle array, the reference's particle layout."""
        out = np.empty((self.n, 4), np.float32)
        out[:, :3] = self.pos
        out[:, 3] = q
        return out


def _nfw_mass(x):
    return np.log1p(x) - x / (1.0 + x)


def _nfw_radii(rng, n, r_s, r_max):
    """Inverse-CDF sampling of NFW radii by bisection on M(<x)."""
    xmax = r_max / r_s
    target = rng.random(n) * _nfw_mass(xmax)
    lo = np.zeros(n)
    hi = np.full(n, xmax)
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        below = _nfw_mass(mid) < target
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return 0.5 * (lo + hi) * r_s


def _directions(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def internal_energy_from_temperature(T, xe):
    """Inverse of get_temperature (quantities.cl:38-61) in float64."""
    mu = 4.0 / (1.0 + 3.0 * X_H + 4.0 * X_H * xe)
    return T / ((5.0 / 3.0 - 1.0) * mu * 121.1475502)


def generate(n, box, halos, seed, background=0.1):
    rng = np.random.Generator(np.random.PCG64(seed))
    n_bg = int(round(background * n))
    n_nfw = n - n_bg
    weights = np.array([h.weight for h in halos], float)
    counts = np.floor(weights / weights.sum() * n_nfw).astype(int)
    counts[0] += n_nfw - counts.sum()
    pos = []
    for h, k in zip(halos, counts):
        r = _nfw_radii(rng, k, h.r_s, h.r_max)
        pos.append(np.asarray(h.center)[None, :] + r[:, None] * _directions(rng, k))
    pos.append(rng.random((n_bg, 3)) * box)
    pos = np.concatenate(pos, axis=0)
    # Every cell takes density and temperature from its nearest halo centre.
    centers = np.array([h.center for h in halos], float)
    rs = np.array([h.r_s for h in halos], float)
    d = np.linalg.norm(pos[:, None, :] - centers[None, :, :], axis=2)
    which = np.argmin(d / rs[None, :], axis=1)
    r = d[np.arange(pos.shape[0]), which]
    x = np.maximum(r / rs[which], 1e-3)
    rho = RHO_S / (x * (1.0 + x) ** 2) * rng.lognormal(0.0, 0.3, pos.shape[0])
    T = T0 * (1.0 + r / rs[which]) ** -0.5 * rng.lognormal(0.0, 0.2, pos.shape[0])
    xe = np.full(pos.shape[0], 1.16)
    u = internal_energy_from_temperature(T, xe)
    return CellSet(pos=pos.astype(np.float32), rho=rho.astype(np.float32),
                   u=u.astype(np.float32), xe=xe.astype(np.float32),
                   temperature=T.astype(np.float32), box=float(box), halos=list(halos))


# Workloads (seed_k = 20170 + k)

def plain_density_cells(n=262_144):
    """Projected-density workload: 256 k cells, NFW r_s = 300 kpc, c = 5
    (r_max = 1.5 Mpc), in a 3 Mpc cube."""
    box = 3000.0
    return generate(n, box, [Halo((box / 2,) * 3, 300.0, 1500.0)], seed=20170)


def xray_cells(n=4_194_304, seed=20171):
    """X-ray workload: 4 M cells, NFW r_s = 400 kpc truncated at 3 Mpc, in a
    6 Mpc cube (shared by the band-map, batched and adjoint workloads)."""
    box = 6000.0
    return generate(n, box, [Halo((box / 2,) * 3, 400.0, 3000.0)], seed=seed)


def scale_cells(n=67_108_864):
    """Scale workload: 64 M cells, two NFW halos with mass ratio 3:1 (r_s 450
    and 300 kpc) 1.5 Mpc apart plus 10 % background, in an 8 Mpc cube."""
    box = 8000.0
    c = box / 2
    halos = [Halo((c - 750.0, c, c), 450.0, 3000.0, 3.0),
             Halo((c + 750.0, c, c), 300.0, 3000.0, 1.0)]
    return generate(n, box, halos, seed=20174)


def small_cells(n, seed=7, box=1000.0, r_s=100.0):
    """Small clustered set for parity tests (seconds on the oracle)."""
    return generate(n, box, [Halo((box / 2,) * 3, r_s, box / 2)], seed=seed)


def gaussian_random_field_at(pos, box, sigma=0.1, ell=200.0, n=256, seed=20174):
    """Seeded Gaussian random field on an n^3 periodic grid over [0, box]^3
    (white noise filtered by exp(-k^2 ell^2 / 2) in Fourier space, then scaled
    to standard deviation sigma), trilinearly interpolated at pos (N, 3).
    The target perturbation of the adjoint workload: log T -> log T + field."""
    rng = np.random.Generator(np.random.PCG64(seed))
    white = rng.standard_normal((n, n, n))
    k = 2.0 * np.pi * np.fft.fftfreq(n, d=box / n)
    kz = 2.0 * np.pi * np.fft.rfftfreq(n, d=box / n)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2
    f = np.fft.irfftn(np.fft.rfftn(white) * np.exp(-0.5 * k2 * ell * ell), s=(n, n, n))
    f *= sigma / f.std()
    g = np.asarray(pos, np.float64) / box * n - 0.5      # cell-centred samples
    i0 = np.floor(g).astype(np.int64)
    t = g - i0
    out = np.zeros(len(g))
    for dx in (0, 1):
        wx = t[:, 0] if dx else 1.0 - t[:, 0]
        for dy in (0, 1):
            wy = t[:, 1] if dy else 1.0 - t[:, 1]
            for dz in (0, 1):
                wz = t[:, 2] if dz else 1.0 - t[:, 2]
                idx = (i0 + np.array([dx, dy, dz])) % n
                out += wx * wy * wz * f[idx[:, 0], idx[:, 1], idx[:, 2]]
    return out


def perturbed_internal_energy(cells, field):
    """u for log T + field (T is proportional to u at fixed x_e)."""
    return (cells.u.astype(np.float64) * np.exp(field)).astype(np.float32)


def synthetic_arf(n=1024, x_min=0.105322271585, dx=0.010644, seed=20175):
    """A seeded stand-in for an X-ray telescope's effective area [cm^2] on the
    reference ARF's energy grid (n samples from x_min in steps of dx): a
    log-normal bump peaking near 1.3 keV, an absorption edge at 2.1 keV, next
    to nothing below 0.25 keV, and 1 % sample noise. The reference's own
    table (the Chandra Cycle 19 ACIS-I ARF) lives in its sources; this
    library loads whatever table the caller passes to ``ilc_arf_load``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    e = x_min + dx * np.arange(n, dtype=np.float64)
    area = 600.0 * np.exp(-((np.log(e) - np.log(1.3)) / 0.9) ** 2)
    area *= np.where(e > 2.1, 0.8, 1.0)
    area *= 1.0 / (1.0 + np.exp(-(e - 0.3) / 0.03))
    area *= 1.0 + 0.01 * rng.standard_normal(n)
    return area.astype(np.float32)


def chandra_spectrum_channels(num_frames, arf_min_energy=0.1053223, arf_num_bins=1024,
                              arf_bin_width=0.010644):
    """Channel energies and widths of the frames of a Chandra spectrum
    (chandra_spectrum_quantity_generator::operator(), spectrum.cpp:45-65):
    frame i sits at arf_min + i * (arf_max - arf_min) / num_frames, computed
    in double, with the width of one ARF bin; arf_max = arf_min +
    arf_num_bins * arf_bin_width (chandra::arf::arf_max_energy). Defaults: the
    reference's arf_min_energy(), get_num_arf_bins() and arf_bin_width()."""
    arf_max = arf_min_energy + arf_num_bins * arf_bin_width
    width = (arf_max - arf_min_energy) / float(num_frames)
    e = np.array([arf_min_energy + i * width for i in range(num_frames)], np.float64)
    return e.astype(np.float32), np.full(num_frames, arf_bin_width, np.float32)
