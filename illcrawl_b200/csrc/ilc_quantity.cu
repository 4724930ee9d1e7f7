// ilc_quantity.cu -- per-cell quantity transforms of the X-ray path
// (quantities.cl:38-136, 156-260, 354-675) with the thermally averaged Gaunt
// factor table (gaunt_factor.cpp:30-41) resident in shared memory and the
// Chandra ARF (chandra.cpp, class chandra::arf) read through the read-only
// cache.
//
// The OpenCL image lookup (read_imagef, CLK_FILTER_LINEAR, CLK_ADDRESS_CLAMP,
// unnormalised coordinates; tabulated_function.cl:26-59) is done in software
// with exact fp32 weights: the sample at u blends texels floor(u-0.5) and
// floor(u-0.5)+1 with weight frac(u-0.5); texels outside the table read 0.
#include "ilc_device.cuh"
#include "ilc_internal.h"
#include "ilc_quantity.cuh"

namespace ilc {

namespace {

__device__ __forceinline__ void load_table(float* dst, const float* __restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// xray_flux (quantities.cl:354-385); kPhoton: xray_photon_flux
// (quantities.cl:640-675), the band integral of emission / photon energy,
// converted from per m^2 to per cm^2.
template <bool kPhoton>
__global__ void __launch_bounds__(256)
xray_flux_kernel(const float* __restrict__ table, GauntView G, const float* __restrict__ rho,
                 const float* __restrict__ u, const float* __restrict__ xe, uint64_t n, float z,
                 float dL, float emin, float emax, int num_samples, float* __restrict__ out,
                 int stride) {
  __shared__ float t[kMaxTable];
  load_table(t, table, G.w * G.h);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float T = temperature(u[i], xe[i]);
    const float f = band_flux<kPhoton>(t, G, (1.f + z) * emin, (1.f + z) * emax,
                                       1.f / (float)num_samples, T, xe[i], rho[i], dL);
    out[i * stride] = kPhoton ? f * 1.e-4f : f;
  }
}

// chandra_xray_total_count_rate (quantities.cl:510-557): the count rate summed
// in channel order over every ARF channel k, at energy x0 + k * dx with
// width dx. The channel energy is the same for all threads of a warp, so the
// ARF reads are broadcasts.
__global__ void __launch_bounds__(256)
chandra_total_kernel(const float* __restrict__ table, GauntView G, const float* __restrict__ arf,
                     ArfView A, const float* __restrict__ rho, const float* __restrict__ u,
                     const float* __restrict__ xe, uint64_t n, float z, float dL,
                     float* __restrict__ out) {
  __shared__ float t[kMaxTable];
  load_table(t, table, G.w * G.h);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float T = temperature(u[i], xe[i]);
    const float x = xe[i], r = rho[i];
    float em = 0.0f;
    for (int k = 0; k < A.n; ++k) {
      const float e = A.x0 + (float)k * A.dx;
      em += chandra_rate(t, G, arf, A, e, A.dx, z, T, x, r, dL);
    }
    out[i] = em;
  }
}

// chandra_xray_spectral_count_rate (quantities.cl:584-622): one channel.
__global__ void __launch_bounds__(256)
chandra_bin_kernel(const float* __restrict__ table, GauntView G, const float* __restrict__ arf,
                   ArfView A, const float* __restrict__ rho, const float* __restrict__ u,
                   const float* __restrict__ xe, uint64_t n, float z, float dL, float e,
                   float de, float* __restrict__ out) {
  __shared__ float t[kMaxTable];
  load_table(t, table, G.w * G.h);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float T = temperature(u[i], xe[i]);
    out[i] = chandra_rate(t, G, arf, A, e, de, z, T, xe[i], rho[i], dL);
  }
}

// chandra_xray_spectral_count_rate for n_bins channels at once (the quantity
// of each frame of chandra_spectrum_quantity_generator, spectrum.cpp:45-65),
// cell-major out[i * n_bins + b] as ilc_render_batched reads it.
__global__ void __launch_bounds__(256)
chandra_bins_kernel(const float* __restrict__ table, GauntView G, const float* __restrict__ arf,
                    ArfView A, const float* __restrict__ rho, const float* __restrict__ u,
                    const float* __restrict__ xe, uint64_t n, float z, float dL,
                    const float* __restrict__ e, const float* __restrict__ de, int n_bins,
                    float* __restrict__ out) {
  __shared__ float t[kMaxTable];
  load_table(t, table, G.w * G.h);
  const uint64_t total = n * (uint64_t)n_bins;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = k / (uint64_t)n_bins;
    const int b = (int)(k - i * (uint64_t)n_bins);
    const float T = temperature(u[i], xe[i]);
    out[k] = chandra_rate(t, G, arf, A, e[b], de[b], z, T, xe[i], rho[i], dL);
  }
}

// xray_spectral_flux (quantities.cl:400-430)
__global__ void __launch_bounds__(256)
xray_bin_kernel(const float* __restrict__ table, GauntView G, const float* __restrict__ rho,
                const float* __restrict__ u, const float* __restrict__ xe, uint64_t n, float z,
                float dL, float e, float de, float* __restrict__ out) {
  __shared__ float t[kMaxTable];
  load_table(t, table, G.w * G.h);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float T = temperature(u[i], xe[i]);
    out[i] = brems(t, G, (1.f + z) * e, (1.f + z) * de, T, xe[i], rho[i], dL);
  }
}

// xray_spectral_flux for n_bins bins at once (the quantity of each frame of
// spectrum_generator, spectrum.cpp:89-109): out[b * n + i] for cell i, bin b.
__global__ void __launch_bounds__(256)
xray_bins_kernel(const float* __restrict__ table, GauntView G, const float* __restrict__ rho,
                 const float* __restrict__ u, const float* __restrict__ xe, uint64_t n, float z,
                 float dL, const float* __restrict__ e, const float* __restrict__ de, int n_bins,
                 float* __restrict__ out) {
  // cell-major output out[i * n_bins + b]: consecutive threads write
  // consecutive bins of a cell, then the next cell
  __shared__ float t[kMaxTable];
  load_table(t, table, G.w * G.h);
  const uint64_t total = n * (uint64_t)n_bins;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = k / (uint64_t)n_bins;
    const int b = (int)(k - i * (uint64_t)n_bins);
    const float T = temperature(u[i], xe[i]);
    out[k] = brems(t, G, (1.f + z) * e[b], (1.f + z) * de[b], T, xe[i], rho[i], dL);
  }
}

// mean_temperature (quantities.cl:268-284)
__global__ void temperature_kernel(const float* __restrict__ u, const float* __restrict__ xe,
                                   uint64_t n, float* __restrict__ out) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i < n) out[i] = temperature(u[i], xe[i]);
}

unsigned persistent_blocks(uint64_t n) {
  const uint64_t want = (n + 255) / 256;
  return (unsigned)(want < 148 * 16 ? want : 148 * 16);
}

}  // namespace

cudaError_t quantity_xray_flux_launch(Context& c, const float* rho, const float* u,
                                      const float* xe, uint64_t n, float z, float dL,
                                      float emin, float emax, int num_samples, float* out,
                                      int out_stride) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  xray_flux_kernel<false><<<persistent_blocks(n), 256, 0, c.stream>>>(
      c.gaunt.as<float>(), G, rho, u, xe, n, z, dL, emin, emax, num_samples, out, out_stride);
  ++c.launches;
  return cudaGetLastError();
}

cudaError_t quantity_xray_photon_flux_launch(Context& c, const float* rho, const float* u,
                                             const float* xe, uint64_t n, float z, float dL,
                                             float emin, float emax, int num_samples,
                                             float* out) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  xray_flux_kernel<true><<<persistent_blocks(n), 256, 0, c.stream>>>(
      c.gaunt.as<float>(), G, rho, u, xe, n, z, dL, emin, emax, num_samples, out, 1);
  ++c.launches;
  return cudaGetLastError();
}

cudaError_t quantity_chandra_total_launch(Context& c, const float* rho, const float* u,
                                          const float* xe, uint64_t n, float z, float dL,
                                          float* out) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  ArfView A{c.arf_n, c.arf_x0, c.arf_dx};
  chandra_total_kernel<<<persistent_blocks(n), 256, 0, c.stream>>>(
      c.gaunt.as<float>(), G, c.arf.as<float>(), A, rho, u, xe, n, z, dL, out);
  ++c.launches;
  return cudaGetLastError();
}

cudaError_t quantity_chandra_bin_launch(Context& c, const float* rho, const float* u,
                                        const float* xe, uint64_t n, float z, float dL, float e,
                                        float de, float* out) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  ArfView A{c.arf_n, c.arf_x0, c.arf_dx};
  chandra_bin_kernel<<<persistent_blocks(n), 256, 0, c.stream>>>(
      c.gaunt.as<float>(), G, c.arf.as<float>(), A, rho, u, xe, n, z, dL, e, de, out);
  ++c.launches;
  return cudaGetLastError();
}

cudaError_t quantity_chandra_bins_launch(Context& c, const float* rho, const float* u,
                                         const float* xe, uint64_t n, float z, float dL,
                                         const float* e, const float* de, int n_bins,
                                         float* out) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  ArfView A{c.arf_n, c.arf_x0, c.arf_dx};
  chandra_bins_kernel<<<persistent_blocks(n * (uint64_t)n_bins), 256, 0, c.stream>>>(
      c.gaunt.as<float>(), G, c.arf.as<float>(), A, rho, u, xe, n, z, dL, e, de, n_bins, out);
  ++c.launches;
  return cudaGetLastError();
}

cudaError_t quantity_xray_bin_launch(Context& c, const float* rho, const float* u,
                                     const float* xe, uint64_t n, float z, float dL, float e,
                                     float de, float* out) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  ++c.launches;
  xray_bin_kernel<<<persistent_blocks(n), 256, 0, c.stream>>>(c.gaunt.as<float>(), G, rho, u,
                                                              xe, n, z, dL, e, de, out);
  return cudaGetLastError();
}

cudaError_t quantity_xray_bins_launch(Context& c, const float* rho, const float* u,
                                      const float* xe, uint64_t n, float z, float dL,
                                      const float* e, const float* de, int n_bins, float* out) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  ++c.launches;
  xray_bins_kernel<<<persistent_blocks(n * (uint64_t)n_bins), 256, 0, c.stream>>>(c.gaunt.as<float>(), G, rho, u, xe,
                                                               n, z, dL, e, de, n_bins, out);
  return cudaGetLastError();
}

cudaError_t quantity_temperature_launch(Context& c, const float* u, const float* xe,
                                        uint64_t n, float* out) {
  ++c.launches;
  temperature_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(u, xe, n, out);
  return cudaGetLastError();
}

}  // namespace ilc
