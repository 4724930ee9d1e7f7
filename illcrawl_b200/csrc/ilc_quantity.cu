// ilc_quantity.cu -- per-cell quantity transforms of the X-ray path
// (quantities.cl:38-136, 156-239, 354-430) with the thermally averaged Gaunt
// factor table (gaunt_factor.cpp:30-41) resident in shared memory.
//
// The OpenCL image lookup (read_imagef, CLK_FILTER_LINEAR, CLK_ADDRESS_CLAMP,
// unnormalised coordinates; tabulated_function.cl:26-59) is done in software
// with exact fp32 weights: the sample at u blends texels floor(u-0.5) and
// floor(u-0.5)+1 with weight frac(u-0.5); texels outside the table read 0.
#include "ilc_device.cuh"
#include "ilc_internal.h"

namespace ilc {

namespace {

constexpr int kMaxTable = 81 * 146;

struct GauntView {
  int w, h;
  float x0, y0, dx, dy;
};

__device__ __forceinline__ float texel(const float* __restrict__ t, const GauntView& G, int i,
                                       int j) {
  if (i < 0 || j < 0 || i >= G.w || j >= G.h) return 0.0f;
  return t[j * G.w + i];
}

__device__ __forceinline__ float gaunt_sample(const float* __restrict__ t, const GauntView& G,
                                              float u, float v) {
  if (!(u == u) || !(v == v)) return 0.0f;
  u = fminf(fmaxf(u, -4.0f), (float)(G.w + 4));
  v = fminf(fmaxf(v, -4.0f), (float)(G.h + 4));
  const float us = u - 0.5f, vs = v - 0.5f;
  const float fu = floorf(us), fv = floorf(vs);
  const int i0 = (int)fu, j0 = (int)fv;
  const float a = us - fu, b = vs - fv;
  const float ia = 1.0f - a, ib = 1.0f - b;
  return ((ia * ib * texel(t, G, i0, j0) + a * ib * texel(t, G, i0 + 1, j0)) +
          ia * b * texel(t, G, i0, j0 + 1)) +
         a * b * texel(t, G, i0 + 1, j0 + 1);
}

// Constants of quantities.cl:29-36.
constexpr float kXH = 0.76f;
constexpr float kB = 8.61733e-5f;
constexpr float kRyd = 13.605f;

__device__ __forceinline__ float temperature(float u, float xe) {
  const float mu = 4.0f / (1.0f + 3.0f * kXH + 4.0f * kXH * xe);
  return (5.f / 3.f - 1.0f) * u * mu * 121.1475502f;
}

__device__ __forceinline__ float g_ff(const float* t, const GauntView& G, float E, float T,
                                      float Z) {
  const float gam2 = Z * Z * kRyd / (kB * T);
  const float u = 1.e3f * E / (kB * T);
  const float rx = (ilc_logf(gam2) - G.x0) / G.dx;
  const float ry = (ilc_logf(u) - G.y0) / G.dy;
  return gaunt_sample(t, G, rx, ry);
}

__device__ __forceinline__ float brems(const float* t, const GauntView& G, float E, float dE,
                                       float T, float xe, float rho, float r) {
  const float ion = 4.046263f * rho * xe;
  const float Z = 1.0f;
  const float Tinv = 1000.f / (kB * T);
  const float r2 = r * r;
  const float rs = 1.0f / sqrtf(T);
  return 0.002535f * dE * Z * Z * ion * ion * g_ff(t, G, E, T, Z) * rs * ilc_expf(-E * Tinv) /
         r2;
}

// integrate_spectral_flux(XRAY_FLUX): (rel_tol, 1) passed as (absolute,
// relative) tolerance, epsilon 0, step bounds [1e-3, 100].
__device__ __forceinline__ float band_flux(const float* t, const GauntView& G, float Emin,
                                           float Emax, float reltol, float T, float xe,
                                           float rho, float dL) {
  float em = 0.0f, E = Emin;
  const float end = Emax;
  float dE = (end - E) * reltol;
  float k1 = brems(t, G, E, 1.0f, T, xe, rho, dL);
  float p[4];
  rkf_points(E, dE, p);
  int guard = 0;
  while (E < end && guard < 100000) {
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) v[j] = brems(t, G, p[j], 1.0f, T, xe, rho, dL);
    rkf_advance_ref32(em, E, dE, k1, reltol, 1.0f, end, v, 0.0f, 1.e-3f, 100.f, p);
    ++guard;
  }
  return em;
}

__device__ __forceinline__ void load_table(float* dst, const float* __restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// xray_flux (quantities.cl:354-385)
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
    out[i * stride] = band_flux(t, G, (1.f + z) * emin, (1.f + z) * emax,
                                1.f / (float)num_samples, T, xe[i], rho[i], dL);
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
  xray_flux_kernel<<<persistent_blocks(n), 256, 0, c.stream>>>(
      c.gaunt.as<float>(), G, rho, u, xe, n, z, dL, emin, emax, num_samples, out, out_stride);
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

cudaError_t quantity_temperature_launch(Context& c, const float* u, const float* xe,
                                        uint64_t n, float* out) {
  ++c.launches;
  temperature_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(u, xe, n, out);
  return cudaGetLastError();
}

}  // namespace ilc
