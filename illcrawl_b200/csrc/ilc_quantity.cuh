// ilc_quantity.cuh -- per-cell X-ray quantities of the reference
// (quantities.cl:38-136, 156-239) as device functions, shared by the quantity
// kernels and the adjoint.
//
// The OpenCL image lookup (read_imagef, CLK_FILTER_LINEAR, CLK_ADDRESS_CLAMP,
// unnormalised coordinates; tabulated_function.cl:26-59) is done in software
// with exact fp32 weights: the sample at u blends texels floor(u-0.5) and
// floor(u-0.5)+1 with weight frac(u-0.5); texels outside the table read 0.
#pragma once

#include "ilc_device.cuh"

namespace ilc {

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

// integrate_spectral_flux (quantities.cl:156-239): (rel_tol, 1) passed as
// (absolute, relative) tolerance, epsilon 0, step bounds [1e-3, 100].
// kPhoton = PHOTON_FLUX: every emission sample is divided by its energy.
template <bool kPhoton = false>
__device__ __forceinline__ float band_flux(const float* t, const GauntView& G, float Emin,
                                           float Emax, float reltol, float T, float xe,
                                           float rho, float dL) {
  float em = 0.0f, E = Emin;
  const float end = Emax;
  float dE = (end - E) * reltol;
  float k1 = brems(t, G, E, 1.0f, T, xe, rho, dL);
  if (kPhoton) k1 = k1 / E;
  float p[4];
  rkf_points(E, dE, p);
  int guard = 0;
  while (E < end && guard < 100000) {
    float v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[j] = brems(t, G, p[j], 1.0f, T, xe, rho, dL);
      if (kPhoton) v[j] = v[j] / p[j];
    }
    rkf_advance_ref32(em, E, dE, k1, reltol, 1.0f, end, v, 0.0f, 1.e-3f, 100.f, p);
    ++guard;
  }
  return em;
}

// A 1D tabulated function (util::tabulated_function, tabulated_function.hpp:
// 35-103): n samples from x0 in steps of dx. Used for the Chandra ARF.
struct ArfView {
  int n;
  float x0, dx;
};

// evaluate_tabulated_function (tabulated_function.cl:31-44): the 1D form of
// the software image lookup above; samples outside the table read 0.
__device__ __forceinline__ float tab1d(const float* __restrict__ t, const ArfView& A, float x) {
  float u = (x - A.x0) / A.dx;
  if (!(u == u)) return 0.0f;
  u = fminf(fmaxf(u, -4.0f), (float)(A.n + 4));
  const float us = u - 0.5f;
  const float fu = floorf(us);
  const int i0 = (int)fu;
  const float a = us - fu;
  const float t0 = (i0 >= 0 && i0 < A.n) ? __ldg(t + i0) : 0.0f;
  const float t1 = (i0 + 1 >= 0 && i0 + 1 < A.n) ? __ldg(t + i0 + 1) : 0.0f;
  return (1.0f - a) * t0 + a * t1;
}

// get_chandra_xray_count_rate_with_temp (quantities.cl:432-460): the photon
// count rate of the channel (E, dE) at redshift z times the ARF at E
// (cm^2 -> m^2), get_spectral_brems_count_rate (quantities.cl:251-260) being
// the emission divided by the redshifted energy.
__device__ __forceinline__ float chandra_rate(const float* t, const GauntView& G,
                                              const float* __restrict__ arf, const ArfView& A,
                                              float E, float dE, float z, float T, float xe,
                                              float rho, float dL) {
  const float av = tab1d(arf, A, E) * 1.e-4f;
  const float Ez = (1.f + z) * E;
  return brems(t, G, Ez, (1.f + z) * dE, T, xe, rho, dL) / Ez * av;
}

}  // namespace ilc
