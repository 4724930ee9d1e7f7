// ilc_adjoint_cell.cuh -- per-cell X-ray band flux with its derivatives with
// respect to ln T and ln rho, for the adjoint.
//
// The band flux is the adaptive energy integration of quantities.cl:156-239.
// Its step sizes move with T and rho (the controller's error estimate scales
// with the integrand), so the derivatives are taken in forward mode through
// the whole integration: the value part repeats the forward's operations and
// decisions exactly (so q is bit-identical to xray_flux_kernel's), and every
// state variable carries a double tangent -- through the sqrt(sqrt()) step
// factor, the clamps (zero tangent when clamped) and the final-step fix.
#pragma once

#include "ilc_device.cuh"

namespace ilc {

struct GauntViewD {
  int w, h;
  float x0, y0, dx, dy;
};

__device__ __forceinline__ double texel_d(const float* __restrict__ t, const GauntViewD& G, int i,
                                          int j) {
  if (i < 0 || j < 0 || i >= G.w || j >= G.h) return 0.0;
  return (double)t[j * G.w + i];
}

// Bilinear blend (OpenCL linear filter, clamp-to-border 0) and its partials.
__device__ __forceinline__ void gaunt_d(const float* t, const GauntViewD& G, double u, double v,
                                        double* g, double* gu, double* gv) {
  *g = *gu = *gv = 0.0;
  if (!(u == u) || !(v == v)) return;
  u = fmin(fmax(u, -4.0), (double)(G.w + 4));
  v = fmin(fmax(v, -4.0), (double)(G.h + 4));
  const double us = u - 0.5, vs = v - 0.5;
  const double fu = floor(us), fv = floor(vs);
  const int i0 = (int)fu, j0 = (int)fv;
  const double a = us - fu, b = vs - fv;
  const double t00 = texel_d(t, G, i0, j0), t10 = texel_d(t, G, i0 + 1, j0);
  const double t01 = texel_d(t, G, i0, j0 + 1), t11 = texel_d(t, G, i0 + 1, j0 + 1);
  *g = (((1 - a) * (1 - b) * t00 + a * (1 - b) * t10) + (1 - a) * b * t01) + a * b * t11;
  *gu = (1 - b) * (t10 - t00) + b * (t11 - t01);
  *gv = (1 - a) * (t01 - t00) + a * (t11 - t10);
}

// Partial derivatives of the spectral emission (dE = 1) at fixed rho, xe:
//   base = A T^-1/2 exp(-E Tinv)/r^2, Tinv = 1000/(kB T)
//   d/dlnT = base (g (E Tinv - 1/2) - (g_u/dx + g_v/dy));  d/dlnrho = 2 brems
//   d/dE   = base (-g Tinv + g_v/(dy E))
__device__ __forceinline__ void brems_tangent(const float* t, const GauntViewD& G, double E,
                                              double T, double xe, double rho, double r,
                                              int which, double* d_param, double* d_E,
                                              double value) {
  const double kB = 8.61733e-5;
  const double ion = 4.046263 * rho * xe;
  const double Tinv = 1000.0 / (kB * T);
  const double ux = (log(13.605 / (kB * T)) - (double)G.x0) / (double)G.dx;
  const double vy = (log(1.e3 * E / (kB * T)) - (double)G.y0) / (double)G.dy;
  double g, gu, gv;
  gaunt_d(t, G, ux, vy, &g, &gu, &gv);
  const double base = 0.002535 * ion * ion / sqrt(T) * exp(-E * Tinv) / (r * r);
  *d_param = which == 0 ? base * (g * (E * Tinv - 0.5) - (gu / (double)G.dx + gv / (double)G.dy))
                        : 2.0 * value;
  *d_E = base * (-g * Tinv + gv / ((double)G.dy * E));
}

__device__ __forceinline__ double sgnd(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

}  // namespace ilc
