// ilc_device.cuh -- device-side building blocks of the nn8 + RKF projection path.
//
// Every expression below is evaluated in the order written in the reference
// OpenCL kernels, with no FMA contraction (the translation units are built with
// -fmad=false) except where the reference itself calls fma(). Under that rule
// the kernels reproduce the CPU restatement of the reference bit for bit.
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace ilc {

// ---------------------------------------------------------------------------
// scalar helpers
// ---------------------------------------------------------------------------

// float -> int, truncating, saturating, NaN -> 0 (cvt.rzi.s32.f32).
__device__ __forceinline__ int to_int_sat(float f) { return __float2int_rz(f); }
__device__ __forceinline__ int to_int_sat(double f) { return __double2int_rz(f); }
// Cell indices are clamped so that adding a spiral offset cannot overflow.
__device__ __forceinline__ int clamp_cell(int c) { return min(max(c, -(1 << 30)), 1 << 30); }

// Natural logarithm, single precision: exponent/mantissa split with the
// mantissa folded into (1/sqrt2, sqrt2], ln(m) = 2*atanh(s), s = (m-1)/(m+1),
// as the odd series 2s(1 + s^2/3 + ... + s^10/11) in Horner form, plus e*ln2
// with a Cody-Waite hi/lo split of ln2.
__device__ __forceinline__ float ilc_logf(float x) {
  if (x != x) return x;
  if (x < 0.0f) return __int_as_float(0x7fc00000);
  if (x == 0.0f) return __int_as_float(0xff800000);
  if (x == __int_as_float(0x7f800000)) return x;
  int e = 0;
  if (x < 1.17549435e-38f) { x = x * 16777216.0f; e = -24; }
  const unsigned b = __float_as_uint(x);
  e += (int)((b >> 23) & 0xffu) - 127;
  float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421356f) { m = m * 0.5f; e = e + 1; }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  float p = 0.0909090909f;
  p = p * s2 + 0.111111111f;
  p = p * s2 + 0.142857143f;
  p = p * s2 + 0.2f;
  p = p * s2 + 0.333333333f;
  p = p * s2 + 1.0f;
  const float lm = (2.0f * s) * p;
  const float fe = (float)e;
  return fe * 0.693145751953125f + (lm + fe * 1.42860682e-06f);
}

// Exponential, single precision: Cody-Waite reduction x = n*ln2 + r with
// n = rint(x*log2(e)), exp(r) by its degree-7 Taylor polynomial (Horner), and
// the scaling by 2^n assembled from exponent bits (two factors if subnormal).
__device__ __forceinline__ float ilc_expf(float x) {
  if (x != x) return x;
  if (x > 88.7228394f) return __int_as_float(0x7f800000);
  if (x < -103.972084f) return 0.0f;
  const float n = rintf(x * 1.44269504f);
  const float r = (x - n * 0.693145751953125f) - n * 1.42860682e-06f;
  float p = 1.98412698e-04f;
  p = p * r + 1.38888889e-03f;
  p = p * r + 8.33333333e-03f;
  p = p * r + 4.16666667e-02f;
  p = p * r + 1.66666667e-01f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  int ni = (int)n;
  if (ni > 127) { p = p * __uint_as_float(0x7f000000u); ni -= 127; }
  if (ni < -126) { p = p * __uint_as_float(0x00800000u); ni += 126; }
  return p * __uint_as_float((unsigned)(ni + 127) << 23);
}

// ---------------------------------------------------------------------------
// particle grid view (particle_grid.hpp:40-131)
// ---------------------------------------------------------------------------
struct GridView {
  float min0, min1, min2;     // grid min corner (float cast of the host double)
  float cs0, cs1, cs2;        // cell sizes
  float half0, half1, half2;  // 0.5f * cell sizes
  float cell_radius;          // 0.5f * sqrtf(dot(cs, cs))
  int n0, n1, n2;             // cells per axis
  const int2* __restrict__ cells;     // [begin, end) per cell
  const float4* __restrict__ parts;   // (x, y, z, q) in cell order
  // Sub-box codes for exact candidate pruning: per sorted particle one byte,
  // sx + 4 sy + 16 sz, its quarter of the cell per axis (read 16 at a time
  // from a 16-byte aligned buffer padded to a multiple of 16 bytes).
  const uint32_t* __restrict__ codes;
  float inv_w0, inv_w1, inv_w2;       // 4 / cell size
  float margin;                       // slack covering float rounding (cell size / 1024)
};

// Per-thread walk statistics (algorithmic traffic accounting).
struct WalkStats {
  uint32_t cells = 0;
  uint32_t cands = 0;
};

// Slot state of one query: the reference's 8-entry (distance, value) lists.
template <bool kIds> struct Slots {
  float d[8];
  float v[8];
  int id[8];
  float R;      // search radius = max slot distance
  float R2up;   // R*R rounded up: candidates with d^2 above it cannot enter
  int mi;       // first slot holding the maximum

  __device__ __forceinline__ void init() {
#pragma unroll
    for (int j = 0; j < 8; ++j) { d[j] = FLT_MAX; v[j] = 0.0f; if (kIds) id[j] = -1; }
    rescan();
  }
  // search radius and max slot (volumetric_nn8_reconstruction.cl:135-143)
  __device__ __forceinline__ void rescan() {
    float r = 0.0f;
    int m = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      if (d[j] > r) m = j;
      r = fmaxf(r, d[j]);
    }
    R = r;
    mi = m;
    R2up = __fmul_ru(r, r);
  }
  __device__ __forceinline__ void insert(float dist, float val, int pid) {
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (j == mi) { d[j] = dist; v[j] = val; if (kIds) id[j] = pid; }
    rescan();
  }
};

// The reference's nn8 walk for one query (volumetric_nn8_reconstruction.cl:128-204).
// spiral: the 8 x 125 cell-offset table (shared memory).
template <bool kIds>
__device__ __forceinline__ void nn8_walk(const GridView& g, const char4* __restrict__ spiral,
                                         float qx, float qy, float qz, Slots<kIds>& s,
                                         WalkStats& st) {
  const int cx = clamp_cell(to_int_sat(floorf((qx - g.min0) / g.cs0)));
  const int cy = clamp_cell(to_int_sat(floorf((qy - g.min1) / g.cs1)));
  const int cz = clamp_cell(to_int_sat(floorf((qz - g.min2) / g.cs2)));
  const float mx = g.min0 + (float)cx * g.cs0;
  const float my = g.min1 + (float)cy * g.cs1;
  const float mz = g.min2 + (float)cz * g.cs2;
  int sx = to_int_sat(floorf((qx - mx) / g.half0));
  int sy = to_int_sat(floorf((qy - my) / g.half1));
  int sz = to_int_sat(floorf((qz - mz) / g.half2));
  sx = min(max(sx, 0), 1);
  sy = min(max(sy, 0), 1);
  sz = min(max(sz, 0), 1);
  const char4* order = spiral + (sx + 2 * sy + 4 * sz) * 125;
  for (int it = 0; it < 125; ++it) {
    const char4 o = order[it];
    const int ix = cx + o.x, iy = cy + o.y, iz = cz + o.z;
    const float ex = ((g.min0 + (float)ix * g.cs0) + g.half0) - qx;
    const float ey = ((g.min1 + (float)iy * g.cs1) + g.half1) - qy;
    const float ez = ((g.min2 + (float)iz * g.cs2) + g.half2) - qz;
    const float r = s.R + g.cell_radius;
    if ((ex * ex + ey * ey) + ez * ez > r * r) break;
    if ((unsigned)ix >= (unsigned)g.n0 || (unsigned)iy >= (unsigned)g.n1 ||
        (unsigned)iz >= (unsigned)g.n2)
      continue;
    const size_t key = (size_t)ix + (size_t)iy * (size_t)g.n0 +
                       (size_t)iz * (size_t)g.n0 * (size_t)g.n1;
    const int2 be = __ldg(&g.cells[key]);
    st.cells += 1;
    st.cands += (uint32_t)max(be.y - be.x, 0);
    for (int p = be.x; p < be.y; ++p) {
      const float4 P = __ldg(&g.parts[p]);
      const float fx = P.x - qx, fy = P.y - qy, fz = P.z - qz;
      const float d2 = (fx * fx + fy * fy) + fz * fz;
      if (d2 <= s.R2up) {
        const float dist = sqrtf(d2);
        if (dist < s.R) s.insert(dist, P.w, p);
      }
    }
  }
}

// get_weight3d + finalize (volumetric_nn8_reconstruction.cl:44-50,212-270)
__device__ __forceinline__ float weight3d(float d) {
  const float i2 = 1.0f / (d * d);
  const float i4 = i2 * i2;
  return (i4 * i4) * i2;
}

template <bool kIds> __device__ __forceinline__ float nn8_finalize(const Slots<kIds>& s) {
  float w[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) w[j] = weight3d(s.d[j]);
  float ws = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) ws = ws + w[j];
  float dot = 0.0f;
#pragma unroll
  for (int j = 0; j < 8; ++j) dot = __fmaf_rn(w[j], s.v[j], dot);
  float res = 0.0f;
  if (ws != 0.0f && dot != 0.0f) res = dot / ws;
  return res;
}

__device__ __forceinline__ float nn8_value(const GridView& g, const char4* spiral, float x,
                                           float y, float z, WalkStats& st) {
  Slots<false> s;
  s.init();
  nn8_walk<false>(g, spiral, x, y, z, s, st);
  return nn8_finalize(s);
}

// Copies the 8 x 125 spiral table into shared memory (block-wide).
__device__ __forceinline__ void load_spiral(char4* dst, const char4* __restrict__ src) {
  for (int i = threadIdx.x + threadIdx.y * blockDim.x; i < 1000;
       i += blockDim.x * blockDim.y)
    dst[i] = src[i];
  __syncthreads();
}

// ---------------------------------------------------------------------------
// RKF4(5) step (integration.cl:34-131)
// ---------------------------------------------------------------------------
constexpr float kEps = 0.01f, kHmin = 0.2f, kHmax = 100.f;

__device__ __forceinline__ void rkf_points(float z, float h, float p[4]) {
  p[0] = z + 3.f / 8.f * h;
  p[1] = z + 12.f / 13.f * h;
  p[2] = z + h;
  p[3] = z + 0.5f * h;
}

// fp32 controller exactly as the reference (pow(x, 0.25f) as sqrtf(sqrtf(x))).
__device__ __forceinline__ void rkf_advance_ref32(float& I, float& z, float& h, float& k1,
                                                  float atol, float rtol, float end,
                                                  const float e[4], float eps, float hmin,
                                                  float hmax, float next[4]) {
  float d4 = 25.f / 216.f * k1 + 1408.f / 2565.f * e[0] + 2197.f / 4101.f * e[1] -
             1.f / 5.f * e[2];
  float d5 = 16.f / 135.f * k1 + 6656.f / 12825.f * e[0] + 28561.f / 56430.f * e[1] -
             9.f / 50.f * e[2] + 2.f / 55.f * e[3];
  d4 *= h;
  d5 *= h;
  const float est4 = I + d4;
  const float old = z;
  z += h;
  float s = 2.0f;
  if (d4 != d5) {
    const float err = fabsf(d5 - d4);
    const float srt = fabsf(I / z * rtol);
    const float ot = fmaxf(atol, srt);
    s = sqrtf(sqrtf(ot * h / (2.0f * err)));
  }
  float nh = s * h;
  if (nh < hmin) nh = hmin;
  else if (nh > hmax) nh = hmax;
  s = nh / h;
  if (s < 0.95f) {
    z = old;
  } else {
    I = est4;
    k1 = e[2];
  }
  h = nh;
  if (z + h >= end) h = end - z + eps;
  rkf_points(z, h, next);
}

// FP64 controller over the fp32 state (increments, error, tolerance and
// acceptance in double; I, z, h, k1 and the evaluation points fp32).
__device__ __forceinline__ void rkf_advance_fp64(float& I, float& z, float& h, float& k1,
                                                 double atol, double rtol, float end,
                                                 const float e[4], float eps, float hmin,
                                                 float hmax, float next[4]) {
  const double hd = (double)h;
  double d4 = 25.0 / 216.0 * (double)k1 + 1408.0 / 2565.0 * (double)e[0] +
              2197.0 / 4101.0 * (double)e[1] - 1.0 / 5.0 * (double)e[2];
  double d5 = 16.0 / 135.0 * (double)k1 + 6656.0 / 12825.0 * (double)e[0] +
              28561.0 / 56430.0 * (double)e[1] - 9.0 / 50.0 * (double)e[2] +
              2.0 / 55.0 * (double)e[3];
  d4 *= hd;
  d5 *= hd;
  const float est4 = (float)((double)I + d4);
  const float old = z;
  const float znew = z + h;
  double s = 2.0;
  if (d4 != d5) {
    const double err = fabs(d5 - d4);
    const double srt = fabs((double)I / (double)znew * rtol);
    const double ot = fmax(atol, srt);
    s = sqrt(sqrt(ot * hd / (2.0 * err)));
  }
  double nh = s * hd;
  if (nh < (double)hmin) nh = (double)hmin;
  else if (nh > (double)hmax) nh = (double)hmax;
  s = nh / hd;
  if (s < 0.95) {
    z = old;
  } else {
    z = znew;
    I = est4;
    k1 = e[2];
  }
  h = (float)nh;
  if (z + h >= end) h = end - z + eps;
  rkf_points(z, h, next);
}

// ---------------------------------------------------------------------------
// camera plane (integration.cl:190-235): pixel corner and ray direction
// ---------------------------------------------------------------------------
struct CamView {
  float look0, look1, look2;
  float b00, b01, b02;
  float b10, b11, b12;
  float min0, min1, min2;
  float ps;
  int nx, ny;
};

__device__ __forceinline__ void pixel_corner(const CamView& c, int ix, int iy, float& px,
                                             float& py, float& pz) {
  const float tx = (float)ix * c.ps, ty = (float)iy * c.ps;
  px = (c.min0 + tx * c.b00) + ty * c.b10;
  py = (c.min1 + tx * c.b01) + ty * c.b11;
  pz = (c.min2 + tx * c.b02) + ty * c.b12;
}

}  // namespace ilc
