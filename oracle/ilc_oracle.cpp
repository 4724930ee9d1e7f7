// ilc_oracle.cpp -- CPU restatement of illcrawl's volumetric projection path.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker: tests/, the smoke
// check in __graft_entry__.py and the cpu_baseline leg of bench.py load it to
// compare the CUDA product against. Nothing in illcrawl_b200/ links it or
// falls back to it.
//
// What it restates (reference file:line in the illcrawl sources):
//   grid build ............ particle_grid.cpp:25-119,151-252, particle_grid.cl:45-190, util.cl:24-49
//   spiral walk table ..... particle_grid_iteration_order.cl:25-1048 (regenerated, see spiral_table())
//   nn8 search + finalize . volumetric_nn8_reconstruction.cl:44-270
//   camera ................ camera.cpp:27-41,124-155, math.hpp:85-149
//   line-of-sight RKF ..... integration.cl:34-259, integration.cpp:161-307,
//                           volumetric_integration.cpp:32-88
//   X-ray quantities ...... quantities.cl:29-136,156-239,354-430,701-711
//   Gaunt lookup .......... tabulated_function.cl:26-59, gaunt_factor.cpp:30-41
//
// Parity status: parity unpinned. The reference ships no tests, golden vectors
// or fixtures for this path, and its OpenCL kernels cannot be run here. The
// reference-pinned artefacts are its tables: the spiral table (checked for
// equality against the reference file), the Gaunt table (the reference data
// file itself) and the Chandra ARF (extracted from the reference source into
// a test fixture). Everything else is pinned to the op order declared here:
// every expression is evaluated left to right exactly as written in the OpenCL
// source, with no contraction into FMA except where the source calls fma()
// (compile with -ffp-contract=off). Declared deviations from the OpenCL text:
//   * pow(x, 0.25f) in rkf_advance is evaluated as sqrtf(sqrtf(x));
//   * log/exp in the Gaunt lookup and emissivity use ilc_logf/ilc_expf below
//     (textbook methods, named there) instead of the vendor builtins;
//   * rsqrt(T) is 1.0f/sqrtf(T);
//   * OpenCL linear image filtering is emulated with exact fp32 weights;
//   * the subcell index is clamped to [0,1] per axis (the reference reads past
//     its table when rounding puts a point on a cell's far edge);
//   * float->int conversions saturate and map NaN to 0 (CUDA cvt.rzi semantics).
// The double instantiation (precision = 1) is the FP64 oracle: the same
// algorithm with every device-side quantity in double.

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace orc {

// --------------------------------------------------------------------------
// Scalar helpers
// --------------------------------------------------------------------------

static inline float f_bits(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
static inline uint32_t bits_f(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }

// float -> int32 with saturation, NaN -> 0 (matches CUDA's cvt.rzi.s32.f32).
static inline int to_int_sat(float f) {
  if (f != f) return 0;
  if (f >= 2147483648.0f) return INT_MAX;
  if (f <= -2147483648.0f) return INT_MIN;
  return (int)f;
}
static inline int to_int_sat(double f) {
  if (f != f) return 0;
  if (f >= 2147483648.0) return INT_MAX;
  if (f <= -2147483648.0) return INT_MIN;
  return (int)f;
}
// Cell indices are clamped so that adding a spiral offset cannot overflow.
static inline int clamp_cell(int c) {
  return std::min(std::max(c, -(1 << 30)), 1 << 30);
}

// Natural logarithm, single precision. Method: exponent/mantissa split with
// the mantissa folded into (1/sqrt2, sqrt2], then ln(m) = 2*atanh(s) with
// s = (m-1)/(m+1) summed as the odd power series 2s(1 + s^2/3 + ... + s^10/11)
// (Horner form), and e*ln2 added with the Cody-Waite hi/lo split of ln2.
static inline float ilc_logf(float x) {
  if (x != x) return x;
  if (x < 0.0f) return NAN;
  if (x == 0.0f) return -INFINITY;
  if (x == INFINITY) return INFINITY;
  int e = 0;
  if (x < 1.17549435e-38f) { x = x * 16777216.0f; e = -24; }
  uint32_t b = bits_f(x);
  e += (int)((b >> 23) & 0xffu) - 127;
  float m = f_bits((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421356f) { m = m * 0.5f; e = e + 1; }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  float p = 0.0909090909f;          // 1/11
  p = p * s2 + 0.111111111f;        // 1/9
  p = p * s2 + 0.142857143f;        // 1/7
  p = p * s2 + 0.2f;                // 1/5
  p = p * s2 + 0.333333333f;        // 1/3
  p = p * s2 + 1.0f;
  const float lm = (2.0f * s) * p;
  const float fe = (float)e;
  return fe * 0.693145751953125f + (lm + fe * 1.42860682e-06f);
}

// Exponential, single precision. Method: Cody-Waite reduction x = n*ln2 + r
// with n = rint(x*log2(e)) and ln2 split into hi/lo parts, exp(r) by its
// Taylor polynomial to degree 7 in Horner form, then scaling by 2^n built from
// the exponent bits (two factors when the result is subnormal).
static inline float ilc_expf(float x) {
  if (x != x) return x;
  if (x > 88.7228394f) return INFINITY;
  if (x < -103.972084f) return 0.0f;
  const float n = rintf(x * 1.44269504f);
  const float r = (x - n * 0.693145751953125f) - n * 1.42860682e-06f;
  float p = 1.98412698e-04f;        // 1/5040
  p = p * r + 1.38888889e-03f;      // 1/720
  p = p * r + 8.33333333e-03f;      // 1/120
  p = p * r + 4.16666667e-02f;      // 1/24
  p = p * r + 1.66666667e-01f;      // 1/6
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  int ni = (int)n;
  if (ni > 127) { p = p * f_bits(0x7f000000u); ni -= 127; }
  if (ni < -126) { p = p * f_bits(0x00800000u); ni += 126; }
  return p * f_bits((uint32_t)(ni + 127) << 23);
}

template <class R> struct mathf;
template <> struct mathf<float> {
  static float log(float x) { return ilc_logf(x); }
  static float exp(float x) { return ilc_expf(x); }
  static float sqrt(float x) { return sqrtf(x); }
  static float floor(float x) { return floorf(x); }
  static float fabs(float x) { return fabsf(x); }
  static float fmax(float a, float b) { return fmaxf(a, b); }
  static float fma(float a, float b, float c) { return fmaf(a, b, c); }
  static float maxval() { return FLT_MAX; }
};
template <> struct mathf<double> {
  static double log(double x) { return std::log(x); }
  static double exp(double x) { return std::exp(x); }
  static double sqrt(double x) { return std::sqrt(x); }
  static double floor(double x) { return std::floor(x); }
  static double fabs(double x) { return std::fabs(x); }
  static double fmax(double a, double b) { return std::fmax(a, b); }
  static double fma(double a, double b, double c) { return std::fma(a, b, c); }
  // The double oracle keeps the reference's "unset" marker MAXFLOAT.
  static double maxval() { return (double)FLT_MAX; }
};

// --------------------------------------------------------------------------
// Spiral iteration table (particle_grid_iteration_order.cl:25-1048).
// For each of the 8 subcells (id = sx + 2*sy + 4*sz) the 125 cell offsets in
// [-2,2]^3, enumerated with x outermost and z innermost, stable-sorted by the
// distance between the subcell centre (+-0.25 cell) and the offset cell centre.
// --------------------------------------------------------------------------
static void spiral_table(int8_t out[8][125][3]) {
  for (int sz = 0; sz < 2; ++sz)
    for (int sy = 0; sy < 2; ++sy)
      for (int sx = 0; sx < 2; ++sx) {
        const int id = sx + 2 * sy + 4 * sz;
        const double c[3] = {sx ? 0.25 : -0.25, sy ? 0.25 : -0.25, sz ? 0.25 : -0.25};
        struct E { int d[3]; double dist; };
        std::vector<E> v;
        for (int dx = -2; dx <= 2; ++dx)
          for (int dy = -2; dy <= 2; ++dy)
            for (int dz = -2; dz <= 2; ++dz) {
              const double a = dx - c[0], b = dy - c[1], g = dz - c[2];
              v.push_back(E{{dx, dy, dz}, std::sqrt(a * a + b * b + g * g)});
            }
        std::stable_sort(v.begin(), v.end(),
                         [](const E& l, const E& r) { return l.dist < r.dist; });
        for (int i = 0; i < 125; ++i)
          for (int k = 0; k < 3; ++k) out[id][i][k] = (int8_t)v[i].d[k];
      }
}

static int8_t g_spiral[8][125][3];
static bool g_spiral_ready = false;
static void ensure_spiral() {
  if (!g_spiral_ready) { spiral_table(g_spiral); g_spiral_ready = true; }
}

// --------------------------------------------------------------------------
// Particle grid (particle_grid.cpp:25-119 ctor, :151-252 build_tiles/sort).
// --------------------------------------------------------------------------
struct Grid {
  float min[3];
  float cs[3];
  int32_t n[3];
  uint64_t total;
  std::vector<float> sorted;       // float4 (x,y,z,q) in cell order
  std::vector<int32_t> cells;      // int2 [begin, end) per grid cell
  std::vector<uint32_t> s2u;       // sorted index -> original index
  std::vector<uint64_t> keys;      // cell key per sorted particle
};

// key = ix + iy*nx + iz*nx*ny from floor((p - min)/cs)  (particle_grid.cl:45-93)
static inline uint64_t cell_key(const Grid& g, const float* p) {
  int idx[3];
  for (int i = 0; i < 3; ++i) idx[i] = to_int_sat(floorf((p[i] - g.min[i]) / g.cs[i]));
  return (uint64_t)(int64_t)idx[0] + (uint64_t)(int64_t)idx[1] * (uint64_t)g.n[0] +
         (uint64_t)(int64_t)idx[2] * (uint64_t)g.n[0] * (uint64_t)g.n[1];
}

// Host-side grid parameters, in double, exactly as particle_grid.cpp:54-103.
static int grid_params(const float* p, size_t n, size_t target, Grid* g) {
  if (n == 0) return 1;
  double mn[3], mx[3];
  for (int j = 0; j < 3; ++j) mn[j] = mx[j] = (double)p[j];
  for (size_t k = 0; k < n; ++k)
    for (int i = 0; i < 3; ++i) {
      const double c = (double)p[4 * k + i];
      if (!std::isfinite(c)) return 2;
      if (c < mn[i]) mn[i] = c;
      if (c > mx[i]) mx[i] = c;
    }
  double vol = 1.0;
  for (int i = 0; i < 3; ++i) {
    mn[i] -= 0.1;
    mx[i] += 0.1;
    vol *= (mx[i] - mn[i]);
  }
  const double cell_volume = (double)target / (double)n * vol;
  const double w = std::cbrt(cell_volume);
  g->total = 1;
  for (int i = 0; i < 3; ++i) {
    g->n[i] = (int32_t)std::ceil((mx[i] - mn[i]) / w);
    g->min[i] = (float)mn[i];
    g->cs[i] = (float)w;
    g->total *= (uint64_t)g->n[i];
  }
  return 0;
}

static int grid_build(const float* p, size_t n, Grid* g) {
  int st = grid_params(p, n, 8, g);
  if (st) return st;
  std::vector<uint64_t> key(n);
  for (size_t i = 0; i < n; ++i) {
    key[i] = cell_key(*g, p + 4 * i);
    if (key[i] >= g->total) return 3;
  }
  // boost::compute::sort_by_key(keys, iota) is a stable radix sort
  // (particle_grid.cpp:225-252); std::stable_sort gives the same permutation.
  std::vector<uint32_t> perm(n);
  for (size_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
  std::stable_sort(perm.begin(), perm.end(),
                   [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
  g->sorted.resize(4 * n);
  g->s2u = perm;
  g->keys.resize(n);
  for (size_t i = 0; i < n; ++i) {
    std::memcpy(&g->sorted[4 * i], p + 4 * (size_t)perm[i], 16);
    g->keys[i] = key[perm[i]];
  }
  // grid3d_determine_cells_begin / _end over a zero-filled cell buffer
  // (particle_grid.cpp:110-113, particle_grid.cl:114-190).
  g->cells.assign(2 * g->total, 0);
  for (size_t i = 0; i < n; ++i) {
    const uint64_t k = g->keys[i];
    if (i == 0 || g->keys[i - 1] != k) g->cells[2 * k] = (int32_t)i;
    if (i + 1 == n || g->keys[i + 1] != k) g->cells[2 * k + 1] = (int32_t)(i + 1);
  }
  return 0;
}

// --------------------------------------------------------------------------
// nn8 search (volumetric_nn8_reconstruction.cl:87-210) and finalize (:212-270)
// --------------------------------------------------------------------------
template <class R> struct Slots {
  R d[8];
  R v[8];
  int32_t id[8];
};

template <class R> static inline void rescan(const Slots<R>& s, R& radius, int& maxi) {
  radius = (R)0;
  maxi = 0;
  for (int j = 0; j < 8; ++j) {
    if (s.d[j] > radius) maxi = j;
    radius = mathf<R>::fmax(radius, s.d[j]);
  }
}

struct SearchStats { uint64_t cells = 0, candidates = 0; };

template <class R>
static void nn8_search(const Grid& g, R qx, R qy, R qz, Slots<R>& s, SearchStats* st) {
  typedef mathf<R> M;
  const R gmin[3] = {(R)g.min[0], (R)g.min[1], (R)g.min[2]};
  const R gcs[3] = {(R)g.cs[0], (R)g.cs[1], (R)g.cs[2]};
  const R q[3] = {qx, qy, qz};
  int c[3];
  R cmin[3];
  for (int i = 0; i < 3; ++i) {
    c[i] = clamp_cell(to_int_sat(M::floor((q[i] - gmin[i]) / gcs[i])));
    cmin[i] = gmin[i] + (R)c[i] * gcs[i];
  }
  const R cell_radius = (R)0.5 * M::sqrt((gcs[0] * gcs[0] + gcs[1] * gcs[1]) + gcs[2] * gcs[2]);
  R radius;
  int maxi;
  rescan(s, radius, maxi);
  int sub[3];
  for (int i = 0; i < 3; ++i) {
    const R hcs = (R)0.5 * gcs[i];
    int si = to_int_sat(M::floor((q[i] - cmin[i]) / hcs));
    sub[i] = si < 0 ? 0 : (si > 1 ? 1 : si);
  }
  const int subcell = sub[0] + 2 * sub[1] + 4 * sub[2];
  const int8_t(*order)[3] = g_spiral[subcell];
  for (int it = 0; it < 125; ++it) {
    const int cc[3] = {c[0] + order[it][0], c[1] + order[it][1], c[2] + order[it][2]};
    R e[3];
    for (int i = 0; i < 3; ++i) {
      const R center = (gmin[i] + (R)cc[i] * gcs[i]) + (R)0.5 * gcs[i];
      e[i] = center - q[i];
    }
    const R r = radius + cell_radius;
    if ((e[0] * e[0] + e[1] * e[1]) + e[2] * e[2] > r * r) break;
    if (cc[0] < 0 || cc[1] < 0 || cc[2] < 0 || cc[0] >= g.n[0] || cc[1] >= g.n[1] ||
        cc[2] >= g.n[2])
      continue;
    const uint64_t key = (uint64_t)cc[0] + (uint64_t)cc[1] * (uint64_t)g.n[0] +
                         (uint64_t)cc[2] * (uint64_t)g.n[0] * (uint64_t)g.n[1];
    const int32_t b = g.cells[2 * key], en = g.cells[2 * key + 1];
    if (st) { st->cells += 1; st->candidates += (uint64_t)(en > b ? en - b : 0); }
    for (int32_t p = b; p < en; ++p) {
      const float* P = &g.sorted[4 * (size_t)p];
      const R fx = (R)P[0] - q[0], fy = (R)P[1] - q[1], fz = (R)P[2] - q[2];
      const R dist = M::sqrt((fx * fx + fy * fy) + fz * fz);
      if (dist < radius) {
        s.d[maxi] = dist;
        s.v[maxi] = (R)P[3];
        s.id[maxi] = p;
        rescan(s, radius, maxi);
      }
    }
  }
}

template <class R> static inline void slots_init(Slots<R>& s) {
  for (int j = 0; j < 8; ++j) { s.d[j] = mathf<R>::maxval(); s.v[j] = (R)0; s.id[j] = -1; }
}

// get_weight3d (volumetric_nn8_reconstruction.cl:44-50)
template <class R> static inline R weight3d(R d) {
  const R i2 = (R)1 / (d * d);
  const R i4 = i2 * i2;
  return (i4 * i4) * i2;
}

template <class R> static inline R nn8_finalize(const Slots<R>& s) {
  R w[8];
  for (int j = 0; j < 8; ++j) w[j] = weight3d(s.d[j]);
  R ws = (R)0;
  for (int j = 0; j < 8; ++j) ws += w[j];
  R dot = (R)0;
  for (int j = 0; j < 8; ++j) dot = mathf<R>::fma(w[j], s.v[j], dot);
  R res = (R)0;
  if (ws != (R)0 && dot != (R)0) res = dot / ws;
  return res;
}

template <class R> static inline R nn8_value(const Grid& g, R x, R y, R z, SearchStats* st) {
  Slots<R> s;
  slots_init(s);
  nn8_search(g, x, y, z, s, st);
  return nn8_finalize(s);
}

// --------------------------------------------------------------------------
// Camera (camera.cpp:27-41, :124-155) -- host side, double
// --------------------------------------------------------------------------
struct Camera {
  double position[3];
  double look_at[3];
  double roll;
  double screen_width;
  int32_t nx, ny;
};

struct CamDev {       // what the device kernels receive (float4 casts)
  float look[3], b0[3], b1[3], minp[3];
  float ps;
  double ps_d;        // pixel size in double (scaling and FP64 oracle)
  double look_d[3], b0_d[3], b1_d[3], minp_d[3];
};

static inline double dot3(const double* a, const double* b) {
  double r = 0.0;
  for (int i = 0; i < 3; ++i) r += a[i] * b[i];
  return r;
}
static inline void cross3(const double* a, const double* b, double* o) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

static void camera_setup(const Camera& cam, CamDev* d) {
  const double ps = cam.screen_width / (double)cam.nx;
  double v1[3] = {0, 0, 1};
  if (cam.look_at[0] == v1[0] && cam.look_at[1] == v1[1] && cam.look_at[2] == v1[2]) {
    v1[0] = 0; v1[1] = 1; v1[2] = 0;
  }
  double a[3], b[3];
  cross3(v1, cam.look_at, a);
  cross3(cam.look_at, a, b);
  // math::matrix_create_rotation_matrix(look_at, roll)  (math.hpp:109-138)
  const double a1 = cam.look_at[0], a2 = cam.look_at[1], a3 = cam.look_at[2];
  const double a1a2 = a1 * a2, a1a3 = a1 * a3, a2a3 = a2 * a3;
  const double ca = std::cos(cam.roll), sa = std::sin(cam.roll);
  const double fc = 1.0 - ca;
  const double m[3][3] = {{a1 * a1 * fc + ca, a1a2 * fc - a3 * sa, a1a3 * fc + a2 * sa},
                          {a1a2 * fc + a3 * sa, a2 * a2 * fc + ca, a2a3 * fc - a1 * sa},
                          {a1a3 * fc - a2 * sa, a2a3 * fc + a1 * sa, a3 * a3 * fc + ca}};
  double ra[3], rb[3];
  for (int i = 0; i < 3; ++i) { ra[i] = dot3(m[i], a); rb[i] = dot3(m[i], b); }
  const double la = 1. / std::sqrt(dot3(ra, ra)), lb = 1. / std::sqrt(dot3(rb, rb));
  double b0[3], b1[3], mp[3];
  for (int i = 0; i < 3; ++i) { b0[i] = la * ra[i]; b1[i] = lb * rb[i]; }
  for (int i = 0; i < 3; ++i) mp[i] = cam.position[i];
  for (int i = 0; i < 3; ++i) mp[i] -= ((double)cam.nx / 2.0) * ps * b0[i];
  for (int i = 0; i < 3; ++i) mp[i] -= ((double)cam.ny / 2.0) * ps * b1[i];
  for (int i = 0; i < 3; ++i) {
    d->look[i] = (float)cam.look_at[i]; d->b0[i] = (float)b0[i];
    d->b1[i] = (float)b1[i]; d->minp[i] = (float)mp[i];
    d->look_d[i] = cam.look_at[i]; d->b0_d[i] = b0[i];
    d->b1_d[i] = b1[i]; d->minp_d[i] = mp[i];
  }
  d->ps = (float)ps;
  d->ps_d = ps;
}

// --------------------------------------------------------------------------
// RKF4(5) line-of-sight integrator (integration.cl:34-188,
// integration.cpp:161-233) -- one integrator per pixel, run sequentially
// per ray (each ray's state depends only on its own evaluations, so the
// reference's lock-step host loop is equivalent to a per-ray loop).
// --------------------------------------------------------------------------
enum { CTRL_REF32 = 0, CTRL_FP64 = 1, CTRL_DOUBLE = 2 };

struct RayResult {
  float value;
  int32_t steps;      // integrand evaluations of 4 points (accepted + rejected)
  int32_t accepted;
  int32_t status;     // 0 ok, 1 step limit
};

// Evaluation points of one step (integration.cl:38-47).
template <class R> static inline void rkf_points(R z, R h, R out[4]) {
  out[0] = z + (R)3 / (R)8 * h;
  out[1] = z + (R)12 / (R)13 * h;
  out[2] = z + h;
  out[3] = z + (R)0.5 * h;
}

// rkf_advance, fp32 arithmetic exactly as integration.cl:49-131 (R = float)
// or the same expression tree in double (R = double, the FP64 oracle).
template <class R>
static inline void rkf_advance_ref(R& I, R& z, R& h, R& k1, R atol, R rtol, R end, const R e[4],
                                   R eps, R hmin, R hmax, R next[4]) {
  typedef mathf<R> M;
  R d4 = (R)25 / (R)216 * k1 + (R)1408 / (R)2565 * e[0] + (R)2197 / (R)4101 * e[1] -
         (R)1 / (R)5 * e[2];
  R d5 = (R)16 / (R)135 * k1 + (R)6656 / (R)12825 * e[0] + (R)28561 / (R)56430 * e[1] -
         (R)9 / (R)50 * e[2] + (R)2 / (R)55 * e[3];
  d4 *= h;
  d5 *= h;
  const R est4 = I + d4;
  const R old = z;
  z += h;
  R s = (R)2;
  if (d4 != d5) {
    const R err = M::fabs(d5 - d4);
    const R srt = M::fabs(I / z * rtol);
    const R ot = M::fmax(atol, srt);
    s = M::sqrt(M::sqrt(ot * h / ((R)2 * err)));
  }
  R nh = s * h;
  if (nh < hmin) nh = hmin;
  else if (nh > hmax) nh = hmax;
  s = nh / h;
  if (s < (R)0.95) {
    z = old;
  } else {
    I = est4;
    k1 = e[2];
  }
  h = nh;
  if (z + h >= end) h = end - z + eps;
  rkf_points(z, h, next);
}

// FP64 step controller over fp32 state: the increments, the error estimate,
// the tolerance and the acceptance test are evaluated in double; the state
// (I, z, h, k1) and the evaluation points stay fp32. The expression tree is
// the reference's with the constants in double (the 2197/4101 weight kept).
static inline void rkf_advance_fp64(float& I, float& z, float& h, float& k1, double atol,
                                    double rtol, float end, const float e[4], float eps,
                                    float hmin, float hmax, float next[4]) {
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
    const double err = std::fabs(d5 - d4);
    const double srt = std::fabs((double)I / (double)znew * rtol);
    const double ot = std::fmax(atol, srt);
    s = std::sqrt(std::sqrt(ot * hd / (2.0 * err)));
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

static const float kEps = 0.01f, kHmin = 0.2f, kHmax = 100.f;  // integration.cl:34-36

// Pixel corner on the camera plane and the 4 query points (integration.cl:190-235).
template <class R> struct RayGeom { R pix[3]; R look[3]; };

static inline void ray_geom_f(const CamDev& c, int ix, int iy, RayGeom<float>& g) {
  const float tx = (float)ix * c.ps, ty = (float)iy * c.ps;
  for (int i = 0; i < 3; ++i) {
    g.pix[i] = (c.minp[i] + tx * c.b0[i]) + ty * c.b1[i];
    g.look[i] = c.look[i];
  }
}
static inline void ray_geom_d(const CamDev& c, int ix, int iy, RayGeom<double>& g) {
  const double tx = (double)ix * c.ps_d, ty = (double)iy * c.ps_d;
  for (int i = 0; i < 3; ++i) {
    g.pix[i] = (c.minp_d[i] + tx * c.b0_d[i]) + ty * c.b1_d[i];
    g.look[i] = c.look_d[i];
  }
}

template <class R>
static inline R eval_point(const Grid& g, const RayGeom<R>& rg, R zq, SearchStats* st) {
  const R x = rg.pix[0] + zq * rg.look[0];
  const R y = rg.pix[1] + zq * rg.look[1];
  const R z = rg.pix[2] + zq * rg.look[2];
  return nn8_value<R>(g, x, y, z, st);
}

// Records the accepted step sizes of one ray (for frozen replay).
struct StepLog { std::vector<float>* h = nullptr; };

static RayResult integrate_ray_f(const Grid& g, const RayGeom<float>& rg, float z0, float end,
                                 double atol, double rtol, int ctrl, int64_t max_steps,
                                 SearchStats* st, std::vector<float>* log) {
  // parallel_runge_kutta_fehlberg ctor: I = 0, z = z0, h = 1, k1 = 0
  // (integration.cpp:161-233). The first points are rkf_points(z0, 1) in
  // float; for z0 = 0 they equal the ctor's double expressions cast to float
  // (integration.cpp:220-225) bit for bit.
  float I = 0.f, z = z0, h = 1.0f, k1 = 0.0f;
  float pts[4];
  rkf_points<float>(z0, 1.0f, pts);
  RayResult rr{0.f, 0, 0, 0};
  const float fa = (float)atol, fr = (float)rtol;
  while (z < end) {
    if (rr.steps >= max_steps) { rr.status = 1; break; }
    float e[4];
    for (int j = 0; j < 4; ++j) e[j] = eval_point<float>(g, rg, pts[j], st);
    const float zb = z, hb = h;
    if (ctrl == CTRL_REF32)
      rkf_advance_ref<float>(I, z, h, k1, fa, fr, end, e, kEps, kHmin, kHmax, pts);
    else
      rkf_advance_fp64(I, z, h, k1, atol, rtol, end, e, kEps, kHmin, kHmax, pts);
    rr.steps += 1;
    if (z != zb) { rr.accepted += 1; if (log) log->push_back(hb); }
  }
  rr.value = I;
  return rr;
}

static RayResult integrate_ray_d(const Grid& g, const RayGeom<double>& rg, double z0,
                                 double end, double atol, double rtol, int64_t max_steps,
                                 SearchStats* st) {
  double I = 0., z = z0, h = 1.0, k1 = 0.0;
  double pts[4] = {z0 + 3. / 8. * 1.0, z0 + 12. / 13. * 1.0, z0 + 1.0, z0 + 0.5};
  RayResult rr{0.f, 0, 0, 0};
  while (z < end) {
    if (rr.steps >= max_steps) { rr.status = 1; break; }
    double e[4];
    for (int j = 0; j < 4; ++j) e[j] = eval_point<double>(g, rg, pts[j], st);
    const double zb = z;
    rkf_advance_ref<double>(I, z, h, k1, atol, rtol, end, e, (double)kEps, (double)kHmin,
                            (double)kHmax, pts);
    rr.steps += 1;
    if (z != zb) rr.accepted += 1;
  }
  rr.value = (float)I;
  return rr;
}

// Frozen step sequence: the accepted steps replayed (every step accepted,
// I += delta4 with k1 chained from the previous step's k5). With a uniform
// sequence h = z_range / n_steps this is the fixed-step mode.
template <class R>
static R replay_ray(const Grid& g, const RayGeom<R>& rg, R z0, const float* hs, int64_t nsteps,
                    SearchStats* st) {
  R I = (R)0, z = z0, k1 = (R)0;
  for (int64_t i = 0; i < nsteps; ++i) {
    const R h = (R)hs[i];
    R p[4];
    rkf_points<R>(z, h, p);
    R e[4];
    for (int j = 0; j < 4; ++j) e[j] = eval_point<R>(g, rg, p[j], st);
    R d4 = (R)25 / (R)216 * k1 + (R)1408 / (R)2565 * e[0] + (R)2197 / (R)4101 * e[1] -
           (R)1 / (R)5 * e[2];
    d4 *= h;
    I = I + d4;
    z += h;
    k1 = e[2];
  }
  return I;
}

// --------------------------------------------------------------------------
// X-ray quantities (quantities.cl:29-136, 156-239, 354-430)
// --------------------------------------------------------------------------
struct Gaunt {
  const float* t;  // row-major: t[y*w + x], x = log(gam2) axis, y = log(u) axis
  int w, h;
  float x0, y0, dx, dy;
};

// read_imagef with CLK_NORMALIZED_COORDS_FALSE | CLK_ADDRESS_CLAMP |
// CLK_FILTER_LINEAR on a CL_R float image: texel centres at i + 0.5, so the
// sample at coordinate u blends texels floor(u-0.5) and floor(u-0.5)+1 with
// weight frac(u-0.5); texels outside the image read the border value 0.
template <class R> static inline R texel(const Gaunt& G, int i, int j) {
  if (i < 0 || j < 0 || i >= G.w || j >= G.h) return (R)0;
  return (R)G.t[(size_t)j * G.w + i];
}

template <class R> static inline R gaunt_sample(const Gaunt& G, R u, R v) {
  typedef mathf<R> M;
  if (!(u == u) || !(v == v)) return (R)0;
  // Coordinates far outside the table only ever read the border.
  u = std::min(std::max(u, (R)-4), (R)(G.w + 4));
  v = std::min(std::max(v, (R)-4), (R)(G.h + 4));
  const R us = u - (R)0.5, vs = v - (R)0.5;
  const R fu = M::floor(us), fv = M::floor(vs);
  const int i0 = (int)fu, j0 = (int)fv;
  const R a = us - fu, b = vs - fv;
  const R ia = (R)1 - a, ib = (R)1 - b;
  return ((ia * ib * texel<R>(G, i0, j0) + a * ib * texel<R>(G, i0 + 1, j0)) +
          ia * b * texel<R>(G, i0, j0 + 1)) +
         a * b * texel<R>(G, i0 + 1, j0 + 1);
}

// evaluate_tabulated_function2d (tabulated_function.cl:46-59)
template <class R> static inline R tab2d(const Gaunt& G, R px, R py) {
  const R rx = (px - (R)G.x0) / (R)G.dx;
  const R ry = (py - (R)G.y0) / (R)G.dy;
  return gaunt_sample<R>(G, rx, ry);
}

template <class R> struct XC;  // constants in the precision of the instantiation
template <> struct XC<float> {
  static float XH() { return 0.76f; }
  static float kB() { return 8.61733e-5f; }
  static float gam() { return 5.f / 3.f; }
  static float Ryd() { return 13.605f; }
  static float conv() { return 121.1475502f; }
  static float nconv() { return 4.046263f; }
  static float pref() { return 0.002535f; }
  static float kilo() { return 1.e3f; }
};
template <> struct XC<double> {
  static double XH() { return 0.76; }
  static double kB() { return 8.61733e-5; }
  static double gam() { return 5. / 3.; }
  static double Ryd() { return 13.605; }
  static double conv() { return 121.1475502; }
  static double nconv() { return 4.046263; }
  static double pref() { return 0.002535; }
  static double kilo() { return 1.e3; }
};

template <class R> static inline R mean_molecular_weight(R xe) {
  typedef XC<R> C;
  return (R)4 / ((R)1 + (R)3 * C::XH() + (R)4 * C::XH() * xe);
}
template <class R> static inline R temperature(R u, R xe) {
  typedef XC<R> C;
  const R mu = mean_molecular_weight(xe);
  return (C::gam() - (R)1) * u * mu * C::conv();
}
template <class R> static inline R g_ff(const Gaunt& G, R E, R T, R Z) {
  typedef XC<R> C;
  const R gam2 = Z * Z * C::Ryd() / (C::kB() * T);
  const R u = C::kilo() * E / (C::kB() * T);
  return tab2d<R>(G, mathf<R>::log(gam2), mathf<R>::log(u));
}
template <class R>
static inline R brems(const Gaunt& G, R E, R dE, R T, R xe, R rho, R r) {
  typedef XC<R> C;
  const R ion = C::nconv() * rho * xe;
  const R Z = (R)1;
  const R Tinv = (R)1000 / (C::kB() * T);
  const R r2 = r * r;
  const R rs = (R)1 / mathf<R>::sqrt(T);
  return (R)C::pref() * dE * Z * Z * ion * ion * g_ff<R>(G, E, T, Z) * rs *
         mathf<R>::exp(-E * Tinv) / r2;
}
// integrate_spectral_flux (quantities.cl:156-239): the call of rkf_advance
// passes (rel_tol, 1) as (absolute, relative) tolerance, epsilon 0, step
// bounds [1e-3, 100]. photon (type PHOTON_FLUX): the emission at the range
// start and at every evaluation point is divided by that energy.
template <class R>
static inline R band_flux(const Gaunt& G, R Emin, R Emax, R reltol, R T, R xe, R rho, R dL,
                          bool photon = false) {
  R em = (R)0, E = Emin;
  const R end = Emax;
  R dE = (end - E) * reltol;
  R k1 = brems<R>(G, E, (R)1, T, xe, rho, dL);
  if (photon) k1 /= E;
  R p[4];
  rkf_points<R>(E, dE, p);
  int guard = 0;
  while (E < end && guard < 100000) {
    R v[4];
    for (int j = 0; j < 4; ++j) {
      v[j] = brems<R>(G, p[j], (R)1, T, xe, rho, dL);
      if (photon) v[j] /= p[j];
    }
    rkf_advance_ref<R>(em, E, dE, k1, reltol, (R)1, end, v, (R)0, (R)1.e-3f, (R)100, p);
    ++guard;
  }
  return em;
}

// util::tabulated_function (tabulated_function.hpp:35-103): n samples from x0
// in steps of dx; the Chandra ARF (chandra.cpp, chandra::arf) is one.
struct Arf {
  const float* t;
  int n;
  float x0, dx;
};

// evaluate_tabulated_function (tabulated_function.cl:31-44): read_imagef on a
// 1D CL_R image with the same sampler as the Gaunt table (texel centres at
// i + 0.5, linear blend, border 0).
template <class R> static inline R arf_sample(const Arf& A, R x) {
  typedef mathf<R> M;
  R u = (x - (R)A.x0) / (R)A.dx;
  if (!(u == u)) return (R)0;
  u = std::min(std::max(u, (R)-4), (R)(A.n + 4));
  const R us = u - (R)0.5;
  const R fu = M::floor(us);
  const int i0 = (int)fu;
  const R a = us - fu;
  const R t0 = (i0 >= 0 && i0 < A.n) ? (R)A.t[i0] : (R)0;
  const R t1 = (i0 + 1 >= 0 && i0 + 1 < A.n) ? (R)A.t[i0 + 1] : (R)0;
  return ((R)1 - a) * t0 + a * t1;
}

template <class R> static inline R cm2_to_m2();
template <> inline float cm2_to_m2<float>() { return 1.e-4f; }
template <> inline double cm2_to_m2<double>() { return 1.e-4; }

// get_chandra_xray_count_rate_with_temp (quantities.cl:432-460) with
// get_spectral_brems_count_rate (quantities.cl:251-260): emission at the
// redshifted channel / redshifted energy * ARF(E) [cm^2 -> m^2].
template <class R>
static inline R chandra_rate(const Gaunt& G, const Arf& A, R E, R dE, R z, R T, R xe, R rho,
                             R dL) {
  const R av = arf_sample<R>(A, E) * cm2_to_m2<R>();
  const R Ez = ((R)1 + z) * E;
  return brems<R>(G, Ez, ((R)1 + z) * dE, T, xe, rho, dL) / Ez * av;
}

// ---- derivatives for the adjoint -------------------------------------------
// Partial derivatives of the spectral emission (dE = 1) at fixed rho, xe:
//   with Tinv = 1000/(kB T), texel coordinates u = (ln(Ryd/(kB T)) - x0)/dx and
//   v = (ln(1e3 E/(kB T)) - y0)/dy, base = A T^-1/2 exp(-E Tinv) / r^2:
//   d/dlnT = base * (g * (E Tinv - 1/2) - (g_u/dx + g_v/dy))
//   d/dE   = base * (-g Tinv + g_v / (dy E))
// g_u, g_v: partial derivatives of the bilinear blend inside the texel.
template <class R>
static inline void gaunt_grad_uv(const Gaunt& G, R u, R v, R* gu, R* gv) {
  typedef mathf<R> M;
  *gu = *gv = (R)0;
  if (!(u == u) || !(v == v)) return;
  u = std::min(std::max(u, (R)-4), (R)(G.w + 4));
  v = std::min(std::max(v, (R)-4), (R)(G.h + 4));
  const R us = u - (R)0.5, vs = v - (R)0.5;
  const R fu = M::floor(us), fv = M::floor(vs);
  const int i0 = (int)fu, j0 = (int)fv;
  const R a = us - fu, b = vs - fv;
  const R t00 = texel<R>(G, i0, j0), t10 = texel<R>(G, i0 + 1, j0);
  const R t01 = texel<R>(G, i0, j0 + 1), t11 = texel<R>(G, i0 + 1, j0 + 1);
  *gu = ((R)1 - b) * (t10 - t00) + b * (t11 - t01);
  *gv = ((R)1 - a) * (t01 - t00) + a * (t11 - t10);
}

// value (the forward's own expression) and its lnT / E partials (double).
template <class R>
static inline void brems_partials(const Gaunt& G, R E, R T, R xe, R rho, R r, R* val,
                                  double* d_lnT, double* d_E) {
  typedef XC<R> C;
  *val = brems<R>(G, E, (R)1, T, xe, rho, r);
  const double Ed = (double)E, Td = (double)T;
  const double kB = (double)C::kB();
  const double ion = (double)C::nconv() * (double)rho * (double)xe;
  const double Tinv = 1000.0 / (kB * Td);
  const double ux = (std::log((double)C::Ryd() / (kB * Td)) - (double)G.x0) / (double)G.dx;
  const double vy = (std::log((double)C::kilo() * Ed / (kB * Td)) - (double)G.y0) / (double)G.dy;
  const double g = gaunt_sample<double>(G, ux, vy);
  double gu, gv;
  gaunt_grad_uv<double>(G, ux, vy, &gu, &gv);
  const double base = (double)C::pref() * ion * ion / std::sqrt(Td) * std::exp(-Ed * Tinv) /
                      ((double)r * (double)r);
  *d_lnT = base * (g * (Ed * Tinv - 0.5) - (gu / (double)G.dx + gv / (double)G.dy));
  *d_E = base * (-g * Tinv + gv / ((double)G.dy * Ed));
}

static inline double sgn(double x) { return x > 0 ? 1.0 : (x < 0 ? -1.0 : 0.0); }

// integrate_spectral_flux(XRAY_FLUX) in forward mode: the values follow the
// forward exactly (same ops, same decisions), and every state variable carries
// its derivative with respect to ln T, through the step controller as well
// (the energy steps are adaptive, so they move with T): the sqrt-sqrt factor,
// the clamps (derivative 0 when clamped) and the final-step adjustment.
// which = 0: tangent along ln T; which = 1: along ln rho (brems ~ rho^2, so its
// partial is 2*brems; the energy steps still move with rho through the error
// estimate when the absolute tolerance dominates).
template <class R>
static inline void band_flux_tangent(const Gaunt& G, R Emin, R Emax, R reltol, R T, R xe, R rho,
                                     R dL, int which, R* q, double* dq) {
  const R atol = reltol, rtol = (R)1, eps = (R)0, hmin = (R)1.e-3f, hmax = (R)100;
  R I = (R)0, z = Emin, h = (Emax - Emin) * reltol, k1;
  double dI = 0, dz = 0, dh = 0, dk1, dkE;
  const R end = Emax;
  brems_partials<R>(G, z, T, xe, rho, dL, &k1, &dk1, &dkE);
  if (which == 1) dk1 = 2.0 * (double)k1;
  R p[4];
  double dp[4] = {0, 0, 0, 0};
  rkf_points<R>(z, h, p);
  const double c[4] = {3. / 8., 12. / 13., 1.0, 0.5};
  int guard = 0;
  while (z < end && guard < 100000) {
    R e[4];
    double de[4];
    for (int j = 0; j < 4; ++j) {
      double pl, pe;
      brems_partials<R>(G, p[j], T, xe, rho, dL, &e[j], &pl, &pe);
      if (which == 1) pl = 2.0 * (double)e[j];
      de[j] = pl + pe * dp[j];
    }
    // rkf_advance_ref with tangents
    R b4 = (R)25 / (R)216 * k1 + (R)1408 / (R)2565 * e[0] + (R)2197 / (R)4101 * e[1] -
           (R)1 / (R)5 * e[2];
    R b5 = (R)16 / (R)135 * k1 + (R)6656 / (R)12825 * e[0] + (R)28561 / (R)56430 * e[1] -
           (R)9 / (R)50 * e[2] + (R)2 / (R)55 * e[3];
    const double db4 = 25. / 216. * dk1 + 1408. / 2565. * de[0] + 2197. / 4101. * de[1] -
                       1. / 5. * de[2];
    const double db5 = 16. / 135. * dk1 + 6656. / 12825. * de[0] + 28561. / 56430. * de[1] -
                       9. / 50. * de[2] + 2. / 55. * de[3];
    const double dd4 = db4 * (double)h + (double)b4 * dh;
    const double dd5 = db5 * (double)h + (double)b5 * dh;
    const R d4 = b4 * h, d5 = b5 * h;
    const R est4 = I + d4;
    const double dest4 = dI + dd4;
    const R old = z;
    const double dold = dz;
    z += h;
    dz += dh;
    R s = (R)2;
    double ds = 0;
    if (d4 != d5) {
      const R err = mathf<R>::fabs(d5 - d4);
      const double derr = sgn((double)d5 - (double)d4) * (dd5 - dd4);
      const R ratio = I / z * rtol;
      const R srt = mathf<R>::fabs(ratio);
      const double dsrt = sgn((double)ratio) * (double)rtol *
                          (dI / (double)z - (double)I * dz / ((double)z * (double)z));
      const R ot = mathf<R>::fmax(atol, srt);
      const double dot_ = srt > atol ? dsrt : 0.0;
      s = mathf<R>::sqrt(mathf<R>::sqrt(ot * h / ((R)2 * err)));
      ds = (double)s * 0.25 * (dot_ / (double)ot + dh / (double)h - derr / (double)err);
    }
    R nh = s * h;
    double dnh = ds * (double)h + (double)s * dh;
    if (nh < hmin) { nh = hmin; dnh = 0; }
    else if (nh > hmax) { nh = hmax; dnh = 0; }
    s = nh / h;
    if (s < (R)0.95) {
      z = old;
      dz = dold;
    } else {
      I = est4;
      dI = dest4;
      k1 = e[2];
      dk1 = de[2];
    }
    h = nh;
    dh = dnh;
    if (z + h >= end) { h = end - z + eps; dh = -dz; }
    rkf_points<R>(z, h, p);
    for (int j = 0; j < 4; ++j) dp[j] = dz + c[j] * dh;
    ++guard;
  }
  *q = I;
  *dq = dI;
}

// Adjoint of one ray over its frozen accepted steps: every accepted step adds
// h*(25/216 k1 + 1408/2565 e0 + 2197/4101 e1 - 1/5 e2) to I, k1 being the
// previous step's e2 (0 before the first step), and each e is the finalize
// of its 8 slots, sum(w v)/sum(w) -> d e / d v_p = w_p / sum(w).
template <class R>
static void adjoint_ray(const Grid& g, const RayGeom<R>& rg, R z0, const float* hs,
                        int64_t nsteps, R gI, double* grad) {
  R z = z0;
  Slots<R> prev;
  bool have_prev = false;
  for (int64_t i = 0; i < nsteps; ++i) {
    const R h = (R)hs[i];
    R p[4];
    rkf_points<R>(z, h, p);
    const R coef[3] = {h * (R)1408 / (R)2565, h * (R)2197 / (R)4101, -h / (R)5};
    Slots<R> s[3];
    for (int j = 0; j < 3; ++j) {
      slots_init(s[j]);
      nn8_search<R>(g, rg.pix[0] + p[j] * rg.look[0], rg.pix[1] + p[j] * rg.look[1],
                    rg.pix[2] + p[j] * rg.look[2], s[j], nullptr);
    }
    auto scatter = [&](const Slots<R>& sl, R c) {
      R w[8], ws = (R)0;
      for (int t = 0; t < 8; ++t) { w[t] = weight3d(sl.d[t]); ws += w[t]; }
      if (ws == (R)0 || !(ws == ws)) return;
      for (int t = 0; t < 8; ++t) {
        if (sl.id[t] < 0 || w[t] == (R)0) continue;
        const double add = (double)(gI * c * (w[t] / ws));
#pragma omp atomic
        grad[sl.id[t]] += add;
      }
    };
    for (int j = 0; j < 3; ++j) scatter(s[j], coef[j]);
    if (have_prev) scatter(prev, h * (R)25 / (R)216);
    prev = s[2];
    have_prev = true;
    z += h;
  }
}

}  // namespace orc

// ==========================================================================
// C interface used by the Python test harness (ctypes)
// ==========================================================================
using namespace orc;

// --------------------------------------------------------------------------
// Batched render: many cameras (jobs), aperture masks, per-ray chords and V
// value channels per cell in one pass. Not a reference function: it restates
// the batched kernel's definition so the kernel can be checked bit for bit.
// With V = 1, no mask and no chord it equals orc_render in the FP64
// controller mode. The reference renders a spectrum as one projection per
// energy bin (spectrum.cpp:89-109, animation.cpp:264-283); here the V
// channels of a ray share one step sequence, driven by a joint FP64
// controller: per channel the single-channel error ratio
//   x_c = max(atol, |I_c/z' rtol|) h / (2 |d5_c - d4_c|)   (16 if d4_c == d5_c)
// and s = (min_c x_c)^(1/4), which is the smallest of the per-channel step
// factors (sqrt is monotone, so the min commutes with it exactly); a step
// is accepted only when every channel would accept it.
// --------------------------------------------------------------------------
struct Job {
  Camera cam;
  double z_range;          // depth when no chord sphere is set
  double aperture;         // > 0: pixel centres farther than this from the screen centre are masked
  double centre[3];        // chord sphere
  double radius;           // > 0: integrate over the ray's chord of the sphere
  double min_chord;        // chords shorter than this are widened about their midpoint
  float scale;             // output = I * scale
  int32_t pad;
  uint64_t offset;         // element offset of the job's V x ny x nx block
};

struct RaySpan { int masked; float origin[3]; float len; };

// Mask, chord and float origin of one ray; every step is a plain IEEE
// double or float operation (no contraction), as the kernel evaluates it.
static void ray_span(const Job& j, const CamDev& d, int ix, int iy, RaySpan* r) {
  r->masked = 0;
  if (j.aperture > 0.0) {
    const double dx = ((double)ix + 0.5 - 0.5 * (double)j.cam.nx) * d.ps_d;
    const double dy = ((double)iy + 0.5 - 0.5 * (double)j.cam.ny) * d.ps_d;
    if (dx * dx + dy * dy > j.aperture * j.aperture) r->masked = 1;
  }
  RayGeom<float> rg;
  ray_geom_f(d, ix, iy, rg);
  if (!(j.radius > 0.0)) {
    for (int i = 0; i < 3; ++i) r->origin[i] = rg.pix[i];
    r->len = (float)j.z_range;
    return;
  }
  RayGeom<double> gd;
  ray_geom_d(d, ix, iy, gd);
  double w[3];
  for (int i = 0; i < 3; ++i) w[i] = j.centre[i] - gd.pix[i];
  const double t = (w[0] * d.look_d[0] + w[1] * d.look_d[1]) + w[2] * d.look_d[2];
  const double ww = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2];
  const double b2 = ww - t * t;
  const double r2 = j.radius * j.radius;
  double half = b2 < r2 ? std::sqrt(r2 - b2) : 0.0;
  const double mh = 0.5 * j.min_chord;
  if (half < mh) half = mh;
  double z0 = t - half;
  const double z1 = t + half;
  if (z0 < 0.0) z0 = 0.0;
  r->len = z1 > z0 ? (float)(z1 - z0) : 0.0f;
  const float z0f = (float)z0;
  for (int i = 0; i < 3; ++i) r->origin[i] = rg.pix[i] + z0f * d.look[i];
}

// Joint FP64 controller over V fp32 channels (see above); for V = 1 it is
// rkf_advance_fp64 operation for operation.
static void rkf_advance_multi(float* I, float& z, float& h, float* k1, int V, double atol,
                              double rtol, float end, const float* e, float eps, float hmin,
                              float hmax, float next[4], float* est) {
  const double hd = (double)h;
  const float znew = z + h;
  double xmin = 0.0;
  for (int c = 0; c < V; ++c) {
    const double e0 = (double)e[c], e1 = (double)e[V + c], e2 = (double)e[2 * V + c],
                 e3 = (double)e[3 * V + c];
    double d4 = 25.0 / 216.0 * (double)k1[c] + 1408.0 / 2565.0 * e0 + 2197.0 / 4101.0 * e1 -
                1.0 / 5.0 * e2;
    double d5 = 16.0 / 135.0 * (double)k1[c] + 6656.0 / 12825.0 * e0 +
                28561.0 / 56430.0 * e1 - 9.0 / 50.0 * e2 + 2.0 / 55.0 * e3;
    d4 *= hd;
    d5 *= hd;
    est[c] = (float)((double)I[c] + d4);
    double x = 16.0;
    if (d4 != d5) {
      const double err = std::fabs(d5 - d4);
      const double srt = std::fabs((double)I[c] / (double)znew * rtol);
      const double ot = std::fmax(atol, srt);
      x = ot * hd / (2.0 * err);
    }
    if (c == 0 || x < xmin) xmin = x;
  }
  double s = std::sqrt(std::sqrt(xmin));
  double nh = s * hd;
  if (nh < (double)hmin) nh = (double)hmin;
  else if (nh > (double)hmax) nh = (double)hmax;
  s = nh / hd;
  if (!(s < 0.95)) {
    z = znew;
    for (int c = 0; c < V; ++c) { I[c] = est[c]; k1[c] = e[2 * V + c]; }
  }
  h = (float)nh;
  if (z + h >= end) h = end - z + eps;
  rkf_points<float>(z, h, next);
}

// Channel values at one point: nn8 slots (sorted indices) applied to each
// channel with nn8_finalize's operation order; empty slots carry value 0.
template <class R>
static void eval_channels(const Grid& g, const float* vs, int V, R x, R y, R z, R* out,
                          SearchStats* st) {
  Slots<R> s;
  slots_init(s);
  nn8_search<R>(g, x, y, z, s, st);
  R w[8];
  for (int j = 0; j < 8; ++j) w[j] = weight3d(s.d[j]);
  R ws = (R)0;
  for (int j = 0; j < 8; ++j) ws += w[j];
  for (int c = 0; c < V; ++c) {
    R dot = (R)0;
    for (int j = 0; j < 8; ++j) {
      const R v = s.id[j] >= 0 ? (R)vs[(size_t)s.id[j] * V + c] : (R)0;
      dot = mathf<R>::fma(w[j], v, dot);
    }
    out[c] = (ws != (R)0 && dot != (R)0) ? dot / ws : (R)0;
  }
}

static RayResult integrate_multi(const Grid& g, const float* vs, int V, const RaySpan& sp,
                                 const float* look, double atol, double rtol,
                                 int64_t max_steps, SearchStats* st, float* I) {
  std::vector<float> k1(V, 0.0f), e(4 * (size_t)V), est(V);
  for (int c = 0; c < V; ++c) I[c] = 0.0f;
  float z = 0.0f, h = 1.0f;
  float pts[4];
  rkf_points<float>(0.0f, 1.0f, pts);
  RayResult rr{0.f, 0, 0, 0};
  while (z < sp.len) {
    if (rr.steps >= max_steps) { rr.status = 1; break; }
    for (int j = 0; j < 4; ++j)
      eval_channels<float>(g, vs, V, sp.origin[0] + pts[j] * look[0],
                           sp.origin[1] + pts[j] * look[1], sp.origin[2] + pts[j] * look[2],
                           &e[(size_t)j * V], st);
    const float zb = z;
    rkf_advance_multi(I, z, h, k1.data(), V, atol, rtol, sp.len, e.data(), kEps, kHmin, kHmax,
                      pts, est.data());
    rr.steps += 1;
    if (z != zb) rr.accepted += 1;
  }
  return rr;
}

// FP64 accuracy reference of one channel of a batched ray: the channel on
// its own (its own step sequence, as the reference's per-bin projection),
// everything in double from the double pixel position and chord.
static float integrate_channel_d(const Grid& g, const float* vs, int V, int c, const Job& j,
                                 const CamDev& d, int ix, int iy, double atol, double rtol,
                                 int64_t max_steps, int* status) {
  RayGeom<double> rg;
  ray_geom_d(d, ix, iy, rg);
  double z0 = 0.0, len = j.z_range;
  if (j.radius > 0.0) {
    double w[3];
    for (int i = 0; i < 3; ++i) w[i] = j.centre[i] - rg.pix[i];
    const double t = (w[0] * d.look_d[0] + w[1] * d.look_d[1]) + w[2] * d.look_d[2];
    const double b2 = ((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]) - t * t;
    double half = b2 < j.radius * j.radius ? std::sqrt(j.radius * j.radius - b2) : 0.0;
    if (half < 0.5 * j.min_chord) half = 0.5 * j.min_chord;
    z0 = t - half;
    const double z1 = t + half;
    if (z0 < 0.0) z0 = 0.0;
    len = z1 > z0 ? z1 - z0 : 0.0;
  }
  double o[3];
  for (int i = 0; i < 3; ++i) o[i] = rg.pix[i] + z0 * rg.look[i];
  double I = 0., z = 0., h = 1.0, k1 = 0.0;
  double pts[4] = {3. / 8., 12. / 13., 1.0, 0.5};
  int64_t steps = 0;
  *status = 0;
  while (z < len) {
    if (steps >= max_steps) { *status = 1; break; }
    double e[4];
    for (int q = 0; q < 4; ++q)
      eval_channels<double>(g, vs + c, V, o[0] + pts[q] * rg.look[0], o[1] + pts[q] * rg.look[1],
                            o[2] + pts[q] * rg.look[2], &e[q], nullptr);
    rkf_advance_ref<double>(I, z, h, k1, atol, rtol, len, e, (double)kEps, (double)kHmin,
                            (double)kHmax, pts);
    ++steps;
  }
  return (float)I;
}

extern "C" {

typedef struct {
  double position[3];
  double look_at[3];
  double roll;
  double screen_width;
  int32_t nx, ny;
} orc_camera;

int orc_spiral_table(int8_t* out) {
  int8_t t[8][125][3];
  spiral_table(t);
  std::memcpy(out, t, sizeof(t));
  return 0;
}

float orc_logf(float x) { return ilc_logf(x); }
float orc_expf(float x) { return ilc_expf(x); }

void* orc_grid_build(const float* xyzq, int64_t n, int32_t* status) {
  ensure_spiral();
  Grid* g = new Grid();
  int st = grid_build(xyzq, (size_t)n, g);
  if (status) *status = st;
  if (st) { delete g; return nullptr; }
  return g;
}

void orc_grid_free(void* h) { delete (Grid*)h; }

int orc_grid_info(void* h, float* min3, float* cs3, int32_t* n3, uint64_t* total) {
  Grid* g = (Grid*)h;
  for (int i = 0; i < 3; ++i) { min3[i] = g->min[i]; cs3[i] = g->cs[i]; n3[i] = g->n[i]; }
  *total = g->total;
  return 0;
}

int orc_grid_export(void* h, int32_t* cells, uint32_t* s2u, float* sorted, uint64_t* keys) {
  Grid* g = (Grid*)h;
  if (cells) std::memcpy(cells, g->cells.data(), g->cells.size() * 4);
  if (s2u) std::memcpy(s2u, g->s2u.data(), g->s2u.size() * 4);
  if (sorted) std::memcpy(sorted, g->sorted.data(), g->sorted.size() * 4);
  if (keys) std::memcpy(keys, g->keys.data(), g->keys.size() * 8);
  return 0;
}

// nn8 queries: out value, and optionally the 8 slots (original particle index,
// distance) in slot order. precision 0 = fp32 restatement, 1 = FP64 oracle.
int orc_nn8_query(void* h, const float* pts, int64_t n, int precision, float* out,
                  int32_t* idx8, float* d8, uint64_t* stats2, int nthreads) {
  Grid* g = (Grid*)h;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  uint64_t cells = 0, cands = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : cells, cands)
  for (int64_t i = 0; i < n; ++i) {
    SearchStats st;
    const float* q = pts + 4 * i;
    if (precision == 0) {
      Slots<float> s;
      slots_init(s);
      nn8_search<float>(*g, q[0], q[1], q[2], s, &st);
      out[i] = nn8_finalize(s);
      for (int j = 0; j < 8; ++j) {
        if (idx8) idx8[8 * i + j] = s.id[j] < 0 ? -1 : (int32_t)g->s2u[s.id[j]];
        if (d8) d8[8 * i + j] = s.d[j];
      }
    } else {
      Slots<double> s;
      slots_init(s);
      nn8_search<double>(*g, (double)q[0], (double)q[1], (double)q[2], s, &st);
      out[i] = (float)nn8_finalize(s);
      for (int j = 0; j < 8; ++j) {
        if (idx8) idx8[8 * i + j] = s.id[j] < 0 ? -1 : (int32_t)g->s2u[s.id[j]];
        if (d8) d8[8 * i + j] = (float)s.d[j];
      }
    }
    cells += st.cells;
    cands += st.candidates;
  }
  if (stats2) { stats2[0] = cells; stats2[1] = cands; }
  return 0;
}

// nn8 with explicit running lists (fp32): merge = 0 starts from empty lists,
// merge = 1 continues list_d / list_v / list_id (n x 8, original indices), as
// the reference's multi-block reconstruction (volumetric_nn8_reconstruction.cl:112-126).
int orc_nn8_query_lists(void* h, const float* pts, int64_t n, int merge, float* list_d,
                        float* list_v, int32_t* list_id, float* out, int nthreads) {
  Grid* g = (Grid*)h;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    const float* q = pts + 4 * i;
    Slots<float> s;
    if (merge) {
      for (int j = 0; j < 8; ++j) {
        s.d[j] = list_d[8 * i + j];
        s.v[j] = list_v[8 * i + j];
        const int32_t o = list_id[8 * i + j];
        s.id[j] = o >= 0 ? (int32_t)(0x80000000u | (uint32_t)o) : -1;
      }
    } else {
      slots_init(s);
    }
    nn8_search<float>(*g, q[0], q[1], q[2], s, nullptr);
    out[i] = nn8_finalize(s);
    for (int j = 0; j < 8; ++j) {
      const int32_t id = s.id[j];
      list_d[8 * i + j] = s.d[j];
      list_v[8 * i + j] = s.v[j];
      list_id[8 * i + j] =
          id == -1 ? -1 : (id < 0 ? (int32_t)((uint32_t)id & 0x7fffffffu) : (int32_t)g->s2u[id]);
    }
  }
  return 0;
}

// Camera basis as the device receives it: look, b0, b1, min corner (float) + pixel size.
int orc_camera_setup(const orc_camera* c, float* out13) {
  Camera cam;
  std::memcpy(&cam, c, sizeof(Camera));
  CamDev d;
  camera_setup(cam, &d);
  for (int i = 0; i < 3; ++i) {
    out13[i] = d.look[i]; out13[3 + i] = d.b0[i]; out13[6 + i] = d.b1[i];
    out13[9 + i] = d.minp[i];
  }
  out13[12] = d.ps;
  return 0;
}

// Adaptive render of selected pixels (pix = iy*nx + ix). mode: 0 = fp32 with
// the reference controller, 1 = fp32 with the FP64 controller, 2 = FP64
// oracle. out: raw line integrals (before the dA scaling).
int orc_render(void* h, const orc_camera* c, double z_range, double atol, double rtol, int mode,
               int64_t max_steps, const int64_t* pix, int64_t npix, float* out,
               int32_t* steps, int32_t* accepted, uint64_t* stats2, int nthreads) {
  Grid* g = (Grid*)h;
  Camera cam;
  std::memcpy(&cam, c, sizeof(Camera));
  CamDev d;
  camera_setup(cam, &d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  uint64_t cells = 0, cands = 0;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : cells, cands, bad)
  for (int64_t k = 0; k < npix; ++k) {
    const int64_t p = pix ? pix[k] : k;
    const int ix = (int)(p % cam.nx), iy = (int)(p / cam.nx);
    SearchStats st;
    RayResult rr;
    if (mode == CTRL_DOUBLE) {
      RayGeom<double> rg;
      ray_geom_d(d, ix, iy, rg);
      rr = integrate_ray_d(*g, rg, 0.0, z_range, atol, rtol, max_steps, &st);
    } else {
      RayGeom<float> rg;
      ray_geom_f(d, ix, iy, rg);
      rr = integrate_ray_f(*g, rg, 0.0f, (float)z_range, atol, rtol, mode, max_steps, &st,
                           nullptr);
    }
    out[k] = rr.value;
    if (steps) steps[k] = rr.steps;
    if (accepted) accepted[k] = rr.accepted;
    bad += rr.status;
    cells += st.cells;
    cands += st.candidates;
  }
  if (stats2) { stats2[0] = cells; stats2[1] = cands; }
  return bad ? 1 : 0;
}

// Fixed-step (frozen uniform sequence) render: n_steps steps of z_range/n_steps.
int orc_render_fixed(void* h, const orc_camera* c, double z_range, int64_t n_steps,
                     int precision, const int64_t* pix, int64_t npix, float* out,
                     uint64_t* stats2, int nthreads) {
  Grid* g = (Grid*)h;
  Camera cam;
  std::memcpy(&cam, c, sizeof(Camera));
  CamDev d;
  camera_setup(cam, &d);
  const float hf = (float)(z_range / (double)n_steps);
  std::vector<float> hs((size_t)n_steps, hf);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  uint64_t cells = 0, cands = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : cells, cands)
  for (int64_t k = 0; k < npix; ++k) {
    const int64_t p = pix ? pix[k] : k;
    const int ix = (int)(p % cam.nx), iy = (int)(p / cam.nx);
    SearchStats st;
    if (precision == 0) {
      RayGeom<float> rg;
      ray_geom_f(d, ix, iy, rg);
      out[k] = replay_ray<float>(*g, rg, 0.0f, hs.data(), n_steps, &st);
    } else {
      RayGeom<double> rg;
      ray_geom_d(d, ix, iy, rg);
      out[k] = (float)replay_ray<double>(*g, rg, 0.0, hs.data(), n_steps, &st);
    }
    cells += st.cells;
    cands += st.candidates;
  }
  if (stats2) { stats2[0] = cells; stats2[1] = cands; }
  return 0;
}

// Adaptive render that also returns each ray's accepted step sizes
// (hs_out: capacity cap per ray, count in nacc), then used for frozen replay.
int orc_render_record(void* h, const orc_camera* c, double z_range, double atol, double rtol,
                      int mode, int64_t max_steps, const int64_t* pix, int64_t npix,
                      float* out, float* hs_out, int64_t cap, int32_t* nacc, int nthreads) {
  Grid* g = (Grid*)h;
  Camera cam;
  std::memcpy(&cam, c, sizeof(Camera));
  CamDev d;
  camera_setup(cam, &d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : bad)
  for (int64_t k = 0; k < npix; ++k) {
    const int64_t p = pix ? pix[k] : k;
    const int ix = (int)(p % cam.nx), iy = (int)(p / cam.nx);
    RayGeom<float> rg;
    ray_geom_f(d, ix, iy, rg);
    std::vector<float> log;
    RayResult rr = integrate_ray_f(*g, rg, 0.0f, (float)z_range, atol, rtol, mode, max_steps,
                                   nullptr, &log);
    out[k] = rr.value;
    const int64_t m = std::min<int64_t>((int64_t)log.size(), cap);
    for (int64_t i = 0; i < m; ++i) hs_out[k * cap + i] = log[i];
    nacc[k] = (int32_t)log.size();
    bad += rr.status + (log.size() > (size_t)cap ? 1 : 0);
  }
  return bad ? 1 : 0;
}

// Frozen replay of given per-ray step sequences (hs: npix x cap, counts n).
int orc_render_replay(void* h, const orc_camera* c, const int64_t* pix, int64_t npix,
                      const float* hs, int64_t cap, const int32_t* n, int precision, float* out,
                      double* out_d, int nthreads) {
  Grid* g = (Grid*)h;
  Camera cam;
  std::memcpy(&cam, c, sizeof(Camera));
  CamDev d;
  camera_setup(cam, &d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t k = 0; k < npix; ++k) {
    const int64_t p = pix ? pix[k] : k;
    const int ix = (int)(p % cam.nx), iy = (int)(p / cam.nx);
    if (precision == 0) {
      RayGeom<float> rg;
      ray_geom_f(d, ix, iy, rg);
      out[k] = replay_ray<float>(*g, rg, 0.0f, hs + k * cap, n[k], nullptr);
    } else {
      RayGeom<double> rg;
      ray_geom_d(d, ix, iy, rg);
      const double v = replay_ray<double>(*g, rg, 0.0, hs + k * cap, n[k], nullptr);
      out[k] = (float)v;
      if (out_d) out_d[k] = v;
    }
  }
  return 0;
}

// The scale applied after integration (volumetric_integration.cpp:74-87):
// out *= (float)length_conversion * (float)dA_eff, where dA_eff is the
// quantity's effective_line_of_sight_integration_dA of (pixel_area*area_conv,
// length_conv*z_range): mode 0 -> dA, 1 -> 1.0 (projected density),
// 2 -> 1/range (mean quantities).
float orc_los_scale(const orc_camera* c, double z_range, double length_conv,
                    double area_conv, int dA_mode) {
  const double ps = c->screen_width / (double)c->nx;
  const float pixel_area = (float)(ps * ps);
  const float lc = (float)length_conv;
  const double dA_in = (double)pixel_area * area_conv;
  const double range = (double)lc * z_range;
  double dA;
  if (dA_mode == 0) dA = dA_in;
  else if (dA_mode == 1) dA = 1.0;
  else dA = 1.0 / range;
  const float dAf = (float)dA;
  return lc * dAf;
}

// Per-cell quantities. table: w x h row-major Gaunt factors.
static Gaunt make_gaunt(const float* table, int w, int hgt) {
  return Gaunt{table, w, hgt, -6.f, -16.f, 0.2f, 0.2f};
}

float orc_gaunt_lookup(const float* table, int w, int hgt, float lg, float lu) {
  Gaunt G = make_gaunt(table, w, hgt);
  return tab2d<float>(G, lg, lu);
}

int orc_temperature(const float* u, const float* xe, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = temperature<float>(u[i], xe[i]);
  return 0;
}

// xray_flux kernel (quantities.cl:354-385).
int orc_xray_band(const float* table, int w, int hgt, const float* rho, const float* u,
                  const float* xe, int64_t n, float z, float dL, float Emin, float Emax,
                  int num_samples, int precision, float* out, int nthreads) {
  Gaunt G = make_gaunt(table, w, hgt);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (precision == 0) {
      const float T = temperature<float>(u[i], xe[i]);
      out[i] = band_flux<float>(G, (1.f + z) * Emin, (1.f + z) * Emax, 1.f / (float)num_samples,
                                T, xe[i], rho[i], dL);
    } else {
      const double T = temperature<double>(u[i], xe[i]);
      const double zz = z;
      out[i] = (float)band_flux<double>(G, (1. + zz) * Emin, (1. + zz) * Emax,
                                        1. / (double)num_samples, T, xe[i], rho[i], dL);
    }
  }
  return 0;
}

// xray_flux and its derivatives with respect to ln T and ln rho (forward mode
// through the adaptive energy integration).
int orc_xray_band_grad(const float* table, int w, int hgt, const float* rho, const float* u,
                       const float* xe, int64_t n, float z, float dL, float Emin, float Emax,
                       int num_samples, int precision, float* q_out, double* dq_out,
                       double* dqr_out, int nthreads) {
  Gaunt G = make_gaunt(table, w, hgt);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (precision == 0) {
      const float T = temperature<float>(u[i], xe[i]);
      float q;
      double dq, dqr;
      band_flux_tangent<float>(G, (1.f + z) * Emin, (1.f + z) * Emax, 1.f / (float)num_samples,
                               T, xe[i], rho[i], dL, 0, &q, &dq);
      band_flux_tangent<float>(G, (1.f + z) * Emin, (1.f + z) * Emax, 1.f / (float)num_samples,
                               T, xe[i], rho[i], dL, 1, &q, &dqr);
      q_out[i] = q;
      dq_out[i] = dq;
      dqr_out[i] = dqr;
    } else {
      const double T = temperature<double>(u[i], xe[i]);
      double q, dq, dqr;
      band_flux_tangent<double>(G, (1. + z) * Emin, (1. + z) * Emax, 1. / (double)num_samples,
                                T, xe[i], rho[i], dL, 0, &q, &dq);
      band_flux_tangent<double>(G, (1. + z) * Emin, (1. + z) * Emax, 1. / (double)num_samples,
                                T, xe[i], rho[i], dL, 1, &q, &dqr);
      q_out[i] = (float)q;
      dq_out[i] = dq;
      dqr_out[i] = dqr;
    }
  }
  return 0;
}

// Adjoint over frozen per-ray step sequences (hs: npix x cap, counts n): adds
// gI[k] * dI_k/dq_p into grad (n_particles, ORIGINAL particle order).
int orc_adjoint(void* h, const orc_camera* c, const int64_t* pix, int64_t npix, const float* hs,
                int64_t cap, const int32_t* n, const double* gI, int precision, double* grad,
                int nthreads) {
  Grid* g = (Grid*)h;
  Camera cam;
  std::memcpy(&cam, c, sizeof(Camera));
  CamDev d;
  camera_setup(cam, &d);
  const size_t np = g->s2u.size();
  std::vector<double> gs(np, 0.0);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t k = 0; k < npix; ++k) {
    const int64_t p = pix ? pix[k] : k;
    const int ix = (int)(p % cam.nx), iy = (int)(p / cam.nx);
    if (precision == 0) {
      RayGeom<float> rg;
      ray_geom_f(d, ix, iy, rg);
      adjoint_ray<float>(*g, rg, 0.0f, hs + k * cap, n[k], (float)gI[k], gs.data());
    } else {
      RayGeom<double> rg;
      ray_geom_d(d, ix, iy, rg);
      adjoint_ray<double>(*g, rg, 0.0, hs + k * cap, n[k], gI[k], gs.data());
    }
  }
  for (size_t i = 0; i < np; ++i) grad[g->s2u[i]] += gs[i];
  return 0;
}

// xray_spectral_flux kernel (quantities.cl:400-430), one energy bin.
int orc_xray_bin(const float* table, int w, int hgt, const float* rho, const float* u,
                 const float* xe, int64_t n, float z, float dL, float E, float dE, int precision,
                 float* out, int nthreads) {
  Gaunt G = make_gaunt(table, w, hgt);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (precision == 0) {
      const float T = temperature<float>(u[i], xe[i]);
      out[i] = brems<float>(G, (1.f + z) * E, (1.f + z) * dE, T, xe[i], rho[i], dL);
    } else {
      const double T = temperature<double>(u[i], xe[i]);
      out[i] = (float)brems<double>(G, (1. + z) * E, (1. + z) * dE, T, xe[i], rho[i], dL);
    }
  }
  return 0;
}


// xray_photon_flux kernel (quantities.cl:640-675): photons/s/kpc^3/cm^2.
int orc_xray_photon_flux(const float* table, int w, int hgt, const float* rho, const float* u,
                         const float* xe, int64_t n, float z, float dL, float Emin, float Emax,
                         int num_samples, int precision, float* out, int nthreads) {
  Gaunt G = make_gaunt(table, w, hgt);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (precision == 0) {
      const float T = temperature<float>(u[i], xe[i]);
      out[i] = band_flux<float>(G, (1.f + z) * Emin, (1.f + z) * Emax, 1.f / (float)num_samples,
                                T, xe[i], rho[i], dL, true) * 1.e-4f;
    } else {
      const double T = temperature<double>(u[i], xe[i]);
      const double zz = z;
      out[i] = (float)(band_flux<double>(G, (1. + zz) * Emin, (1. + zz) * Emax,
                                         1. / (double)num_samples, T, xe[i], rho[i], dL, true) *
                       1.e-4);
    }
  }
  return 0;
}

// chandra_xray_total_count_rate kernel (quantities.cl:510-557): the channel
// count rates of every ARF channel k (energy x0 + k * dx, width dx) summed in
// channel order.
int orc_chandra_count_rate(const float* table, int w, int hgt, const float* arf, int n_arf,
                           float ax0, float adx, const float* rho, const float* u,
                           const float* xe, int64_t n, float z, float dL, int precision,
                           float* out, int nthreads) {
  Gaunt G = make_gaunt(table, w, hgt);
  const Arf A{arf, n_arf, ax0, adx};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (precision == 0) {
      const float T = temperature<float>(u[i], xe[i]);
      float em = 0.0f;
      for (int k = 0; k < n_arf; ++k)
        em += chandra_rate<float>(G, A, ax0 + (float)k * adx, adx, z, T, xe[i], rho[i], dL);
      out[i] = em;
    } else {
      const double T = temperature<double>(u[i], xe[i]);
      double em = 0.0;
      for (int k = 0; k < n_arf; ++k)
        em += chandra_rate<double>(G, A, (double)ax0 + (double)k * (double)adx, (double)adx,
                                   (double)z, T, xe[i], rho[i], dL);
      out[i] = (float)em;
    }
  }
  return 0;
}

// chandra_xray_spectral_count_rate kernel (quantities.cl:584-622): one channel.
int orc_chandra_spectral_count_rate(const float* table, int w, int hgt, const float* arf,
                                    int n_arf, float ax0, float adx, const float* rho,
                                    const float* u, const float* xe, int64_t n, float z,
                                    float dL, float E, float dE, int precision, float* out,
                                    int nthreads) {
  Gaunt G = make_gaunt(table, w, hgt);
  const Arf A{arf, n_arf, ax0, adx};
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    if (precision == 0) {
      const float T = temperature<float>(u[i], xe[i]);
      out[i] = chandra_rate<float>(G, A, E, dE, z, T, xe[i], rho[i], dL);
    } else {
      const double T = temperature<double>(u[i], xe[i]);
      out[i] = (float)chandra_rate<double>(G, A, E, dE, z, T, xe[i], rho[i], dL);
    }
  }
  return 0;
}

// Batched render (see Job). values: n x V, cell-major, original cell order.
// rays == nullptr: every pixel of every job into images at the job offsets
// (channel-major V x ny x nx), masked pixels 0. Otherwise rays holds
// (job, pixel) pairs and out receives nrays x V. precision 0: the batched
// fp32 kernel's definition; 1: each channel on its own in double.
// stats4: steps, accepted steps, cells visited, candidates.
int orc_render_batched(void* h, const float* values, int32_t V, const void* jobs_v,
                       int32_t n_jobs, double atol, double rtol, int64_t max_steps,
                       const int64_t* rays, int64_t nrays, int precision, float* out,
                       uint64_t* stats4, int nthreads) {
  Grid* g = (Grid*)h;
  const Job* jobs = (const Job*)jobs_v;
  const int64_t n = (int64_t)g->s2u.size();
  std::vector<float> vs((size_t)n * V);
  for (int64_t p = 0; p < n; ++p)
    for (int c = 0; c < V; ++c) vs[(size_t)p * V + c] = values[(size_t)g->s2u[p] * V + c];
  std::vector<CamDev> cams(n_jobs);
  for (int k = 0; k < n_jobs; ++k) camera_setup(jobs[k].cam, &cams[k]);
  std::vector<int64_t> list;
  if (!rays) {
    for (int k = 0; k < n_jobs; ++k)
      for (int64_t p = 0; p < (int64_t)jobs[k].cam.nx * jobs[k].cam.ny; ++p) {
        list.push_back(k);
        list.push_back(p);
      }
    rays = list.data();
    nrays = (int64_t)list.size() / 2;
  }
  if (nthreads > 0) omp_set_num_threads(nthreads);
  uint64_t st_steps = 0, st_acc = 0, st_cells = 0, st_cands = 0;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : st_steps, st_acc, st_cells, st_cands, bad)
  for (int64_t k = 0; k < nrays; ++k) {
    const Job& j = jobs[rays[2 * k]];
    const CamDev& d = cams[rays[2 * k]];
    const int64_t p = rays[2 * k + 1];
    const int ix = (int)(p % j.cam.nx), iy = (int)(p / j.cam.nx);
    std::vector<float> I(V, 0.0f);
    RaySpan sp;
    ray_span(j, d, ix, iy, &sp);
    if (!sp.masked) {
      if (precision == 0) {
        SearchStats st;
        RayResult rr = integrate_multi(*g, vs.data(), V, sp, d.look, atol, rtol, max_steps, &st,
                                       I.data());
        bad += rr.status;
        st_steps += rr.steps;
        st_acc += rr.accepted;
        st_cells += st.cells;
        st_cands += st.candidates;
      } else {
        for (int c = 0; c < V; ++c) {
          int status = 0;
          I[c] = integrate_channel_d(*g, vs.data(), V, c, j, d, ix, iy, atol, rtol, max_steps,
                                     &status);
          bad += status;
        }
      }
    }
    for (int c = 0; c < V; ++c) {
      const float v = sp.masked ? 0.0f : I[c] * j.scale;
      if (list.empty())
        out[(size_t)k * V + c] = v;
      else
        out[j.offset + (size_t)c * j.cam.nx * j.cam.ny + (size_t)p] = v;
    }
  }
  if (stats4) { stats4[0] = st_steps; stats4[1] = st_acc; stats4[2] = st_cells; stats4[3] = st_cands; }
  return bad ? 1 : 0;
}

// Ray span of one pixel of a job (mask, float origin, length) for tests.
int orc_ray_span(const void* job_v, int32_t ix, int32_t iy, int32_t* masked, float* origin3,
                 float* len) {
  const Job& j = *(const Job*)job_v;
  CamDev d;
  camera_setup(j.cam, &d);
  RaySpan sp;
  ray_span(j, d, ix, iy, &sp);
  *masked = sp.masked;
  for (int i = 0; i < 3; ++i) origin3[i] = sp.origin[i];
  *len = sp.len;
  return 0;
}


// Cell ingestion of reconstructing_data_crawler::run
// (reconstructing_data_crawler.cpp:170-230): float coordinates widened to
// double, coordinate_system::correct_periodicity (coordinate_system.hpp:25-47)
// against the cutout box widened by `border`, volume_cutout::contains_point
// with zero tolerance (reconstructing_data_crawler.cpp:49-60), kept cells in
// input order with the corrected coordinates cast to float
// (to_device_vector4, cl_types.hpp:55-61). Returns the number kept.
int64_t orc_ingest_cells(const float* xyz, const float* q, int64_t n, const double* center,
                         const double* extent, const double* periodic, double border,
                         float* out_xyzq, uint32_t* out_index) {
  double bmin[3], bmax[3];
  for (int j = 0; j < 3; ++j) {
    bmin[j] = center[j] - 0.5 * extent[j];  // get_bounding_box_min_corner
    bmax[j] = center[j] + 0.5 * extent[j];
  }
  int64_t k = 0;
  for (int64_t i = 0; i < n; ++i) {
    double c[3];
    for (int j = 0; j < 3; ++j) c[j] = (double)xyz[3 * i + j];
    for (int j = 0; j < 3; ++j) {
      const double gmin = bmin[j] - border, gmax = bmax[j] + border;
      if (gmin <= c[j] - periodic[j] && c[j] - periodic[j] <= gmax)
        c[j] -= periodic[j];
      else if (gmin <= c[j] + periodic[j] && c[j] + periodic[j] <= gmax)
        c[j] += periodic[j];
    }
    bool in = true;
    for (int j = 0; j < 3; ++j) {
      if (c[j] < (center[j] - 0.5 * extent[j] - 0.0)) in = false;
      if (c[j] > (center[j] + 0.5 * extent[j] + 0.0)) in = false;
    }
    if (!in) continue;
    for (int j = 0; j < 3; ++j) out_xyzq[4 * k + j] = (float)c[j];
    out_xyzq[4 * k + 3] = q ? q[i] : 0.0f;
    if (out_index) out_index[k] = (uint32_t)i;
    ++k;
  }
  return k;
}


// volumetric_slice::create_slice (volumetric_slice.cpp:31-101) with no extra
// samples: nn8 value at camera::get_pixel_coordinate(x, y) (camera.cpp:49-54,
// double, cast to float), output = 0 + dV * value / 1 in double, cast to float.
int orc_volumetric_slice(void* h, const orc_camera* c, double dV, float* out, int nthreads) {
  Grid* g = (Grid*)h;
  Camera cam;
  std::memcpy(&cam, c, sizeof(Camera));
  CamDev d;
  camera_setup(cam, &d);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  const int64_t npix = (int64_t)cam.nx * cam.ny;
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < npix; ++p) {
    const double xs = (double)(p % cam.nx), ys = (double)(p / cam.nx);
    float q[3];
    for (int j = 0; j < 3; ++j)
      q[j] = (float)((d.minp_d[j] + xs * d.ps_d * d.b0_d[j]) + ys * d.ps_d * d.b1_d[j]);
    const float v = nn8_value<float>(*g, q[0], q[1], q[2], nullptr);
    const float acc = 0.0f;
    out[p] = (float)((double)acc + dV * (double)v / 1.0);
  }
  return 0;
}

// ---- Monte-Carlo radial profile -----------------------------------------
// distributed_mc_radial_profile (profile.cpp:26-355) with the sampler of
// random.cpp:28-86 drawing from a counter-based hash instead of the
// reference's std::random_device-seeded std::mt19937: draw j of sample k is
// the top 53 bits of mix(mix(seed ^ mix(k)) + j), mix = the SplitMix64 output
// function (Steele, Lea, Flood 2014).
static inline uint64_t prof_mix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
static inline double prof_draw(uint64_t seed, uint64_t k, uint64_t j) {
  const uint64_t h = prof_mix(prof_mix(seed ^ prof_mix(k)) + j);
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}
// Cube root from +, *, / and exact exponent scaling (so that it is the same
// on any IEEE machine): u = m 2^(3q), m in [0.5, 4), eight Newton steps from 1.
static inline double prof_cbrt(double u) {
  if (!(u > 0.0)) return 0.0;
  int e;
  double m = std::frexp(u, &e);
  int r = e % 3;
  if (r < 0) r += 3;
  m = std::ldexp(m, r);
  e -= r;
  double y = 1.0;
  for (int i = 0; i < 8; ++i) y = (2.0 * y + m / (y * y)) / 3.0;
  return std::ldexp(y, e / 3);
}

// profile.cpp:320-355 (shells) and 93-128 (generate_num_samples).
static bool prof_shells(double R, int N, double density, std::vector<double>& rmin,
                        std::vector<double>& rmax, std::vector<double>& vol,
                        std::vector<uint64_t>& count) {
  if (!(R > 0.0) || !std::isfinite(R) || N < 1 || N > (1 << 20) || !(density > 0.0) ||
      !std::isfinite(density))
    return false;
  const unsigned n = (unsigned)N;
  auto radius = [&](unsigned i) { return i * (R / n); };
  rmin.resize(n); rmax.resize(n); vol.resize(n); count.resize(n);
  for (unsigned i = 0; i < n; ++i) {
    rmin[i] = i == 0 ? 0.0 : 0.5 * (radius(i - 1) + radius(i));
    rmax[i] = 0.5 * (radius(i + 1) + radius(i));
    vol[i] = 4. / 3 * M_PI * (rmax[i] * rmax[i] * rmax[i] - rmin[i] * rmin[i] * rmin[i]);
  }
  double expected = 0.0, sq = 0.0;
  for (unsigned i = 0; i < n; ++i) expected += vol[i] * density;
  for (unsigned i = 0; i < n; ++i) sq += vol[i] * vol[i];
  const double norm = expected / sq;
  uint64_t total = 0;
  for (unsigned i = 0; i < n; ++i) {
    const double want = norm * (vol[i] * vol[i]);
    if (!(want < 1099511627776.0)) return false;
    count[i] = (uint64_t)want;
    if (count[i] == 0) count[i] = 1;
    total += count[i];
    if (total > 1099511627776ull) return false;
  }
  return true;
}

int orc_mc_profile_shells(double R, int N, double density, double* radii, uint64_t* counts) {
  std::vector<double> a, b, v;
  std::vector<uint64_t> c;
  if (!prof_shells(R, N, density, a, b, v, c)) return 1;
  for (int i = 0; i < N; ++i) {
    if (radii) radii[i] = i * (R / (unsigned)N);
    if (counts) counts[i] = c[i];
  }
  return 0;
}

// The profile: sample k (shells in order) uniform in its shell
// (uniform_spherical_shell, random.cpp:67-86, with Marsaglia's surface point
// of random.cpp:28-45: at most 64 attempts, then the pole), cast to float as
// to_device_vector4 (cl_types.hpp:55-61); nn8 value summed per shell in
// double in sample order (profile.cpp:212-225); times the effective dV of
// apply_volume_factor (profile.cpp:236-256), mode 0 dV * conv, mode 1
// (dV * conv) / (V * conv).
int orc_mc_radial_profile(void* h, const double* center, double R, int N, double density,
                          uint64_t seed, int mode, double conv, double* profile, float* pts,
                          float* vals, int nthreads) {
  Grid* g = (Grid*)h;
  std::vector<double> rmin, rmax, vol;
  std::vector<uint64_t> count;
  if (!prof_shells(R, N, density, rmin, rmax, vol, count) || (mode != 0 && mode != 1)) return 1;
  std::vector<uint64_t> first(N + 1, 0);
  for (int i = 0; i < N; ++i) first[i + 1] = first[i] + count[i];
  const uint64_t total = first[N];
  std::vector<float> v(total);
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)total; ++k) {
    const int s = (int)(std::upper_bound(first.begin(), first.end(), (uint64_t)k) -
                        first.begin()) - 1;
    double x1 = 0.0, x2 = 0.0, r = 0.0;
    for (int a = 0; a < 64; ++a) {
      const double t1 = -1. + (1. - -1.) * prof_draw(seed, (uint64_t)k, 2 * a);
      const double t2 = -1. + (1. - -1.) * prof_draw(seed, (uint64_t)k, 2 * a + 1);
      const double rr = t1 * t1 + t2 * t2;
      if (rr <= 1.) {
        x1 = t1; x2 = t2; r = rr;
        break;
      }
    }
    const double sq = std::sqrt(1. - r);
    const double p[3] = {2 * x1 * sq, 2 * x2 * sq, 1 - 2 * r};
    const double u_min = rmin[s] * rmin[s] * rmin[s], u_max = rmax[s] * rmax[s] * rmax[s];
    const double u = u_min + (u_max - u_min) * prof_draw(seed, (uint64_t)k, 128);
    const double rad = prof_cbrt(u);
    float q[3];
    for (int j = 0; j < 3; ++j) q[j] = (float)(rad * p[j] + center[j]);
    v[k] = nn8_value<float>(*g, q[0], q[1], q[2], nullptr);
    if (pts) {
      for (int j = 0; j < 3; ++j) pts[4 * k + j] = q[j];
      pts[4 * k + 3] = 0.0f;
    }
    if (vals) vals[k] = v[k];
  }
  for (int s = 0; s < N; ++s) {
    double sum = 0.0;
    for (uint64_t k = first[s]; k < first[s + 1]; ++k) sum += (double)v[k];
    const double dV = vol[s] / (double)count[s];
    const double eff = mode == 0 ? dV * conv : (dV * conv) / (vol[s] * conv);
    profile[s] = sum * eff;
  }
  return 0;
}

}  // extern "C"
