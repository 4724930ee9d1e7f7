// ilc_random.cuh -- reproducible random numbers for the sampled nn8 consumers
// (volumetric slices with extra samples, Monte-Carlo radial profiles).
//
// The reference draws these from std::mt19937 seeded by std::random_device
// (random.hpp:33-63), so no two of its runs share samples. Here every draw is
// a counter-based hash of (seed, sample index, draw index): any sample can be
// produced by any thread in any order, and the CPU oracle produces the same
// bits. The hash is the SplitMix64 output function (Steele, Lea, Flood 2014;
// the constants are Vigna's published ones).
#pragma once

#include <cstdint>

namespace ilc {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Uniform double in [0, 1) from the top 53 bits (exact: an integer times 2^-53).
__host__ __device__ __forceinline__ double unit_double(uint64_t h) {
  return (double)(h >> 11) * (1.0 / 9007199254740992.0);
}

// Draw j of sample k: independent streams per sample.
__host__ __device__ __forceinline__ double sample_draw(uint64_t seed, uint64_t k, uint64_t j) {
  return unit_double(mix64(mix64(seed ^ mix64(k)) + j));
}

// Cube root of u >= 0 from IEEE +, *, / and exact exponent scaling only, so
// that host and device agree to the bit: u = m 2^(3q) with m in [0.5, 4),
// eight Newton steps y <- (2y + m / y^2) / 3 from y = 1 (quadratic
// convergence; within an ulp of the true root), then y 2^q.
__host__ __device__ __forceinline__ double cbrt_newton(double u) {
  if (!(u > 0.0)) return 0.0;
  int e;
  double m = frexp(u, &e);
  int r = e % 3;
  if (r < 0) r += 3;
  m = ldexp(m, r);
  e -= r;
  double y = 1.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) y = (2.0 * y + m / (y * y)) / 3.0;
  return ldexp(y, e / 3);
}

// random::sampler::uniform_spherical_shell (random.cpp:67-86): a point on the
// unit sphere by Marsaglia's method (uniform_sphere_surface, random.cpp:28-45:
// x1, x2 uniform in [-1, 1) until r = x1^2 + x2^2 <= 1, then
// (2 x1 sqrt(1 - r), 2 x2 sqrt(1 - r), 1 - 2r)), scaled by cbrt(u) with u
// uniform in [r_min^3, r_max^3), plus the centre; in double, cast to float as
// math::to_device_vector4 does (cl_types.hpp:55-61). Attempt a of the surface
// draw uses draws 2a and 2a + 1; after 64 rejections (probability 2e-43) the
// pole (0, 0, 1) is taken. The radius uses draw 128.
// Shell of global sample g: the lo with prefix[lo] <= g < prefix[lo + 1]
// (prefix: n_shells + 1 increasing entries from 0, g < prefix[n_shells]).
__host__ __device__ __forceinline__ int find_shell(const uint64_t* prefix, int n_shells,
                                                   uint64_t g) {
  int lo = 0, hi = n_shells;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (prefix[mid] <= g) lo = mid; else hi = mid;
  }
  return lo;
}

struct ShellPoint {
  float x, y, z;
};

__host__ __device__ __forceinline__ ShellPoint shell_sample(uint64_t seed, uint64_t k,
                                                            double u_min, double u_max,
                                                            const double c[3]) {
  double x1 = 0.0, x2 = 0.0, r = 0.0;
  for (int a = 0; a < 64; ++a) {
    const double t1 = -1.0 + (1.0 - -1.0) * sample_draw(seed, k, 2 * a);
    const double t2 = -1.0 + (1.0 - -1.0) * sample_draw(seed, k, 2 * a + 1);
    const double rr = t1 * t1 + t2 * t2;
    if (rr <= 1.0) {
      x1 = t1;
      x2 = t2;
      r = rr;
      break;
    }
  }
  const double s = sqrt(1.0 - r);
  const double p0 = 2.0 * x1 * s, p1 = 2.0 * x2 * s, p2 = 1.0 - 2.0 * r;
  const double u = u_min + (u_max - u_min) * sample_draw(seed, k, 128);
  const double rad = cbrt_newton(u);
  ShellPoint out;
  out.x = (float)(rad * p0 + c[0]);
  out.y = (float)(rad * p1 + c[1]);
  out.z = (float)(rad * p2 + c[2]);
  return out;
}

}  // namespace ilc
