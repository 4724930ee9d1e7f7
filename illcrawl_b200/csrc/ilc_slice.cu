// ilc_slice.cu -- volumetric_slice::create_slice (volumetric_slice.cpp:31-101):
// the nn8 reconstruction at every pixel of a camera plane, plus optional
// jittered extra samples per pixel, scaled by the quantity's effective dV.
//
// Sample 0 of pixel (x, y) is camera::get_pixel_coordinate(x, y)
// (camera.cpp:49-54) in double, cast to float. The reference draws the extra
// samples' offsets from std::random_device (not reproducible); here they come
// from a counter-based hash of (seed, sample, pixel), uniform in [-0.5, 0.5)
// pixel, so a slice is reproducible for a given seed.
#include <algorithm>

#include "ilc_internal.h"
#include "ilc_random.cuh"

namespace ilc {
namespace {

struct SlicePlane {
  double minp[3], b0[3], b1[3];
  double ps;
  int nx, ny;
};

__device__ __forceinline__ double unit_offset(uint64_t h) {  // [-0.5, 0.5)
  return (double)(h >> 11) * (1.0 / 9007199254740992.0) - 0.5;
}

__global__ void slice_points_kernel(SlicePlane P, int samples, uint64_t seed,
                                    float4* __restrict__ pts) {
  const uint64_t npix = (uint64_t)P.nx * (uint64_t)P.ny;
  const uint64_t total = npix * (uint64_t)samples;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i = k / npix, p = k - i * npix;
    double xs = (double)(p % (uint64_t)P.nx), ys = (double)(p / (uint64_t)P.nx);
    if (i > 0) {
      const uint64_t h = mix64(seed ^ mix64(k));
      xs += unit_offset(h);
      ys += unit_offset(mix64(h));
    }
    double c[3];
#pragma unroll
    for (int j = 0; j < 3; ++j) c[j] = (P.minp[j] + xs * P.ps * P.b0[j]) + ys * P.ps * P.b1[j];
    pts[k] = make_float4((float)c[0], (float)c[1], (float)c[2], 0.0f);
  }
}

// output[p] += dV * value / samples for every sample in order, as the
// reference accumulates (a float pixel, each increment computed in double).
__global__ void slice_accumulate_kernel(const float* __restrict__ vals, uint64_t npix,
                                        int samples, double dV, float* __restrict__ out) {
  for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < npix;
       p += (uint64_t)gridDim.x * blockDim.x) {
    float acc = 0.0f;
    for (int i = 0; i < samples; ++i)
      acc = (float)((double)acc + dV * (double)vals[(uint64_t)i * npix + p] / (double)samples);
    out[p] = acc;
  }
}

}  // namespace

cudaError_t slice_launch(Context& c, const double plane[13], int nx, int ny, int samples,
                         uint64_t seed, double dV, float* out) {
  cudaError_t e;
  SlicePlane P;
  for (int j = 0; j < 3; ++j) {
    P.b0[j] = plane[3 + j];
    P.b1[j] = plane[6 + j];
    P.minp[j] = plane[9 + j];
  }
  P.ps = plane[12];
  P.nx = nx;
  P.ny = ny;
  const uint64_t npix = (uint64_t)nx * (uint64_t)ny, total = npix * (uint64_t)samples;
  if ((e = c.in_b.ensure(total * 16)) || (e = c.out_b.ensure(total * 4))) return e;
  const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 16);
  slice_points_kernel<<<blocks, 256, 0, c.stream>>>(P, samples, seed, c.in_b.as<float4>());
  ++c.launches;
  if ((e = cudaGetLastError())) return e;
  if ((e = nn8_query_launch(c, c.in_b.as<float4>(), total, false, c.out_b.as<float>(), nullptr,
                            nullptr)))
    return e;
  const unsigned b2 = (unsigned)std::min<uint64_t>((npix + 255) / 256, 148ull * 16);
  slice_accumulate_kernel<<<b2, 256, 0, c.stream>>>(c.out_b.as<float>(), npix, samples, dV, out);
  ++c.launches;
  return cudaGetLastError();
}

}  // namespace ilc
