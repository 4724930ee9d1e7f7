// ilc_profile.cu -- distributed_mc_radial_profile (profile.cpp:26-355): a
// Monte-Carlo radial profile of the reconstructed quantity around a centre.
//
// Shell i spans [mid(r_{i-1}, r_i), mid(r_i, r_{i+1})] with r_i = i R / N
// (shell 0 starts at 0; profile.cpp:320-355) and gets n_i = max(1,
// floor(norm V_i^2)) samples, norm = sample_density sum(V) / sum(V^2)
// (generate_num_samples, profile.cpp:93-128). Sample k of the whole profile
// (shells in order) is uniform in its shell (shell_sample in ilc_random.cuh);
// its nn8 value is summed into the shell in double and the sum is scaled by
// the quantity's effective dV (apply_volume_factor, profile.cpp:236-256).
//
// On the device: samples are made and evaluated in batches of whole segments
// (at most 8192 consecutive samples of one shell) so that memory stays
// bounded as in the reference's _max_batch_size batches; each segment is
// reduced by one block in a fixed order and the host adds the segment sums of
// a shell in segment order, so the result does not depend on the batch size.
#include <algorithm>

#include "ilc_internal.h"
#include "ilc_random.cuh"

namespace ilc {
namespace {

constexpr int kReduceThreads = 256;

// Sample points of global samples [g0, g0 + n): shell by binary search over
// the shell prefix (prefix[0] = 0 < prefix[1] < ... < prefix[N] = total).
__global__ void profile_points_kernel(const uint64_t* __restrict__ prefix, int n_shells,
                                      const double* __restrict__ u_min,
                                      const double* __restrict__ u_max, double cx, double cy,
                                      double cz, uint64_t seed, uint64_t g0, uint64_t n,
                                      float4* __restrict__ pts) {
  const double c[3] = {cx, cy, cz};
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = g0 + k;
    const int s = find_shell(prefix, n_shells, g);
    const ShellPoint p = shell_sample(seed, g, u_min[s], u_max[s], c);
    pts[k] = make_float4(p.x, p.y, p.z, 0.0f);
  }
}

// One block per segment: sum of vals[seg.begin - g0, seg.end - g0) in double,
// strided per thread, then a fixed shared-memory tree.
__global__ void __launch_bounds__(kReduceThreads)
profile_segment_sum_kernel(const ulonglong2* __restrict__ segs, uint64_t g0,
                           const float* __restrict__ vals, double* __restrict__ sums) {
  __shared__ double part[kReduceThreads];
  const ulonglong2 s = segs[blockIdx.x];
  double acc = 0.0;
  for (uint64_t g = s.x + threadIdx.x; g < s.y; g += kReduceThreads)
    acc += (double)vals[g - g0];
  part[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = part[0];
}

}  // namespace

cudaError_t profile_points_launch(Context& c, const uint64_t* prefix, int n_shells,
                                  const double* u_min, const double* u_max,
                                  const double center[3], uint64_t seed, uint64_t g0, uint64_t n,
                                  float4* pts) {
  const unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
  profile_points_kernel<<<blocks, 256, 0, c.stream>>>(prefix, n_shells, u_min, u_max, center[0],
                                                      center[1], center[2], seed, g0, n, pts);
  ++c.launches;
  return cudaGetLastError();
}

cudaError_t profile_segment_sum_launch(Context& c, const ulonglong2* segs, uint32_t n_segs,
                                       uint64_t g0, const float* vals, double* sums) {
  profile_segment_sum_kernel<<<n_segs, kReduceThreads, 0, c.stream>>>(segs, g0, vals, sums);
  ++c.launches;
  return cudaGetLastError();
}

}  // namespace ilc
