// ilc_ingest.cu -- device-side cell ingestion: the per-row loop of
// reconstructing_data_crawler::run (reconstructing_data_crawler.cpp:170-230).
//
// Every cell's float coordinates are widened to double, moved by one period
// along each axis where that brings them into the cutout box widened by the
// border (coordinate_system.hpp:25-47), and kept if the corrected point lies
// in the cutout box (volume_cutout::contains_point,
// reconstructing_data_crawler.cpp:49-60). Kept cells are written in input
// order -- the order the reference appends them to its particle vector, which
// the grid's stable sort then preserves within each cell -- as float4
// (x, y, z, q) with the corrected coordinates cast to float
// (to_device_vector4, cl_types.hpp:55-61), plus their input index.
//
// Two passes over the cells: per-block counts, an exclusive scan of the
// counts, then a scatter that ranks each kept cell inside its block with warp
// ballots.
#include "ilc_internal.h"

namespace ilc {
namespace {

constexpr int kIngestThreads = 256;

__device__ __forceinline__ bool within(double x, double lo, double hi) {
  return lo <= x && x <= hi;
}

// Periodic correction and containment test of cell i; c receives the
// corrected coordinates.
__device__ __forceinline__ bool correct_and_test(const float* __restrict__ xyz, uint64_t i,
                                                 const CutoutParams& p, double c[3]) {
  bool in = true;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double x = (double)xyz[3 * i + j];
    if (within(x - p.period[j], p.glo[j], p.ghi[j]))
      x -= p.period[j];
    else if (within(x + p.period[j], p.glo[j], p.ghi[j]))
      x += p.period[j];
    c[j] = x;
    if (x < p.lo[j] || x > p.hi[j]) in = false;
  }
  return in;
}

__global__ void __launch_bounds__(kIngestThreads)
ingest_count_kernel(const float* __restrict__ xyz, uint64_t n, CutoutParams p,
                    uint32_t* __restrict__ block_counts) {
  const uint64_t i = blockIdx.x * (uint64_t)kIngestThreads + threadIdx.x;
  double c[3];
  const bool keep = i < n && correct_and_test(xyz, i, p, c);
  const int cnt = __syncthreads_count(keep);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = (uint32_t)cnt;
}

__global__ void __launch_bounds__(kIngestThreads)
ingest_scatter_kernel(const float* __restrict__ xyz, const float* __restrict__ q, uint64_t n,
                      CutoutParams p, const uint32_t* __restrict__ block_offsets,
                      float4* __restrict__ out, uint32_t* __restrict__ out_index,
                      unsigned long long* __restrict__ n_out) {
  __shared__ uint32_t warp_counts[kIngestThreads / 32];
  const uint64_t i = blockIdx.x * (uint64_t)kIngestThreads + threadIdx.x;
  double c[3] = {0.0, 0.0, 0.0};
  const bool keep = i < n && correct_and_test(xyz, i, p, c);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned ball = __ballot_sync(0xffffffffu, keep);
  if (lane == 0) warp_counts[warp] = __popc(ball);
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += warp_counts[w];
  if (keep) {
    const uint64_t k = (uint64_t)block_offsets[blockIdx.x] + before +
                       __popc(ball & ((1u << lane) - 1u));
    out[k] = make_float4((float)c[0], (float)c[1], (float)c[2], q ? q[i] : 0.0f);
    if (out_index) out_index[k] = (uint32_t)i;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
    uint32_t tot = 0;
    for (int w = 0; w < kIngestThreads / 32; ++w) tot += warp_counts[w];
    *n_out = (unsigned long long)block_offsets[blockIdx.x] + tot;
  }
}

}  // namespace

cudaError_t ingest_launch(Context& c, const float* xyz, const float* q, uint64_t n,
                          const CutoutParams& p, float4* out, uint32_t* out_index,
                          unsigned long long* n_out) {
  cudaError_t e;
  const uint64_t blocks = (n + kIngestThreads - 1) / kIngestThreads;
  if ((e = c.hist.ensure(blocks * 4 + 64))) return e;
  uint32_t* counts = c.hist.as<uint32_t>();
  ingest_count_kernel<<<(unsigned)blocks, kIngestThreads, 0, c.stream>>>(xyz, n, p, counts);
  ++c.launches;
  if ((e = cudaGetLastError())) return e;
  if ((e = exclusive_scan_u32(c, counts, blocks))) return e;
  ingest_scatter_kernel<<<(unsigned)blocks, kIngestThreads, 0, c.stream>>>(
      xyz, q, n, p, counts, out, out_index, n_out);
  ++c.launches;
  return cudaGetLastError();
}

}  // namespace ilc
