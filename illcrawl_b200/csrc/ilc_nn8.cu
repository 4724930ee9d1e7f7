// ilc_nn8.cu -- nn8 reconstruction at arbitrary query points: the fused
// volumetric_nn8_reconstruction + finalize kernels
// (volumetric_nn8_reconstruction.cl:87-270), one thread per query.
//
// merge = false starts from empty lists (is_first_run); merge = true continues
// from the lists the previous call left, which is how the reference combines
// particle blocks (volumetric_nn8_reconstruction.cl:112-126).
#include "ilc_device.cuh"
#include "ilc_internal.h"

namespace ilc {

namespace {

__global__ void __launch_bounds__(256)
nn8_query_kernel(GridView g, const char4* __restrict__ spiral_g, const float4* __restrict__ pts,
                 uint64_t n, int merge, float* __restrict__ list_d, float* __restrict__ list_v,
                 int32_t* __restrict__ list_id, float* __restrict__ out,
                 int32_t* __restrict__ idx8, float* __restrict__ d8,
                 const uint32_t* __restrict__ s2u, unsigned long long* __restrict__ stats) {
  __shared__ char4 spiral[1000];
  load_spiral(spiral, spiral_g);
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  WalkStats st;
  if (i < n) {
    const float4 q = pts[i];
    Slots<true> s;
    if (merge) {
      // Lists carry original indices; entries kept from the previous call are
      // tagged with the top bit so they are not mapped through this grid's s2u.
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        s.d[j] = list_d[8 * i + j];
        s.v[j] = list_v[8 * i + j];
        const int32_t o = list_id[8 * i + j];
        s.id[j] = o >= 0 ? (int32_t)(0x80000000u | (uint32_t)o) : -1;
      }
      s.rescan();
    } else {
      s.init();
    }
    nn8_walk<true>(g, spiral, q.x, q.y, q.z, s, st);
    out[i] = nn8_finalize(s);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int32_t id = s.id[j];
      const int32_t orig =
          id == -1 ? -1 : (id < 0 ? (int32_t)((uint32_t)id & 0x7fffffffu) : (int32_t)s2u[id]);
      list_d[8 * i + j] = s.d[j];
      list_v[8 * i + j] = s.v[j];
      list_id[8 * i + j] = orig;
      if (idx8) idx8[8 * i + j] = orig;
      if (d8) d8[8 * i + j] = s.d[j];
    }
  }
  // warp-aggregated traffic counters
  unsigned long long c = st.cells, k = st.cands;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, off);
    k += __shfl_xor_sync(0xffffffffu, k, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&stats[3], c);
    atomicAdd(&stats[4], k);
  }
}

}  // namespace

GridView make_grid_view(const Context& c);

cudaError_t nn8_query_launch(Context& c, const float4* pts, uint64_t n, bool merge, float* out,
                             int32_t* idx8, float* d8) {
  cudaError_t e;
  if ((e = c.list_d.ensure(n * 32)) || (e = c.list_v.ensure(n * 32)) ||
      (e = c.list_id.ensure(n * 32)) || (e = c.flags.ensure(kFlagsBytes)))
    return e;
  if ((e = cudaMemsetAsync(c.flags.p, 0, kFlagsBytes, c.stream))) return e;
  c.list_n = n;
  const GridView g = make_grid_view(c);
  const unsigned blocks = (unsigned)((n + 255) / 256);
  unsigned long long* stats =
      reinterpret_cast<unsigned long long*>(c.flags.as<char>() + 64);
  ++c.launches;
  nn8_query_kernel<<<blocks, 256, 0, c.stream>>>(
      g, c.spiral.as<char4>(), pts, n, merge ? 1 : 0, c.list_d.as<float>(), c.list_v.as<float>(),
      c.list_id.as<int32_t>(), out, idx8, d8, c.s2u.as<uint32_t>(), stats);
  return cudaGetLastError();
}

}  // namespace ilc
