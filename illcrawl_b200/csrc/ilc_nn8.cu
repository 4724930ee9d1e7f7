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

// ---------------------------------------------------------------------------
// Warp-cooperative form of the same walk: one warp per query.
//
// Lanes 0-7 hold the 8 (distance, value, index) slots. The spiral is taken 32
// cells at a time (lane L: cell it0 + L): each lane computes its cell's
// centre distance and loads its cell range; the candidates of those cells,
// concatenated in spiral and index order, are tested 32 at a time (lane k:
// candidate k) against the squared radius held at the start of the round
// (R only shrinks, so a candidate that fails it cannot be inserted), and
// __ballot_sync collects the hits. The hits are then inserted one after the
// other in candidate order with the reference's test (d^2 <= R*R rounded up,
// sqrt(d^2) < R, replace the first maximal slot), and the early break is
// applied at every cell in order with the radius of that moment: a ballot of
// the cells whose centre is beyond R + cell radius gives, after each
// insertion, the first cell the walk stops at. The slots therefore go through
// the same insertions as in the one-thread walk, and the result is the same
// bit for bit. The maximum slot is found with __reduce_max_sync over the
// distances' bit patterns (non-negative floats order as unsigned integers)
// and the first slot holding it with a ballot.
// ---------------------------------------------------------------------------
constexpr unsigned kFull = 0xffffffffu;

struct WarpSlots {
  float d, v;   // this lane's slot (lanes 0-7)
  int32_t id;
  float R, R2up, rr;
  int mi;
};

__device__ __forceinline__ void warp_rescan(WarpSlots& s, int lane, float crad) {
  const unsigned bits = __reduce_max_sync(kFull, lane < 8 ? __float_as_uint(s.d) : 0u);
  s.R = __uint_as_float(bits);
  s.mi = __ffs(__ballot_sync(kFull, lane < 8 && __float_as_uint(s.d) == bits)) - 1;
  s.R2up = __fmul_ru(s.R, s.R);
  const float b = s.R + crad;
  s.rr = b * b;
}

__device__ __forceinline__ void nn8_walk_warp(const GridView& g, const char4* __restrict__ spiral,
                                              float qx, float qy, float qz, WarpSlots& s,
                                              int lane, WalkStats& st) {
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
  const float crad = g.cell_radius;
  for (int it0 = 0; it0 < 125; it0 += 32) {
    // this lane's cell of the chunk
    const int it = it0 + lane;
    const bool valid = it < 125;
    float cd = 0.0f;
    bool ing = false;
    int bx = 0, nc = 0;
    if (valid) {
      const char4 o = order[it];
      const int ix = cx + o.x, iy = cy + o.y, iz = cz + o.z;
      const float ex = ((g.min0 + (float)ix * g.cs0) + g.half0) - qx;
      const float ey = ((g.min1 + (float)iy * g.cs1) + g.half1) - qy;
      const float ez = ((g.min2 + (float)iz * g.cs2) + g.half2) - qz;
      cd = (ex * ex + ey * ey) + ez * ez;
      ing = (unsigned)ix < (unsigned)g.n0 && (unsigned)iy < (unsigned)g.n1 &&
            (unsigned)iz < (unsigned)g.n2;
      if (ing) {
        const size_t key = (size_t)ix + (size_t)iy * (size_t)g.n0 +
                           (size_t)iz * (size_t)g.n0 * (size_t)g.n1;
        const int2 be = __ldg(&g.cells[key]);
        bx = be.x;
        nc = max(be.y - be.x, 0);
      }
    }
    const unsigned validm = __ballot_sync(kFull, valid);
    const unsigned ingm = __ballot_sync(kFull, ing);
    // inclusive / exclusive prefix of the candidate counts over the chunk
    int incl = nc;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, off);
      if (lane >= off) incl += t;
    }
    const int excl = incl - nc;
    const int total = __shfl_sync(kFull, incl, 31);
    // cells (in chunk order) that end the walk at the current radius
    unsigned bm = __ballot_sync(kFull, valid && cd > s.rr);
    int cur = 0;         // first cell of the chunk whose break test is still due
    int brk = -1;        // cell the walk stops at (-1: none in this chunk)
    for (int base = 0; base < total && brk < 0; base += 32) {
      const int gk = base + lane;
      // cell of candidate gk: the last chunk cell whose exclusive prefix is <= gk
      int c = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const int t = c + step;
        const int e = __shfl_sync(kFull, excl, t < 32 ? t : 31);
        if (t < 32 && e <= gk) c = t;
      }
      const int cbx = __shfl_sync(kFull, bx, c);
      const int cex = __shfl_sync(kFull, excl, c);
      float d2 = 0.0f, val = 0.0f;
      int p = -1;
      bool hit = false;
      if (gk < total) {
        p = cbx + (gk - cex);
        const float4 P = __ldg(&g.parts[p]);
        const float fx = P.x - qx, fy = P.y - qy, fz = P.z - qz;
        d2 = (fx * fx + fy * fy) + fz * fz;
        val = P.w;
        hit = d2 <= s.R2up;
      }
      unsigned hm = __ballot_sync(kFull, hit);
      while (hm) {
        const int k = __ffs(hm) - 1;
        hm &= hm - 1;
        const int ck = __shfl_sync(kFull, c, k);
        const float d2k = __shfl_sync(kFull, d2, k);
        const float vk = __shfl_sync(kFull, val, k);
        const int pk = __shfl_sync(kFull, p, k);
        if (ck >= cur) {  // break tests of the cells up to candidate k's cell
          const unsigned due = bm & (0xffffffffu >> (31 - ck)) & (0xffffffffu << cur);
          if (due) {
            brk = __ffs(due) - 1;
            break;
          }
          cur = ck + 1;
        }
        if (d2k <= s.R2up) {
          const float dist = sqrtf(d2k);
          if (dist < s.R) {
            if (lane == s.mi) {
              s.d = dist;
              s.v = vk;
              s.id = pk;
            }
            warp_rescan(s, lane, crad);
            bm = __ballot_sync(kFull, valid && cd > s.rr);
          }
        }
      }
    }
    if (brk < 0 && cur < 32) {  // break tests of the cells after the last hit
      const unsigned due = bm & (0xffffffffu << cur);
      if (due) brk = __ffs(due) - 1;
    }
    // statistics: the in-grid cells before the break and their candidates
    const unsigned seen = brk < 0 ? validm : (brk == 0 ? 0u : (0xffffffffu >> (32 - brk)));
    st.cells += __popc(ingm & seen);
    st.cands += brk < 0 ? (uint32_t)total : (uint32_t)__shfl_sync(kFull, excl, brk);
    if (brk >= 0) return;
  }
}

__global__ void __launch_bounds__(256)
nn8_query_warp_kernel(GridView g, const char4* __restrict__ spiral_g,
                      const float4* __restrict__ pts, uint64_t n, int merge,
                      float* __restrict__ list_d, float* __restrict__ list_v,
                      int32_t* __restrict__ list_id, float* __restrict__ out,
                      int32_t* __restrict__ idx8, float* __restrict__ d8,
                      const uint32_t* __restrict__ s2u, unsigned long long* __restrict__ stats) {
  __shared__ char4 spiral[1000];
  load_spiral(spiral, spiral_g);
  const int lane = threadIdx.x & 31;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  WalkStats st;
  for (uint64_t i = blockIdx.x * (uint64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); i < n;
       i += warps) {
    const float4 q = pts[i];
    WarpSlots s;
    s.d = FLT_MAX;
    s.v = 0.0f;
    s.id = -1;
    if (merge && lane < 8) {
      s.d = list_d[8 * i + lane];
      s.v = list_v[8 * i + lane];
      const int32_t o = list_id[8 * i + lane];
      s.id = o >= 0 ? (int32_t)(0x80000000u | (uint32_t)o) : -1;
    }
    warp_rescan(s, lane, g.cell_radius);
    nn8_walk_warp(g, spiral, q.x, q.y, q.z, s, lane, st);
    // finalize in slot order (volumetric_nn8_reconstruction.cl:212-270)
    const float w = weight3d(s.d);
    float ws = 0.0f, dot = 0.0f;
#pragma unroll
    for (int t = 0; t < 8; ++t) ws = ws + __shfl_sync(kFull, w, t);
#pragma unroll
    for (int t = 0; t < 8; ++t)
      dot = __fmaf_rn(__shfl_sync(kFull, w, t), __shfl_sync(kFull, s.v, t), dot);
    if (lane == 0) out[i] = (ws != 0.0f && dot != 0.0f) ? dot / ws : 0.0f;
    if (lane < 8) {
      const int32_t id = s.id;
      const int32_t orig =
          id == -1 ? -1 : (id < 0 ? (int32_t)((uint32_t)id & 0x7fffffffu) : (int32_t)s2u[id]);
      list_d[8 * i + lane] = s.d;
      list_v[8 * i + lane] = s.v;
      list_id[8 * i + lane] = orig;
      if (idx8) idx8[8 * i + lane] = orig;
      if (d8) d8[8 * i + lane] = s.d;
    }
  }
  if (lane == 0) {
    atomicAdd(&stats[3], (unsigned long long)st.cells);
    atomicAdd(&stats[4], (unsigned long long)st.cands);
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
  if (c.query_engine == ILC_QUERY_WARP) {
    // one warp per query; persistent blocks of 8 warps, as many as are resident
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, nn8_query_warp_kernel, 256, 0);
    const uint64_t cap = (uint64_t)(sms > 0 ? sms : 148) * (uint64_t)(per_sm > 0 ? per_sm : 1);
    const uint64_t want = (n + 7) / 8;
    const unsigned wb = (unsigned)(want < cap ? (want > 0 ? want : 1) : cap);
    nn8_query_warp_kernel<<<wb, 256, 0, c.stream>>>(
        g, c.spiral.as<char4>(), pts, n, merge ? 1 : 0, c.list_d.as<float>(),
        c.list_v.as<float>(), c.list_id.as<int32_t>(), out, idx8, d8, c.s2u.as<uint32_t>(),
        stats);
  } else {
    nn8_query_kernel<<<blocks, 256, 0, c.stream>>>(
        g, c.spiral.as<char4>(), pts, n, merge ? 1 : 0, c.list_d.as<float>(),
        c.list_v.as<float>(), c.list_id.as<int32_t>(), out, idx8, d8, c.s2u.as<uint32_t>(),
        stats);
  }
  return cudaGetLastError();
}

}  // namespace ilc
