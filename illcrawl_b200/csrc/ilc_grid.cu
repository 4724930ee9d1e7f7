// ilc_grid.cu -- particle grid build on the device (particle_grid.cpp:25-252,
// particle_grid.cl:45-190, util.cl:24-49).
//
// Pipeline: bounding box (exact float min/max) -> host grid parameters in
// double, as the reference -> cell keys -> stable LSD radix sort of (key,
// original index) -> gather of the float4 particles into cell order -> cell
// [begin, end) ranges by adjacent difference over a zero-filled cell array.
// The stable sort gives the permutation boost::compute::sort_by_key gives, so
// keys, permutation and cell ranges are bit-identical to the reference's.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "ilc_device.cuh"
#include "ilc_internal.h"

namespace ilc {

namespace {

// Order-preserving map float -> uint32 (for atomicMin/atomicMax on floats).
__device__ __forceinline__ unsigned f2ord(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float ord2f_bits(unsigned o, unsigned* bits) {
  const unsigned u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
  *bits = u;
  return 0.0f;
}

__global__ void bbox_kernel(const float4* __restrict__ in, uint64_t n, unsigned* __restrict__ acc) {
  // acc[0..2] min (ordered), acc[3..5] max (ordered), acc[6] nonfinite flag
  unsigned mn[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
  unsigned mx[3] = {0u, 0u, 0u};
  unsigned bad = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float4 p = in[i];
    const float c[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (!isfinite(c[k])) { bad = 1; continue; }
      const unsigned o = f2ord(c[k]);
      mn[k] = min(mn[k], o);
      mx[k] = max(mx[k], o);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      mn[k] = min(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], off));
      mx[k] = max(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], off));
    }
  }
  bad = __any_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicMin(&acc[k], mn[k]);
      atomicMax(&acc[3 + k], mx[k]);
    }
    if (bad) atomicOr(&acc[6], 1u);
  }
}

struct KeyGrid {
  float min0, min1, min2, cs0, cs1, cs2;
  int n0, n1;
  uint64_t total;
};

// grid3d_generate_sort_keys (particle_grid.cl:96-112): key = ix + iy*nx + iz*nx*ny
// with (int)floor((p - min)/cs). Keys outside [0, total) raise a flag.
__global__ void keys_kernel(const float4* __restrict__ in, uint64_t n, KeyGrid g,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                            uint32_t* __restrict__ flags) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 p = in[i];
  const int ix = to_int_sat(floorf((p.x - g.min0) / g.cs0));
  const int iy = to_int_sat(floorf((p.y - g.min1) / g.cs1));
  const int iz = to_int_sat(floorf((p.z - g.min2) / g.cs2));
  const uint64_t key = (uint64_t)(int64_t)ix + (uint64_t)(int64_t)iy * (uint64_t)g.n0 +
                       (uint64_t)(int64_t)iz * (uint64_t)g.n0 * (uint64_t)g.n1;
  if (key >= g.total) {
    atomicOr(flags, FLAG_KEY_RANGE);
    keys[i] = 0;
  } else {
    keys[i] = (uint32_t)key;
  }
  vals[i] = (uint32_t)i;
}

// ---------------- stable LSD radix sort, 8-bit digits ----------------------
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
constexpr int kWarps = kSortThreads / 32;

// Per-tile digit histogram, stored digit-major: hist[digit * tiles + tile].
__global__ void radix_hist_kernel(const uint32_t* __restrict__ keys, uint64_t n, int shift,
                                  uint32_t tiles, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const uint64_t i = base + (uint64_t)it * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of m entries by one block of 1024 threads (chunked).
__global__ void scan_kernel(uint32_t* __restrict__ a, uint64_t m) {
  __shared__ uint32_t part[1024];
  const uint64_t chunk = (m + 1023) / 1024;
  const uint64_t b = threadIdx.x * chunk, e = min(m, b + chunk);
  uint32_t s = 0;
  for (uint64_t i = b; i < e; ++i) s += a[i];
  part[threadIdx.x] = s;
  __syncthreads();
  // Hillis-Steele inclusive scan over the 1024 partials
  for (int off = 1; off < 1024; off <<= 1) {
    const uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
  for (uint64_t i = b; i < e; ++i) {
    const uint32_t v = a[i];
    a[i] = run;
    run += v;
  }
}

// Multi-block exclusive scan for long arrays (the radix histogram holds
// 256 x tiles entries: 8.4 M at 67 M particles). Three coalesced passes:
// per-chunk sums, a scan of the chunk sums by scan_kernel, then every chunk
// scanned in place from its offset. Same result as scan_kernel (integer sums).
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 16;                           // consecutive entries per thread
constexpr uint64_t kScanChunk = kScanThreads * kScanPer;  // 16,384 entries per block

// Block-wide exclusive scan of one value per thread (1024 threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, off);
    if (lane >= off) inc += t;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_tot[lane];
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, w, off);
      if (lane >= off) w += t;
    }
    warp_tot[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  return (warp ? warp_tot[warp - 1] : 0u) + inc - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_sums_kernel(const uint32_t* __restrict__ a,
                                                                 uint64_t m,
                                                                 uint32_t* __restrict__ sums) {
  __shared__ uint32_t warp_tot[32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanChunk;
  uint32_t s = 0;
#pragma unroll
  for (int it = 0; it < kScanPer; ++it) {
    const uint64_t i = base + (uint64_t)it * kScanThreads + threadIdx.x;
    if (i < m) s += a[i];
  }
  const uint32_t ex = block_exclusive_scan(s, warp_tot);
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = ex + s;
}

__global__ void __launch_bounds__(kScanThreads) scan_chunks_kernel(uint32_t* __restrict__ a,
                                                                   uint64_t m,
                                                                   const uint32_t* __restrict__ offs) {
  __shared__ uint32_t warp_tot[32];
  const uint64_t b = (uint64_t)blockIdx.x * kScanChunk + (uint64_t)threadIdx.x * kScanPer;
  uint32_t v[kScanPer];
  if (b + kScanPer <= m) {  // 64-byte aligned: the array and every chunk start are
    const uint4* p = reinterpret_cast<const uint4*>(a + b);
#pragma unroll
    for (int q = 0; q < kScanPer / 4; ++q) {
      const uint4 t = p[q];
      v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) v[k] = b + k < m ? a[b + k] : 0u;
  }
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) s += v[k];
  uint32_t run = block_exclusive_scan(s, warp_tot) + offs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    const uint32_t t = v[k];
    v[k] = run;
    run += t;
  }
  if (b + kScanPer <= m) {
    uint4* p = reinterpret_cast<uint4*>(a + b);
#pragma unroll
    for (int q = 0; q < kScanPer / 4; ++q)
      p[q] = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  } else {
#pragma unroll
    for (int k = 0; k < kScanPer; ++k)
      if (b + k < m) a[b + k] = v[k];
  }
}

// Number of chunk sums the multi-block scan of m entries needs.
inline uint64_t scan_chunks(uint64_t m) { return (m + kScanChunk - 1) / kScanChunk; }

// Exclusive scan of a[0, m) in place on stream st; `sums` holds
// scan_chunks(m) entries (unused when m fits one chunk). a must be 16-byte
// aligned. Returns the number of kernels launched.
int scan_u32(uint32_t* a, uint64_t m, uint32_t* sums, cudaStream_t st) {
  if (m <= kScanChunk) {
    scan_kernel<<<1, 1024, 0, st>>>(a, m);
    return 1;
  }
  const unsigned nb = (unsigned)scan_chunks(m);
  scan_sums_kernel<<<nb, kScanThreads, 0, st>>>(a, m, sums);
  scan_kernel<<<1, 1024, 0, st>>>(sums, nb);
  scan_chunks_kernel<<<nb, kScanThreads, 0, st>>>(a, m, sums);
  return 3;
}

// Stable scatter: items of a tile are ranked in index order (warp-contiguous
// chunks of 256, lane-striped), per digit, then placed at the tile's scanned
// digit offset.
__global__ void radix_scatter_kernel(const uint32_t* __restrict__ kin,
                                     const uint32_t* __restrict__ vin, uint64_t n, int shift,
                                     uint32_t tiles, const uint32_t* __restrict__ hist,
                                     uint32_t* __restrict__ kout, uint32_t* __restrict__ vout) {
  __shared__ uint32_t wcount[kWarps][256];
  __shared__ uint32_t goff[256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kWarps * 256; i += kSortThreads) (&wcount[0][0])[i] = 0;
  goff[threadIdx.x] = hist[(uint64_t)threadIdx.x * tiles + blockIdx.x];
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile + (uint64_t)warp * (32 * kSortItems);
  uint32_t k[kSortItems], v[kSortItems], rank[kSortItems];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const uint64_t i = base + (uint64_t)it * 32 + lane;
    const bool ok = i < n;
    k[it] = ok ? kin[i] : 0u;
    v[it] = ok ? vin[i] : 0u;
    const unsigned digit = ok ? ((k[it] >> shift) & 255u) : (256u + lane);
    const unsigned peers = __match_any_sync(0xffffffffu, digit);
    const unsigned before = __popc(peers & lt);
    const unsigned leader = __ffs(peers) - 1;
    uint32_t cnt = 0;
    if (ok) cnt = wcount[warp][digit];
    rank[it] = cnt + before;
    __syncwarp();
    if (ok && lane == (int)leader) wcount[warp][digit] = cnt + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {  // per digit: counts -> exclusive offsets across warps
    const int d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      const uint32_t t = wcount[w][d];
      wcount[w][d] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < kSortItems; ++it) {
    const uint64_t i = base + (uint64_t)it * 32 + lane;
    if (i < n) {
      const unsigned digit = (k[it] >> shift) & 255u;
      const uint32_t pos = goff[digit] + wcount[warp][digit] + rank[it];
      kout[pos] = k[it];
      vout[pos] = v[it];
    }
  }
}

// grid3d_sort_particles_into_cells + sorted->unsorted map
__global__ void gather_kernel(const float4* __restrict__ in, const uint32_t* __restrict__ perm,
                              uint64_t n, float4* __restrict__ out, uint32_t* __restrict__ s2u) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = perm[i];
  out[i] = in[j];
  s2u[i] = j;
}

// grid3d_determine_cells_begin / _end on the sorted keys
__global__ void cell_ranges_kernel(const uint32_t* __restrict__ sk, uint64_t n,
                                   int2* __restrict__ cells) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t k = sk[i];
  if (i == 0 || sk[i - 1] != k) cells[k].x = (int)i;
  if (i + 1 == n || sk[i + 1] != k) cells[k].y = (int)(i + 1);
}

// Sub-box code of every sorted particle: which quarter of its cell it lies in
// per axis (clamped to 0..3), packed sx + 4 sy + 16 sz. The nn8 walk uses it
// only to skip candidates that lie, by more than a rounding margin, outside
// the cube of the current search radius around the query points: those could
// never be inserted, so skipping them leaves every result unchanged.
__global__ void codes_kernel(const float4* __restrict__ parts, const uint32_t* __restrict__ sk,
                             uint64_t n, KeyGrid kg, uint8_t* __restrict__ codes) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t k = sk[i];
  const uint32_t kx = k % (uint32_t)kg.n0, kyz = k / (uint32_t)kg.n0;
  const uint32_t ky = kyz % (uint32_t)kg.n1, kz = kyz / (uint32_t)kg.n1;
  const float4 p = parts[i];
  const float c[3] = {p.x, p.y, p.z};
  const float mn[3] = {kg.min0 + (float)kx * kg.cs0, kg.min1 + (float)ky * kg.cs1,
                       kg.min2 + (float)kz * kg.cs2};
  const float iw[3] = {4.0f / kg.cs0, 4.0f / kg.cs1, 4.0f / kg.cs2};
  int q[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float t = (c[a] - mn[a]) * iw[a];
    q[a] = t > 0.0f ? min((int)t, 3) : 0;
  }
  codes[i] = (uint8_t)(q[0] | (q[1] << 2) | (q[2] << 4));
}

inline unsigned grid_blocks(uint64_t n, int threads) {
  return (unsigned)((n + threads - 1) / threads);
}

}  // namespace

cudaError_t grid_bbox(Context& c, const float4* in, uint64_t n, float* mn3, float* mx3,
                      bool* nonfinite) {
  cudaError_t e = c.hist.ensure(64);
  if (e) return e;
  unsigned init[8] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u, 0u};
  e = cudaMemcpyAsync(c.hist.p, init, sizeof(init), cudaMemcpyHostToDevice, c.stream);
  if (e) return e;
  const unsigned blocks = (unsigned)std::min<uint64_t>(grid_blocks(n, 256), 148 * 8);
  bbox_kernel<<<blocks, 256, 0, c.stream>>>(in, n, c.hist.as<unsigned>());
  ++c.launches;
  e = cudaGetLastError();
  if (e) return e;
  unsigned out[8];
  e = cudaMemcpyAsync(out, c.hist.p, sizeof(out), cudaMemcpyDeviceToHost, c.stream);
  if (e) return e;
  e = cudaStreamSynchronize(c.stream);
  if (e) return e;
  for (int k = 0; k < 3; ++k) {
    unsigned b;
    ord2f_bits(out[k], &b);
    std::memcpy(&mn3[k], &b, 4);
    ord2f_bits(out[3 + k], &b);
    std::memcpy(&mx3[k], &b, 4);
  }
  *nonfinite = out[6] != 0;
  return cudaSuccess;
}

cudaError_t exclusive_scan_u32(Context& c, uint32_t* a, uint64_t m) {
  ++c.launches;
  scan_kernel<<<1, 1024, 0, c.stream>>>(a, m);
  return cudaGetLastError();
}

cudaError_t grid_build_device(Context& c, const float4* in, uint64_t n) {
  cudaError_t e;
  const GridParams& g = c.gp;
  if ((e = c.keys_a.ensure(n * 4)) || (e = c.keys_b.ensure(n * 4)) ||
      (e = c.vals_a.ensure(n * 4)) || (e = c.vals_b.ensure(n * 4)) ||
      (e = c.parts.ensure(n * 16)) || (e = c.s2u.ensure(n * 4)) ||
      (e = c.codes.ensure(((n + 15) / 16) * 16 + 16)) || (e = c.cells.ensure(g.total * 8)) ||
      (e = c.flags.ensure(kFlagsBytes)))
    return e;
  const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
  // histogram, then the scan's chunk sums
  if ((e = c.hist.ensure(tiles * 256 * 4 + 4 * scan_chunks(tiles * 256) + 64))) return e;
  uint32_t* chunk_sums = c.hist.as<uint32_t>() + tiles * 256;
  if ((e = cudaMemsetAsync(c.flags.p, 0, kFlagsBytes, c.stream))) return e;

  KeyGrid kg{g.min[0], g.min[1], g.min[2], g.cs[0], g.cs[1], g.cs[2], g.n[0], g.n[1], g.total};
  keys_kernel<<<grid_blocks(n, 256), 256, 0, c.stream>>>(in, n, kg, c.keys_a.as<uint32_t>(),
                                                          c.vals_a.as<uint32_t>(),
                                                          c.flags.as<uint32_t>());
  if ((e = cudaGetLastError())) return e;

  int bits = 1;
  while (bits < 32 && (1ull << bits) < g.total) ++bits;
  uint32_t *ka = c.keys_a.as<uint32_t>(), *kb = c.keys_b.as<uint32_t>();
  uint32_t *va = c.vals_a.as<uint32_t>(), *vb = c.vals_b.as<uint32_t>();
  for (int shift = 0; shift < bits; shift += 8) {
    radix_hist_kernel<<<(unsigned)tiles, kSortThreads, 0, c.stream>>>(
        ka, n, shift, (uint32_t)tiles, c.hist.as<uint32_t>());
    c.launches += 2 + scan_u32(c.hist.as<uint32_t>(), tiles * 256, chunk_sums, c.stream);
    radix_scatter_kernel<<<(unsigned)tiles, kSortThreads, 0, c.stream>>>(
        ka, va, n, shift, (uint32_t)tiles, c.hist.as<uint32_t>(), kb, vb);
    if ((e = cudaGetLastError())) return e;
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  gather_kernel<<<grid_blocks(n, 256), 256, 0, c.stream>>>(in, va, n, c.parts.as<float4>(),
                                                            c.s2u.as<uint32_t>());
  c.sorted_keys = ka;
  if ((e = cudaMemsetAsync(c.cells.p, 0, g.total * 8, c.stream))) return e;
  cell_ranges_kernel<<<grid_blocks(n, 256), 256, 0, c.stream>>>(ka, n, c.cells.as<int2>());
  codes_kernel<<<grid_blocks(n, 256), 256, 0, c.stream>>>(c.parts.as<float4>(), ka, n, kg,
                                                           c.codes.as<uint8_t>());
  c.launches += 4;  // keys, gather, cell ranges, codes
  return cudaGetLastError();
}

// Spiral iteration table (particle_grid_iteration_order.cl:25-1048): per subcell
// id = sx + 2*sy + 4*sz, the 125 offsets of [-2,2]^3 enumerated x-outermost,
// stable-sorted by distance from the subcell centre (+-0.25) to the cell centre.
void spiral_table(int8_t out[8][125][3]) {
  for (int sz = 0; sz < 2; ++sz)
    for (int sy = 0; sy < 2; ++sy)
      for (int sx = 0; sx < 2; ++sx) {
        const double cc[3] = {sx ? 0.25 : -0.25, sy ? 0.25 : -0.25, sz ? 0.25 : -0.25};
        struct Off { int d[3]; double r; };
        std::vector<Off> v;
        v.reserve(125);
        for (int dx = -2; dx <= 2; ++dx)
          for (int dy = -2; dy <= 2; ++dy)
            for (int dz = -2; dz <= 2; ++dz) {
              const double a = dx - cc[0], b = dy - cc[1], q = dz - cc[2];
              v.push_back(Off{{dx, dy, dz}, std::sqrt(a * a + b * b + q * q)});
            }
        std::stable_sort(v.begin(), v.end(), [](const Off& l, const Off& r) { return l.r < r.r; });
        const int id = sx + 2 * sy + 4 * sz;
        for (int i = 0; i < 125; ++i)
          for (int k = 0; k < 3; ++k) out[id][i][k] = (int8_t)v[i].d[k];
      }
}

}  // namespace ilc

// ---------------------------------------------------------------------------
// Allocation-free grid build.
//
// Some callers cannot allocate device memory at the point where they need a
// grid: real-time loops with a fixed memory budget, or hosts whose allocator
// owns every device buffer. ilc_grid_build_noalloc builds the same particle
// grid as ilc_nn8_setup_particles without any allocation: the caller passes
// device buffers for the inputs and outputs, and the sort's scratch space is
// this file-scope device array, sized for at most ILC_NOALLOC_MAX_PARTICLES
// particles (about 16.5 MiB, held on every GPU that loads the library until
// the process exits). The grid parameters are computed on the host from the
// bounding box, so the call waits on its stream before it returns.
// ---------------------------------------------------------------------------
namespace ilc {
namespace {

constexpr uint64_t kNoAllocMax = 1ull << 20;  // ILC_NOALLOC_MAX_PARTICLES
constexpr uint64_t kNoAllocTiles = (kNoAllocMax + 2047) / 2048;
// [0, 64): bounding-box words; [64, 128): flags; then keys a/b, values a/b,
// and the radix histogram.
constexpr size_t kOffKeysA = 256;
constexpr size_t kOffKeysB = kOffKeysA + 4 * kNoAllocMax;
constexpr size_t kOffValsA = kOffKeysB + 4 * kNoAllocMax;
constexpr size_t kOffValsB = kOffValsA + 4 * kNoAllocMax;
constexpr size_t kOffHist = kOffValsB + 4 * kNoAllocMax;
constexpr size_t kScratchBytes = kOffHist + 4 * 256 * kNoAllocTiles;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device, looked up once per device
// with that device current (in host code the symbol is only a host-side
// stand-in for the array, not a device address).
// Every thread that looks it up stores the same value, so relaxed atomics
// suffice to make concurrent first calls well defined.
constexpr int kMaxDevices = 64;
static std::atomic<void*> g_noalloc_ptr[kMaxDevices];

}  // namespace
}  // namespace ilc

extern "C" ilc_status ilc_grid_build_noalloc(const float* particles, uint64_t n,
                                             float* sorted_particles, int32_t* cells,
                                             uint64_t cells_capacity,
                                             uint32_t* sorted_to_unsorted, ilc_grid_desc* desc,
                                             void* stream) {
  using namespace ilc;
  if (!particles || !sorted_particles || !cells || !sorted_to_unsorted || !desc || n == 0)
    return ILC_ERR_INVALID_ARGUMENT;
  if (n > kNoAllocMax) return ILC_ERR_INVALID_ARGUMENT;  // beyond the scratch array
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ILC_ERR_CUDA;
  void* sp = g_noalloc_ptr[dev].load(std::memory_order_relaxed);
  if (!sp) {
    if (cudaGetSymbolAddress(&sp, g_noalloc_scratch) != cudaSuccess || !sp) return ILC_ERR_CUDA;
    g_noalloc_ptr[dev].store(sp, std::memory_order_relaxed);
  }
  unsigned char* s = static_cast<unsigned char*>(sp);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float4* in = reinterpret_cast<const float4*>(particles);
  unsigned* acc = reinterpret_cast<unsigned*>(s);
  uint32_t* flags = reinterpret_cast<uint32_t*>(s + 64);
  // bounding box (the words must start at +/- extremes, the flags at zero)
  const unsigned init[8] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0u, 0u};
  if (cudaMemcpyAsync(acc, init, sizeof(init), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemsetAsync(flags, 0, 64, st) != cudaSuccess)
    return ILC_ERR_CUDA;
  bbox_kernel<<<(unsigned)std::min<uint64_t>(grid_blocks(n, 256), 148 * 8), 256, 0, st>>>(in, n,
                                                                                         acc);
  unsigned box[8];
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(box, acc, sizeof(box), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return ILC_ERR_CUDA;
  if (box[6]) return ILC_ERR_NONFINITE_INPUT;
  // grid parameters in double, as particle_grid.cpp:54-103
  double mn[3], mx[3], vol = 1.0;
  for (int k = 0; k < 3; ++k) {
    unsigned b;
    float f;
    ord2f_bits(box[k], &b);
    std::memcpy(&f, &b, 4);
    mn[k] = (double)f - 0.1;
    ord2f_bits(box[3 + k], &b);
    std::memcpy(&f, &b, 4);
    mx[k] = (double)f + 0.1;
    vol *= (mx[k] - mn[k]);
  }
  const double w = std::cbrt((double)8 / (double)n * vol);
  KeyGrid kg;
  int32_t nc[3];
  uint64_t total = 1;
  for (int k = 0; k < 3; ++k) {
    const double c = std::ceil((mx[k] - mn[k]) / w);
    nc[k] = (c >= 1.0 && c <= 2147483647.0) ? (int32_t)c : 0;  // 0: rejected below
    desc->min_corner[k] = (float)mn[k];
    desc->cell_sizes[k] = (float)w;
    desc->num_cells[k] = nc[k];
    total *= (uint64_t)(nc[k] > 0 ? nc[k] : 0);
    if (total >= (1ull << 32)) total = 1ull << 32;  // rejected below; no wrap
  }
  desc->total_cells = total;
  desc->num_particles = n;
  if (total == 0 || total >= (1ull << 32)) return ILC_ERR_GRID_TOO_LARGE;
  if (total > cells_capacity) return ILC_ERR_INVALID_ARGUMENT;  // desc says how many are needed
  kg.min0 = desc->min_corner[0]; kg.min1 = desc->min_corner[1]; kg.min2 = desc->min_corner[2];
  kg.cs0 = desc->cell_sizes[0]; kg.cs1 = desc->cell_sizes[1]; kg.cs2 = desc->cell_sizes[2];
  kg.n0 = nc[0]; kg.n1 = nc[1];
  kg.total = total;
  uint32_t* ka = reinterpret_cast<uint32_t*>(s + kOffKeysA);
  uint32_t* kb = reinterpret_cast<uint32_t*>(s + kOffKeysB);
  uint32_t* va = reinterpret_cast<uint32_t*>(s + kOffValsA);
  uint32_t* vb = reinterpret_cast<uint32_t*>(s + kOffValsB);
  uint32_t* hist = reinterpret_cast<uint32_t*>(s + kOffHist);
  keys_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(in, n, kg, ka, va, flags);
  const uint64_t tiles = (n + kSortTile - 1) / kSortTile;
  int bits = 1;
  while (bits < 32 && (1ull << bits) < total) ++bits;
  for (int shift = 0; shift < bits; shift += 8) {
    radix_hist_kernel<<<(unsigned)tiles, kSortThreads, 0, st>>>(ka, n, shift, (uint32_t)tiles,
                                                                 hist);
    scan_kernel<<<1, 1024, 0, st>>>(hist, tiles * 256);
    radix_scatter_kernel<<<(unsigned)tiles, kSortThreads, 0, st>>>(ka, va, n, shift,
                                                                   (uint32_t)tiles, hist, kb, vb);
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  gather_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(in, va, n,
                                                      reinterpret_cast<float4*>(sorted_particles),
                                                      sorted_to_unsorted);
  if (cudaMemsetAsync(cells, 0, total * 8, st) != cudaSuccess) return ILC_ERR_CUDA;
  cell_ranges_kernel<<<grid_blocks(n, 256), 256, 0, st>>>(ka, n, reinterpret_cast<int2*>(cells));
  uint32_t f = 0;
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(&f, flags, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return ILC_ERR_CUDA;
  if (f & FLAG_KEY_RANGE) return ILC_ERR_INTERNAL;
  return ILC_OK;
}
