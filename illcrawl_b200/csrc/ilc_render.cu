// ilc_render.cu -- line-of-sight projection over the camera plane: the whole
// parallel_runge_kutta_fehlberg host loop (integration.cpp:84-307,
// volumetric_integration.cpp:32-88) as one kernel launch.
//
// Each thread owns one pixel's integrator and runs its RKF4(5) steps to the
// end of the ray, evaluating the 4 integrand points of every step with the
// nn8 walk inline. A ray's state depends only on its own evaluations, so this
// is the same computation as the reference's lock-step loop with stream
// compaction, without its per-iteration host synchronisations.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "ilc_device.cuh"
#include "ilc_internal.h"
#include "ilc_walk4.cuh"

namespace ilc {

GridView make_grid_view(const Context& c) {
  GridView g;
  std::memset(&g, 0, sizeof(g));  // padding too: the bytes key the batched launch graph
  g.min0 = c.gp.min[0]; g.min1 = c.gp.min[1]; g.min2 = c.gp.min[2];
  g.cs0 = c.gp.cs[0]; g.cs1 = c.gp.cs[1]; g.cs2 = c.gp.cs[2];
  g.half0 = 0.5f * c.gp.cs[0]; g.half1 = 0.5f * c.gp.cs[1]; g.half2 = 0.5f * c.gp.cs[2];
  g.cell_radius = 0.5f * sqrtf((c.gp.cs[0] * c.gp.cs[0] + c.gp.cs[1] * c.gp.cs[1]) +
                               c.gp.cs[2] * c.gp.cs[2]);
  g.n0 = c.gp.n[0]; g.n1 = c.gp.n[1]; g.n2 = c.gp.n[2];
  g.cells = c.cells.as<int2>();
  g.parts = c.parts.as<float4>();
  g.codes = c.codes.as<uint32_t>();
  g.inv_w0 = 4.0f / c.gp.cs[0];
  g.inv_w1 = 4.0f / c.gp.cs[1];
  g.inv_w2 = 4.0f / c.gp.cs[2];
  // slack for the float rounding of cell keys and cell boxes: a 1024th of a
  // cell, and at least 8 ulp of the largest coordinate of the grid
  float ext = 0.0f;
  for (int k = 0; k < 3; ++k)
    ext = std::fmax(ext, std::fmax(std::fabs(c.gp.min[k]),
                                   std::fabs(c.gp.min[k] + (float)c.gp.n[k] * c.gp.cs[k])));
  g.margin = std::fmax(std::fmax(std::fmax(c.gp.cs[0], c.gp.cs[1]), c.gp.cs[2]) / 1024.0f,
                       ext * 9.5367431640625e-07f);
  return g;
}

namespace {

struct RenderK {
  CamView cam;
  float z0, z_end;
  double atol, rtol;
  int controller;
  int64_t fixed_steps;
  float fixed_h;
  const float* replay_h;    // frozen per-ray sequences (ray-major, rec_cap each)
  const int32_t* replay_n;  // steps per ray
  int64_t max_steps;
  float window;     // z window of the adaptive schedule (<= 0: none)
  int row_stride;   // render every row_stride-th row of tiles (1 = all)
  int row0;         // first pixel row (a multiple of the tile height)
  int row_end;      // one past the last pixel row
  float* rec_h;     // optional: accepted step sizes per ray (ray-major, rec_cap each)
  int32_t* rec_n;   // optional: number of accepted steps per ray
  int64_t rec_cap;
  float scale;
  int apply_scale;
  float* out;
  double* out_d;        // optional (frozen replay): the line integrals summed in double
  uint64_t* ray_stats;  // optional: per ray (steps, accepted, cells visited, candidates)
  unsigned* queue;      // persistent launch: tile counter (nullptr: one block per tile)
  unsigned ntiles, tiles_x;
};

// Pixel tiling: a block of 128 threads covers 16 x 8 pixels; each warp an
// 8 x 4 tile, so the 32 rays of a warp are spatial neighbours.
constexpr int kRenderThreads = 128;
constexpr int kTileX = 16, kTileY = 8;
__device__ __forceinline__ void block_pixel(int row_stride, int row0, int bx, int by, int& ix,
                                            int& iy) {
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  ix = bx * kTileX + (warp & 1) * 8 + (lane & 7);
  iy = row0 + by * row_stride * kTileY + (warp >> 1) * 4 + (lane >> 3);
}

// One 16 x 8 tile of rays, all threads of the block (the adaptive branch
// synchronises the block at every z window).
__device__ __forceinline__ void render_tile(const RenderK& a, const GridView& g,
                                            const char4* __restrict__ spiral, SlotMem& slot_mem,
                                            uint32_t* __restrict__ flags,
                                            unsigned long long* __restrict__ stats, int bx,
                                            int by) {
  int ix, iy;
  block_pixel(a.row_stride, a.row0, bx, by, ix, iy);
  const bool active = ix < a.cam.nx && iy < a.row_end;
  // per-ray arrays are indexed from the launch's first row
  const int64_t lray = (int64_t)(iy - a.row0) * a.cam.nx + ix;
  WalkStats ws;
  unsigned long long steps = 0, acc = 0;
  bool at_limit = false;
  float px = 0.0f, py = 0.0f, pz = 0.0f;
  if (active) pixel_corner(a.cam, ix, iy, px, py, pz);
  const float lx = a.cam.look0, ly = a.cam.look1, lz = a.cam.look2;
  float I = 0.0f, z = a.z0, h = 1.0f, k1 = 0.0f;
  double Id = 0.0;  // out_d: the same increments summed in double
  float pts[4];
  if (a.replay_h) {
    if (active) {
      // Frozen per-ray sequence: the given steps, every one accepted.
      const int64_t nr = a.replay_n[lray];
      const int32_t n = (int32_t)(nr < 0 ? 0 : (nr > a.rec_cap ? a.rec_cap : nr));
      const float* hs = a.replay_h + lray * a.rec_cap;
      for (int32_t s = 0; s < n; ++s) {
        h = hs[s];
        rkf_points(z, h, pts);
        float e[4];
        nn8_step4(g, spiral, slot_mem, px, py, pz, lx, ly, lz, pts, e, ws);
        float d4 = 25.f / 216.f * k1 + 1408.f / 2565.f * e[0] + 2197.f / 4101.f * e[1] -
                   1.f / 5.f * e[2];
        d4 *= h;
        I = I + d4;
        if (a.out_d) Id += (double)d4;
        z += h;
        k1 = e[2];
      }
      steps = acc = (unsigned long long)(n > 0 ? n : 0);
    }
  } else if (a.fixed_steps > 0) {
    if (active) {
      // Frozen uniform sequence: every step accepted, I += delta4.
      h = a.fixed_h;
      for (int64_t s = 0; s < a.fixed_steps; ++s) {
        rkf_points(z, h, pts);
        float e[4];
        nn8_step4(g, spiral, slot_mem, px, py, pz, lx, ly, lz, pts, e, ws);
        float d4 = 25.f / 216.f * k1 + 1408.f / 2565.f * e[0] + 2197.f / 4101.f * e[1] -
                   1.f / 5.f * e[2];
        d4 *= h;
        I = I + d4;
        z += h;
        k1 = e[2];
      }
      steps = acc = (unsigned long long)a.fixed_steps;
    }
  } else {
    // Adaptive stepping, scheduled in z windows: every ray of the block runs
    // its steps up to the window's end, then the block moves on together, so
    // the rays in flight on an SM query one slab of the grid at a time. The
    // windows only order the work; each ray's step sequence is unchanged.
    rkf_points(z, h, pts);
    const float fa = (float)a.atol, fr = (float)a.rtol;
    bool run = active;
    float wend = a.window > 0.0f ? a.z0 + a.window : a.z_end;
    while (__syncthreads_or(run && z < a.z_end)) {
      while (run && z < a.z_end && z < wend) {
        if ((int64_t)steps >= a.max_steps) { at_limit = true; run = false; break; }
        float e[4];
        nn8_step4(g, spiral, slot_mem, px, py, pz, lx, ly, lz, pts, e, ws);
        const float zb = z, hb = h;
        if (a.controller == ILC_CONTROLLER_REF32)
          rkf_advance_ref32(I, z, h, k1, fa, fr, a.z_end, e, kEps, kHmin, kHmax, pts);
        else
          rkf_advance_fp64(I, z, h, k1, a.atol, a.rtol, a.z_end, e, kEps, kHmin, kHmax, pts);
        ++steps;
        if (z != zb) {
          if (a.rec_h && (int64_t)acc < a.rec_cap)
            a.rec_h[lray * a.rec_cap + (int64_t)acc] = hb;
          ++acc;
        }
      }
      wend = a.window > 0.0f ? wend + a.window : a.z_end;
    }
    if (active && a.rec_n) {
      a.rec_n[lray] = (int32_t)min((int64_t)acc, a.rec_cap);
      if ((int64_t)acc > a.rec_cap) atomicOr(flags, FLAG_REC_OVERFLOW);
    }
  }
  if (active && a.out) a.out[(size_t)iy * a.cam.nx + ix] = a.apply_scale ? I * a.scale : I;
  if (active && a.out_d)
    a.out_d[(size_t)iy * a.cam.nx + ix] = a.apply_scale ? Id * (double)a.scale : Id;
  if (active && a.ray_stats) {
    uint64_t* r = a.ray_stats + 4 * lray;
    r[0] = steps;
    r[1] = acc;
    r[2] = ws.cells;
    r[3] = ws.cands;
  }
  if (at_limit) atomicOr(flags, FLAG_STEP_LIMIT);
  // warp-aggregated statistics
  unsigned long long c = ws.cells, k = ws.cands, st = steps, ac = acc, mx = steps,
                     lim = at_limit ? 1ull : 0ull;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    c += __shfl_xor_sync(0xffffffffu, c, off);
    k += __shfl_xor_sync(0xffffffffu, k, off);
    st += __shfl_xor_sync(0xffffffffu, st, off);
    ac += __shfl_xor_sync(0xffffffffu, ac, off);
    lim += __shfl_xor_sync(0xffffffffu, lim, off);
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&stats[0], st);
    atomicAdd(&stats[1], ac);
    atomicAdd(&stats[2], 4ull * st);
    atomicAdd(&stats[3], c);
    atomicAdd(&stats[4], k);
    atomicMax(&stats[5], mx);
    atomicAdd(&stats[6], lim);
  }
}

// Persistent: the resident blocks take tiles (row-major) from a queue until
// none is left, so the blocks that finish early take on more tiles instead of
// idling while the slowest tiles of a wave finish. Without a queue, one block
// per tile.
template <int kMinBlocks>
__global__ void __launch_bounds__(kRenderThreads, kMinBlocks)
render_kernel(RenderK a, GridView g, const char4* __restrict__ spiral_g,
              uint32_t* __restrict__ flags, unsigned long long* __restrict__ stats) {
  __shared__ char4 spiral[1000];
  __shared__ SlotMem slot_mem;
  __shared__ unsigned next_tile;
  load_spiral(spiral, spiral_g);
  if (!a.queue) {
    render_tile(a, g, spiral, slot_mem, flags, stats, blockIdx.x, blockIdx.y);
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) next_tile = atomicAdd(a.queue, 1u);
    __syncthreads();
    const unsigned t = next_tile;
    __syncthreads();
    if (t >= a.ntiles) break;
    render_tile(a, g, spiral, slot_mem, flags, stats, (int)(t % a.tiles_x),
                (int)(t / a.tiles_x));
  }
}

}  // namespace

cudaError_t render_launch(Context& c, const RenderArgs& a, float* kernel_ms) {
  cudaError_t e;
  if ((e = c.flags.ensure(kFlagsBytes))) return e;
  if ((e = cudaMemsetAsync(c.flags.p, 0, kFlagsBytes, c.stream))) return e;
  RenderK k;
  k.cam.look0 = a.cam[0]; k.cam.look1 = a.cam[1]; k.cam.look2 = a.cam[2];
  k.cam.b00 = a.cam[3]; k.cam.b01 = a.cam[4]; k.cam.b02 = a.cam[5];
  k.cam.b10 = a.cam[6]; k.cam.b11 = a.cam[7]; k.cam.b12 = a.cam[8];
  k.cam.min0 = a.cam[9]; k.cam.min1 = a.cam[10]; k.cam.min2 = a.cam[11];
  k.cam.ps = a.cam[12];
  k.cam.nx = a.nx; k.cam.ny = a.ny;
  k.z0 = a.z0; k.z_end = a.z_end;
  k.atol = a.atol; k.rtol = a.rtol;
  k.controller = a.controller;
  k.fixed_steps = a.fixed_steps;
  k.fixed_h = a.fixed_h;
  k.replay_h = a.replay_h;
  k.replay_n = a.replay_n;
  k.max_steps = c.max_steps;
  k.window = a.window_override >= 0.0f ? a.window_override : c.z_window;
  k.row_stride = a.row_stride > 1 ? a.row_stride : 1;
  k.row0 = a.row0;
  k.row_end = a.rows > 0 ? std::min(a.ny, a.row0 + a.rows) : a.ny;
  k.rec_h = a.rec_h;
  k.rec_n = a.rec_n;
  k.rec_cap = a.rec_cap;
  k.scale = a.scale;
  k.apply_scale = a.apply_scale ? 1 : 0;
  k.out = a.out;
  k.out_d = a.out_d;
  k.ray_stats = a.ray_stats;
  const GridView g = make_grid_view(c);
  const int tile_rows = (k.row_end - k.row0 + kTileY - 1) / kTileY;
  dim3 grid((a.nx + kTileX - 1) / kTileX, (tile_rows + k.row_stride - 1) / k.row_stride);
  const int occ = a.occupancy_override >= 0 ? a.occupancy_override : c.render_occupancy;
  k.queue = nullptr;
  k.tiles_x = grid.x;
  k.ntiles = grid.x * grid.y;
  {
    // persistent blocks, as many as are resident
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    cudaError_t oe =
        occ == 5   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_kernel<5>,
                                                                   kRenderThreads, 0)
        : occ == 4 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_kernel<4>,
                                                                   kRenderThreads, 0)
        : occ == 3 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_kernel<3>,
                                                                   kRenderThreads, 0)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, render_kernel<1>,
                                                                   kRenderThreads, 0);
    const unsigned resident = (unsigned)((sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1));
    if (oe == cudaSuccess && k.ntiles > resident) {
      if ((e = c.tile_queue.ensure(256))) return e;
      if ((e = cudaMemsetAsync(c.tile_queue.p, 0, 4, c.stream))) return e;
      k.queue = c.tile_queue.as<unsigned>();
      grid = dim3(resident, 1);
    }
  }
  if (!c.ev0) {
    if ((e = cudaEventCreate(&c.ev0)) || (e = cudaEventCreate(&c.ev1))) return e;
  }
  cudaEventRecord(c.ev0, c.stream);
  ++c.launches;
  unsigned long long* stats = reinterpret_cast<unsigned long long*>(c.flags.as<char>() + 64);
  if (occ == 5)
    render_kernel<5><<<grid, kRenderThreads, 0, c.stream>>>(k, g, c.spiral.as<char4>(),
                                                            c.flags.as<uint32_t>(), stats);
  else if (occ == 4)
    render_kernel<4><<<grid, kRenderThreads, 0, c.stream>>>(k, g, c.spiral.as<char4>(),
                                                            c.flags.as<uint32_t>(), stats);
  else if (occ == 3)
    render_kernel<3><<<grid, kRenderThreads, 0, c.stream>>>(k, g, c.spiral.as<char4>(),
                                                            c.flags.as<uint32_t>(), stats);
  else
    render_kernel<1><<<grid, kRenderThreads, 0, c.stream>>>(k, g, c.spiral.as<char4>(),
                                                            c.flags.as<uint32_t>(), stats);
  if ((e = cudaGetLastError())) return e;
  cudaEventRecord(c.ev1, c.stream);
  if (kernel_ms) {
    if ((e = cudaEventSynchronize(c.ev1))) return e;
    cudaEventElapsedTime(kernel_ms, c.ev0, c.ev1);
  }
  return cudaSuccess;
}

}  // namespace ilc
