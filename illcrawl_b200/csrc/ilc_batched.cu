// ilc_batched.cu -- batched render: many cameras (jobs), aperture masks,
// per-ray chords and V value channels per cell (e.g. 128 X-ray energy bins)
// in one persistent launch fed by a work queue of 32-ray tiles.
//
// The reference renders each (camera, energy bin) as a separate projection
// with its own host loop (animation.cpp:29-100,264-283; spectrum.cpp:89-109).
// Here every warp takes the next tile from a global queue until the queue is
// empty, so rays of very different length (masked apertures, chords of a
// sphere) keep all SMs busy, and the V channels of a ray share one nn8 walk
// per integrand point: the walk yields the 8 neighbours' sorted indices and
// weights once, and the channel values are gathered from a cell-major table
// (one 4*V-byte row per neighbour, read coalesced by the warp).
//
// Step control: one step sequence per ray for all channels, from the joint
// FP64 controller (per channel the single-channel error ratio, minimum over
// channels, accept only if every channel accepts). With V = 1 this is the
// single-ray FP64 controller operation for operation, so a one-channel job
// without mask or chord reproduces the plain render bit for bit.
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <string>
#include <vector>

#include "ilc_device.cuh"
#include "ilc_internal.h"
#include "ilc_walk4.cuh"

namespace ilc {

GridView make_grid_view(const Context& c);  // ilc_render.cu

namespace {

constexpr int kBThreads = 128;
constexpr unsigned kFull = 0xffffffffu;

struct BatchK {
  const JobDev* jobs;
  int n_jobs;
  uint64_t n_items;
  int V;
  const float* chan;
  float* out;
  float* state;   // multi-channel: per ray slot I[V], k1[V], candidate I[V], k5[V]
  double atol, rtol;
  int64_t max_steps;
  int tile_w;
  float window;
  const uint32_t* order;
  unsigned long long* queue;
  int axis_z;       // every job looks along z (look x and y exactly 0)
};

// Largest k with jobs[k].item_begin <= item.
__device__ __forceinline__ int find_job(const JobDev* __restrict__ jobs, int n, uint64_t item) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].item_begin <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Aperture mask, chord of the job's sphere and the ray's float origin.
// Every operation is a single IEEE double or float operation (no
// contraction), in the order the host-side definition uses.
__device__ __forceinline__ void ray_span(const JobDev& j, int ix, int iy, bool& masked,
                                         float o[3], float& len) {
  masked = false;
  if (j.aperture > 0.0) {
    const double dx = ((double)ix + 0.5 - 0.5 * (double)j.nx) * j.ps_d;
    const double dy = ((double)iy + 0.5 - 0.5 * (double)j.ny) * j.ps_d;
    if (dx * dx + dy * dy > j.aperture * j.aperture) masked = true;
  }
  const float tx = (float)ix * j.ps, ty = (float)iy * j.ps;
  float pix[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) pix[i] = (j.minp[i] + tx * j.b0[i]) + ty * j.b1[i];
  if (!(j.radius > 0.0)) {
#pragma unroll
    for (int i = 0; i < 3; ++i) o[i] = pix[i];
    len = (float)j.z_range;
    return;
  }
  const double txd = (double)ix * j.ps_d, tyd = (double)iy * j.ps_d;
  double w[3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
    w[i] = j.centre[i] - ((j.minp_d[i] + txd * j.b0_d[i]) + tyd * j.b1_d[i]);
  const double t = (w[0] * j.look_d[0] + w[1] * j.look_d[1]) + w[2] * j.look_d[2];
  const double ww = (w[0] * w[0] + w[1] * w[1]) + w[2] * w[2];
  const double b2 = ww - t * t;
  const double r2 = j.radius * j.radius;
  double half = b2 < r2 ? sqrt(r2 - b2) : 0.0;
  const double mh = 0.5 * j.min_chord;
  if (half < mh) half = mh;
  double z0 = t - half;
  const double z1 = t + half;
  if (z0 < 0.0) z0 = 0.0;
  len = z1 > z0 ? (float)(z1 - z0) : 0.0f;
  const float z0f = (float)z0;
#pragma unroll
  for (int i = 0; i < 3; ++i) o[i] = pix[i] + z0f * j.look[i];
}

// Weights of point J's slots (get_weight3d) and their sum, in slot order.
template <int J>
__device__ __forceinline__ void slot_weights(const Step4& s, float w[8], float& ws) {
#pragma unroll
  for (int t = 0; t < 8; ++t) w[t] = weight3d(s4_d(s, J, t));
  ws = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) ws = ws + w[t];
}

// Single-channel value of point J (nn8 finalize order), from the channel
// table or, without one, from the particles' q.
template <int J>
__device__ __forceinline__ float value1(const Step4& s, const float* __restrict__ chan,
                                        const float4* __restrict__ parts) {
  float w[8], ws;
  slot_weights<J>(s, w, ws);
  float dot = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int id = __float_as_int(s4_v(s, J, t));
    const float v = id < 0 ? 0.0f : (chan ? __ldg(&chan[id]) : __ldg(&parts[id].w));
    dot = __fmaf_rn(w[t], v, dot);
  }
  return (ws != 0.0f && dot != 0.0f) ? dot / ws : 0.0f;
}

// Hands point J's slots to the warp: the distances become weights in place
// (the indices stay), and their sum goes to wsum.
template <int J>
__device__ __forceinline__ void slots_to_weights(const Step4& s, float& wsum) {
  float w[8], ws;
  slot_weights<J>(s, w, ws);
#pragma unroll
  for (int t = 0; t < 8; ++t) s4_d(s, J, t) = w[t];
  wsum = ws;
}

// One channel's FP64 step candidate: returns I + delta4 (as the accepted
// value) and sets x to the channel's error ratio
// max(atol, |I/z' rtol|) h / (2 |delta5 - delta4|), or 16 if delta4 == delta5.
__device__ __forceinline__ float channel_step(float Ic, float k1c, float e0, float e1, float e2,
                                              float e3, double hd, float znew, double atol,
                                              double rtol, double& x) {
  double d4 = 25.0 / 216.0 * (double)k1c + 1408.0 / 2565.0 * (double)e0 +
              2197.0 / 4101.0 * (double)e1 - 1.0 / 5.0 * (double)e2;
  double d5 = 16.0 / 135.0 * (double)k1c + 6656.0 / 12825.0 * (double)e0 +
              28561.0 / 56430.0 * (double)e1 - 9.0 / 50.0 * (double)e2 + 2.0 / 55.0 * (double)e3;
  d4 *= hd;
  d5 *= hd;
  x = 16.0;
  if (d4 != d5) {
    const double err = fabs(d5 - d4);
    const double srt = fabs((double)Ic / (double)znew * rtol);
    const double ot = fmax(atol, srt);
    x = ot * hd / (2.0 * err);
  }
  return (float)((double)Ic + d4);
}

// kMulti: V > 1 channels from the table. kOwnVal (V = 1 without a channel
// table): the slots carry the particles' own q, as the render kernel's walk
// does, so no value is looked up by index afterwards.
template <bool kMulti, int kMinBlocks, bool kOwnVal, bool kAxis = false>
__global__ void __launch_bounds__(kBThreads, kMinBlocks)
batched_kernel(BatchK a, GridView g, const char4* __restrict__ spiral_g,
               uint32_t* __restrict__ flags, unsigned long long* __restrict__ stats) {
  __shared__ char4 spiral[1000];
  // slot arrays of the walks; for V > 1 also the hand-over to the warp:
  // weights in the distance rows, indices in the value rows, sums in slot_ws
  __shared__ SlotMem slot_mem;
  __shared__ float slot_ws[kMulti ? 4 : 1][kBThreads];
  // the block's work counters (steps, accepted, -, cells, candidates, max
  // steps of a ray, rays at the step limit), added per tile: kept out of the
  // registers the walk needs
  __shared__ unsigned long long blk_stats[7];
  if (threadIdx.x < 7) blk_stats[threadIdx.x] = 0ull;
  load_spiral(spiral, spiral_g);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tw = a.tile_w, th = a.tile_w > 0 ? 32 / a.tile_w : 1;
  float* wstate = kMulti ? a.state + ((size_t)blockIdx.x * kBThreads + (size_t)warp * 32) *
                                         4 * (size_t)a.V
                         : nullptr;
  for (;;) {
    unsigned long long item = 0;
    if (lane == 0) item = atomicAdd(a.queue, 1ull);
    item = __shfl_sync(kFull, item, 0);
    if (item >= a.n_items) break;
    if (a.order) item = a.order[item];
    const JobDev& J = a.jobs[find_job(a.jobs, a.n_jobs, item)];
    const uint64_t t = item - J.item_begin;
    int ix, iy;
    bool inside;
    if (tw > 0) {  // compact tile of tw x th pixels
      const int tx = (int)(t % (uint64_t)J.tiles_x), ty = (int)(t / (uint64_t)J.tiles_x);
      ix = tx * tw + lane % tw;
      iy = ty * th + lane / tw;
      inside = ix < J.nx && iy < J.ny;
    } else {       // strided: pixels t, t + T, t + 2T, ... (T = items of the job)
      const uint64_t pix = t + (uint64_t)lane * (uint64_t)J.tiles_x;
      inside = pix < (uint64_t)J.nx * (uint64_t)J.ny;
      ix = inside ? (int)(pix % (uint64_t)J.nx) : J.nx;
      iy = inside ? (int)(pix / (uint64_t)J.nx) : J.ny;
    }
    bool masked = true;
    float o[3] = {0.0f, 0.0f, 0.0f}, len = 0.0f;
    if (inside) ray_span(J, ix, iy, masked, o, len);
    const float lx = J.look[0], ly = J.look[1], lz = J.look[2];
    bool run = inside && !masked;
    float z = 0.0f, h = 1.0f, I = 0.0f, k1 = 0.0f;
    float pts[4];
    rkf_points(0.0f, 1.0f, pts);
    uint32_t rs = 0, ra = 0;
    WalkStats ws;
    if (kMulti) {
      for (int i = lane; i < 32 * 4 * a.V; i += 32) wstate[i] = 0.0f;
      __syncwarp();
    }
    // z windows: the rays of the warp step up to the window's end, then the
    // warp moves on together, so its 32 rays query one slab of the grid at a
    // time. This orders the work only; each ray's steps are unchanged.
    float wend = a.window > 0.0f ? a.window : FLT_MAX;
    while (__any_sync(kFull, run && z < len)) {
      if (!__any_sync(kFull, run && z < len && z < wend)) {
        wend += a.window;
        continue;
      }
      if (run && z < len && z < wend && (int64_t)rs >= a.max_steps) {
        atomicAdd(&blk_stats[6], 1ull);
        run = false;
      }
      const bool go = run && z < len && z < wend;
      if (go) {
        Step4 s;
        s4_bind(s, slot_mem);
        nn8_walk_step4<!kOwnVal, kAxis>(g, spiral, o[0], o[1], o[2], lx, ly, lz, pts, s, ws);
        if (!kMulti) {
          float e[4];
          if (kOwnVal) {
            e[0] = s4_finalize<0>(s);
            e[1] = s4_finalize<1>(s);
            e[2] = s4_finalize<2>(s);
            e[3] = s4_finalize<3>(s);
          } else {
            e[0] = value1<0>(s, a.chan, g.parts);
            e[1] = value1<1>(s, a.chan, g.parts);
            e[2] = value1<2>(s, a.chan, g.parts);
            e[3] = value1<3>(s, a.chan, g.parts);
          }
          const float zb = z;
          rkf_advance_fp64(I, z, h, k1, a.atol, a.rtol, len, e, kEps, kHmin, kHmax, pts);
          ++rs;
          if (z != zb) ++ra;
        } else {
          slots_to_weights<0>(s, slot_ws[0][threadIdx.x]);
          slots_to_weights<1>(s, slot_ws[1][threadIdx.x]);
          slots_to_weights<2>(s, slot_ws[2][threadIdx.x]);
          slots_to_weights<3>(s, slot_ws[3][threadIdx.x]);
        }
      }
      if (kMulti) {
        __syncwarp();
        unsigned gom = __ballot_sync(kFull, go);
        bool my_acc = false;
        double my_nh = 0.0;
        while (gom) {
          const int r = __ffs(gom) - 1;
          gom &= gom - 1;
          const float zr = __shfl_sync(kFull, z, r), hr = __shfl_sync(kFull, h, r);
          const int tr = warp * 32 + r;  // ray r's thread: its slot columns
          float* Is = wstate + (size_t)r * 4 * a.V;
          float* Ks = Is + a.V;
          const double hd = (double)hr;
          const float znew = zr + hr;
          double xl = __longlong_as_double(0x7ff0000000000000ll);  // +inf
          bool x0nan = false;
          // candidate values (I + delta4, k5) go to the ray's scratch half
          // and are committed once the warp knows the step is accepted
          float* Es = Ks + a.V;
          float* E2s = Es + a.V;
          if ((a.V & 3) == 0) {
            // rows of V = 4G floats: lane handles float4 groups lane, lane+32, ...
            // (channels 4g..4g+3), one 16-byte load per neighbour and group
            const int G = a.V >> 2;
            const float4* __restrict__ chan4 = reinterpret_cast<const float4*>(a.chan);
#pragma unroll 1
            for (int gi = lane; gi < G; gi += 32) {
              float ev[4][4];
#pragma unroll
              for (int p = 0; p < 4; ++p) {
                float dot[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                  const int id = __float_as_int(slot_mem.v[p * 8 + q][tr]);
                  const float4 v = id >= 0 ? __ldg(&chan4[(size_t)id * G + gi])
                                           : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                  const float wq = slot_mem.d[p * 8 + q][tr];
                  dot[0] = __fmaf_rn(wq, v.x, dot[0]);
                  dot[1] = __fmaf_rn(wq, v.y, dot[1]);
                  dot[2] = __fmaf_rn(wq, v.z, dot[2]);
                  dot[3] = __fmaf_rn(wq, v.w, dot[3]);
                }
                const float wsum = slot_ws[p][tr];
#pragma unroll
                for (int k = 0; k < 4; ++k)
                  ev[p][k] = (wsum != 0.0f && dot[k] != 0.0f) ? dot[k] / wsum : 0.0f;
              }
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const int c = 4 * gi + k;
                double x;
                Es[c] = channel_step(Is[c], Ks[c], ev[0][k], ev[1][k], ev[2][k], ev[3][k], hd,
                                     znew, a.atol, a.rtol, x);
                E2s[c] = ev[2][k];
                if (c == 0 && isnan(x)) x0nan = true;
                xl = fmin(xl, x);
              }
            }
          } else {
#pragma unroll 1
            for (int c = lane; c < a.V; c += 32) {
              float ev[4];
#pragma unroll
              for (int p = 0; p < 4; ++p) {
                float dot = 0.0f;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                  const int id = __float_as_int(slot_mem.v[p * 8 + q][tr]);
                  const float v = id >= 0 ? __ldg(&a.chan[(size_t)id * a.V + c]) : 0.0f;
                  dot = __fmaf_rn(slot_mem.d[p * 8 + q][tr], v, dot);
                }
                const float wsum = slot_ws[p][tr];
                ev[p] = (wsum != 0.0f && dot != 0.0f) ? dot / wsum : 0.0f;
              }
              double x;
              Es[c] = channel_step(Is[c], Ks[c], ev[0], ev[1], ev[2], ev[3], hd, znew, a.atol,
                                   a.rtol, x);
              E2s[c] = ev[2];
              if (c == 0 && isnan(x)) x0nan = true;
              xl = fmin(xl, x);
            }
          }
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) xl = fmin(xl, __shfl_xor_sync(kFull, xl, off));
          // The host-side definition takes x_0 and then every smaller x_c:
          // a NaN x_0 gives NaN, any other NaN is passed over.
          const bool n0 = __shfl_sync(kFull, x0nan, 0);
          const double xmin = n0 ? __longlong_as_double(0x7ff8000000000000ll) : xl;
          double sc = sqrt(sqrt(xmin));
          double nh = sc * hd;
          if (nh < (double)kHmin) nh = (double)kHmin;
          else if (nh > (double)kHmax) nh = (double)kHmax;
          sc = nh / hd;
          const bool accept = !(sc < 0.95);
          if (accept) {
#pragma unroll 1
            for (int c = lane; c < a.V; c += 32) {
              Is[c] = Es[c];
              Ks[c] = E2s[c];
            }
          }
          if (lane == r) {
            my_acc = accept;
            my_nh = nh;
          }
        }
        __syncwarp();
        if (go) {
          const float znew = z + h;
          if (my_acc) z = znew;
          h = (float)my_nh;
          if (z + h >= len) h = len - z + kEps;
          rkf_points(z, h, pts);
          ++rs;
          if (my_acc) ++ra;
        }
      }
    }
    // outputs of the tile
    if (!kMulti) {
      if (inside)
        a.out[J.out_offset + (size_t)iy * J.nx + ix] = masked ? 0.0f : I * J.scale;
    } else {
      __syncwarp();
      const size_t plane = (size_t)J.nx * (size_t)J.ny;
      for (int r = 0; r < 32; ++r) {
        const int ixr = __shfl_sync(kFull, ix, r), iyr = __shfl_sync(kFull, iy, r);
        const bool in_r = __shfl_sync(kFull, inside, r), m_r = __shfl_sync(kFull, masked, r);
        if (!in_r) continue;
        const float* Is = wstate + (size_t)r * 4 * a.V;
        for (int c = lane; c < a.V; c += 32)
          a.out[J.out_offset + (size_t)c * plane + (size_t)iyr * J.nx + ixr] =
              m_r ? 0.0f : Is[c] * J.scale;
      }
      __syncwarp();
    }
    atomicAdd(&blk_stats[0], (unsigned long long)rs);
    atomicAdd(&blk_stats[1], (unsigned long long)ra);
    atomicAdd(&blk_stats[3], (unsigned long long)ws.cells);
    atomicAdd(&blk_stats[4], (unsigned long long)ws.cands);
    atomicMax(&blk_stats[5], (unsigned long long)rs);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (blk_stats[6]) atomicOr(flags, FLAG_STEP_LIMIT);
    atomicAdd(&stats[0], blk_stats[0]);
    atomicAdd(&stats[1], blk_stats[1]);
    atomicAdd(&stats[2], 4ull * blk_stats[0]);
    atomicAdd(&stats[3], blk_stats[3]);
    atomicAdd(&stats[4], blk_stats[4]);
    atomicMax(&stats[5], blk_stats[5]);
    atomicAdd(&stats[6], blk_stats[6]);
  }
}

__global__ void channels_sort_kernel(const float* __restrict__ in,
                                     const uint32_t* __restrict__ s2u, uint64_t n, int V,
                                     float* __restrict__ out) {
  const uint64_t total = n * (uint64_t)V;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = i / (uint64_t)V, c = i - p * (uint64_t)V;
    out[i] = in[(uint64_t)s2u[p] * V + c];
  }
}

// Per-tile cost estimate of one job: every particle in front of the camera
// (and within its depth when the job has no chord) adds its cell's
// occupancy to the tile its pixel column falls in, so tiles whose rays cross
// many particles in dense cells -- the long, expensive rays -- score high.
__global__ void tile_cost_kernel(const float4* __restrict__ parts,
                                 const uint32_t* __restrict__ keys,
                                 const int2* __restrict__ cells, uint64_t n, JobDev J, int tw,
                                 int th, float* __restrict__ cost) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float4 p = parts[i];
    const float dx = p.x - J.minp[0], dy = p.y - J.minp[1], dz = p.z - J.minp[2];
    const float u = (dx * J.b0[0] + dy * J.b0[1] + dz * J.b0[2]) / J.ps;
    const float v = (dx * J.b1[0] + dy * J.b1[1] + dz * J.b1[2]) / J.ps;
    const float t = dx * J.look[0] + dy * J.look[1] + dz * J.look[2];
    if (!(u >= 0.0f) || !(v >= 0.0f) || !(u < (float)J.nx) || !(v < (float)J.ny)) continue;
    if (!(t >= 0.0f) || (!(J.radius > 0.0) && !(t <= (float)J.z_range))) continue;
    const int ix = (int)u, iy = (int)v;
    const int2 be = cells[keys[i]];
    const uint64_t item = tw > 0 ? (uint64_t)(iy / th) * J.tiles_x + (uint64_t)(ix / tw)
                                 : ((uint64_t)iy * J.nx + ix) % (uint64_t)J.tiles_x;
    atomicAdd(&cost[J.item_begin + item], (float)(be.y - be.x));
  }
}

template <bool kMulti, int kMinBlocks>
int persistent_blocks(const Context& c) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
                                                batched_kernel<kMulti, kMinBlocks, false>,
                                                kBThreads, 0);
  if (sms <= 0) sms = 148;
  if (per_sm <= 0) per_sm = 1;
  return sms * per_sm;
}

template <bool kMulti, int kMinBlocks>
cudaError_t launch_variant(Context& c, const BatchK& k, const GridView& g, int blocks) {
  unsigned long long* stats = reinterpret_cast<unsigned long long*>(c.flags.as<char>() + 64);
  if constexpr (!kMulti) {
    if (!k.chan) {
      if (k.axis_z)
        batched_kernel<false, kMinBlocks, true, true><<<blocks, kBThreads, 0, c.stream>>>(
            k, g, c.spiral.as<char4>(), c.flags.as<uint32_t>(), stats);
      else
        batched_kernel<false, kMinBlocks, true><<<blocks, kBThreads, 0, c.stream>>>(
            k, g, c.spiral.as<char4>(), c.flags.as<uint32_t>(), stats);
      return cudaGetLastError();
    }
  }
  batched_kernel<kMulti, kMinBlocks, false><<<blocks, kBThreads, 0, c.stream>>>(
      k, g, c.spiral.as<char4>(), c.flags.as<uint32_t>(), stats);
  return cudaGetLastError();
}

int variant_blocks(const Context& c, bool multi, int occ) {
  if (multi)
    return occ == 5   ? persistent_blocks<true, 5>(c)
           : occ == 4 ? persistent_blocks<true, 4>(c)
           : occ == 3 ? persistent_blocks<true, 3>(c)
                      : persistent_blocks<true, 1>(c);
  return occ == 5   ? persistent_blocks<false, 5>(c)
         : occ == 4 ? persistent_blocks<false, 4>(c)
         : occ == 3 ? persistent_blocks<false, 3>(c)
                    : persistent_blocks<false, 1>(c);
}

cudaError_t enqueue(Context& c, const BatchK& k, const GridView& g, int occ, int blocks) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(c.flags.p, 0, kFlagsBytes, c.stream))) return e;
  if ((e = cudaMemsetAsync(c.queue.p, 0, 8, c.stream))) return e;
  if (k.V == 1)
    return occ == 5   ? launch_variant<false, 5>(c, k, g, blocks)
           : occ == 4 ? launch_variant<false, 4>(c, k, g, blocks)
           : occ == 3 ? launch_variant<false, 3>(c, k, g, blocks)
                      : launch_variant<false, 1>(c, k, g, blocks);
  return occ == 5   ? launch_variant<true, 5>(c, k, g, blocks)
         : occ == 4 ? launch_variant<true, 4>(c, k, g, blocks)
         : occ == 3 ? launch_variant<true, 3>(c, k, g, blocks)
                    : launch_variant<true, 1>(c, k, g, blocks);
}

}  // namespace

cudaError_t channels_sort_launch(Context& c, const float* in, uint64_t n, int V, float* out) {
  const uint64_t total = n * (uint64_t)V;
  const unsigned blocks = (unsigned)std::min<uint64_t>((total + 255) / 256, 148ull * 16);
  ++c.launches;
  channels_sort_kernel<<<blocks > 0 ? blocks : 1, 256, 0, c.stream>>>(in, c.s2u.as<uint32_t>(),
                                                                       n, V, out);
  return cudaGetLastError();
}

cudaError_t batched_order(Context& c, BatchArgs& a, const std::vector<JobDev>& jobs) {
  cudaError_t e;
  const uint64_t m = a.n_items;
  if ((e = c.item_cost.ensure(m * 4)) || (e = c.item_order.ensure(m * 4))) return e;
  if ((e = cudaMemsetAsync(c.item_cost.p, 0, m * 4, c.stream))) return e;
  const int tw = a.tile_w, th = a.tile_w > 0 ? 32 / a.tile_w : 1;
  const uint64_t n = c.n_particles;
  const unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 8);
  for (const JobDev& j : jobs) {
    tile_cost_kernel<<<blocks > 0 ? blocks : 1, 256, 0, c.stream>>>(
        c.parts.as<float4>(), c.sorted_keys, c.cells.as<int2>(), n, j, tw, th,
        c.item_cost.as<float>());
    ++c.launches;
  }
  if ((e = cudaGetLastError())) return e;
  std::vector<float> cost(m);
  if ((e = cudaMemcpyAsync(cost.data(), c.item_cost.p, m * 4, cudaMemcpyDeviceToHost,
                           c.stream)) ||
      (e = cudaStreamSynchronize(c.stream)))
    return e;
  std::vector<uint32_t> order(m);
  for (uint64_t i = 0; i < m; ++i) order[i] = (uint32_t)i;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t x, uint32_t y) { return cost[x] > cost[y]; });
  if ((e = cudaMemcpyAsync(c.item_order.p, order.data(), m * 4, cudaMemcpyHostToDevice,
                           c.stream)) ||
      (e = cudaStreamSynchronize(c.stream)))
    return e;
  a.order = c.item_order.as<uint32_t>();
  return cudaSuccess;
}

// The launch sequence (reset of the flags and the queue, persistent kernel)
// runs as a CUDA graph, instantiated once per set of launch parameters and
// replayed while they stay the same (repeated frames of one job set).
cudaError_t batched_launch(Context& c, const BatchArgs& a, float* kernel_ms) {
  cudaError_t e;
  if ((e = c.flags.ensure(kFlagsBytes))) return e;
  if ((e = c.queue.ensure(256))) return e;
  BatchK k;
  std::memset(&k, 0, sizeof(k));  // the bytes are the graph's key
  k.jobs = a.jobs;
  k.n_jobs = a.n_jobs;
  k.n_items = a.n_items;
  k.V = a.V;
  k.chan = a.chan;
  k.out = a.out;
  k.atol = a.atol;
  k.rtol = a.rtol;
  k.max_steps = c.max_steps;
  k.tile_w = a.tile_w;
  k.window = a.window;
  k.order = a.order;
  k.queue = c.queue.as<unsigned long long>();
  k.axis_z = a.axis_z ? 1 : 0;
  const int occ = a.occupancy;
  const int blocks = variant_blocks(c, a.V > 1, occ);
  if (a.V > 1) {
    if ((e = c.chan_state.ensure((size_t)blocks * kBThreads * 4 * (size_t)k.V * 4))) return e;
    k.state = c.chan_state.as<float>();
  }
  const GridView g = make_grid_view(c);
  if (!c.ev0) {
    if ((e = cudaEventCreate(&c.ev0)) || (e = cudaEventCreate(&c.ev1))) return e;
  }
  std::string key(reinterpret_cast<const char*>(&k), sizeof(k));
  key.append(reinterpret_cast<const char*>(&g), sizeof(g));
  key.append(reinterpret_cast<const char*>(&occ), sizeof(occ));
  key.append(reinterpret_cast<const char*>(&blocks), sizeof(blocks));
  if (!c.batch_exec || key != c.batch_key) {
    if (c.batch_exec) {
      cudaGraphExecDestroy(c.batch_exec);
      c.batch_exec = nullptr;
    }
    c.batch_key.clear();
    cudaGraph_t graph = nullptr;
    if ((e = cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal))) return e;
    const cudaError_t el = enqueue(c, k, g, occ, blocks);
    e = cudaStreamEndCapture(c.stream, &graph);
    if (el) {
      if (graph) cudaGraphDestroy(graph);
      return el;
    }
    if (e) return e;
    e = cudaGraphInstantiate(&c.batch_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e) {
      c.batch_exec = nullptr;
      return e;
    }
    c.batch_key = key;
  }
  cudaEventRecord(c.ev0, c.stream);
  ++c.launches;
  if ((e = cudaGraphLaunch(c.batch_exec, c.stream))) return e;
  cudaEventRecord(c.ev1, c.stream);
  if (kernel_ms) {
    if ((e = cudaEventSynchronize(c.ev1))) return e;
    cudaEventElapsedTime(kernel_ms, c.ev0, c.ev1);
  }
  return cudaSuccess;
}

}  // namespace ilc
