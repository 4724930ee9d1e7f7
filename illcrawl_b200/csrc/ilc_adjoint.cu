// ilc_adjoint.cu -- gradient of an image loss with respect to per-cell log
// density and log temperature, through the nn8 reconstruction and the RKF
// line-of-sight integral, with the neighbour choice fixed and the step
// sequence frozen from the forward pass (checkpointed per ray, or recomputed).
//
// With fixed neighbours and frozen steps a pixel is linear in the per-cell
// values q: every accepted step adds h (25/216 k1 + 1408/2565 e0 +
// 2197/4101 e1 - 1/5 e2) (integration.cl:63-67,118), k1 being the previous
// accepted step's e2 (0 before the first), and every e is the nn8 finalize
// sum(w v)/sum(w) (volumetric_nn8_reconstruction.cl:212-270), so
// d e / d v_p = w_p / sum(w). The adjoint replays each ray's steps, evaluates
// e0, e1, e2 (e3 only enters the error estimate) and scatters
// dL/dI * coefficient * w_p / sum(w) into dL/dq_p. The per-cell chain rule
// then multiplies by dq/dln rho and dq/dln T of the adaptive band flux
// (ilc_adjoint_cell.cuh).
#include "ilc_adjoint_cell.cuh"
#include "ilc_device.cuh"
#include "ilc_internal.h"
#include "ilc_quantity.cuh"
#include "ilc_walk4.cuh"

namespace ilc {

namespace {

// q (bit-identical to xray_flux_kernel), dq/dlnT, dq/dlnrho for one cell.
template <int kWhich>
__device__ void band_flux_tangent(const float* t, const GauntView& G, float Emin, float Emax,
                                  float reltol, float T, float xe, float rho, float dL, float* q,
                                  double* dq) {
  const GauntViewD GD{G.w, G.h, G.x0, G.y0, G.dx, G.dy};
  const float atol = reltol, rtol = 1.0f, eps = 0.0f, hmin = 1.e-3f, hmax = 100.f;
  float I = 0.0f, z = Emin, h = (Emax - Emin) * reltol;
  double dI = 0, dz = 0, dh = 0, dk1, dkE;
  const float end = Emax;
  float k1 = brems(t, G, z, 1.0f, T, xe, rho, dL);
  brems_tangent(t, GD, z, T, xe, rho, dL, kWhich, &dk1, &dkE, (double)k1);
  float p[4];
  double dp[4] = {0, 0, 0, 0};
  rkf_points(z, h, p);
  const double c[4] = {3. / 8., 12. / 13., 1.0, 0.5};
  int guard = 0;
  while (z < end && guard < 100000) {
    float e[4];
    double de[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      e[j] = brems(t, G, p[j], 1.0f, T, xe, rho, dL);
      double pl, pe;
      brems_tangent(t, GD, p[j], T, xe, rho, dL, kWhich, &pl, &pe, (double)e[j]);
      de[j] = pl + pe * dp[j];
    }
    const float b4 = 25.f / 216.f * k1 + 1408.f / 2565.f * e[0] + 2197.f / 4101.f * e[1] -
                     1.f / 5.f * e[2];
    const float b5 = 16.f / 135.f * k1 + 6656.f / 12825.f * e[0] + 28561.f / 56430.f * e[1] -
                     9.f / 50.f * e[2] + 2.f / 55.f * e[3];
    const double db4 = 25. / 216. * dk1 + 1408. / 2565. * de[0] + 2197. / 4101. * de[1] -
                       1. / 5. * de[2];
    const double db5 = 16. / 135. * dk1 + 6656. / 12825. * de[0] + 28561. / 56430. * de[1] -
                       9. / 50. * de[2] + 2. / 55. * de[3];
    const double dd4 = db4 * (double)h + (double)b4 * dh;
    const double dd5 = db5 * (double)h + (double)b5 * dh;
    const float d4 = b4 * h, d5 = b5 * h;
    const float est4 = I + d4;
    const double dest4 = dI + dd4;
    const float old = z;
    const double dold = dz;
    z += h;
    dz += dh;
    float s = 2.0f;
    double ds = 0;
    if (d4 != d5) {
      const float err = fabsf(d5 - d4);
      const double derr = sgnd((double)d5 - (double)d4) * (dd5 - dd4);
      const float ratio = I / z * rtol;
      const float srt = fabsf(ratio);
      const double dsrt = sgnd((double)ratio) * (double)rtol *
                          (dI / (double)z - (double)I * dz / ((double)z * (double)z));
      const float ot = fmaxf(atol, srt);
      const double dot_ = srt > atol ? dsrt : 0.0;
      s = sqrtf(sqrtf(ot * h / (2.0f * err)));
      ds = (double)s * 0.25 * (dot_ / (double)ot + dh / (double)h - derr / (double)err);
    }
    float nh = s * h;
    double dnh = ds * (double)h + (double)s * dh;
    if (nh < hmin) { nh = hmin; dnh = 0; }
    else if (nh > hmax) { nh = hmax; dnh = 0; }
    s = nh / h;
    if (s < 0.95f) {
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
    rkf_points(z, h, p);
#pragma unroll
    for (int j = 0; j < 4; ++j) dp[j] = dz + c[j] * dh;
    ++guard;
  }
  *q = I;
  *dq = dI;
}

__global__ void __launch_bounds__(256)
xray_flux_grad_kernel(const float* __restrict__ table, GauntView G, const float* __restrict__ rho,
                      const float* __restrict__ u, const float* __restrict__ xe, uint64_t n,
                      float z, float dL, float emin, float emax, int num_samples,
                      float* __restrict__ q_out, int q_stride, float* __restrict__ dq_lnT,
                      float* __restrict__ dq_lnrho) {
  __shared__ float t[81 * 146];
  for (int i = threadIdx.x; i < G.w * G.h; i += blockDim.x) t[i] = table[i];
  __syncthreads();
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const float T = temperature(u[i], xe[i]);
    const float e0 = (1.f + z) * emin, e1 = (1.f + z) * emax, rt = 1.f / (float)num_samples;
    float q;
    double dT, dR;
    band_flux_tangent<0>(t, G, e0, e1, rt, T, xe[i], rho[i], dL, &q, &dT);
    band_flux_tangent<1>(t, G, e0, e1, rt, T, xe[i], rho[i], dL, &q, &dR);
    q_out[i * q_stride] = q;
    dq_lnT[i] = (float)dT;
    dq_lnrho[i] = (float)dR;
  }
}

// L = sum over pixels of (log I - log I_target)^2 on the scaled image; the
// seed per ray is dL/dI_raw = 2 (log I - log I_target) / I_raw. Pixels with a
// non-positive value or target are left out of the loss (log undefined).
__global__ void loss_seed_kernel(const float* __restrict__ img, const float* __restrict__ target,
                                 int64_t npix, float scale, float* __restrict__ seed,
                                 double* __restrict__ loss) {
  double part = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npix;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float I = img[i], tg = target[i];
    float s = 0.0f;
    if (I > 0.0f && tg > 0.0f && isfinite(I) && isfinite(tg)) {
      const double r = log((double)I) - log((double)tg);
      part += r * r;
      const double raw = (double)I / (double)scale;
      s = (float)(2.0 * r / raw);
    }
    seed[i] = s;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, part);
}

// d e / d v_p = w_p / sum(w) for the 8 slots of one evaluation (0 where the
// finalize has no weight): scatter4 adds c * that to grad at the sorted
// particle index of point J's slots. The accumulator is double: a cell's
// gradient sums contributions of both signs from many rays, and fp32
// accumulation loses digits to cancellation.
template <int J>
__device__ __forceinline__ void scatter4(const Step4& s, float c, double* __restrict__ grad) {
  if (c == 0.0f) return;
  float w[8];
  float ws = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    w[t] = weight3d(s4_d(s, J, t));
    ws = ws + w[t];
  }
  if (!(ws > 0.0f) || !isfinite(ws)) return;
  const double f = (double)c / (double)ws;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int id = __float_as_int(s4_v(s, J, t));
    if (id >= 0 && w[t] != 0.0f) atomicAdd(&grad[id], f * (double)w[t]);
  }
}

// Point 2's slots of the previous step (it is the next step's k1).
struct PrevSlots {
  float d[8];
  int id[8];
};

__device__ __forceinline__ void scatter_prev(const PrevSlots& s, float c,
                                             double* __restrict__ grad) {
  if (c == 0.0f) return;
  float w[8];
  float ws = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    w[t] = weight3d(s.d[t]);
    ws = ws + w[t];
  }
  if (!(ws > 0.0f) || !isfinite(ws)) return;
  const double f = (double)c / (double)ws;
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (s.id[t] >= 0 && w[t] != 0.0f) atomicAdd(&grad[s.id[t]], f * (double)w[t]);
}

__device__ __forceinline__ void keep_prev(const Step4& s, PrevSlots& p) {
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    p.d[t] = s4_d(s, 2, t);
    p.id[t] = __float_as_int(s4_v(s, 2, t));
  }
}

// nn8 value of point J (finalize order) with the values read by index.
template <int J>
__device__ __forceinline__ float value_by_id(const Step4& s, const float4* __restrict__ parts) {
  float w[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) w[t] = weight3d(s4_d(s, J, t));
  float ws = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) ws = ws + w[t];
  float dot = 0.0f;
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int id = __float_as_int(s4_v(s, J, t));
    dot = __fmaf_rn(w[t], id >= 0 ? __ldg(&parts[id].w) : 0.0f, dot);
  }
  return (ws != 0.0f && dot != 0.0f) ? dot / ws : 0.0f;
}

struct AdjK {
  CamView cam;
  float z0, z_end;
  double atol, rtol;
  int controller;
  int64_t max_steps;
  int mode;                        // ILC_ADJOINT_CHECKPOINT / _RECOMPUTE
  const float* __restrict__ rec_h;  // checkpoint: accepted step sizes, ray-major
  const int32_t* __restrict__ rec_n;
  int64_t rec_cap;
  const float* __restrict__ seed;  // dL/dI_raw per pixel (whole image)
  double* __restrict__ grad;       // dL/dq per sorted particle
  int row0, row_end;               // pixel rows of this launch; rec_* indexed from row0
  unsigned* queue;                 // persistent launch: tile counter (nullptr: block per tile)
  unsigned ntiles, tiles_x;
};

// The rays of one 16 x 8 tile (one per thread; no block synchronisation).
__device__ __forceinline__ void adjoint_tile(const AdjK& a, const GridView& g,
                                             const char4* __restrict__ spiral, SlotMem& slot_mem,
                                             uint32_t* __restrict__ flags,
                                             unsigned long long* __restrict__ stats, int bx,
                                             int by) {
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  const int ix = bx * 16 + (warp & 1) * 8 + (lane & 7);
  const int iy = a.row0 + by * 8 + (warp >> 1) * 4 + (lane >> 3);
  if (ix >= a.cam.nx || iy >= a.row_end) return;
  const int64_t ray = (int64_t)(iy - a.row0) * a.cam.nx + ix;  // in the launch's rows
  const float gi = a.seed[(int64_t)iy * a.cam.nx + ix];
  if (gi == 0.0f) return;
  float px, py, pz;
  pixel_corner(a.cam, ix, iy, px, py, pz);
  const float lx = a.cam.look0, ly = a.cam.look1, lz = a.cam.look2;
  WalkStats ws;
  unsigned long long steps = 0;
  PrevSlots prev;
  bool have_prev = false;
  float z = a.z0;
  if (a.mode == ILC_ADJOINT_CHECKPOINT) {
    const int32_t n = a.rec_n[ray];
    const float* hs = a.rec_h + ray * a.rec_cap;
    for (int32_t i = 0; i < n; ++i) {
      const float h = hs[i];
      float p[4];
      rkf_points(z, h, p);
      Step4 s;
      s4_bind(s, slot_mem);
      nn8_walk_step4<true>(g, spiral, px, py, pz, lx, ly, lz, p, s, ws);
      scatter4<0>(s, gi * (h * 1408.f / 2565.f), a.grad);
      scatter4<1>(s, gi * (h * 2197.f / 4101.f), a.grad);
      scatter4<2>(s, gi * (-h / 5.f), a.grad);
      if (have_prev) scatter_prev(prev, gi * (h * 25.f / 216.f), a.grad);
      keep_prev(s, prev);
      have_prev = true;
      z += h;
      ++steps;
    }
  } else {
    // Recompute: run the forward controller again; accepted steps scatter.
    float I = 0.0f, h = 1.0f, k1 = 0.0f;
    float pts[4];
    rkf_points(z, h, pts);
    const float fa = (float)a.atol, fr = (float)a.rtol;
    while (z < a.z_end) {
      if ((int64_t)steps >= a.max_steps) { atomicOr(flags, FLAG_STEP_LIMIT); break; }
      Step4 s;
      s4_bind(s, slot_mem);
      nn8_walk_step4<true>(g, spiral, px, py, pz, lx, ly, lz, pts, s, ws);
      const float e[4] = {value_by_id<0>(s, g.parts), value_by_id<1>(s, g.parts),
                          value_by_id<2>(s, g.parts), value_by_id<3>(s, g.parts)};
      const float zb = z, hb = h;
      if (a.controller == ILC_CONTROLLER_REF32)
        rkf_advance_ref32(I, z, h, k1, fa, fr, a.z_end, e, kEps, kHmin, kHmax, pts);
      else
        rkf_advance_fp64(I, z, h, k1, a.atol, a.rtol, a.z_end, e, kEps, kHmin, kHmax, pts);
      ++steps;
      if (z != zb) {
        scatter4<0>(s, gi * (hb * 1408.f / 2565.f), a.grad);
        scatter4<1>(s, gi * (hb * 2197.f / 4101.f), a.grad);
        scatter4<2>(s, gi * (-hb / 5.f), a.grad);
        if (have_prev) scatter_prev(prev, gi * (hb * 25.f / 216.f), a.grad);
        keep_prev(s, prev);
        have_prev = true;
      }
    }
  }
  unsigned long long c = ws.cells, k = ws.cands;
  atomicAdd(&stats[0], steps);
  atomicAdd(&stats[3], c);
  atomicAdd(&stats[4], k);
}

// Persistent: the resident blocks take tiles from a queue (one block per tile
// without one), as the render kernel does.
__global__ void __launch_bounds__(128)
adjoint_kernel(AdjK a, GridView g, const char4* __restrict__ spiral_g,
               uint32_t* __restrict__ flags, unsigned long long* __restrict__ stats) {
  __shared__ char4 spiral[1000];
  __shared__ SlotMem slot_mem;
  __shared__ unsigned next_tile;
  load_spiral(spiral, spiral_g);
  if (!a.queue) {
    adjoint_tile(a, g, spiral, slot_mem, flags, stats, blockIdx.x, blockIdx.y);
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) next_tile = atomicAdd(a.queue, 1u);
    __syncthreads();
    const unsigned t = next_tile;
    __syncthreads();
    if (t >= a.ntiles) break;
    adjoint_tile(a, g, spiral, slot_mem, flags, stats, (int)(t % a.tiles_x),
                 (int)(t / a.tiles_x));
  }
}

// dL/dln rho and dL/dln T in the original particle order.
__global__ void cell_grad_kernel(const double* __restrict__ grad_sorted,
                                 const uint32_t* __restrict__ s2u, uint64_t n,
                                 const float* __restrict__ dq_lnrho,
                                 const float* __restrict__ dq_lnT, float* __restrict__ g_lnrho,
                                 float* __restrict__ g_lnT) {
  const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t o = s2u[i];
  const double gq = grad_sorted[i];
  g_lnrho[o] = (float)(gq * (double)dq_lnrho[o]);
  g_lnT[o] = (float)(gq * (double)dq_lnT[o]);
}

}  // namespace

GridView make_grid_view(const Context& c);

cudaError_t adjoint_cell_launch(Context& c, const float* rho, const float* u, const float* xe,
                                uint64_t n, float z, float dL, float emin, float emax,
                                int num_samples, float* q_out, int q_stride, float* dq_lnT,
                                float* dq_lnrho) {
  GauntView G{c.gw, c.gh, c.gx0, c.gy0, c.gdx, c.gdy};
  const uint64_t want = (n + 255) / 256;
  const unsigned blocks = (unsigned)(want < 148 * 16 ? want : 148 * 16);
  ++c.launches;
  xray_flux_grad_kernel<<<blocks, 256, 0, c.stream>>>(c.gaunt.as<float>(), G, rho, u, xe, n, z,
                                                       dL, emin, emax, num_samples, q_out,
                                                       q_stride, dq_lnT, dq_lnrho);
  return cudaGetLastError();
}

cudaError_t adjoint_seed_launch(Context& c, const float* img, const float* target, int64_t npix,
                                float scale, float* seed, double* loss, bool reset_loss) {
  if (reset_loss) {
    cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(double), c.stream);
    if (e) return e;
  }
  ++c.launches;
  loss_seed_kernel<<<148 * 4, 256, 0, c.stream>>>(img, target, npix, scale, seed, loss);
  return cudaGetLastError();
}

cudaError_t adjoint_ray_launch(Context& c, const RenderArgs& r, int mode, const float* seed,
                               double* grad, float* kernel_ms) {
  cudaError_t e;
  if ((e = c.flags.ensure(kFlagsBytes))) return e;
  if ((e = cudaMemsetAsync(c.flags.p, 0, kFlagsBytes, c.stream))) return e;
  AdjK k;
  k.cam.look0 = r.cam[0]; k.cam.look1 = r.cam[1]; k.cam.look2 = r.cam[2];
  k.cam.b00 = r.cam[3]; k.cam.b01 = r.cam[4]; k.cam.b02 = r.cam[5];
  k.cam.b10 = r.cam[6]; k.cam.b11 = r.cam[7]; k.cam.b12 = r.cam[8];
  k.cam.min0 = r.cam[9]; k.cam.min1 = r.cam[10]; k.cam.min2 = r.cam[11];
  k.cam.ps = r.cam[12];
  k.cam.nx = r.nx; k.cam.ny = r.ny;
  k.z0 = r.z0; k.z_end = r.z_end;
  k.atol = r.atol; k.rtol = r.rtol;
  k.controller = r.controller;
  k.max_steps = c.max_steps;
  k.mode = mode;
  k.rec_h = r.rec_h;
  k.rec_n = r.rec_n;
  k.rec_cap = r.rec_cap;
  k.seed = seed;
  k.grad = grad;
  k.row0 = r.row0;
  k.row_end = r.rows > 0 ? (r.row0 + r.rows < r.ny ? r.row0 + r.rows : r.ny) : r.ny;
  const GridView g = make_grid_view(c);
  dim3 grid((r.nx + 15) / 16, (k.row_end - k.row0 + 7) / 8);
  k.queue = nullptr;
  k.tiles_x = grid.x;
  k.ntiles = grid.x * grid.y;
  {
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device);
    const cudaError_t oe =
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel, 128, 0);
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
  adjoint_kernel<<<grid, 128, 0, c.stream>>>(
      k, g, c.spiral.as<char4>(), c.flags.as<uint32_t>(),
      reinterpret_cast<unsigned long long*>(c.flags.as<char>() + 64));
  if ((e = cudaGetLastError())) return e;
  cudaEventRecord(c.ev1, c.stream);
  if (kernel_ms) {
    if ((e = cudaEventSynchronize(c.ev1))) return e;
    cudaEventElapsedTime(kernel_ms, c.ev0, c.ev1);
  }
  return cudaSuccess;
}

cudaError_t adjoint_chain_launch(Context& c, const double* grad, uint64_t n, const float* dq_lnrho,
                                 const float* dq_lnT, float* g_lnrho, float* g_lnT) {
  ++c.launches;
  cell_grad_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(
      grad, c.s2u.as<uint32_t>(), n, dq_lnrho, dq_lnT, g_lnrho, g_lnT);
  return cudaGetLastError();
}

}  // namespace ilc
