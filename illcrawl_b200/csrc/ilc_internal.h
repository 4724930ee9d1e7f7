// ilc_internal.h -- host-side state shared by the CUDA translation units and the
// C ABI: the context (stream, device buffers, last error) and kernel launchers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ilc.h"

namespace ilc {

// Grow-only device buffer: reallocated only when a call needs more room, so a
// render loop does not allocate per call (the reference reallocates its nn8
// list buffers on every setup_evaluation_points).
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// Host copy of the particle grid parameters (particle_grid.cpp:54-103).
struct GridParams {
  float min[3];
  float cs[3];
  int32_t n[3];
  uint64_t total;
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string error;
  int64_t max_steps = 1 << 20;  // per-ray RKF step cap
  uint64_t checkpoint_budget = 0;  // adjoint: device bytes for step checkpoints (0: a quarter
                                   // of the device's memory)
  float z_window = 0.0f;        // adaptive render: z window of the block schedule (0 = none)
  int32_t render_occupancy = 4; // adaptive render: blocks per SM (0 = register-limited)
  int32_t render_engine = ILC_ENGINE_PERSISTENT;  // FP64 adaptive renders: kernel used
  int32_t query_engine = ILC_QUERY_THREAD;        // ilc_nn8_query: one thread or one warp per query

  // particle grid
  bool has_grid = false;
  uint64_t n_particles = 0;
  GridParams gp{};
  DevBuf parts;      // float4 sorted particles
  DevBuf cells;      // int2 per grid cell
  DevBuf s2u;        // uint32 sorted -> original index
  DevBuf codes;      // uint8 sub-box code per sorted particle (candidate pruning)
  const uint32_t* sorted_keys = nullptr;  // cell key per sorted particle (keys_a or keys_b)
  DevBuf keys_a, keys_b, vals_a, vals_b, hist, tmp_in;  // build scratch

  // Gaunt table
  bool has_gaunt = false;
  DevBuf gaunt;
  int32_t gw = 0, gh = 0;
  float gx0 = 0, gy0 = 0, gdx = 0, gdy = 0;

  // Chandra ARF (1D tabulated function)
  bool has_arf = false;
  DevBuf arf;
  int32_t arf_n = 0;
  float arf_x0 = 0, arf_dx = 0;

  // nn8 running lists for multi-block merging (volumetric_reconstruction_backend_nn8.cpp:57-66)
  DevBuf list_d, list_v, list_id;
  uint64_t list_n = 0;

  // generic per-call staging
  DevBuf in_a, in_b, in_c, out_a, out_b, out_c;
  DevBuf tile_queue;  // persistent one-block-per-tile kernels: tile counter
  DevBuf spiral;     // char4[1000]
  DevBuf flags;      // uint32 error flags + uint64 stats
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  uint64_t launches = 0;  // kernels this context has launched

  // adjoint: step checkpoints, per-cell derivatives, gradient accumulator
  DevBuf rec_h, rec_n, adj_dT, adj_dR, adj_grad, adj_seed, adj_loss;

  // Monte-Carlo radial profile: shell table, segments, segment sums
  DevBuf prof_tab, prof_seg, prof_sum;

  // batched render: job table, sorted channel table, channel state, queue
  DevBuf jobs, chan_sorted, chan_state, queue, item_cost, item_order;
  int32_t batch_tile_w = 8;       // batched work item: tile_w x (32 / tile_w) pixels
  int32_t batch_occupancy = 4;    // batched kernel: blocks per SM (0 = register-limited)
  float batch_window = 40.0f;     // batched kernel: per-warp z window (0 = none)
  bool batch_cost_order = true;   // hand out the costliest tiles first
  cudaGraphExec_t batch_exec = nullptr;  // the batched launch sequence as a CUDA graph
  std::string batch_key;                 // launch parameters it was captured with
};

// Error flags written by kernels (bit mask in flags[0]).
enum : uint32_t {
  FLAG_KEY_RANGE = 1u,
  FLAG_STEP_LIMIT = 2u,
  FLAG_NONFINITE = 4u,
  FLAG_REC_OVERFLOW = 8u,
};

// Stats block layout behind the flags word (uint64 counters).
struct DevStats {
  unsigned long long steps;
  unsigned long long accepted;
  unsigned long long queries;
  unsigned long long cells;
  unsigned long long cands;
  unsigned long long max_steps;
  unsigned long long rays_at_limit;
  unsigned long long pad;
};
constexpr size_t kFlagsBytes = 64 + sizeof(DevStats);

// launchers (return cudaError_t of the launch sequence)
cudaError_t grid_bbox(Context& c, const float4* in, uint64_t n, float* mn3, float* mx3,
                      bool* nonfinite);
cudaError_t grid_build_device(Context& c, const float4* in, uint64_t n);
// In-place exclusive prefix sum of m uint32 (one block; for per-block counts).
cudaError_t exclusive_scan_u32(Context& c, uint32_t* a, uint64_t m);

// Cell ingestion (ilc_ingest.cu): periodic correction and volume cutout of
// n cells, compacted in input order into (x, y, z, q) float4 and the original
// indices; *n_out (device uint64) receives the number kept.
struct CutoutParams {
  double lo[3], hi[3];     // cutout box: center -/+ extent / 2
  double glo[3], ghi[3];   // box widened by the border (periodic correction)
  double period[3];
};
// volumetric_slice::create_slice (ilc_slice.cu); plane = camera_plane's double
// output (look, basis0, basis1, min corner, pixel size); out: device image.
cudaError_t slice_launch(Context& c, const double plane[13], int nx, int ny, int samples,
                         uint64_t seed, double dV, float* out);
cudaError_t ingest_launch(Context& c, const float* xyz, const float* q, uint64_t n,
                          const CutoutParams& p, float4* out, uint32_t* out_index,
                          unsigned long long* n_out);
cudaError_t nn8_query_launch(Context& c, const float4* pts, uint64_t n, bool merge,
                             float* out, int32_t* idx8, float* d8);
cudaError_t quantity_xray_flux_launch(Context& c, const float* rho, const float* u,
                                      const float* xe, uint64_t n, float z, float dL,
                                      float emin, float emax, int num_samples, float* out,
                                      int out_stride = 1);
cudaError_t quantity_xray_bin_launch(Context& c, const float* rho, const float* u,
                                     const float* xe, uint64_t n, float z, float dL, float e,
                                     float de, float* out);
cudaError_t quantity_xray_bins_launch(Context& c, const float* rho, const float* u,
                                      const float* xe, uint64_t n, float z, float dL,
                                      const float* e, const float* de, int n_bins, float* out);
cudaError_t quantity_temperature_launch(Context& c, const float* u, const float* xe,
                                        uint64_t n, float* out);
cudaError_t profile_points_launch(Context& c, const uint64_t* prefix, int n_shells,
                                  const double* u_min, const double* u_max,
                                  const double center[3], uint64_t seed, uint64_t g0, uint64_t n,
                                  float4* pts);
cudaError_t profile_segment_sum_launch(Context& c, const ulonglong2* segs, uint32_t n_segs,
                                       uint64_t g0, const float* vals, double* sums);
cudaError_t quantity_xray_photon_flux_launch(Context& c, const float* rho, const float* u,
                                             const float* xe, uint64_t n, float z, float dL,
                                             float emin, float emax, int num_samples,
                                             float* out);
cudaError_t quantity_chandra_total_launch(Context& c, const float* rho, const float* u,
                                          const float* xe, uint64_t n, float z, float dL,
                                          float* out);
cudaError_t quantity_chandra_bin_launch(Context& c, const float* rho, const float* u,
                                        const float* xe, uint64_t n, float z, float dL, float e,
                                        float de, float* out);
cudaError_t quantity_chandra_bins_launch(Context& c, const float* rho, const float* u,
                                         const float* xe, uint64_t n, float z, float dL,
                                         const float* e, const float* de, int n_bins,
                                         float* out);

struct RenderArgs {
  float cam[13];        // look(3), b0(3), b1(3), min corner(3), pixel size
  int32_t nx, ny;
  float z0, z_end;
  double atol, rtol;
  int32_t controller;   // ILC_CONTROLLER_*
  int64_t fixed_steps;  // > 0: fixed-step mode
  float fixed_h;        // step of the fixed-step mode, (float)(z_range / fixed_steps)
  float scale;          // multiplier applied to each pixel
  bool apply_scale;
  float* out;           // device image
  double* out_d = nullptr;  // frozen replay: device image of the increments summed in double
  float window_override = -1.0f;  // >= 0: z window for this launch (autotuner)
  int occupancy_override = -1;    // >= 0: occupancy variant for this launch (autotuner)
  int row_stride = 1;             // > 1: only every row_stride-th tile row (autotuner)
  float* rec_h = nullptr;         // adjoint checkpoint: accepted step sizes per ray
  int32_t* rec_n = nullptr;
  int64_t rec_cap = 0;
  const float* replay_h = nullptr;    // frozen replay: per-ray step sizes (rec_cap each)
  const int32_t* replay_n = nullptr;  // frozen replay: steps per ray
  uint64_t* ray_stats = nullptr;      // optional: per ray (steps, accepted, cells, candidates)
  int32_t row0 = 0;   // first pixel row of this launch (a multiple of 8)
  int32_t rows = 0;   // pixel rows of this launch (0: to the last row); per-ray arrays
                      // (rec_h, rec_n, replay_*, ray_stats) are indexed from row0
};

// Adjoint of the X-ray band map (ilc_adjoint.cu).
// q (stride q_stride floats), dq/dlnT and dq/dlnrho per cell, original order.
cudaError_t adjoint_cell_launch(Context& c, const float* rho, const float* u, const float* xe,
                                uint64_t n, float z, float dL, float emin, float emax,
                                int num_samples, float* q_out, int q_stride, float* dq_lnT,
                                float* dq_lnrho);
// loss (double, accumulated) and dL/dI_raw seed per pixel
cudaError_t adjoint_seed_launch(Context& c, const float* img, const float* target, int64_t npix,
                                float scale, float* seed, double* loss, bool reset_loss = true);
// replay (checkpoint) or recompute the rays of the band [a.row0, a.row0 + a.rows)
// and scatter dL/dq (sorted order); seed is indexed by the full image's pixels
cudaError_t adjoint_ray_launch(Context& c, const RenderArgs& a, int mode, const float* seed,
                               double* grad, float* kernel_ms);
// dL/dln rho, dL/dln T in the original order
cudaError_t adjoint_chain_launch(Context& c, const double* grad, uint64_t n, const float* dq_lnrho,
                                 const float* dq_lnT, float* g_lnrho, float* g_lnT);
cudaError_t render_launch(Context& c, const RenderArgs& a, float* kernel_ms);

// One camera of a batched render, as the kernel reads it.
struct JobDev {
  float look[3], b0[3], b1[3], minp[3];
  float ps;
  int32_t nx, ny, tiles_x;
  double look_d[3], b0_d[3], b1_d[3], minp_d[3];
  double ps_d;
  double z_range, aperture, centre[3], radius, min_chord;
  float scale;
  int32_t pad;
  uint64_t out_offset;
  uint64_t item_begin;   // first work item (tile) of the job
};

struct BatchArgs {
  const JobDev* jobs;     // device
  int32_t n_jobs;
  uint64_t n_items;
  int32_t V;
  const float* chan;      // device, sorted order, n x V (V = 1: nullptr = particles' q)
  float* out;             // device images
  double atol, rtol;
  int32_t tile_w;         // 1, 2, 4, 8, 16 or 32
  int32_t occupancy;      // 0, 3 or 4
  float window;           // per-warp z window (0 = none)
  const uint32_t* order;  // device: work item handed out q-th (nullptr = natural order)
  bool axis_z = false;    // every job looks along z (look x and y exactly 0)
};
// Estimated cost per work item of a batched render (the particles projected
// into each tile's pixel columns, weighted by their cell's occupancy), and
// the item order by decreasing cost.
cudaError_t batched_order(Context& c, BatchArgs& a, const std::vector<JobDev>& jobs);
// Sorted channel table: out[p * V + c] = in[s2u[p] * V + c].
cudaError_t channels_sort_launch(Context& c, const float* in, uint64_t n, int V, float* out);
cudaError_t batched_launch(Context& c, const BatchArgs& a, float* kernel_ms);

// Spiral table (8 subcells x 125 offsets), generated on the host.
void spiral_table(int8_t out[8][125][3]);

}  // namespace ilc
