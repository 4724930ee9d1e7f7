// ilc_capi.cu -- the extern "C" boundary (include/ilc.h) over the CUDA path.
//
// Host-side arithmetic that the reference does on the CPU in double (grid
// parameters, camera basis, image scaling) is done here the same way, so the
// device receives the same float parameters the reference's kernels receive.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "ilc_internal.h"
#include "ilc_random.cuh"

struct ilc_ctx {
  ilc::Context c;
};

namespace ilc {
namespace {

ilc_status fail(Context& c, ilc_status st, const std::string& msg) {
  c.error = msg;
  return st;
}

ilc_status cuda_fail(Context& c, cudaError_t e, const char* where) {
  const ilc_status st =
      e == cudaErrorMemoryAllocation ? ILC_ERR_OUT_OF_MEMORY : ILC_ERR_CUDA;
  c.error = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  return st;
}

#define ILC_CUDA(ctx, expr, where)               \
  do {                                           \
    cudaError_t e_ = (expr);                     \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, where); \
  } while (0)

// Stages a caller array on the device: returns the device pointer to use.
cudaError_t stage_in(Context& c, DevBuf& buf, const void* src, size_t bytes, int is_device,
                     const void** out) {
  if (is_device) {
    *out = src;
    return cudaSuccess;
  }
  cudaError_t e = buf.ensure(bytes);
  if (e) return e;
  e = cudaMemcpyAsync(buf.p, src, bytes, cudaMemcpyHostToDevice, c.stream);
  *out = buf.p;
  return e;
}

cudaError_t out_ptr(DevBuf& buf, void* dst, size_t bytes, int is_device, void** out) {
  if (is_device) {
    *out = dst;
    return cudaSuccess;
  }
  cudaError_t e = buf.ensure(bytes);
  *out = buf.p;
  return e;
}

cudaError_t finish_out(Context& c, void* dst, const void* dev, size_t bytes, int is_device) {
  if (!is_device && bytes) {
    cudaError_t e = cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDeviceToHost, c.stream);
    if (e) return e;
  }
  return cudaStreamSynchronize(c.stream);
}

// particle_grid ctor (particle_grid.cpp:54-103): bounding box +-0.1 in double,
// cell width cbrt(8/N * V), n_cells = ceil(extent / width), float casts.
void make_grid_params(const float mn_f[3], const float mx_f[3], uint64_t n, GridParams* g) {
  double mn[3], mx[3];
  for (int i = 0; i < 3; ++i) { mn[i] = (double)mn_f[i]; mx[i] = (double)mx_f[i]; }
  double vol = 1.0;
  for (int i = 0; i < 3; ++i) {
    mn[i] -= 0.1;
    mx[i] += 0.1;
    vol *= (mx[i] - mn[i]);
  }
  const double cell_volume = (double)8 / (double)n * vol;
  const double w = std::cbrt(cell_volume);
  g->total = 1;
  for (int i = 0; i < 3; ++i) {
    // cells per axis; 0 (rejected by the caller) when it does not fit an
    // int32 or is not a positive number (the float -> int cast would be undefined)
    const double nc = std::ceil((mx[i] - mn[i]) / w);
    g->n[i] = (nc >= 1.0 && nc <= 2147483647.0) ? (int32_t)nc : 0;
    g->min[i] = (float)mn[i];
    g->cs[i] = (float)w;
    g->total *= (uint64_t)g->n[i];
    if (g->total >= (1ull << 32)) g->total = 1ull << 32;  // rejected by the caller; no wrap
  }
}

// camera::update_basis_vectors / update_min_position (camera.cpp:124-155,
// math.hpp:85-149), in double, then cast to float.
void camera_plane(const ilc_camera& cam, float out[13], double* outd = nullptr) {
  auto dot3 = [](const double* a, const double* b) {
    double r = 0.0;
    for (int i = 0; i < 3; ++i) r += a[i] * b[i];
    return r;
  };
  auto cross3 = [](const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  const double ps = cam.screen_width / (double)cam.num_pix_x;
  double v1[3] = {0, 0, 1};
  if (cam.look_at[0] == v1[0] && cam.look_at[1] == v1[1] && cam.look_at[2] == v1[2]) {
    v1[0] = 0; v1[1] = 1; v1[2] = 0;
  }
  double a[3], b[3];
  cross3(v1, cam.look_at, a);
  cross3(cam.look_at, a, b);
  const double a1 = cam.look_at[0], a2 = cam.look_at[1], a3 = cam.look_at[2];
  const double a1a2 = a1 * a2, a1a3 = a1 * a3, a2a3 = a2 * a3;
  const double ca = std::cos(cam.roll), sa = std::sin(cam.roll);
  const double fc = 1.0 - ca;
  const double m[3][3] = {{a1 * a1 * fc + ca, a1a2 * fc - a3 * sa, a1a3 * fc + a2 * sa},
                          {a1a2 * fc + a3 * sa, a2 * a2 * fc + ca, a2a3 * fc - a1 * sa},
                          {a1a3 * fc - a2 * sa, a2a3 * fc + a1 * sa, a3 * a3 * fc + ca}};
  double ra[3], rb[3];
  for (int i = 0; i < 3; ++i) { ra[i] = dot3(m[i], a); rb[i] = dot3(m[i], b); }
  const double la = 1. / std::sqrt(dot3(ra, ra)), lb = 1. / std::sqrt(dot3(rb, rb));
  double b0[3], b1[3], mp[3];
  for (int i = 0; i < 3; ++i) { b0[i] = la * ra[i]; b1[i] = lb * rb[i]; }
  for (int i = 0; i < 3; ++i) mp[i] = cam.position[i];
  for (int i = 0; i < 3; ++i) mp[i] -= ((double)cam.num_pix_x / 2.0) * ps * b0[i];
  for (int i = 0; i < 3; ++i) mp[i] -= ((double)cam.num_pix_y / 2.0) * ps * b1[i];
  for (int i = 0; i < 3; ++i) {
    out[i] = (float)cam.look_at[i];
    out[3 + i] = (float)b0[i];
    out[6 + i] = (float)b1[i];
    out[9 + i] = (float)mp[i];
  }
  out[12] = (float)ps;
  if (outd) {
    for (int i = 0; i < 3; ++i) {
      outd[i] = cam.look_at[i];
      outd[3 + i] = b0[i];
      outd[6 + i] = b1[i];
      outd[9 + i] = mp[i];
    }
    outd[12] = ps;
  }
}

float los_scale(const ilc_camera& cam, double z_range, const ilc_los_scaling& s) {
  const double ps = cam.screen_width / (double)cam.num_pix_x;
  const float pixel_area = (float)(ps * ps);
  const float lc = (float)s.length_conversion;
  const double dA_in = (double)pixel_area * s.area_conversion;
  const double range = (double)lc * z_range;
  double dA;
  if (s.dA_mode == ILC_DA_PIXEL_AREA) dA = dA_in;
  else if (s.dA_mode == ILC_DA_UNIT) dA = 1.0;
  else dA = 1.0 / range;
  const float dAf = (float)dA;
  return lc * dAf;
}

bool camera_ok(const ilc_camera* cam) {
  if (!cam || cam->num_pix_x <= 0 || cam->num_pix_y <= 0) return false;
  if (!(cam->screen_width > 0.0)) return false;
  const double l2 = cam->look_at[0] * cam->look_at[0] + cam->look_at[1] * cam->look_at[1] +
                    cam->look_at[2] * cam->look_at[2];
  return l2 > 0.0 && std::isfinite(l2);
}

ilc_status read_flags(Context& c, uint32_t* flags, DevStats* stats) {
  char buf[kFlagsBytes];
  ILC_CUDA(c, cudaMemcpyAsync(buf, c.flags.p, kFlagsBytes, cudaMemcpyDeviceToHost, c.stream),
           "read flags");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "read flags");
  std::memcpy(flags, buf, 4);
  if (stats) std::memcpy(stats, buf + 64, sizeof(DevStats));
  return ILC_OK;
}

// Grid over the n float4 particles already in c.tmp_in (setup_particles).
ilc_status build_grid_staged(Context& c, uint64_t n) {
  c.has_grid = false;
  float mn[3], mx[3];
  bool nonfinite = false;
  ILC_CUDA(c, grid_bbox(c, c.tmp_in.as<float4>(), n, mn, mx, &nonfinite), "bounding box");
  if (nonfinite) return fail(c, ILC_ERR_NONFINITE_INPUT, "non-finite particle coordinates");
  GridParams g;
  make_grid_params(mn, mx, n, &g);
  if (g.total >= (1ull << 32) || g.n[0] <= 0 || g.n[1] <= 0 || g.n[2] <= 0)
    return fail(c, ILC_ERR_GRID_TOO_LARGE, "grid has more than 2^32 cells");
  c.gp = g;
  ILC_CUDA(c, grid_build_device(c, c.tmp_in.as<float4>(), n), "grid build");
  uint32_t flags = 0;
  ilc_status st = read_flags(c, &flags, nullptr);
  if (st) return st;
  if (flags & FLAG_KEY_RANGE) return fail(c, ILC_ERR_INTERNAL, "particle outside its grid");
  c.n_particles = n;
  c.has_grid = true;
  return ILC_OK;
}

// Job table of a batched render on the device (values not staged).
ilc_status batched_jobs(Context& c, int32_t V, const ilc_job* jobs, int32_t n_jobs,
                        ilc_tolerance tol, uint64_t images_len, BatchArgs* a) {
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "batched render before setup_particles");
  if (V < 1 || V > 256 || !jobs || n_jobs < 1)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid batched render arguments (1 <= V <= 256)");
  if (!(tol.absolute >= 0.0) || !(tol.relative >= 0.0) ||
      (tol.absolute <= 0.0 && tol.relative <= 0.0))
    return fail(c, ILC_ERR_INVALID_ARGUMENT,
                "either the absolute or the relative tolerance has to be > 0");
  std::vector<JobDev> jd((size_t)n_jobs);
  const int tw = c.batch_tile_w, th = c.batch_tile_w > 0 ? 32 / c.batch_tile_w : 1;
  uint64_t items = 0;
  for (int32_t k = 0; k < n_jobs; ++k) {
    const ilc_job& j = jobs[k];
    if (!camera_ok(&j.camera)) return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid job camera");
    const bool chord = j.sphere_radius > 0.0;
    if (!std::isfinite(j.aperture_radius) || !std::isfinite(j.sphere_radius) ||
        !std::isfinite(j.min_chord) || !std::isfinite(j.sphere_center[0]) ||
        !std::isfinite(j.sphere_center[1]) || !std::isfinite(j.sphere_center[2]) ||
        (!chord && !(j.z_range > 0.0 && std::isfinite(j.z_range))))
      return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid job range, chord or aperture");
    const uint64_t plane = (uint64_t)j.camera.num_pix_x * (uint64_t)j.camera.num_pix_y;
    if (j.out_offset > images_len || (uint64_t)V * plane > images_len - j.out_offset)
      return fail(c, ILC_ERR_INVALID_ARGUMENT, "job output block beyond images_len");
    JobDev& d = jd[k];
    std::memset(&d, 0, sizeof(d));
    float f[13];
    double dd[13];
    camera_plane(j.camera, f, dd);
    for (int i = 0; i < 3; ++i) {
      d.look[i] = f[i];
      d.b0[i] = f[3 + i];
      d.b1[i] = f[6 + i];
      d.minp[i] = f[9 + i];
      d.look_d[i] = dd[i];
      d.b0_d[i] = dd[3 + i];
      d.b1_d[i] = dd[6 + i];
      d.minp_d[i] = dd[9 + i];
      d.centre[i] = j.sphere_center[i];
    }
    d.ps = f[12];
    d.ps_d = dd[12];
    d.nx = j.camera.num_pix_x;
    d.ny = j.camera.num_pix_y;
    // compact tiles: tiles per row; strided (tw = 0): items of the job
    const uint64_t npix = (uint64_t)d.nx * (uint64_t)d.ny;
    d.tiles_x = tw > 0 ? (d.nx + tw - 1) / tw : (int32_t)((npix + 31) / 32);
    d.z_range = j.z_range;
    d.aperture = j.aperture_radius;
    d.radius = j.sphere_radius;
    d.min_chord = j.min_chord;
    d.scale = j.scale;
    d.out_offset = j.out_offset;
    d.item_begin = items;
    items += tw > 0 ? (uint64_t)d.tiles_x * (uint64_t)((d.ny + th - 1) / th)
                    : (uint64_t)d.tiles_x;
  }
  ILC_CUDA(c, c.jobs.ensure(jd.size() * sizeof(JobDev)), "job table");
  ILC_CUDA(c, cudaMemcpyAsync(c.jobs.p, jd.data(), jd.size() * sizeof(JobDev),
                              cudaMemcpyHostToDevice, c.stream), "job table H2D");
  a->jobs = c.jobs.as<JobDev>();
  a->n_jobs = n_jobs;
  a->n_items = items;
  a->V = V;
  a->chan = nullptr;
  a->atol = tol.absolute;
  a->rtol = tol.relative;
  a->tile_w = c.batch_tile_w;
  a->occupancy = c.batch_occupancy;
  a->window = c.batch_window;
  a->order = nullptr;
  a->axis_z = true;
  for (const JobDev& d : jd)
    if (d.look[0] != 0.0f || d.look[1] != 0.0f) a->axis_z = false;
  if (c.batch_cost_order) ILC_CUDA(c, batched_order(c, *a, jd), "work order");
  return ILC_OK;
}

// Job table plus the sorted channel table of a batched render.
ilc_status batched_prepare(Context& c, const float* values, int32_t V, int values_on_device,
                           const ilc_job* jobs, int32_t n_jobs, ilc_tolerance tol,
                           uint64_t images_len, BatchArgs* a) {
  if (!values) return fail(c, ILC_ERR_INVALID_ARGUMENT, "values is NULL");
  ilc_status st = batched_jobs(c, V, jobs, n_jobs, tol, images_len, a);
  if (st) return st;
  const uint64_t n = c.n_particles;
  const void* dv = nullptr;
  ILC_CUDA(c, stage_in(c, c.in_a, values, n * (uint64_t)V * 4, values_on_device, &dv),
           "values H2D");
  ILC_CUDA(c, c.chan_sorted.ensure(n * (uint64_t)V * 4), "channel table");
  ILC_CUDA(c, channels_sort_launch(c, static_cast<const float*>(dv), n, V,
                                   c.chan_sorted.as<float>()), "channel sort");
  a->chan = c.chan_sorted.as<float>();
  return ILC_OK;
}

bool tile_w_ok(int32_t w) {
  return w == 0 || w == 1 || w == 2 || w == 4 || w == 8 || w == 16 || w == 32;
}

// Optional frozen replay (replay_h/replay_n) or step recording (rec_h/rec_n),
// both device arrays of cap steps per ray; either forces the grid kernel.
struct StepArrays {
  const float* replay_h = nullptr;
  const int32_t* replay_n = nullptr;
  float* rec_h = nullptr;
  int32_t* rec_n = nullptr;
  int64_t cap = 0;
  uint64_t* ray_stats = nullptr;  // per-ray statistics (device)
  double* out_d = nullptr;        // frozen replay summed in double (device image)
};

ilc_status render_common(Context& c, const ilc_camera* cam, double z_range, ilc_tolerance tol,
                         int32_t controller, int64_t fixed_steps,
                         const ilc_los_scaling* scaling, float* image, int is_device,
                         ilc_render_stats* stats, const StepArrays& sa = StepArrays()) {
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "render before setup_particles");
  if (!camera_ok(cam)) return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid camera");
  if (!(z_range > 0.0) || !std::isfinite(z_range) || (!image && !sa.out_d))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid z_range or image");
  if (fixed_steps <= 0 && !sa.replay_h) {
    if (!(tol.absolute >= 0.0) || !(tol.relative >= 0.0) ||
        (tol.absolute <= 0.0 && tol.relative <= 0.0))
      return fail(c, ILC_ERR_INVALID_ARGUMENT,
                  "either the absolute or the relative tolerance has to be > 0");
    if (controller != ILC_CONTROLLER_REF32 && controller != ILC_CONTROLLER_FP64)
      return fail(c, ILC_ERR_INVALID_ARGUMENT, "unknown controller");
  }
  RenderArgs a{};
  camera_plane(*cam, a.cam);
  a.nx = cam->num_pix_x;
  a.ny = cam->num_pix_y;
  a.z0 = 0.0f;
  a.z_end = (float)z_range;
  a.atol = tol.absolute;
  a.rtol = tol.relative;
  a.controller = controller;
  a.fixed_steps = fixed_steps;
  a.fixed_h = fixed_steps > 0 ? (float)(z_range / (double)fixed_steps) : 0.0f;
  a.apply_scale = scaling != nullptr;
  a.scale = scaling ? los_scale(*cam, z_range, *scaling) : 1.0f;
  a.replay_h = sa.replay_h;
  a.replay_n = sa.replay_n;
  a.rec_h = sa.rec_h;
  a.rec_n = sa.rec_n;
  a.rec_cap = sa.cap;
  a.ray_stats = sa.ray_stats;
  a.out_d = sa.out_d;
  const size_t bytes = (size_t)a.nx * (size_t)a.ny * 4;
  void* dimg = nullptr;
  if (image) ILC_CUDA(c, out_ptr(c.out_a, image, bytes, is_device, &dimg), "image buffer");
  a.out = static_cast<float*>(dimg);
  float ms = 0.0f;
  if (c.render_engine == ILC_ENGINE_PERSISTENT && fixed_steps <= 0 &&
      controller == ILC_CONTROLLER_FP64 && !sa.replay_h && !sa.rec_h && !sa.ray_stats) {
    // one job through the persistent work-queue kernel, values = particle q
    ilc_job j{};
    j.camera = *cam;
    j.z_range = z_range;
    j.scale = a.scale;
    BatchArgs ba{};
    ilc_status st = batched_jobs(c, 1, &j, 1, tol, (uint64_t)a.nx * (uint64_t)a.ny, &ba);
    if (st) return st;
    ba.out = a.out;
    ILC_CUDA(c, batched_launch(c, ba, &ms), "render kernel (persistent)");
  } else {
    ILC_CUDA(c, render_launch(c, a, &ms), "render kernel");
  }
  if (image) ILC_CUDA(c, finish_out(c, image, dimg, bytes, is_device), "render");
  uint32_t flags = 0;
  DevStats ds{};
  ilc_status st = read_flags(c, &flags, &ds);
  if (st) return st;
  if (stats) {
    stats->steps = ds.steps;
    stats->accepted_steps = ds.accepted;
    stats->queries = ds.queries;
    stats->cells_visited = ds.cells;
    stats->candidates = ds.cands;
    stats->max_steps_per_ray = ds.max_steps;
    stats->rays_at_step_limit = ds.rays_at_limit;
    stats->kernel_ms = ms;
  }
  if (flags & FLAG_STEP_LIMIT)
    return fail(c, ILC_ERR_STEP_LIMIT, "rays reached the per-ray step limit");
  if (flags & FLAG_REC_OVERFLOW)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "step recording capacity too small");
  return ILC_OK;
}

// distributed_mc_radial_profile's shells (profile.cpp:320-355) and
// generate_num_samples (profile.cpp:93-128), in the reference's double
// arithmetic and summation order.
struct ProfileShells {
  std::vector<double> radius, r_min, r_max, volume;
  std::vector<double> u_min, u_max;     // uniform_spherical_shell's u range (random.cpp:67-74)
  std::vector<uint64_t> count, prefix;  // prefix: num_radii + 1 entries
};

constexpr uint64_t kMaxProfileSamples = 1ull << 40;
constexpr uint64_t kProfileSegment = 8192;       // samples per reduction segment
constexpr uint64_t kProfileBatch = 1ull << 22;   // samples per device batch

bool profile_shells(double max_radius, int32_t num_radii, double density, ProfileShells* S) {
  if (!(max_radius > 0.0) || !std::isfinite(max_radius) || num_radii < 1 ||
      num_radii > (1 << 20) || !(density > 0.0) || !std::isfinite(density))
    return false;
  const unsigned N = (unsigned)num_radii;
  auto radius = [&](unsigned i) { return i * (max_radius / N); };
  S->radius.resize(N);
  S->r_min.resize(N);
  S->r_max.resize(N);
  S->volume.resize(N);
  S->u_min.resize(N);
  S->u_max.resize(N);
  for (unsigned i = 0; i < N; ++i) {
    S->radius[i] = radius(i);
    S->r_min[i] = i == 0 ? 0.0 : 0.5 * (radius(i - 1) + radius(i));
    S->r_max[i] = 0.5 * (radius(i + 1) + radius(i));
    const double a = S->r_min[i], b = S->r_max[i];
    S->volume[i] = 4. / 3 * M_PI * (b * b * b - a * a * a);
    S->u_min[i] = a * a * a;
    S->u_max[i] = b * b * b;
  }
  double expected = 0.0, sum_sq = 0.0;
  for (unsigned i = 0; i < N; ++i) expected += S->volume[i] * density;
  for (unsigned i = 0; i < N; ++i) sum_sq += S->volume[i] * S->volume[i];
  const double norm = expected / sum_sq;
  S->count.resize(N);
  S->prefix.assign(N + 1, 0);
  for (unsigned i = 0; i < N; ++i) {
    const double want = norm * (S->volume[i] * S->volume[i]);
    if (!(want < (double)kMaxProfileSamples)) return false;
    uint64_t n = (uint64_t)want;
    if (n == 0) n = 1;
    S->count[i] = n;
    S->prefix[i + 1] = S->prefix[i] + n;
    if (S->prefix[i + 1] > kMaxProfileSamples) return false;
  }
  return true;
}

}  // namespace
}  // namespace ilc

using namespace ilc;

extern "C" {

ilc_ctx* ilc_create(int device) {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  ilc_ctx* h = new (std::nothrow) ilc_ctx();
  if (!h) return nullptr;
  Context& c = h->c;
  c.device = device;
  if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    return nullptr;
  }
  c.own_stream = true;
  int8_t t[8][125][3];
  spiral_table(t);
  char4 packed[1000];
  for (int s = 0; s < 8; ++s)
    for (int i = 0; i < 125; ++i)
      packed[s * 125 + i] = make_char4(t[s][i][0], t[s][i][1], t[s][i][2], 0);
  if (c.spiral.ensure(sizeof(packed)) ||
      cudaMemcpy(c.spiral.p, packed, sizeof(packed), cudaMemcpyHostToDevice) ||
      c.flags.ensure(kFlagsBytes)) {
    ilc_destroy(h);
    return nullptr;
  }
  return h;
}

void ilc_destroy(ilc_ctx* h) {
  if (!h) return;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (c.stream) cudaStreamSynchronize(c.stream);
  for (DevBuf* b : {&c.parts, &c.cells, &c.s2u, &c.keys_a, &c.keys_b, &c.vals_a, &c.vals_b,
                    &c.hist, &c.tmp_in, &c.gaunt, &c.list_d, &c.list_v, &c.list_id, &c.in_a,
                    &c.in_b, &c.in_c, &c.out_a, &c.out_b, &c.out_c, &c.spiral, &c.flags,
                    &c.rec_h, &c.rec_n, &c.adj_dT, &c.adj_dR, &c.adj_grad, &c.adj_seed,
                    &c.adj_loss, &c.codes, &c.jobs, &c.chan_sorted, &c.chan_state, &c.queue,
                    &c.item_cost, &c.item_order, &c.arf, &c.prof_tab, &c.prof_seg,
                    &c.prof_sum})
    b->release();
  if (c.batch_exec) cudaGraphExecDestroy(c.batch_exec);
  if (c.ev0) cudaEventDestroy(c.ev0);
  if (c.ev1) cudaEventDestroy(c.ev1);
  if (c.own_stream && c.stream) cudaStreamDestroy(c.stream);
  delete h;
}

const char* ilc_last_error(const ilc_ctx* h) { return h ? h->c.error.c_str() : "null context"; }

ilc_status ilc_set_step_limit(ilc_ctx* h, int64_t max_steps) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  if (max_steps <= 0) return fail(h->c, ILC_ERR_INVALID_ARGUMENT, "step limit must be > 0");
  h->c.max_steps = max_steps;
  return ILC_OK;
}

void* ilc_get_stream(ilc_ctx* h) { return h ? (void*)h->c.stream : nullptr; }

ilc_status ilc_set_render_engine(ilc_ctx* h, int32_t engine) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  if (engine != ILC_ENGINE_GRID && engine != ILC_ENGINE_PERSISTENT)
    return fail(h->c, ILC_ERR_INVALID_ARGUMENT, "unknown render engine");
  h->c.render_engine = engine;
  return ILC_OK;
}

ilc_status ilc_set_render_occupancy(ilc_ctx* h, int32_t blocks_per_sm) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  if (blocks_per_sm != 0 && blocks_per_sm != 3 && blocks_per_sm != 4 && blocks_per_sm != 5)
    return fail(h->c, ILC_ERR_INVALID_ARGUMENT, "occupancy must be 0, 3, 4 or 5");
  h->c.render_occupancy = blocks_per_sm;
  return ILC_OK;
}

ilc_status ilc_set_z_window(ilc_ctx* h, float z_window) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  if (!(z_window >= 0.0f) || !std::isfinite(z_window))
    return fail(h->c, ILC_ERR_INVALID_ARGUMENT, "z_window must be finite and >= 0");
  h->c.z_window = z_window;
  return ILC_OK;
}

ilc_status ilc_nn8_setup_particles(ilc_ctx* h, const float* particles, uint64_t n,
                                   int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!particles || n == 0) return fail(c, ILC_ERR_INVALID_ARGUMENT, "no particles");
  if (n >= (1ull << 31)) return fail(c, ILC_ERR_GRID_TOO_LARGE, "more than 2^31 particles");
  c.has_grid = false;
  const void* din = nullptr;
  ILC_CUDA(c, stage_in(c, c.tmp_in, particles, n * 16, is_device, &din), "particles H2D");
  float mn[3], mx[3];
  bool nonfinite = false;
  ILC_CUDA(c, grid_bbox(c, static_cast<const float4*>(din), n, mn, mx, &nonfinite),
           "bounding box");
  if (nonfinite) return fail(c, ILC_ERR_NONFINITE_INPUT, "non-finite particle coordinates");
  GridParams g;
  make_grid_params(mn, mx, n, &g);
  if (g.total >= (1ull << 32) || g.n[0] <= 0 || g.n[1] <= 0 || g.n[2] <= 0)
    return fail(c, ILC_ERR_GRID_TOO_LARGE, "grid has more than 2^32 cells");
  c.gp = g;
  ILC_CUDA(c, grid_build_device(c, static_cast<const float4*>(din), n), "grid build");
  uint32_t flags = 0;
  ilc_status st = read_flags(c, &flags, nullptr);
  if (st) return st;
  if (flags & FLAG_KEY_RANGE) return fail(c, ILC_ERR_INTERNAL, "particle outside its grid");
  c.n_particles = n;
  c.has_grid = true;
  // The nn8 lists survive a new particle block: the next query with
  // merge_previous = 1 continues them (reconstructing_data_crawler.cpp:164-255).
  return ILC_OK;
}

ilc_status ilc_grid_describe(ilc_ctx* h, ilc_grid_desc* out) {
  if (!h || !out) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "no grid");
  for (int i = 0; i < 3; ++i) {
    out->min_corner[i] = c.gp.min[i];
    out->cell_sizes[i] = c.gp.cs[i];
    out->num_cells[i] = c.gp.n[i];
  }
  out->total_cells = c.gp.total;
  out->num_particles = c.n_particles;
  return ILC_OK;
}

ilc_status ilc_grid_export(ilc_ctx* h, int32_t* cells, uint32_t* s2u, float* sorted,
                           int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "no grid");
  const cudaMemcpyKind k = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  if (cells)
    ILC_CUDA(c, cudaMemcpyAsync(cells, c.cells.p, c.gp.total * 8, k, c.stream), "export cells");
  if (s2u)
    ILC_CUDA(c, cudaMemcpyAsync(s2u, c.s2u.p, c.n_particles * 4, k, c.stream), "export s2u");
  if (sorted)
    ILC_CUDA(c, cudaMemcpyAsync(sorted, c.parts.p, c.n_particles * 16, k, c.stream),
             "export particles");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "export");
  return ILC_OK;
}

ilc_status ilc_nn8_query(ilc_ctx* h, const float* points, uint64_t n, int merge_previous,
                         float* out_values, int32_t* out_idx8, float* out_dist8,
                         int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "query before setup_particles");
  if (n == 0) return ILC_OK;
  if (!points || !out_values) return fail(c, ILC_ERR_INVALID_ARGUMENT, "null array");
  if (merge_previous && c.list_n != n)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "merge_previous needs the same point count");
  const void* dp = nullptr;
  void *dv = nullptr, *di = nullptr, *dd = nullptr;
  ILC_CUDA(c, stage_in(c, c.in_a, points, n * 16, is_device, &dp), "points H2D");
  ILC_CUDA(c, out_ptr(c.out_a, out_values, n * 4, is_device, &dv), "values");
  if (out_idx8) ILC_CUDA(c, out_ptr(c.out_b, out_idx8, n * 32, is_device, &di), "idx");
  if (out_dist8) ILC_CUDA(c, out_ptr(c.out_c, out_dist8, n * 32, is_device, &dd), "dist");
  ILC_CUDA(c, nn8_query_launch(c, static_cast<const float4*>(dp), n, merge_previous != 0,
                               static_cast<float*>(dv), static_cast<int32_t*>(di),
                               static_cast<float*>(dd)),
           "nn8 kernel");
  if (!is_device) {
    ILC_CUDA(c, cudaMemcpyAsync(out_values, dv, n * 4, cudaMemcpyDeviceToHost, c.stream), "D2H");
    if (out_idx8)
      ILC_CUDA(c, cudaMemcpyAsync(out_idx8, di, n * 32, cudaMemcpyDeviceToHost, c.stream), "D2H");
    if (out_dist8)
      ILC_CUDA(c, cudaMemcpyAsync(out_dist8, dd, n * 32, cudaMemcpyDeviceToHost, c.stream), "D2H");
  }
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "nn8 query");
  return ILC_OK;
}

ilc_status ilc_gaunt_load(ilc_ctx* h, const float* table, int32_t width, int32_t height,
                          float x0, float y0, float dx, float dy) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!table || width <= 0 || height <= 0 || width * height > 81 * 146 || !(dx > 0.0f) ||
      !(dy > 0.0f))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid Gaunt table (at most 81 x 146 entries)");
  const size_t bytes = (size_t)width * height * 4;
  ILC_CUDA(c, c.gaunt.ensure(bytes), "gaunt alloc");
  ILC_CUDA(c, cudaMemcpyAsync(c.gaunt.p, table, bytes, cudaMemcpyHostToDevice, c.stream),
           "gaunt H2D");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "gaunt");
  c.gw = width; c.gh = height; c.gx0 = x0; c.gy0 = y0; c.gdx = dx; c.gdy = dy;
  c.has_gaunt = true;
  return ILC_OK;
}

static ilc_status quantity_inputs(Context& c, const float* rho, const float* u, const float* xe,
                                  uint64_t n, int is_device, const float** drho,
                                  const float** du, const float** dxe) {
  const void *a = nullptr, *b = nullptr, *d = nullptr;
  if (rho) ILC_CUDA(c, stage_in(c, c.in_a, rho, n * 4, is_device, &a), "rho H2D");
  if (u) ILC_CUDA(c, stage_in(c, c.in_b, u, n * 4, is_device, &b), "u H2D");
  if (xe) ILC_CUDA(c, stage_in(c, c.in_c, xe, n * 4, is_device, &d), "xe H2D");
  *drho = static_cast<const float*>(a);
  *du = static_cast<const float*>(b);
  *dxe = static_cast<const float*>(d);
  return ILC_OK;
}

ilc_status ilc_quantity_xray_flux(ilc_ctx* h, const float* rho, const float* u, const float* xe,
                                  uint64_t n, float redshift, float luminosity_distance,
                                  float e_min, float e_max, int32_t num_samples, float* out,
                                  int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (n == 0) return ILC_OK;
  if (!rho || !u || !xe || !out || num_samples <= 0 || !(e_max >= e_min))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid xray_flux arguments");
  const float *a, *b, *d;
  ilc_status st = quantity_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  void* dout = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, out, n * 4, is_device, &dout), "out");
  ILC_CUDA(c, quantity_xray_flux_launch(c, a, b, d, n, redshift, luminosity_distance, e_min,
                                        e_max, num_samples, static_cast<float*>(dout)),
           "xray_flux kernel");
  ILC_CUDA(c, finish_out(c, out, dout, n * 4, is_device), "xray_flux");
  return ILC_OK;
}

ilc_status ilc_quantity_xray_spectral_flux(ilc_ctx* h, const float* rho, const float* u,
                                           const float* xe, uint64_t n, float redshift,
                                           float luminosity_distance, float energy,
                                           float energy_bin_width, float* out, int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (n == 0) return ILC_OK;
  if (!rho || !u || !xe || !out)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid xray_spectral_flux arguments");
  const float *a, *b, *d;
  ilc_status st = quantity_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  void* dout = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, out, n * 4, is_device, &dout), "out");
  ILC_CUDA(c, quantity_xray_bin_launch(c, a, b, d, n, redshift, luminosity_distance, energy,
                                       energy_bin_width, static_cast<float*>(dout)),
           "xray_spectral_flux kernel");
  ILC_CUDA(c, finish_out(c, out, dout, n * 4, is_device), "xray_spectral_flux");
  return ILC_OK;
}

ilc_status ilc_quantity_xray_photon_flux(ilc_ctx* h, const float* rho, const float* u,
                                         const float* xe, uint64_t n, float redshift,
                                         float luminosity_distance, float e_min, float e_max,
                                         int32_t num_samples, float* out, int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (n == 0) return ILC_OK;
  if (!rho || !u || !xe || !out || num_samples <= 0 || !(e_max >= e_min))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid xray_photon_flux arguments");
  const float *a, *b, *d;
  ilc_status st = quantity_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  void* dout = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, out, n * 4, is_device, &dout), "out");
  ILC_CUDA(c, quantity_xray_photon_flux_launch(c, a, b, d, n, redshift, luminosity_distance,
                                               e_min, e_max, num_samples,
                                               static_cast<float*>(dout)),
           "xray_photon_flux kernel");
  ILC_CUDA(c, finish_out(c, out, dout, n * 4, is_device), "xray_photon_flux");
  return ILC_OK;
}

ilc_status ilc_arf_load(ilc_ctx* h, const float* table, int32_t n, float x_min, float dx) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!table || n <= 0 || n > 65536 || !(dx > 0.0f) || !std::isfinite(dx) ||
      !std::isfinite(x_min))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid ARF table (1 to 65536 samples, dx > 0)");
  const size_t bytes = (size_t)n * 4;
  ILC_CUDA(c, c.arf.ensure(bytes), "arf alloc");
  ILC_CUDA(c, cudaMemcpyAsync(c.arf.p, table, bytes, cudaMemcpyHostToDevice, c.stream),
           "arf H2D");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "arf");
  c.arf_n = n; c.arf_x0 = x_min; c.arf_dx = dx;
  c.has_arf = true;
  return ILC_OK;
}

// Null check and staging of the Chandra quantities' inputs.
static ilc_status chandra_inputs(Context& c, const float* rho, const float* u, const float* xe,
                                 uint64_t n, int is_device, const float** a, const float** b,
                                 const float** d) {
  if (!rho || !u || !xe) return fail(c, ILC_ERR_INVALID_ARGUMENT, "null input array");
  return quantity_inputs(c, rho, u, xe, n, is_device, a, b, d);
}

ilc_status ilc_quantity_chandra_count_rate(ilc_ctx* h, const float* rho, const float* u,
                                           const float* xe, uint64_t n, float redshift,
                                           float luminosity_distance, float* out,
                                           int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (!c.has_arf) return fail(c, ILC_ERR_NO_ARF_TABLE, "ARF table not loaded");
  if (n == 0) return ILC_OK;
  if (!out) return fail(c, ILC_ERR_INVALID_ARGUMENT, "null output");
  const float *a, *b, *d;
  ilc_status st = chandra_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  void* dout = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, out, n * 4, is_device, &dout), "out");
  ILC_CUDA(c, quantity_chandra_total_launch(c, a, b, d, n, redshift, luminosity_distance,
                                            static_cast<float*>(dout)),
           "chandra_count_rate kernel");
  ILC_CUDA(c, finish_out(c, out, dout, n * 4, is_device), "chandra_count_rate");
  return ILC_OK;
}

ilc_status ilc_quantity_chandra_spectral_count_rate(ilc_ctx* h, const float* rho,
                                                    const float* u, const float* xe,
                                                    uint64_t n, float redshift,
                                                    float luminosity_distance, float energy,
                                                    float energy_bin_width, float* out,
                                                    int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (!c.has_arf) return fail(c, ILC_ERR_NO_ARF_TABLE, "ARF table not loaded");
  if (n == 0) return ILC_OK;
  if (!out) return fail(c, ILC_ERR_INVALID_ARGUMENT, "null output");
  const float *a, *b, *d;
  ilc_status st = chandra_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  void* dout = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, out, n * 4, is_device, &dout), "out");
  ILC_CUDA(c, quantity_chandra_bin_launch(c, a, b, d, n, redshift, luminosity_distance, energy,
                                          energy_bin_width, static_cast<float*>(dout)),
           "chandra_spectral_count_rate kernel");
  ILC_CUDA(c, finish_out(c, out, dout, n * 4, is_device), "chandra_spectral_count_rate");
  return ILC_OK;
}

ilc_status ilc_quantity_chandra_spectrum(ilc_ctx* h, const float* rho, const float* u,
                                         const float* xe, uint64_t n, float redshift,
                                         float luminosity_distance, const float* energies,
                                         const float* widths, int32_t n_bins, float* out,
                                         int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (!c.has_arf) return fail(c, ILC_ERR_NO_ARF_TABLE, "ARF table not loaded");
  if (n == 0) return ILC_OK;
  if (!out || !energies || !widths || n_bins < 1)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid chandra_spectrum arguments");
  const float *a, *b, *d;
  ilc_status st = chandra_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  std::vector<float> ed(2 * (size_t)n_bins);
  std::memcpy(ed.data(), energies, 4 * (size_t)n_bins);
  std::memcpy(ed.data() + n_bins, widths, 4 * (size_t)n_bins);
  ILC_CUDA(c, c.out_c.ensure(8 * (size_t)n_bins), "bin table");
  ILC_CUDA(c, cudaMemcpyAsync(c.out_c.p, ed.data(), 8 * (size_t)n_bins, cudaMemcpyHostToDevice,
                              c.stream), "bin table H2D");
  void* dout = nullptr;
  const size_t bytes = n * (size_t)n_bins * 4;
  ILC_CUDA(c, out_ptr(c.out_a, out, bytes, is_device, &dout), "out");
  ILC_CUDA(c, quantity_chandra_bins_launch(c, a, b, d, n, redshift, luminosity_distance,
                                           c.out_c.as<float>(), c.out_c.as<float>() + n_bins,
                                           n_bins, static_cast<float*>(dout)),
           "chandra_spectrum kernel");
  ILC_CUDA(c, finish_out(c, out, dout, bytes, is_device), "chandra_spectrum");
  return ILC_OK;
}

ilc_status ilc_quantity_temperature(ilc_ctx* h, const float* u, const float* xe, uint64_t n,
                                    float* out, int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (n == 0) return ILC_OK;
  if (!u || !xe || !out) return fail(c, ILC_ERR_INVALID_ARGUMENT, "null array");
  const float *a, *b, *d;
  ilc_status st = quantity_inputs(c, nullptr, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  void* dout = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, out, n * 4, is_device, &dout), "out");
  ILC_CUDA(c, quantity_temperature_launch(c, b, d, n, static_cast<float*>(dout)),
           "temperature kernel");
  ILC_CUDA(c, finish_out(c, out, dout, n * 4, is_device), "temperature");
  return ILC_OK;
}

ilc_status ilc_camera_plane(const ilc_camera* cam, float* out13) {
  if (!camera_ok(cam) || !out13) return ILC_ERR_INVALID_ARGUMENT;
  camera_plane(*cam, out13);
  return ILC_OK;
}

ilc_status ilc_render_adaptive(ilc_ctx* h, const ilc_camera* cam, double z_range,
                               ilc_tolerance tol, int32_t controller,
                               const ilc_los_scaling* scaling, float* image, int is_device,
                               ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  cudaSetDevice(h->c.device);
  return render_common(h->c, cam, z_range, tol, controller, 0, scaling, image, is_device, stats);
}

ilc_status ilc_render_fixed(ilc_ctx* h, const ilc_camera* cam, double z_range, int64_t num_steps,
                            const ilc_los_scaling* scaling, float* image, int is_device,
                            ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  cudaSetDevice(h->c.device);
  if (num_steps <= 0) return fail(h->c, ILC_ERR_INVALID_ARGUMENT, "num_steps must be > 0");
  return render_common(h->c, cam, z_range, ilc_tolerance{0.0, 0.0}, ILC_CONTROLLER_REF32,
                       num_steps, scaling, image, is_device, stats);
}

ilc_status ilc_render_record(ilc_ctx* h, const ilc_camera* cam, double z_range,
                             ilc_tolerance tol, int32_t controller, float* step_sizes,
                             int32_t* n_steps, int64_t capacity, int steps_on_device,
                             float* image, int is_device, ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!camera_ok(cam) || !step_sizes || !n_steps || capacity <= 0)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid step recording arguments");
  const uint64_t rays = (uint64_t)cam->num_pix_x * (uint64_t)cam->num_pix_y;
  void *dh = nullptr, *dn = nullptr;
  ILC_CUDA(c, out_ptr(c.out_b, step_sizes, rays * (uint64_t)capacity * 4, steps_on_device, &dh),
           "step buffer");
  ILC_CUDA(c, out_ptr(c.out_c, n_steps, rays * 4, steps_on_device, &dn), "step counts");
  StepArrays sa;
  sa.rec_h = static_cast<float*>(dh);
  sa.rec_n = static_cast<int32_t*>(dn);
  sa.cap = capacity;
  ilc_status st = render_common(c, cam, z_range, tol, controller, 0, nullptr, image, is_device,
                                stats, sa);
  ILC_CUDA(c, finish_out(c, step_sizes, dh, rays * (uint64_t)capacity * 4, steps_on_device),
           "step buffer D2H");
  ILC_CUDA(c, finish_out(c, n_steps, dn, rays * 4, steps_on_device), "step counts D2H");
  return st;
}

ilc_status ilc_render_ray_stats(ilc_ctx* h, const ilc_camera* cam, double z_range,
                                ilc_tolerance tol, int32_t controller,
                                const ilc_los_scaling* scaling, float* image,
                                uint64_t* ray_stats, int is_device, ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!camera_ok(cam) || !ray_stats)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid per-ray statistics arguments");
  const uint64_t bytes = (uint64_t)cam->num_pix_x * (uint64_t)cam->num_pix_y * 32;
  void* dr = nullptr;
  ILC_CUDA(c, out_ptr(c.out_b, ray_stats, bytes, is_device, &dr), "ray statistics buffer");
  StepArrays sa;
  sa.ray_stats = static_cast<uint64_t*>(dr);
  ilc_status st = render_common(c, cam, z_range, tol, controller, 0, scaling, image, is_device,
                                stats, sa);
  ILC_CUDA(c, finish_out(c, ray_stats, dr, bytes, is_device), "ray statistics D2H");
  return st;
}

static ilc_status render_frozen_common(ilc_ctx* h, const ilc_camera* cam, double z_range,
                                       const float* step_sizes, const int32_t* n_steps,
                                       int64_t capacity, int steps_on_device,
                                       const ilc_los_scaling* scaling, float* image,
                                       double* image_d, int is_device, ilc_render_stats* stats);

ilc_status ilc_render_frozen(ilc_ctx* h, const ilc_camera* cam, double z_range,
                             const float* step_sizes, const int32_t* n_steps, int64_t capacity,
                             int steps_on_device, const ilc_los_scaling* scaling, float* image,
                             int is_device, ilc_render_stats* stats) {
  if (!image) return ILC_ERR_INVALID_ARGUMENT;
  return render_frozen_common(h, cam, z_range, step_sizes, n_steps, capacity, steps_on_device,
                              scaling, image, nullptr, is_device, stats);
}

ilc_status ilc_render_frozen_f64(ilc_ctx* h, const ilc_camera* cam, double z_range,
                                 const float* step_sizes, const int32_t* n_steps,
                                 int64_t capacity, int steps_on_device,
                                 const ilc_los_scaling* scaling, double* image, int is_device,
                                 ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!image || !camera_ok(cam)) return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid image");
  const uint64_t bytes = (uint64_t)cam->num_pix_x * (uint64_t)cam->num_pix_y * 8;
  void* dimg = nullptr;
  ILC_CUDA(c, out_ptr(c.out_c, image, bytes, is_device, &dimg), "double image buffer");
  ilc_status st = render_frozen_common(h, cam, z_range, step_sizes, n_steps, capacity,
                                       steps_on_device, scaling, nullptr,
                                       static_cast<double*>(dimg), is_device, stats);
  if (st) return st;
  ILC_CUDA(c, finish_out(c, image, dimg, bytes, is_device), "double image D2H");
  return ILC_OK;
}

static ilc_status render_frozen_common(ilc_ctx* h, const ilc_camera* cam, double z_range,
                                       const float* step_sizes, const int32_t* n_steps,
                                       int64_t capacity, int steps_on_device,
                                       const ilc_los_scaling* scaling, float* image,
                                       double* image_d, int is_device, ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!camera_ok(cam) || !step_sizes || !n_steps || capacity <= 0)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid frozen sequence arguments");
  const uint64_t rays = (uint64_t)cam->num_pix_x * (uint64_t)cam->num_pix_y;
  std::vector<int32_t> hn;
  if (!steps_on_device) {  // a count beyond capacity would read past the ray's row
    hn.assign(n_steps, n_steps + rays);
    for (int32_t v : hn)
      if (v < 0 || v > capacity)
        return fail(c, ILC_ERR_INVALID_ARGUMENT, "n_steps outside [0, capacity]");
  }
  const void *dh = nullptr, *dn = nullptr;
  ILC_CUDA(c, stage_in(c, c.in_b, step_sizes, rays * (uint64_t)capacity * 4, steps_on_device,
                       &dh), "steps H2D");
  ILC_CUDA(c, stage_in(c, c.in_c, n_steps, rays * 4, steps_on_device, &dn), "counts H2D");
  StepArrays sa;
  sa.replay_h = static_cast<const float*>(dh);
  sa.replay_n = static_cast<const int32_t*>(dn);
  sa.cap = capacity;
  sa.out_d = image_d;
  return render_common(c, cam, z_range, ilc_tolerance{0.0, 0.0}, ILC_CONTROLLER_REF32, 0,
                       scaling, image, is_device, stats, sa);
}

float ilc_los_scale(const ilc_camera* cam, double z_range, const ilc_los_scaling* scaling) {
  if (!camera_ok(cam) || !scaling) return 0.0f;
  return los_scale(*cam, z_range, *scaling);
}

ilc_status ilc_project_xray_flux(ilc_ctx* h, const float* cells, const float* rho,
                                 const float* u, const float* xe, uint64_t n, float redshift,
                                 float luminosity_distance, float e_min, float e_max,
                                 int32_t num_samples, const ilc_camera* cam, double z_range,
                                 ilc_tolerance tol, int32_t controller,
                                 const ilc_los_scaling* scaling, float* image, int is_device,
                                 ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (!cells || !rho || !u || !xe || n == 0 || num_samples <= 0 || !(e_max >= e_min))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid band-map arguments");
  if (n >= (1ull << 31)) return fail(c, ILC_ERR_GRID_TOO_LARGE, "more than 2^31 particles");
  // Particle records are assembled in the context's staging buffer, whose q
  // slot the quantity kernel fills (stride 4) -- the crawler's packing step.
  ILC_CUDA(c, c.tmp_in.ensure(n * 16), "particle staging");
  ILC_CUDA(c, cudaMemcpyAsync(c.tmp_in.p, cells, n * 16,
                              is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                              c.stream),
           "cells copy");
  const float *a, *b, *d;
  ilc_status st = quantity_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  ILC_CUDA(c, quantity_xray_flux_launch(c, a, b, d, n, redshift, luminosity_distance, e_min,
                                        e_max, num_samples, c.tmp_in.as<float>() + 3, 4),
           "xray_flux kernel");
  st = build_grid_staged(c, n);
  if (st) return st;
  return render_common(c, cam, z_range, tol, controller, 0, scaling, image, is_device, stats);
}

uint64_t ilc_kernel_launches(const ilc_ctx* h) { return h ? h->c.launches : 0; }

ilc_status ilc_device_alloc(ilc_ctx* h, uint64_t bytes, void** out) {
  if (!h || !out) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  *out = nullptr;
  if (bytes == 0) return ILC_OK;
  cudaSetDevice(c.device);
  ILC_CUDA(c, cudaMalloc(out, bytes), "device alloc");
  return ILC_OK;
}

ilc_status ilc_device_free(ilc_ctx* h, void* p) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  if (!p) return ILC_OK;
  Context& c = h->c;
  cudaSetDevice(c.device);
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "device free");
  ILC_CUDA(c, cudaFree(p), "device free");
  return ILC_OK;
}

ilc_status ilc_copy(ilc_ctx* h, void* dst, const void* src, uint64_t bytes) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  if (bytes == 0) return ILC_OK;
  if (!dst || !src) return fail(c, ILC_ERR_INVALID_ARGUMENT, "null array");
  cudaSetDevice(c.device);
  ILC_CUDA(c, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c.stream), "copy");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "copy");
  return ILC_OK;
}

ilc_status ilc_nn8_query_stats(ilc_ctx* h, uint64_t* cells_visited, uint64_t* candidates) {
  if (!h || !cells_visited || !candidates) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.flags.p) return fail(c, ILC_ERR_INVALID_ARGUMENT, "no query has run on this context");
  uint32_t flags = 0;
  DevStats ds{};
  ilc_status st = read_flags(c, &flags, &ds);
  if (st) return st;
  *cells_visited = ds.cells;
  *candidates = ds.cands;
  return ILC_OK;
}

ilc_status ilc_set_query_engine(ilc_ctx* h, int32_t engine) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  if (engine != ILC_QUERY_THREAD && engine != ILC_QUERY_WARP)
    return fail(h->c, ILC_ERR_INVALID_ARGUMENT, "unknown query engine");
  h->c.query_engine = engine;
  return ILC_OK;
}

ilc_status ilc_set_checkpoint_budget(ilc_ctx* h, uint64_t bytes) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  h->c.checkpoint_budget = bytes;  // 0: a quarter of the device's memory
  return ILC_OK;
}

ilc_status ilc_adjoint_xray_flux(ilc_ctx* h, const float* cells, const float* rho,
                                 const float* u, const float* xe, uint64_t n, float redshift,
                                 float luminosity_distance, float e_min, float e_max,
                                 int32_t num_samples, const ilc_camera* cam, double z_range,
                                 ilc_tolerance tol, int32_t controller,
                                 const ilc_los_scaling* scaling, const float* target, int32_t mode,
                                 float* image, float* dL_dlnrho, float* dL_dlnT, int is_device,
                                 ilc_adjoint_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (!cells || !rho || !u || !xe || !target || !image || !dL_dlnrho || !dL_dlnT || n == 0 ||
      num_samples <= 0 || !(e_max >= e_min) || !camera_ok(cam) || !(z_range > 0.0) ||
      !std::isfinite(z_range))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid adjoint arguments");
  if (mode != ILC_ADJOINT_CHECKPOINT && mode != ILC_ADJOINT_RECOMPUTE)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "unknown adjoint mode");
  if (controller != ILC_CONTROLLER_REF32 && controller != ILC_CONTROLLER_FP64)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "unknown controller");
  if (!(tol.absolute >= 0.0) || !(tol.relative >= 0.0) ||
      (tol.absolute <= 0.0 && tol.relative <= 0.0))
    return fail(c, ILC_ERR_INVALID_ARGUMENT,
                "either the absolute or the relative tolerance has to be > 0");
  if (n >= (1ull << 31)) return fail(c, ILC_ERR_GRID_TOO_LARGE, "more than 2^31 particles");
  const int64_t npix = (int64_t)cam->num_pix_x * cam->num_pix_y;
  cudaEvent_t q0, q1;
  ILC_CUDA(c, cudaEventCreate(&q0), "event");
  ILC_CUDA(c, cudaEventCreate(&q1), "event");
  // 1. per-cell q (into the particles' q slot), dq/dln T, dq/dln rho
  ILC_CUDA(c, c.tmp_in.ensure(n * 16), "particle staging");
  ILC_CUDA(c, cudaMemcpyAsync(c.tmp_in.p, cells, n * 16,
                              is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                              c.stream),
           "cells copy");
  const float *a, *b, *d;
  ilc_status st = quantity_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  ILC_CUDA(c, c.adj_dT.ensure(n * 4), "dq/dlnT");
  ILC_CUDA(c, c.adj_dR.ensure(n * 4), "dq/dlnrho");
  cudaEventRecord(q0, c.stream);
  ILC_CUDA(c, adjoint_cell_launch(c, a, b, d, n, redshift, luminosity_distance, e_min, e_max,
                                  num_samples, c.tmp_in.as<float>() + 3, 4, c.adj_dT.as<float>(),
                                  c.adj_dR.as<float>()),
           "xray_flux derivative kernel");
  cudaEventRecord(q1, c.stream);
  // 2. grid
  st = build_grid_staged(c, n);
  if (st) return st;
  // 3-5. forward render (recording the accepted steps in CHECKPOINT mode),
  // loss and per-pixel seed, adjoint rays: in bands of pixel rows whose step
  // checkpoints (4 B x (ceil(z_range / 0.2 kpc) + 2) per ray, the most
  // accepted steps a ray can take at the minimum step) fit the context's
  // checkpoint budget. The seed of a pixel depends only on its own value, so
  // each band runs forward -> seed -> adjoint before the next one starts.
  RenderArgs ra{};
  camera_plane(*cam, ra.cam);
  ra.nx = cam->num_pix_x;
  ra.ny = cam->num_pix_y;
  ra.z0 = 0.0f;
  ra.z_end = (float)z_range;
  ra.atol = tol.absolute;
  ra.rtol = tol.relative;
  ra.controller = controller;
  ra.apply_scale = scaling != nullptr;
  ra.scale = scaling ? los_scale(*cam, z_range, *scaling) : 1.0f;
  ILC_CUDA(c, c.out_b.ensure((size_t)npix * 4), "image");
  ra.out = c.out_b.as<float>();
  int32_t band_rows = ra.ny;
  if (mode == ILC_ADJOINT_CHECKPOINT) {
    ra.rec_cap = (int64_t)std::ceil(z_range / 0.2) + 2;
    const uint64_t per_row = (uint64_t)ra.nx * (uint64_t)ra.rec_cap * 4;
    uint64_t budget = c.checkpoint_budget;
    if (budget == 0) {
      size_t free_b = 0, total_b = 0;
      ILC_CUDA(c, cudaMemGetInfo(&free_b, &total_b), "device memory size");
      budget = total_b / 4;
    }
    const uint64_t fit = budget / per_row;
    band_rows = (int32_t)std::min<uint64_t>((uint64_t)ra.ny, std::max<uint64_t>(8, fit / 8 * 8));
    ILC_CUDA(c, c.rec_h.ensure((size_t)band_rows * per_row),
             "step checkpoints (use ILC_ADJOINT_RECOMPUTE to avoid them)");
    ILC_CUDA(c, c.rec_n.ensure((size_t)band_rows * ra.nx * 4), "step counts");
    ra.rec_h = c.rec_h.as<float>();
    ra.rec_n = c.rec_n.as<int32_t>();
  }
  const void* dtarget = nullptr;
  ILC_CUDA(c, stage_in(c, c.in_a, target, (size_t)npix * 4, is_device, &dtarget), "target");
  ILC_CUDA(c, c.adj_seed.ensure((size_t)npix * 4), "seed");
  ILC_CUDA(c, c.adj_loss.ensure(8), "loss");
  ILC_CUDA(c, cudaMemsetAsync(c.adj_loss.p, 0, 8, c.stream), "loss");
  ILC_CUDA(c, c.adj_grad.ensure(n * 8), "gradient");
  ILC_CUDA(c, cudaMemsetAsync(c.adj_grad.p, 0, n * 8, c.stream), "gradient");
  float fwd_ms = 0.0f, adj_ms = 0.0f;
  uint64_t fwd_steps = 0, adj_steps = 0;
  uint32_t flags = 0;
  for (int32_t row0 = 0; row0 < ra.ny; row0 += band_rows) {
    ra.row0 = row0;
    ra.rows = std::min(band_rows, ra.ny - row0);
    float ms = 0.0f;
    ILC_CUDA(c, render_launch(c, ra, &ms), "forward render");
    fwd_ms += ms;
    DevStats fs{};
    st = read_flags(c, &flags, &fs);
    if (st) return st;
    if (flags & FLAG_STEP_LIMIT)
      return fail(c, ILC_ERR_STEP_LIMIT, "rays reached the step limit");
    if (flags & FLAG_REC_OVERFLOW) return fail(c, ILC_ERR_INTERNAL, "step checkpoint overflow");
    fwd_steps += fs.steps;
    const size_t off = (size_t)row0 * ra.nx;
    ILC_CUDA(c, adjoint_seed_launch(c, ra.out + off, static_cast<const float*>(dtarget) + off,
                                    (int64_t)ra.rows * ra.nx, ra.scale,
                                    c.adj_seed.as<float>() + off, c.adj_loss.as<double>(),
                                    false),
             "loss kernel");
    ILC_CUDA(c, adjoint_ray_launch(c, ra, mode, c.adj_seed.as<float>(), c.adj_grad.as<double>(),
                                   &ms),
             "adjoint kernel");
    adj_ms += ms;
    DevStats as{};
    st = read_flags(c, &flags, &as);
    if (st) return st;
    if (flags & FLAG_STEP_LIMIT)
      return fail(c, ILC_ERR_STEP_LIMIT, "rays reached the step limit");
    adj_steps += as.steps;
  }
  // 6. chain rule into the caller's arrays
  void *gr = nullptr, *gt = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, dL_dlnrho, n * 4, is_device, &gr), "dL/dlnrho");
  ILC_CUDA(c, out_ptr(c.out_c, dL_dlnT, n * 4, is_device, &gt), "dL/dlnT");
  ILC_CUDA(c, adjoint_chain_launch(c, c.adj_grad.as<double>(), n, c.adj_dR.as<float>(),
                                   c.adj_dT.as<float>(), static_cast<float*>(gr),
                                   static_cast<float*>(gt)),
           "chain rule kernel");
  const cudaMemcpyKind k = is_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  ILC_CUDA(c, cudaMemcpyAsync(image, ra.out, (size_t)npix * 4, k, c.stream), "image out");
  if (!is_device) {
    ILC_CUDA(c, cudaMemcpyAsync(dL_dlnrho, gr, n * 4, cudaMemcpyDeviceToHost, c.stream), "D2H");
    ILC_CUDA(c, cudaMemcpyAsync(dL_dlnT, gt, n * 4, cudaMemcpyDeviceToHost, c.stream), "D2H");
  }
  double loss = 0.0;
  ILC_CUDA(c, cudaMemcpyAsync(&loss, c.adj_loss.p, 8, cudaMemcpyDeviceToHost, c.stream), "loss");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "adjoint");
  float qms = 0.0f;
  cudaEventElapsedTime(&qms, q0, q1);
  cudaEventDestroy(q0);
  cudaEventDestroy(q1);
  if (stats) {
    stats->loss = loss;
    stats->quantity_ms = qms;
    stats->forward_ms = fwd_ms;
    stats->adjoint_ms = adj_ms;
    stats->forward_steps = fwd_steps;
    stats->adjoint_steps = adj_steps;
  }
  return ILC_OK;
}

ilc_status ilc_autotune_render(ilc_ctx* h, const ilc_camera* cam, double z_range,
                               ilc_tolerance tol, int32_t controller, const float* windows,
                               int32_t n_windows, const int32_t* occupancies,
                               int32_t n_occupancies, int32_t sample_stride, float* best_window,
                               int32_t* best_occupancy, float* times_ms) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "autotune before setup_particles");
  if (!camera_ok(cam) || !windows || n_windows <= 0 || !occupancies || n_occupancies <= 0 ||
      sample_stride <= 0 || !best_window || !best_occupancy || !(z_range > 0.0))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid autotune arguments");
  RenderArgs a{};
  camera_plane(*cam, a.cam);
  a.nx = cam->num_pix_x;
  a.ny = cam->num_pix_y;
  a.z0 = 0.0f;
  a.z_end = (float)z_range;
  a.atol = tol.absolute;
  a.rtol = tol.relative;
  a.controller = controller;
  a.apply_scale = false;
  a.scale = 1.0f;
  a.row_stride = sample_stride;
  ILC_CUDA(c, c.out_b.ensure((size_t)a.nx * (size_t)a.ny * 4), "autotune image");
  a.out = c.out_b.as<float>();
  float best_ms = 0.0f;
  bool first = true;
  for (int32_t i = 0; i < n_windows; ++i) {
    if (!(windows[i] >= 0.0f) || !std::isfinite(windows[i]))
      return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid z window candidate");
    for (int32_t j = 0; j < n_occupancies; ++j) {
      if (occupancies[j] != 0 && occupancies[j] != 3 && occupancies[j] != 4 && occupancies[j] != 5)
        return fail(c, ILC_ERR_INVALID_ARGUMENT, "occupancy must be 0, 3, 4 or 5");
      a.window_override = windows[i];
      a.occupancy_override = occupancies[j];
      float ms = 0.0f;
      ILC_CUDA(c, render_launch(c, a, &ms), "autotune render");
      uint32_t flags = 0;
      ilc_status st = read_flags(c, &flags, nullptr);
      if (st) return st;
      if (flags & FLAG_STEP_LIMIT)
        return fail(c, ILC_ERR_STEP_LIMIT, "rays reached the per-ray step limit");
      if (times_ms) times_ms[i * n_occupancies + j] = ms;
      if (first || ms < best_ms) {
        first = false;
        best_ms = ms;
        *best_window = windows[i];
        *best_occupancy = occupancies[j];
      }
    }
  }
  c.z_window = *best_window;
  c.render_occupancy = *best_occupancy;
  return ILC_OK;
}


ilc_status ilc_quantity_xray_spectrum(ilc_ctx* h, const float* rho, const float* u,
                                      const float* xe, uint64_t n, float redshift,
                                      float luminosity_distance, const float* energies,
                                      const float* widths, int32_t n_bins, float* out,
                                      int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_gaunt) return fail(c, ILC_ERR_NO_GAUNT_TABLE, "Gaunt table not loaded");
  if (n == 0) return ILC_OK;
  if (!rho || !u || !xe || !out || !energies || !widths || n_bins < 1)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid xray_spectrum arguments");
  const float *a, *b, *d;
  ilc_status st = quantity_inputs(c, rho, u, xe, n, is_device, &a, &b, &d);
  if (st) return st;
  std::vector<float> ed(2 * (size_t)n_bins);
  std::memcpy(ed.data(), energies, 4 * (size_t)n_bins);
  std::memcpy(ed.data() + n_bins, widths, 4 * (size_t)n_bins);
  ILC_CUDA(c, c.out_c.ensure(8 * (size_t)n_bins), "bin table");
  ILC_CUDA(c, cudaMemcpyAsync(c.out_c.p, ed.data(), 8 * (size_t)n_bins, cudaMemcpyHostToDevice,
                              c.stream), "bin table H2D");
  void* dout = nullptr;
  const size_t bytes = n * (size_t)n_bins * 4;
  ILC_CUDA(c, out_ptr(c.out_a, out, bytes, is_device, &dout), "out");
  ILC_CUDA(c, quantity_xray_bins_launch(c, a, b, d, n, redshift, luminosity_distance,
                                        c.out_c.as<float>(), c.out_c.as<float>() + n_bins,
                                        n_bins, static_cast<float*>(dout)),
           "xray_spectrum kernel");
  ILC_CUDA(c, finish_out(c, out, dout, bytes, is_device), "xray_spectrum");
  return ILC_OK;
}

ilc_status ilc_set_batch_schedule(ilc_ctx* h, int32_t tile_w, int32_t blocks_per_sm,
                                  float z_window, int32_t cost_order) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  if (!tile_w_ok(tile_w) || (blocks_per_sm != 0 && blocks_per_sm != 3 && blocks_per_sm != 4 && blocks_per_sm != 5) ||
      !(z_window >= 0.0f) || !std::isfinite(z_window))
    return fail(h->c, ILC_ERR_INVALID_ARGUMENT,
                "tile_w 0 or 1..32 (powers of 2), occupancy 0, 3, 4 or 5, z_window >= 0");
  h->c.batch_tile_w = tile_w;
  h->c.batch_occupancy = blocks_per_sm;
  h->c.batch_window = z_window;
  h->c.batch_cost_order = cost_order != 0;
  return ILC_OK;
}

ilc_status ilc_render_batched(ilc_ctx* h, const float* values, int32_t n_channels,
                              int values_on_device, const ilc_job* jobs, int32_t n_jobs,
                              ilc_tolerance tol, float* images, uint64_t images_len,
                              int images_on_device, ilc_render_stats* stats) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!images || images_len == 0)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid images buffer");
  BatchArgs a{};
  ilc_status st = batched_prepare(c, values, n_channels, values_on_device, jobs, n_jobs, tol,
                                  images_len, &a);
  if (st) return st;
  void* dimg = nullptr;
  ILC_CUDA(c, out_ptr(c.out_b, images, images_len * 4, images_on_device, &dimg), "images");
  a.out = static_cast<float*>(dimg);
  float ms = 0.0f;
  ILC_CUDA(c, batched_launch(c, a, &ms), "batched render kernel");
  ILC_CUDA(c, finish_out(c, images, dimg, images_len * 4, images_on_device), "batched render");
  uint32_t flags = 0;
  DevStats ds{};
  st = read_flags(c, &flags, &ds);
  if (st) return st;
  if (stats) {
    stats->steps = ds.steps;
    stats->accepted_steps = ds.accepted;
    stats->queries = ds.queries;
    stats->cells_visited = ds.cells;
    stats->candidates = ds.cands;
    stats->max_steps_per_ray = ds.max_steps;
    stats->rays_at_step_limit = ds.rays_at_limit;
    stats->kernel_ms = ms;
  }
  if (flags & FLAG_STEP_LIMIT)
    return fail(c, ILC_ERR_STEP_LIMIT, "rays reached the per-ray step limit");
  return ILC_OK;
}

ilc_status ilc_autotune_batched(ilc_ctx* h, const float* values, int32_t n_channels,
                                int values_on_device, const ilc_job* jobs, int32_t n_jobs,
                                ilc_tolerance tol, const int32_t* tile_ws, int32_t n_tiles,
                                const int32_t* occupancies, int32_t n_occupancies,
                                const float* windows, int32_t n_windows, int32_t* best_tile_w,
                                int32_t* best_occupancy, float* best_window, float* times_ms) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!tile_ws || n_tiles < 1 || !occupancies || n_occupancies < 1 || !windows ||
      n_windows < 1 || !best_tile_w || !best_occupancy || !best_window || !jobs || n_jobs < 1)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid autotune arguments");
  for (int32_t i = 0; i < n_tiles; ++i)
    if (!tile_w_ok(tile_ws[i])) return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid tile_w");
  for (int32_t i = 0; i < n_occupancies; ++i)
    if (occupancies[i] != 0 && occupancies[i] != 3 && occupancies[i] != 4 && occupancies[i] != 5)
      return fail(c, ILC_ERR_INVALID_ARGUMENT, "occupancy must be 0, 3, 4 or 5");
  for (int32_t i = 0; i < n_windows; ++i)
    if (!(windows[i] >= 0.0f) || !std::isfinite(windows[i]))
      return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid z window");
  uint64_t len = 0;
  for (int32_t k = 0; k < n_jobs; ++k) {
    const uint64_t e = jobs[k].out_offset + (uint64_t)n_channels *
                                                (uint64_t)jobs[k].camera.num_pix_x *
                                                (uint64_t)jobs[k].camera.num_pix_y;
    len = std::max(len, e);
  }
  const int32_t keep_w = c.batch_tile_w, keep_o = c.batch_occupancy;
  const float keep_z = c.batch_window;
  const bool keep_order = c.batch_cost_order;
  auto restore = [&]() {
    c.batch_tile_w = keep_w;
    c.batch_occupancy = keep_o;
    c.batch_window = keep_z;
    c.batch_cost_order = keep_order;
  };
  float best = 0.0f;
  bool first = true;
  for (int32_t i = 0; i < n_tiles; ++i) {
    for (int32_t j = 0; j < n_occupancies; ++j) {
      for (int32_t q = 0; q < n_windows; ++q) {
        c.batch_tile_w = tile_ws[i];
        c.batch_occupancy = occupancies[j];
        c.batch_window = windows[q];
        c.batch_cost_order = true;
        BatchArgs a{};
        ilc_status st = batched_prepare(c, values, n_channels, values_on_device, jobs, n_jobs,
                                        tol, len, &a);
        if (st) {
          restore();
          return st;
        }
        ILC_CUDA(c, c.out_b.ensure(len * 4), "autotune images");
        a.out = c.out_b.as<float>();
        float ms = 0.0f;
        ILC_CUDA(c, batched_launch(c, a, &ms), "autotune batched kernel");
        uint32_t flags = 0;
        st = read_flags(c, &flags, nullptr);
        if (st) {
          restore();
          return st;
        }
        if (flags & FLAG_STEP_LIMIT) {
          restore();
          return fail(c, ILC_ERR_STEP_LIMIT, "rays reached the per-ray step limit");
        }
        if (times_ms) times_ms[(i * n_occupancies + j) * n_windows + q] = ms;
        if (first || ms < best) {
          first = false;
          best = ms;
          *best_tile_w = tile_ws[i];
          *best_occupancy = occupancies[j];
          *best_window = windows[q];
        }
      }
    }
  }
  c.batch_tile_w = *best_tile_w;
  c.batch_occupancy = *best_occupancy;
  c.batch_window = *best_window;
  c.batch_cost_order = true;
  return ILC_OK;
}


ilc_status ilc_ingest_cells(ilc_ctx* h, const float* xyz, const float* q, uint64_t n,
                            const double* center, const double* extent, const double* periodic,
                            double border, float* out_xyzq, uint32_t* out_index,
                            uint64_t* n_out, int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!n_out) return fail(c, ILC_ERR_INVALID_ARGUMENT, "n_out is NULL");
  *n_out = 0;
  if (n == 0) return ILC_OK;
  if (!xyz || !center || !extent || !periodic || !out_xyzq)
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid ingest arguments");
  if (n >= (1ull << 32)) return fail(c, ILC_ERR_INVALID_ARGUMENT, "at most 2^32 - 1 cells");
  CutoutParams p;
  for (int j = 0; j < 3; ++j) {
    if (!std::isfinite(center[j]) || !(extent[j] >= 0.0) || !std::isfinite(extent[j]) ||
        !(periodic[j] >= 0.0) || !std::isfinite(periodic[j]))
      return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid cutout center, extent or period");
    // volume_cutout bounding box and the border-widened box of correct_periodicity
    p.lo[j] = center[j] - 0.5 * extent[j];
    p.hi[j] = center[j] + 0.5 * extent[j];
    p.glo[j] = p.lo[j] - border;
    p.ghi[j] = p.hi[j] + border;
    p.period[j] = periodic[j];
  }
  if (!(border >= 0.0) || !std::isfinite(border))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid border");
  const void *dx = nullptr, *dq = nullptr;
  ILC_CUDA(c, stage_in(c, c.in_a, xyz, n * 12, is_device, &dx), "cells H2D");
  if (q) ILC_CUDA(c, stage_in(c, c.in_b, q, n * 4, is_device, &dq), "quantity H2D");
  void *dout = nullptr, *didx = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, out_xyzq, n * 16, is_device, &dout), "ingest output");
  if (out_index) ILC_CUDA(c, out_ptr(c.out_b, out_index, n * 4, is_device, &didx), "index output");
  ILC_CUDA(c, c.out_c.ensure(64), "count");
  ILC_CUDA(c, ingest_launch(c, static_cast<const float*>(dx), static_cast<const float*>(dq), n, p,
                            static_cast<float4*>(dout), static_cast<uint32_t*>(didx),
                            c.out_c.as<unsigned long long>()),
           "ingest kernels");
  unsigned long long kept = 0;
  ILC_CUDA(c, cudaMemcpyAsync(&kept, c.out_c.p, 8, cudaMemcpyDeviceToHost, c.stream), "count D2H");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "ingest");
  if (!is_device) {
    ILC_CUDA(c, cudaMemcpyAsync(out_xyzq, dout, kept * 16, cudaMemcpyDeviceToHost, c.stream),
             "ingest output D2H");
    if (out_index)
      ILC_CUDA(c, cudaMemcpyAsync(out_index, didx, kept * 4, cudaMemcpyDeviceToHost, c.stream),
               "index output D2H");
    ILC_CUDA(c, cudaStreamSynchronize(c.stream), "ingest");
  }
  *n_out = kept;
  return ILC_OK;
}


ilc_status ilc_volumetric_slice(ilc_ctx* h, const ilc_camera* cam, double dV,
                                int32_t additional_samples, uint64_t seed, float* image,
                                int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "slice before setup_particles");
  if (!camera_ok(cam) || !image || additional_samples < 0 || !std::isfinite(dV))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid slice arguments");
  float f[13];
  double d[13];
  camera_plane(*cam, f, d);
  const uint64_t npix = (uint64_t)cam->num_pix_x * (uint64_t)cam->num_pix_y;
  void* dimg = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, image, npix * 4, is_device, &dimg), "slice image");
  ILC_CUDA(c, slice_launch(c, d, cam->num_pix_x, cam->num_pix_y, additional_samples + 1, seed, dV,
                           static_cast<float*>(dimg)),
           "slice kernels");
  ILC_CUDA(c, finish_out(c, image, dimg, npix * 4, is_device), "slice");
  return ILC_OK;
}


ilc_status ilc_volumetric_tomography(ilc_ctx* h, const ilc_camera* cam, double dV,
                                     int64_t initial_z_step, int64_t num_steps, float* cube,
                                     int is_device) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "tomography before setup_particles");
  if (!camera_ok(cam) || !cube || initial_z_step < 0 || num_steps < 0 || !std::isfinite(dV))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid tomography arguments");
  if (num_steps == 0) return ILC_OK;
  const uint64_t npix = (uint64_t)cam->num_pix_x * (uint64_t)cam->num_pix_y;
  void* dcube = nullptr;
  ILC_CUDA(c, out_ptr(c.out_a, cube, npix * (uint64_t)num_steps * 4, is_device, &dcube),
           "tomography cube");
  const double ps = cam->screen_width / (double)cam->num_pix_x;
  for (int64_t z = 0; z < num_steps; ++z) {
    // camera moved along look_at by (initial + z) pixel sizes (volumetric_tomography.cpp:81-82)
    ilc_camera mc = *cam;
    const double t = (double)(initial_z_step + z) * ps;
    for (int j = 0; j < 3; ++j) mc.position[j] = cam->position[j] + t * cam->look_at[j];
    float f[13];
    double d[13];
    camera_plane(mc, f, d);
    ILC_CUDA(c, slice_launch(c, d, cam->num_pix_x, cam->num_pix_y, 1, 0, dV,
                             static_cast<float*>(dcube) + (uint64_t)z * npix),
             "tomography slice");
  }
  ILC_CUDA(c, finish_out(c, cube, dcube, npix * (uint64_t)num_steps * 4, is_device), "tomography");
  return ILC_OK;
}

ilc_status ilc_mc_profile_shells(double max_radius, int32_t num_radii, double sample_density,
                                 double* radii, uint64_t* counts) {
  ProfileShells S;
  if (!profile_shells(max_radius, num_radii, sample_density, &S))
    return ILC_ERR_INVALID_ARGUMENT;
  for (int32_t i = 0; i < num_radii; ++i) {
    if (radii) radii[i] = S.radius[i];
    if (counts) counts[i] = S.count[i];
  }
  return ILC_OK;
}

ilc_status ilc_mc_profile_points(const double center[3], double max_radius, int32_t num_radii,
                                 double sample_density, uint64_t seed, uint64_t first,
                                 uint64_t count, float* points) {
  ProfileShells S;
  if (!center || (count > 0 && !points) ||
      !profile_shells(max_radius, num_radii, sample_density, &S))
    return ILC_ERR_INVALID_ARGUMENT;
  const uint64_t total = S.prefix[(size_t)num_radii];
  if (first > total || count > total - first) return ILC_ERR_INVALID_ARGUMENT;
  for (uint64_t k = 0; k < count; ++k) {
    const uint64_t g = first + k;
    const int s = find_shell(S.prefix.data(), num_radii, g);
    const ShellPoint p = shell_sample(seed, g, S.u_min[s], S.u_max[s], center);
    points[4 * k + 0] = p.x;
    points[4 * k + 1] = p.y;
    points[4 * k + 2] = p.z;
    points[4 * k + 3] = 0.0f;
  }
  return ILC_OK;
}

ilc_status ilc_mc_radial_profile(ilc_ctx* h, const double center[3], double max_radius,
                                 int32_t num_radii, double sample_density, uint64_t seed,
                                 int32_t dV_mode, double volume_conversion, double* profile,
                                 float* sample_points, float* sample_values) {
  if (!h) return ILC_ERR_INVALID_ARGUMENT;
  Context& c = h->c;
  cudaSetDevice(c.device);
  if (!c.has_grid) return fail(c, ILC_ERR_NO_PARTICLES, "profile before setup_particles");
  if (!center || !profile || (dV_mode != ILC_DV_VOLUME && dV_mode != ILC_DV_MEAN) ||
      !std::isfinite(center[0]) || !std::isfinite(center[1]) || !std::isfinite(center[2]) ||
      !std::isfinite(volume_conversion))
    return fail(c, ILC_ERR_INVALID_ARGUMENT, "invalid profile arguments");
  ProfileShells S;
  if (!profile_shells(max_radius, num_radii, sample_density, &S))
    return fail(c, ILC_ERR_INVALID_ARGUMENT,
                "invalid profile shells (radius, 1..2^20 radii, density, at most 2^40 samples)");
  const uint32_t N = (uint32_t)num_radii;
  // device shell table: prefix (N + 1), u_min (N), u_max (N)
  std::vector<char> tab(8 * (size_t)(N + 1) + 16 * (size_t)N);
  uint64_t* t_prefix = reinterpret_cast<uint64_t*>(tab.data());
  double* t_umin = reinterpret_cast<double*>(tab.data() + 8 * (size_t)(N + 1));
  double* t_umax = t_umin + N;
  for (uint32_t i = 0; i <= N; ++i) t_prefix[i] = S.prefix[i];
  for (uint32_t i = 0; i < N; ++i) {
    t_umin[i] = S.u_min[i];
    t_umax[i] = S.u_max[i];
  }
  // reduction segments: at most kProfileSegment consecutive samples of one shell
  std::vector<ulonglong2> segs;
  std::vector<uint32_t> seg_shell;
  for (uint32_t i = 0; i < N; ++i)
    for (uint64_t b = S.prefix[i]; b < S.prefix[i + 1]; b += kProfileSegment) {
      segs.push_back(make_ulonglong2(b, std::min(b + kProfileSegment, S.prefix[i + 1])));
      seg_shell.push_back(i);
    }
  const uint64_t total = S.prefix[N];
  const uint64_t batch_cap = std::min(total, kProfileBatch);
  ILC_CUDA(c, c.prof_tab.ensure(tab.size()), "profile table");
  ILC_CUDA(c, c.prof_seg.ensure(segs.size() * sizeof(ulonglong2)), "profile segments");
  ILC_CUDA(c, c.prof_sum.ensure(segs.size() * 8), "profile sums");
  ILC_CUDA(c, c.in_b.ensure(batch_cap * 16), "profile points");
  ILC_CUDA(c, c.out_b.ensure(batch_cap * 4), "profile values");
  ILC_CUDA(c, cudaMemcpyAsync(c.prof_tab.p, tab.data(), tab.size(), cudaMemcpyHostToDevice,
                              c.stream), "profile table H2D");
  ILC_CUDA(c, cudaMemcpyAsync(c.prof_seg.p, segs.data(), segs.size() * sizeof(ulonglong2),
                              cudaMemcpyHostToDevice, c.stream), "profile segments H2D");
  const uint64_t* d_prefix = c.prof_tab.as<uint64_t>();
  const double* d_umin = reinterpret_cast<const double*>(c.prof_tab.as<char>() + 8 * (size_t)(N + 1));
  const double* d_umax = d_umin + N;
  size_t si = 0;
  while (si < segs.size()) {
    // a batch: the consecutive whole segments that fit in kProfileBatch samples
    const uint64_t g0 = segs[si].x;
    size_t sj = si;
    while (sj < segs.size() && segs[sj].y - g0 <= kProfileBatch) ++sj;
    const uint64_t n = segs[sj - 1].y - g0;
    ILC_CUDA(c, profile_points_launch(c, d_prefix, (int)N, d_umin, d_umax, center, seed, g0, n,
                                      c.in_b.as<float4>()),
             "profile points kernel");
    ILC_CUDA(c, nn8_query_launch(c, c.in_b.as<float4>(), n, false, c.out_b.as<float>(), nullptr,
                                 nullptr),
             "profile nn8 kernel");
    ILC_CUDA(c, profile_segment_sum_launch(c, c.prof_seg.as<ulonglong2>() + si,
                                           (uint32_t)(sj - si), g0, c.out_b.as<float>(),
                                           c.prof_sum.as<double>() + si),
             "profile reduction kernel");
    if (sample_points)
      ILC_CUDA(c, cudaMemcpyAsync(sample_points + 4 * g0, c.in_b.p, n * 16,
                                  cudaMemcpyDeviceToHost, c.stream), "profile points D2H");
    if (sample_values)
      ILC_CUDA(c, cudaMemcpyAsync(sample_values + g0, c.out_b.p, n * 4, cudaMemcpyDeviceToHost,
                                  c.stream), "profile values D2H");
    ILC_CUDA(c, cudaStreamSynchronize(c.stream), "profile batch");
    si = sj;
  }
  std::vector<double> seg_sum(segs.size());
  ILC_CUDA(c, cudaMemcpyAsync(seg_sum.data(), c.prof_sum.p, segs.size() * 8,
                              cudaMemcpyDeviceToHost, c.stream), "profile sums D2H");
  ILC_CUDA(c, cudaStreamSynchronize(c.stream), "profile");
  for (uint32_t i = 0; i < N; ++i) profile[i] = 0.0;
  for (size_t k = 0; k < segs.size(); ++k) profile[seg_shell[k]] += seg_sum[k];
  for (uint32_t i = 0; i < N; ++i) {
    // apply_volume_factor (profile.cpp:236-256)
    const double dV = S.volume[i] / (double)S.count[i];
    const double eff = dV_mode == ILC_DV_VOLUME
                           ? dV * volume_conversion
                           : (dV * volume_conversion) / (S.volume[i] * volume_conversion);
    profile[i] *= eff;
  }
  return ILC_OK;
}

}  // extern "C"
