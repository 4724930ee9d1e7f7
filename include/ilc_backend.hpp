// ilc_backend.hpp -- C++ adapter of the B200 backend to illcrawl's interfaces.
//
// Header-only, over the C ABI of ilc.h. It mirrors:
//   * reconstruction_backend / reconstruction_backends::nn8
//     (reconstruction_backend.hpp:35-58, volumetric_reconstruction_backend_nn8.hpp:36-82):
//     the abstract class reconstruction_backend and its implementation nn8_cuda,
//     with device_buffer (device memory owned through the library) in place of
//     cl::Buffer, so query results stay on the device as in the reference;
//   * volumetric_integration::create_projection (volumetric_integration.cpp:32-88):
//     function create_projection, which runs the whole RKF loop on the device.
// Errors are reported as exceptions (ilc::error), as the reference's
// qcl::check_cl_error / std::runtime_error do.
#ifndef ILC_BACKEND_HPP
#define ILC_BACKEND_HPP

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ilc.h"

namespace ilc {

class error : public std::runtime_error {
 public:
  error(ilc_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  ilc_status status;
};

// Owning handle of an ilc_ctx (one device, one stream).
class context {
 public:
  explicit context(int device = 0) : h_(ilc_create(device)) {
    if (!h_) throw error(ILC_ERR_CUDA, "ilc_create failed: no usable CUDA device");
  }
  ~context() { ilc_destroy(h_); }
  context(const context&) = delete;
  context& operator=(const context&) = delete;
  ilc_ctx* get() const { return h_; }
  void check(ilc_status s) const {
    if (s != ILC_OK) throw error(s, ilc_last_error(h_));
  }

 private:
  ilc_ctx* h_;
};

// A caller-owned array; on_device selects the pointer kind (ilc.h "is_device").
template <class T> struct view {
  T* ptr = nullptr;
  std::size_t n = 0;
  bool on_device = false;
};

// Device memory owned through the library (the role of cl::Buffer in the
// reference's backends). Move-only.
template <class T> class device_buffer {
 public:
  device_buffer() = default;
  device_buffer(context& ctx, std::size_t n) : ctx_(&ctx) { resize(n); }
  ~device_buffer() { release(); }
  device_buffer(const device_buffer&) = delete;
  device_buffer& operator=(const device_buffer&) = delete;
  device_buffer(device_buffer&& o) noexcept : ctx_(o.ctx_), p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  device_buffer& operator=(device_buffer&& o) noexcept {
    if (this != &o) {
      release();
      ctx_ = o.ctx_; p_ = o.p_; n_ = o.n_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  void bind(context& ctx) { ctx_ = &ctx; }
  // Grow-only: keeps the allocation when n fits (contents are not kept on growth).
  void resize(std::size_t n) {
    if (n <= cap_) {
      n_ = n;
      return;
    }
    if (!ctx_) throw error(ILC_ERR_INVALID_ARGUMENT, "device_buffer has no context");
    release();
    void* p = nullptr;
    ctx_->check(ilc_device_alloc(ctx_->get(), (uint64_t)(n * sizeof(T)), &p));
    p_ = static_cast<T*>(p);
    n_ = cap_ = n;
  }
  T* data() const { return p_; }
  std::size_t size() const { return n_; }
  view<const T> cview() const { return view<const T>{p_, n_, true}; }
  void copy_from_host(const T* src, std::size_t n) {
    resize(n);
    ctx_->check(ilc_copy(ctx_->get(), p_, src, (uint64_t)(n * sizeof(T))));
  }
  std::vector<T> to_host() const {
    std::vector<T> out(n_);
    if (n_) ctx_->check(ilc_copy(ctx_->get(), out.data(), p_, (uint64_t)(n_ * sizeof(T))));
    return out;
  }

 private:
  void release() {
    if (p_ && ctx_) ilc_device_free(ctx_->get(), p_);
    p_ = nullptr;
    n_ = cap_ = 0;
  }
  context* ctx_ = nullptr;
  T* p_ = nullptr;
  std::size_t n_ = 0, cap_ = 0;
};

// float4 particle record, the reference's device_vector4 (x, y, z, quantity).
struct particle {
  float s[4];
};

// reconstruction_backend (reconstruction_backend.hpp:35-58) with CUDA device
// buffers in place of cl::Buffer and dataset names in place of H5::DataSet
// handles: additional per-particle datasets arrive as float arrays in the
// order get_required_additional_datasets names them.
class reconstruction_backend {
 public:
  using particle = ilc::particle;
  virtual std::vector<std::string> get_required_additional_datasets() const = 0;
  virtual const device_buffer<float>& retrieve_results() = 0;
  virtual std::string get_backend_name() const = 0;
  virtual void init_backend(std::size_t blocksize) = 0;
  virtual void setup_particles(const std::vector<particle>& particles,
                               const std::vector<view<const float>>& additional_datasets) = 0;
  virtual void setup_evaluation_points(view<const float> evaluation_points,
                                       std::size_t num_points) = 0;
  virtual void run() = 0;
  virtual ~reconstruction_backend() {}
};

// reconstruction_backends::nn8 (volumetric_reconstruction_backend_nn8.hpp:36-82,
// volumetric_reconstruction_backend_nn8.cpp:26-141) over the CUDA context.
// As in the reference, the results stay on the device: retrieve_results()
// hands out the backend's own device buffer (one float per evaluation point),
// valid until the next setup_evaluation_points; results_to_host() copies it.
// Host evaluation points are staged into a device buffer once per
// setup_evaluation_points; device points are borrowed, as the reference
// borrows the caller's cl::Buffer.
class nn8_cuda : public reconstruction_backend {
 public:
  explicit nn8_cuda(context& ctx) : ctx_(ctx), points_dev_(), result_() {
    points_dev_.bind(ctx);
    result_.bind(ctx);
  }

  // No smoothing lengths or other per-particle datasets are needed
  // (volumetric_reconstruction_backend_nn8.cpp:32-35).
  std::vector<std::string> get_required_additional_datasets() const override { return {}; }
  std::string get_backend_name() const override { return "volumetric/nn8_cuda"; }
  void init_backend(std::size_t blocksize) override { blocksize_ = blocksize; }

  void setup_particles(const std::vector<particle>& particles,
                       const std::vector<view<const float>>& = {}) override {
    ctx_.check(ilc_nn8_setup_particles(ctx_.get(), &particles[0].s[0], particles.size(), 0));
  }
  // Particles already on the device (float4 each), or on the host.
  void setup_particles(view<const float> particles_float4) {
    ctx_.check(ilc_nn8_setup_particles(ctx_.get(), particles_float4.ptr, particles_float4.n,
                                       particles_float4.on_device ? 1 : 0));
  }

  void setup_evaluation_points(view<const float> points_float4,
                               std::size_t num_points) override {
    if (points_float4.on_device) {
      points_ = points_float4.ptr;
    } else {
      points_dev_.copy_from_host(points_float4.ptr, num_points * 4);
      points_ = points_dev_.data();
    }
    n_ = num_points;
    first_run_ = true;
    result_.resize(num_points);
  }

  // One particle block; later blocks merge into the running lists.
  void run() override {
    ctx_.check(ilc_nn8_query(ctx_.get(), points_, n_, first_run_ ? 0 : 1, result_.data(),
                             nullptr, nullptr, 1));
    first_run_ = false;
  }

  const device_buffer<float>& retrieve_results() override { return result_; }
  std::vector<float> results_to_host() const { return result_.to_host(); }

 private:
  context& ctx_;
  std::size_t blocksize_ = 0;
  const float* points_ = nullptr;
  std::size_t n_ = 0;
  bool first_run_ = true;
  device_buffer<float> points_dev_;
  device_buffer<float> result_;
};

// volumetric_integration::create_projection: output is num_pix_x * num_pix_y
// floats, row = y; quantities pick dA_mode as their
// effective_line_of_sight_integration_dA does.
inline ilc_render_stats create_projection(context& ctx, const ilc_camera& cam, double z_range,
                                          double abs_tol, double rel_tol,
                                          const ilc_los_scaling& scaling, std::vector<float>& out,
                                          int controller = ILC_CONTROLLER_FP64) {
  out.assign((std::size_t)cam.num_pix_x * (std::size_t)cam.num_pix_y, 0.0f);
  ilc_render_stats st{};
  ctx.check(ilc_render_adaptive(ctx.get(), &cam, z_range, ilc_tolerance{abs_tol, rel_tol},
                                controller, &scaling, out.data(), 0, &st));
  return st;
}

// The crawler's per-row loop (reconstructing_data_crawler.cpp:170-230): cells
// (x, y, z triples) periodically corrected and cut to the volume, kept cells in
// input order as particles with their q.
inline std::vector<particle> ingest_cells(context& ctx, const std::vector<float>& xyz,
                                          const std::vector<float>& q, const double center[3],
                                          const double extent[3], const double periodic[3],
                                          double border = 100.0,
                                          std::vector<uint32_t>* index = nullptr) {
  const uint64_t n = xyz.size() / 3;
  std::vector<particle> out(n);
  std::vector<uint32_t> idx(n);
  uint64_t kept = 0;
  ctx.check(ilc_ingest_cells(ctx.get(), xyz.data(), q.empty() ? nullptr : q.data(), n, center,
                             extent, periodic, border, reinterpret_cast<float*>(out.data()),
                             idx.data(), &kept, 0));
  out.resize(kept);
  if (index) {
    idx.resize(kept);
    *index = std::move(idx);
  }
  return out;
}

// multi_quantity_integrated_projection (animation.cpp:264-283) over a per-cell
// table of n_bins quantities (cell-major, n x n_bins): one batched render of
// every camera. cube: per camera, n_bins slices of num_pix_y x num_pix_x.
inline ilc_render_stats render_table(context& ctx, const std::vector<float>& table, int32_t nb,
                                     std::vector<ilc_job>& jobs, double rel_tol,
                                     std::vector<float>& cube) {
  uint64_t off = 0;
  for (auto& j : jobs) {
    j.out_offset = off;
    off += (uint64_t)nb * (uint64_t)j.camera.num_pix_x * (uint64_t)j.camera.num_pix_y;
  }
  cube.assign(off, 0.0f);
  ilc_render_stats st{};
  ctx.check(ilc_render_batched(ctx.get(), table.data(), nb, 0, jobs.data(), (int32_t)jobs.size(),
                               ilc_tolerance{0.0, rel_tol}, cube.data(), off, 0, &st));
  return st;
}

// spectrum_generator (spectrum.hpp:81-126) for X-ray spectra: the per-cell
// bin table, then render_table. The particles (cell positions) must be set
// up; rho, u, xe are the cells' fields in that order.
inline ilc_render_stats render_xray_spectra(context& ctx, const std::vector<float>& rho,
                                            const std::vector<float>& u,
                                            const std::vector<float>& xe, float redshift,
                                            float luminosity_distance,
                                            const std::vector<float>& energies,
                                            const std::vector<float>& widths,
                                            std::vector<ilc_job>& jobs, double rel_tol,
                                            std::vector<float>& cube) {
  const uint64_t n = rho.size();
  const int32_t nb = (int32_t)energies.size();
  std::vector<float> table(n * (uint64_t)nb);
  ctx.check(ilc_quantity_xray_spectrum(ctx.get(), rho.data(), u.data(), xe.data(), n, redshift,
                                       luminosity_distance, energies.data(), widths.data(), nb,
                                       table.data(), 0));
  return render_table(ctx, table, nb, jobs, rel_tol, cube);
}

// chandra::arf as util::tabulated_function (tabulated_function.hpp:35-103):
// the caller's effective-area samples [cm^2] from x_min [keV] in steps of dx.
inline void load_arf(context& ctx, const std::vector<float>& area, float x_min, float dx) {
  ctx.check(ilc_arf_load(ctx.get(), area.data(), (int32_t)area.size(), x_min, dx));
}

// spectrum_generator with chandra_spectrum_quantity_generator (spectrum.cpp:
// 45-65): channel count rates per cell, then render_table. Needs load_arf.
inline ilc_render_stats render_chandra_spectra(context& ctx, const std::vector<float>& rho,
                                               const std::vector<float>& u,
                                               const std::vector<float>& xe, float redshift,
                                               float luminosity_distance,
                                               const std::vector<float>& energies,
                                               const std::vector<float>& widths,
                                               std::vector<ilc_job>& jobs, double rel_tol,
                                               std::vector<float>& cube) {
  const uint64_t n = rho.size();
  const int32_t nb = (int32_t)energies.size();
  std::vector<float> table(n * (uint64_t)nb);
  ctx.check(ilc_quantity_chandra_spectrum(ctx.get(), rho.data(), u.data(), xe.data(), n,
                                          redshift, luminosity_distance, energies.data(),
                                          widths.data(), nb, table.data(), 0));
  return render_table(ctx, table, nb, jobs, rel_tol, cube);
}

// volumetric_slice::create_slice (volumetric_slice.cpp:31-101), one sample per
// pixel unless additional_samples > 0; image is num_pix_y x num_pix_x.
inline void volumetric_slice(context& ctx, const ilc_camera& cam, double dV,
                             std::vector<float>& image, int additional_samples = 0,
                             uint64_t seed = 0) {
  image.assign((std::size_t)cam.num_pix_x * (std::size_t)cam.num_pix_y, 0.0f);
  ctx.check(ilc_volumetric_slice(ctx.get(), &cam, dV, additional_samples, seed, image.data(), 0));
}

// distributed_mc_radial_profile::operator() (profile.cpp:47-74) on one device:
// the profile of the particles' quantity in num_radii shells around center,
// and the shell radii (get_comoving_profile_radii).
inline std::vector<double> mc_radial_profile(context& ctx, const std::array<double, 3>& center,
                                             double max_radius, int32_t num_radii,
                                             double sample_density, uint64_t seed = 0,
                                             int32_t dV_mode = ILC_DV_VOLUME,
                                             double volume_conversion = 1.0,
                                             std::vector<double>* radii = nullptr) {
  std::vector<double> profile((std::size_t)num_radii, 0.0);
  ctx.check(ilc_mc_radial_profile(ctx.get(), center.data(), max_radius, num_radii,
                                  sample_density, seed, dV_mode, volume_conversion,
                                  profile.data(), nullptr, nullptr));
  if (radii) {
    radii->assign((std::size_t)num_radii, 0.0);
    ctx.check(ilc_mc_profile_shells(max_radius, num_radii, sample_density, radii->data(),
                                    nullptr));
  }
  return profile;
}

// util::fits<float>::save + fits_header::add_entry (fits.hpp:142-258).
inline void write_fits(const std::string& path, const std::vector<float>& data,
                       const std::vector<int64_t>& naxes,
                       const std::vector<ilc_fits_card>& cards = {}) {
  const ilc_status st = ilc_fits_write_image(path.c_str(), data.data(), (int32_t)naxes.size(),
                                             naxes.data(), cards.data(), (int32_t)cards.size());
  if (st != ILC_OK) throw error(st, "could not write " + path);
}

}  // namespace ilc

#endif  // ILC_BACKEND_HPP
