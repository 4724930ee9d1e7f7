// Drives the C++ adapter (include/ilc_backend.hpp) the way illcrawl's crawler
// and volumetric_integration drive their backend: nn8 queries at points and
// one projection. Prints "ok <checksum>" on success.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "ilc_backend.hpp"

int main() {
  try {
    ilc::context ctx(0);
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> u(0.f, 100.f);
    std::vector<ilc::particle> parts(20000);
    for (auto& p : parts) p = ilc::particle{{u(rng), u(rng), u(rng), 1.0f + u(rng) / 100.f}};
    // through the abstract interface, as the crawler holds its backend
    ilc::nn8_cuda impl(ctx);
    ilc::reconstruction_backend& backend = impl;
    backend.init_backend(40000000);
    backend.setup_particles(parts, {});
    std::vector<float> pts(4 * 1000);
    for (auto& v : pts) v = u(rng);
    backend.setup_evaluation_points(ilc::view<const float>{pts.data(), pts.size() / 4, false}, 1000);
    backend.run();
    const ilc::device_buffer<float>& res = backend.retrieve_results();
    if (res.size() != 1000 || res.data() == nullptr) {
      std::printf("device result buffer missing\n");
      return 1;
    }
    const std::vector<float> host_res = res.to_host();
    // the same points already on the device: the results must not differ
    ilc::device_buffer<float> dpts(ctx, pts.size());
    dpts.copy_from_host(pts.data(), pts.size());
    backend.setup_evaluation_points(ilc::view<const float>{dpts.data(), 1000, true}, 1000);
    backend.run();
    if (impl.results_to_host() != host_res) {
      std::printf("device-point query differs from host-point query\n");
      return 1;
    }
    double sum = 0;
    for (float v : host_res) sum += v;
    ilc_camera cam{{50, 50, 0}, {0, 0, 1}, 0.0, 100.0, 16, 16};
    std::vector<float> img;
    ilc::create_projection(ctx, cam, 100.0, 0.0, 1e-3, ilc_los_scaling{1.0, 1.0, ILC_DA_UNIT}, img);
    for (float v : img) sum += v;
    // the crawler's row loop feeding the grid, a slice, a 2-bin spectrum of
    // two cameras, and the image as a FITS file
    std::vector<float> xyz(3 * 20000), q(20000), rho(20000), uu(20000), xe(20000, 1.16f);
    for (std::size_t i = 0; i < q.size(); ++i) {
      for (int j = 0; j < 3; ++j) xyz[3 * i + j] = u(rng);
      q[i] = 1.0f + u(rng) / 100.f;
      rho[i] = 1e4f * q[i];
      uu[i] = 2e5f + 1e3f * u(rng);
    }
    const double centre[3] = {50, 50, 50}, extent[3] = {80, 80, 80}, period[3] = {100, 100, 100};
    std::vector<uint32_t> kept_index;
    auto kept = ilc::ingest_cells(ctx, xyz, q, centre, extent, period, 5.0, &kept_index);
    backend.setup_particles(kept, {});
    std::vector<float> slice;
    ilc::volumetric_slice(ctx, cam, 1.0, slice);
    for (float v : slice) sum += v;
    std::vector<double> radii;
    const auto prof = ilc::mc_radial_profile(ctx, {50.0, 50.0, 50.0}, 30.0, 6, 0.05, 3,
                                             ILC_DV_MEAN, 1.0, &radii);
    for (std::size_t i = 0; i < prof.size(); ++i) sum += prof[i] * 1e-6 + radii[i] * 1e-9;
    std::vector<float> krho, ku, kxe;
    for (uint32_t i : kept_index) {
      krho.push_back(rho[i]);
      ku.push_back(uu[i]);
      kxe.push_back(xe[i]);
    }
    {  // the reference's Gaunt table (rows: log u, 81 columns: log gamma^2)
      std::vector<float> tab;
      if (FILE* f = std::fopen("illcrawl_b200/data/gaunt_factor.dat", "r")) {
        char line[4096];
        while (std::fgets(line, sizeof line, f)) {
          if (line[0] == '#') continue;
          char* p = line;
          char* e = nullptr;
          for (float v = std::strtof(p, &e); e != p; v = std::strtof(p, &e)) {
            tab.push_back(v);
            p = e;
          }
        }
        std::fclose(f);
      }
      if (tab.size() == 81 * 146)
        ctx.check(ilc_gaunt_load(ctx.get(), tab.data(), 81, 146, -6.f, -16.f, 0.2f, 0.2f));
    }
    std::vector<ilc_job> jobs(2);
    for (auto& j : jobs) {
      j = ilc_job{};
      j.camera = cam;
      j.z_range = 100.0;
      j.scale = 1.0f;
    }
    jobs[1].aperture_radius = 30.0;
    std::vector<float> cube;
    try {
      ilc::render_xray_spectra(ctx, krho, ku, kxe, 0.2f, 978500.0f, {1.0f, 2.0f}, {1.0f, 1.0f},
                               jobs, 1e-3, cube);
      for (float v : cube) sum += v * 1e-20;
      // a flat 100 cm^2 effective area over 0.1-6.5 keV in place of the Chandra ARF
      ilc::load_arf(ctx, std::vector<float>(64, 100.0f), 0.1f, 0.1f);
      ilc::render_chandra_spectra(ctx, krho, ku, kxe, 0.2f, 978500.0f, {0.5f, 2.0f},
                                  {0.1f, 0.1f}, jobs, 1e-3, cube);
      for (float v : cube) sum += v * 1e-20;
    } catch (const ilc::error& e) {
      if (e.status != ILC_ERR_NO_GAUNT_TABLE) throw;  // run from elsewhere: no table file
    }
    ilc::write_fits("_build/adapter_demo.fits", img, {16, 16},
                    {ilc_fits_card{"type", ILC_FITS_STRING, 0.0, 0, "image", "Type of this file"}});
    std::printf("ok %.9g\n", sum);
    return std::isfinite(sum) ? 0 : 1;
  } catch (const ilc::error& e) {
    std::printf("error %d %s\n", (int)e.status, e.what());
    return 2;
  }
}
