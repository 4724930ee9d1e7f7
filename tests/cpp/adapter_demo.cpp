// Drives the C++ adapter (include/ilc_backend.hpp) the way illcrawl's crawler
// and volumetric_integration drive their backend: nn8 queries at points and
// one projection. Prints "ok <checksum>" on success.
#include <cmath>
#include <cstdio>
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
    ilc::nn8_cuda backend(ctx);
    backend.init_backend(40000000);
    backend.setup_particles(parts);
    std::vector<float> pts(4 * 1000);
    for (auto& v : pts) v = u(rng);
    backend.setup_evaluation_points(ilc::view<const float>{pts.data(), pts.size() / 4, false}, 1000);
    backend.run();
    double sum = 0;
    for (float v : backend.retrieve_results()) sum += v;
    ilc_camera cam{{50, 50, 0}, {0, 0, 1}, 0.0, 100.0, 16, 16};
    std::vector<float> img;
    ilc::create_projection(ctx, cam, 100.0, 0.0, 1e-3, ilc_los_scaling{1.0, 1.0, ILC_DA_UNIT}, img);
    for (float v : img) sum += v;
    std::printf("ok %.9g\n", sum);
    return std::isfinite(sum) ? 0 : 1;
  } catch (const ilc::error& e) {
    std::printf("error %d %s\n", (int)e.status, e.what());
    return 2;
  }
}
