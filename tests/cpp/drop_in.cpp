// Drives the gravity step through the reference's own C++ interface
// (include/ct2_cosmictiger.hpp), the way src/main.cpp would: options from
// the command line, particle_allocate + particles_init, particle_to_grid,
// kick, drift, kick_step, and the 3D FFT pair.  Prints one line per check and
// exits non-zero on the first failure.
#include <cmath>
#include <cstdio>
#include <vector>

#include "ct2_cosmictiger.hpp"

static int fails = 0;
#define CHECK(cond, msg)                                   \
  do {                                                     \
    const bool ok_ = (cond);                               \
    std::printf("%s %s\n", ok_ ? "ok  " : "FAIL", msg);    \
    if (!ok_) fails++;                                     \
  } while (0)

int main(int argc, char *argv[]) {
  if (!process_options(argc, argv)) return 2;
  const options &opts = get_options();
  const size_t n = opts.nparts;
  CHECK(std::fabs(opts.GM * (double)n - 1.0) < 1e-6, "GM = 1/Ngrid^3 (options.cpp:88)");
  particle_allocate(n);
  particles_init();
  CHECK(particle_count() == n, "particle_count");
  particle_to_grid();
  // every particle sits in the cell whose range holds it
  const int M = particle_cell_dim();
  size_t covered = 0;
  bool inside = true;
  for (int i = 0; i < M; i++)
    for (int j = 0; j < M; j++)
      for (int k = 0; k < M; k++) {
        auto r = particle_get_cell(i, j, k);
        covered += r.second - r.first;
        for (size_t q = r.first; q < r.second && inside; q++) {
          const int sh = 32 - (int)std::lround(std::log2((double)M));
          inside = (int)(particle_x((int)q) >> sh) == i && (int)(particle_y((int)q) >> sh) == j &&
                   (int)(particle_z((int)q) >> sh) == k;
        }
      }
  CHECK(covered == n && inside, "particle_get_cell ranges cover every particle in its own cell");
  CHECK(!particle_cell_neighbors(1, 2, 3).empty(), "particle_cell_neighbors");
  kick_params kp;
  kp.ascending = true;
  kp.descending = true;
  kp.top = true;
  kp.first = false;
  kp.rung = 0;
  kp.t0 = 1e-3f;
  kp.eta = opts.eta;
  kp.max_dt = 1.0f;
  kp.scale = 1.0f;
  const int mr = kick(kp);
  double vmax = 0.0;
  for (size_t i = 0; i < n; i++) vmax = std::fmax(vmax, std::fabs(particle_vx((int)i)));
  CHECK(mr >= 0 && vmax > 0.0, "kick moved velocities and returned a rung");
  const pos_fixed x0 = particle_x(0);
  const float v0 = particle_vx(0);
  drift(1e-3f, 1.0f);
  const pos_fixed expect = x0 + (pos_fixed)(int64_t)(v0 * 1e-3f * 4294967296.0f);
  CHECK(particle_x(0) == expect, "drift is x += fixed32(v dt/scale)");
  int minrung = 0;
  const int mr2 = kick_step(minrung, 0, 1.0, 1.0, 1.0, 1e-3, 0, false);
  CHECK(mr2 >= 0 && minrung >= 0, "kick_step");
  auto counts = particle_rung_counts();
  size_t tot = 0;
  for (auto c : counts) tot += c;
  CHECK(tot == n, "particle_rung_counts");
  // FFT pair: c2r(r2c(x)) = N^3 x
  const int N = 16;
  std::vector<double> x(N * N * N), y(2 * N * N * (N / 2 + 1)), z(N * N * N);
  for (size_t i = 0; i < x.size(); i++) x[i] = std::sin(0.1 * (double)i) + 0.01 * (double)(i % 7);
  fft_r2c_3d(x.data(), y.data(), N);
  fft_c2r_3d(y.data(), z.data(), N);
  double e = 0.0;
  for (size_t i = 0; i < x.size(); i++) e = std::fmax(e, std::fabs(z[i] / (N * N * N) - x[i]));
  CHECK(e < 1e-12, "fft_c2r_3d(fft_r2c_3d(x)) = N^3 x");
  double s0 = 0.0;
  for (double v : x) s0 += v;
  CHECK(std::fabs(y[0] - s0) < 1e-9 * std::fabs(s0) + 1e-9, "r2c DC term in the real plane");
  double adot = cosmos_dadt(0.5), a = 0.5, add = 0.0;
  cosmos_update(add, adot, a, 1e-3);
  CHECK(a > 0.5 && std::isfinite(adot), "cosmos_update advances a");
  std::printf("%s\n", fails ? "FAILED" : "ALL OK");
  return fails ? 1 : 0;
}
