// The reference's C++ interface (include/ct2_cosmictiger.hpp) over the C ABI.
//
// Like the reference (src/particle.cpp:17-25) the particle store is a set of
// process-global host arrays reached through particle_x(i) ... accessors; the
// GPU context holds the working copy.  Any accessor call marks the host copy
// as possibly modified, and the next GPU entry point uploads it first; every
// entry point that moves or reorders particles on the GPU copies the store
// back, so the host arrays always show the reference's state afterwards
// (including the cell order that particle_to_grid leaves behind).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "../../include/ct2_cosmictiger.hpp"
#include "../../include/ct2g.h"

namespace {

options g_opts;
bool g_opts_ready = false;

std::vector<pos_fixed> g_x, g_y, g_z;
std::vector<force_float> g_vx, g_vy, g_vz;
std::vector<char> g_rung;
bool g_host_dirty = true;  // host arrays may differ from the device copy

ct2g_ctx *g_ctx = nullptr;
ct2g_options g_ctx_opts;
bool g_ctx_ready = false;

// caches refreshed after particle_to_grid / kick
std::vector<int64_t> g_cell_begin, g_cell_end;
std::vector<float> g_expansions;
bool g_cells_valid = false, g_exp_valid = false;

void check(int rc, const char *what) {
  if (rc != CT2G_OK) {
    std::string m = std::string(what) + ": " + ct2g_status_string(rc);
    if (g_ctx) m += std::string(" (") + ct2g_last_error(g_ctx) + ")";
    throw ct2_error(rc, m);
  }
}

options default_options() {
  options o;
  o.config_file = "";
  o.hsoft = 1.0f / 50.0f;  // src/options.cpp:53-61 defaults
  o.bwidth = 3.0f;
  o.omega_m = 0.25f;
  o.mass_res = 1e9f;
  o.hubble = 0.7f;
  o.eta = 0.15f;
  o.Theta = 1.0f;
  o.Ngrid = 32;
  o.ppcell = 256;
  o.mesh = 64;
  o.order = 4;
  o.kernel = 0;
  o.GM = o.code_to_cm = o.code_to_g = o.code_to_s = 0.f;
  o.omega_lam = o.omega_r = 0.f;
  o.nparts = 0;
  return o;
}

// derived quantities, src/options.cpp:88-95 (CGS constants from
// cosmictiger/constants.hpp)
void derive(options &o) {
  const double c = 2.99792458e10, G = 6.67259e-8, sigma = 5.67051e-5;
  const double H0 = 1e7 / 3.086e24, M0 = 1.989e33, pi = 3.14159265358979323846;
  const double n3 = (double)o.Ngrid * o.Ngrid * o.Ngrid;
  o.GM = (float)(1.0 / n3);
  o.nparts = o.Ngrid * o.Ngrid * o.Ngrid;
  // M0 * mass_res (~2e42 g by default) overflows the float field, as it does
  // in the reference; the conversions that follow are carried in FP64 so
  // code_to_cm and code_to_s (and the cosmology built on them) stay finite
  const double code_to_g = M0 * (double)o.mass_res;
  o.code_to_g = (float)code_to_g;
  const double Hh = H0 * o.hubble;
  const double code_to_cm = std::cbrt(code_to_g * 8.0 * pi * n3 * G / (3.0 * o.omega_m * Hh * Hh));
  o.code_to_cm = (float)code_to_cm;
  o.code_to_s = (float)(code_to_cm / c);
  // radiation: photons plus Neff = 3.086 neutrino species at (4/11)^(4/3)
  const double Neff = 3.086;
  const double Tcmb = 2.73 * o.Theta;
  o.omega_r = (float)(32.0 * pi / 3.0 * G * sigma * (1.0 + Neff * 7.0 / 8.0 * std::pow(4.0 / 11.0, 4.0 / 3.0)) *
                      std::pow(Tcmb, 4) / (H0 * H0 * c * c * c * o.hubble * o.hubble));
  o.omega_lam = 1.0f - o.omega_r - o.omega_m;
}

void show(const options &o) {
  std::printf("%-20s: %e\n", "bwidth", o.bwidth);
  std::printf("%-20s: %s\n", "config_file", o.config_file.c_str());
  std::printf("%-20s: %e\n", "code_to_cm", o.code_to_cm);
  std::printf("%-20s: %e\n", "code_to_g", o.code_to_g);
  std::printf("%-20s: %e\n", "code_to_s", o.code_to_s);
  std::printf("%-20s: %e\n", "eta", o.eta);
  std::printf("%-20s: %e\n", "GM", o.GM);
  std::printf("%-20s: %e\n", "hsoft", o.hsoft);
  std::printf("%-20s: %e\n", "hubble", o.hubble);
  std::printf("%-20s: %e\n", "omega_lam", o.omega_lam);
  std::printf("%-20s: %e\n", "omega_m", o.omega_m);
  std::printf("%-20s: %e\n", "omega_r", o.omega_r);
  std::printf("%-20s: %e\n", "mass_res", o.mass_res);
  std::printf("%-20s: %li\n", "Ngrid", (long)o.Ngrid);
  std::printf("%-20s: %li\n", "nparts", (long)o.nparts);
  std::printf("%-20s: %i\n", "ppcell", o.ppcell);
  std::printf("%-20s: %e\n", "Theta", o.Theta);
  std::printf("%-20s: %i\n", "mesh", o.mesh);
  std::printf("%-20s: %i\n", "order", o.order);
}

bool assign(options &o, const std::string &key, const std::string &val) {
  try {
    if (key == "config_file") o.config_file = val;
    else if (key == "hsoft") o.hsoft = std::stof(val);
    else if (key == "bwidth") o.bwidth = std::stof(val);
    else if (key == "omega_m") o.omega_m = std::stof(val);
    else if (key == "mass_res") o.mass_res = std::stof(val);
    else if (key == "hubble") o.hubble = std::stof(val);
    else if (key == "eta") o.eta = std::stof(val);
    else if (key == "Theta") o.Theta = std::stof(val);
    else if (key == "Ngrid") o.Ngrid = (size_t)std::stoul(val);
    else if (key == "ppcell") o.ppcell = std::stoi(val);
    else if (key == "mesh") o.mesh = std::stoi(val);
    else if (key == "order") o.order = std::stoi(val);
    else if (key == "kernel") o.kernel = std::stoi(val);
    else return false;
  } catch (const std::exception &) {
    return false;
  }
  return true;
}

std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

void ensure_opts() {
  if (!g_opts_ready) {
    g_opts = default_options();
    derive(g_opts);
    g_opts_ready = true;
  }
}

ct2g_ctx *ctx() {
  ensure_opts();
  ct2g_options o;
  ct2g_default_options(&o);
  o.bwidth = g_opts.bwidth;
  o.hsoft = g_opts.hsoft;
  o.eta = g_opts.eta;
  o.GM = g_opts.GM;
  o.mesh = g_opts.mesh;
  o.order = g_opts.order;
  o.kernel = g_opts.kernel;
  const bool same = g_ctx_ready && o.bwidth == g_ctx_opts.bwidth && o.mesh == g_ctx_opts.mesh &&
                    o.order == g_ctx_opts.order && o.kernel == g_ctx_opts.kernel;
  if (same) {
    if (o.hsoft != g_ctx_opts.hsoft || o.eta != g_ctx_opts.eta || o.GM != g_ctx_opts.GM) {
      check(ct2g_set_params(g_ctx, o.hsoft, o.eta, o.GM), "ct2g_set_params");
      g_ctx_opts = o;
    }
    return g_ctx;
  }
  if (g_ctx) ct2g_destroy(g_ctx);
  g_ctx = nullptr;
  g_ctx_ready = false;
  check(ct2g_create(&o, &g_ctx), "ct2g_create");
  g_ctx_opts = o;
  g_ctx_ready = true;
  g_host_dirty = true;
  return g_ctx;
}

void to_device() {
  ct2g_ctx *c = ctx();
  if (!g_host_dirty) return;
  static_assert(sizeof(char) == sizeof(int8_t), "rung storage");
  check(ct2g_upload_particles(c, g_x.data(), g_y.data(), g_z.data(), g_vx.data(), g_vy.data(),
                              g_vz.data(), reinterpret_cast<const int8_t *>(g_rung.data()),
                              g_x.size()),
        "upload particles");
  g_host_dirty = false;
  g_cells_valid = g_exp_valid = false;
}

void to_host() {
  check(ct2g_download_particles(g_ctx, g_x.data(), g_y.data(), g_z.data(), g_vx.data(),
                                g_vy.data(), g_vz.data(), reinterpret_cast<int8_t *>(g_rung.data()),
                                nullptr),
        "download particles");
  g_host_dirty = false;
}

void invalidate_caches() { g_cells_valid = g_exp_valid = false; }

}  // namespace

// ---------------------------------------------------------------- options --
const options &get_options() {
  ensure_opts();
  return g_opts;
}

void set_options(const options &opts) {
  g_opts = opts;
  derive(g_opts);
  g_opts_ready = true;
}

// process_options (src/options.cpp:44-115): --key=value or --key value on the
// command line, key = value lines in config_file; --help prints the keys.
bool process_options(int argc, char *argv[]) {
  options o = default_options();
  bool rc = true;
  std::vector<std::pair<std::string, std::string>> kv;
  for (int i = 1; i < argc; i++) {
    std::string a = argv[i];
    if (a == "--help") {
      std::printf("options:\n  --config_file --hsoft --bwidth --omega_m --mass_res --hubble --eta "
                  "--Theta --Ngrid --ppcell --mesh --order --kernel\n");
      rc = false;
      continue;
    }
    if (a.rfind("--", 0) != 0) continue;
    a = a.substr(2);
    const size_t eq = a.find('=');
    if (eq != std::string::npos) {
      kv.emplace_back(a.substr(0, eq), a.substr(eq + 1));
    } else if (i + 1 < argc) {
      kv.emplace_back(a, argv[++i]);
    }
  }
  for (auto &p : kv) assign(o, p.first, p.second);
  if (rc && !o.config_file.empty()) {
    std::ifstream f(o.config_file);
    if (!f) {
      std::printf("Configuration file %s not found!\n", o.config_file.c_str());
      return false;
    }
    std::string line;
    while (std::getline(f, line)) {
      const size_t h = line.find('#');
      if (h != std::string::npos) line = line.substr(0, h);
      const size_t eq = line.find('=');
      if (eq == std::string::npos) continue;
      assign(o, trim(line.substr(0, eq)), trim(line.substr(eq + 1)));
    }
    // the command line wins over the file, as with program_options' first store
    for (auto &p : kv) assign(o, p.first, p.second);
  }
  derive(o);
  show(o);
  g_opts = o;
  g_opts_ready = true;
  return rc;
}

// ---------------------------------------------------------------- particles --
void particle_allocate(size_t count) {
  g_x.assign(count, 0);
  g_y.assign(count, 0);
  g_z.assign(count, 0);
  g_vx.assign(count, 0.f);
  g_vy.assign(count, 0.f);
  g_vz.assign(count, 0.f);
  g_rung.assign(count, 0);
  g_host_dirty = true;
  invalidate_caches();
}

// particles_init (src/particle.cpp:364-374): uniform positions from libc rand
// as rand1() = (rand()+0.5)/RAND_MAX (src/util.cpp:3-5), zero velocity, rung 0
void particles_init() {
  for (size_t n = 0; n < g_x.size(); n++) {
    pos_fixed *p[3] = {&g_x[n], &g_y[n], &g_z[n]};
    for (int d = 0; d < 3; d++) {
      const double r = (std::rand() + 0.5) / RAND_MAX;
      *p[d] = (pos_fixed)(uint64_t)(r * 4294967296.0);
    }
    g_vx[n] = g_vy[n] = g_vz[n] = 0.f;
    g_rung[n] = 0;
  }
  g_host_dirty = true;
  invalidate_caches();
}

// Raw SoA particle files (no counterpart in the reference, whose only
// initial-condition path is particles_init): an 8-byte magic "CT2SOA1", the
// count as uint64, then the x, y, z (uint32 fixed point), vx, vy, vz (float)
// and rung (int8) arrays, little-endian, as ct2_b200/ics.py writes them.
namespace {
const char kSoaMagic[8] = {'C', 'T', '2', 'S', 'O', 'A', '1', 0};
}

void particles_save(const std::string &path) {
  std::ofstream f(path, std::ios::binary);
  if (!f) throw ct2_error(CT2G_EINVAL, "particles_save: cannot open " + path);
  const uint64_t n = g_x.size();
  f.write(kSoaMagic, 8);
  f.write(reinterpret_cast<const char *>(&n), 8);
  f.write(reinterpret_cast<const char *>(g_x.data()), 4 * n);
  f.write(reinterpret_cast<const char *>(g_y.data()), 4 * n);
  f.write(reinterpret_cast<const char *>(g_z.data()), 4 * n);
  f.write(reinterpret_cast<const char *>(g_vx.data()), 4 * n);
  f.write(reinterpret_cast<const char *>(g_vy.data()), 4 * n);
  f.write(reinterpret_cast<const char *>(g_vz.data()), 4 * n);
  f.write(g_rung.data(), n);
  if (!f) throw ct2_error(CT2G_EINVAL, "particles_save: write failed for " + path);
}

void particles_load(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw ct2_error(CT2G_EINVAL, "particles_load: cannot open " + path);
  char magic[8];
  uint64_t n = 0;
  f.read(magic, 8);
  f.read(reinterpret_cast<char *>(&n), 8);
  if (!f || std::memcmp(magic, kSoaMagic, 8) != 0)
    throw ct2_error(CT2G_EINVAL, "particles_load: not a particle file: " + path);
  particle_allocate((size_t)n);
  f.read(reinterpret_cast<char *>(g_x.data()), 4 * n);
  f.read(reinterpret_cast<char *>(g_y.data()), 4 * n);
  f.read(reinterpret_cast<char *>(g_z.data()), 4 * n);
  f.read(reinterpret_cast<char *>(g_vx.data()), 4 * n);
  f.read(reinterpret_cast<char *>(g_vy.data()), 4 * n);
  f.read(reinterpret_cast<char *>(g_vz.data()), 4 * n);
  f.read(g_rung.data(), n);
  if (!f) throw ct2_error(CT2G_EINVAL, "particles_load: file too short: " + path);
}

size_t particle_count() { return g_x.size(); }
pos_fixed &particle_x(int i) { g_host_dirty = true; return g_x[i]; }
pos_fixed &particle_y(int i) { g_host_dirty = true; return g_y[i]; }
pos_fixed &particle_z(int i) { g_host_dirty = true; return g_z[i]; }
force_float &particle_vx(int i) { g_host_dirty = true; return g_vx[i]; }
force_float &particle_vy(int i) { g_host_dirty = true; return g_vy[i]; }
force_float &particle_vz(int i) { g_host_dirty = true; return g_vz[i]; }
char &particle_rung(int i) { g_host_dirty = true; return g_rung[i]; }

void particle_to_grid() {
  to_device();
  check(ct2g_particle_to_grid(g_ctx), "particle_to_grid");
  to_host();
  invalidate_caches();
}

void particle_sort_by_rung(int minrung) {
  to_device();
  check(ct2g_sort_by_rung(g_ctx, minrung), "particle_sort_by_rung");
  to_host();
  invalidate_caches();
}

std::vector<size_t> particle_rung_counts() {
  to_device();
  size_t counts[128];
  int nr = 0;
  check(ct2g_rung_counts(g_ctx, counts, 128, &nr), "particle_rung_counts");
  return std::vector<size_t>(counts, counts + nr);
}

std::pair<size_t, size_t> particle_current_range() {
  ctx();
  size_t b = 0, e = 0;
  check(ct2g_current_range(g_ctx, &b, &e), "particle_current_range");
  if (!g_ctx || e == 0) e = g_x.size();
  return {b, e};
}

void particle_pop_rungs() { check(ct2g_pop_rungs(ctx()), "particle_pop_rungs"); invalidate_caches(); }
void particle_push_rungs() { check(ct2g_push_rungs(ctx()), "particle_push_rungs"); }

void particle_set_minrung(int minrung) {
  to_device();
  check(ct2g_set_minrung(g_ctx, minrung), "particle_set_minrung");
  to_host();
}

int particle_cell_dim() { return get_options().mesh; }

std::pair<size_t, size_t> particle_get_cell(int i, int j, int k) {
  const int M = particle_cell_dim();
  if (!g_cells_valid) {
    g_cell_begin.resize((size_t)M * M * M);
    g_cell_end.resize((size_t)M * M * M);
    check(ct2g_download_cells(ctx(), g_cell_begin.data(), g_cell_end.data()), "particle_get_cell");
    g_cells_valid = true;
  }
  const size_t c = ((size_t)i * M + j) * M + k;
  return {(size_t)g_cell_begin[c], (size_t)g_cell_end[c]};
}

// particle_cell_neighbors (src/particle.cpp:302-318), with the sphere test on
// the offsets and the wrapped neighbour's range pushed
std::vector<std::pair<size_t, size_t>> particle_cell_neighbors(int i, int j, int k) {
  const int M = particle_cell_dim();
  const double bw = get_options().bwidth;
  const int B = (int)std::floor(bw);
  std::vector<std::pair<size_t, size_t>> out;
  for (int a = -B; a <= B; a++)
    for (int b = -B; b <= B; b++)
      for (int c = -B; c <= B; c++)
        if ((double)(a * a + b * b + c * c) <= bw * bw)
          out.push_back(particle_get_cell((i + a + M) % M, (j + b + M) % M, (k + c + M) % M));
  return out;
}

std::vector<double> particle_get_expansion(int i, int j, int k) {
  const int M = particle_cell_dim();
  const int p = get_options().order;
  const int nc = (p + 1) * (p + 2) * (p + 3) / 6;
  if (!g_exp_valid) {
    g_expansions.resize((size_t)nc * M * M * M);
    int rc = ct2g_download_expansions(ctx(), g_expansions.data());
    if (rc == CT2G_ESTATE) {
      check(ct2g_compute_expansions(g_ctx), "particle_get_expansion");
      rc = ct2g_download_expansions(g_ctx, g_expansions.data());
    }
    check(rc, "particle_get_expansion");
    g_exp_valid = true;
  }
  std::vector<double> L(nc);
  const size_t c = ((size_t)i * M + j) * M + k, C = (size_t)M * M * M;
  for (int n = 0; n < nc; n++) L[n] = g_expansions[(size_t)n * C + c];
  return L;
}

// ---------------------------------------------------------------- kick/drift --
int kick(const kick_params &params) {
  const bool was_dirty = g_host_dirty;
  to_device();
  // a fresh upload invalidates the grid; rebinning unchanged positions is the
  // identity, so redo it as the reference's caller already did
  if (was_dirty) check(ct2g_particle_to_grid(g_ctx), "kick: particle_to_grid");
  ct2g_kick_params kp;
  kp.ascending = params.ascending;
  kp.descending = params.descending;
  kp.top = params.top;
  kp.first = params.first;
  kp.rung = params.rung;
  kp.t0 = params.t0;
  kp.eta = params.eta;
  kp.max_dt = params.max_dt;
  kp.scale = params.scale;
  int mr = 0;
  check(ct2g_kick(g_ctx, &kp, &mr), "kick");
  to_host();
  return mr;
}

void drift(float dt, float scale) {
  to_device();
  check(ct2g_drift(g_ctx, dt, scale), "drift");
  to_host();
  invalidate_caches();
}

int kick_step(int &minrung, int max_rung, double scale, double adot, double tau, double t0,
              int minrung0, bool nocrop) {
  to_device();
  int mr = 0;
  check(ct2g_kick_step(g_ctx, &minrung, max_rung, scale, adot, tau, t0, minrung0, nocrop ? 1 : 0,
                       &mr),
        "kick_step");
  to_host();
  invalidate_caches();
  return mr;
}

// ---------------------------------------------------------------- FFT --
void fft_r2c_3d(fft_float *xin, fft_float *xout, int N) {
  check(ct2g_fft_r2c_3d(ctx(), xin, xout, N, 1), "fft_r2c_3d");
}

void fft_c2r_3d(fft_float *xin, fft_float *xout, int N) {
  check(ct2g_fft_c2r_3d(ctx(), xin, xout, N, 1), "fft_c2r_3d");
}

// ---------------------------------------------------------------- 1D FFT --
static_assert(sizeof(fft_simd) == 4 * sizeof(double), "fft_simd is four doubles");
static_assert(sizeof(ct2::complex<fft_simd>) == 8 * sizeof(double), "complex<fft_simd> layout");

void fft_real(fft_float *X, int N, int dir) {
  check(ct2g_fft1d_real(ctx(), X, N, 1, dir), "fft_real");
}

void fft_real(fft_simd *X, int N, int dir) {
  check(ct2g_fft1d_real(ctx(), reinterpret_cast<double *>(X), N, 4, dir), "fft_real");
}

void fft_complex(ct2::complex<fft_simd> *X, int N, int dir) {
  check(ct2g_fft1d_complex(ctx(), reinterpret_cast<double *>(X), N, 4, dir), "fft_complex");
}

void scramble(fft_float *X, int N1, int N2, int N3) {
  check(ct2g_scramble(ctx(), X, N1, N2, N3), "scramble");
}

void transpose_yz(fft_float *X, int N) { check(ct2g_transpose_yz(ctx(), X, N), "transpose_yz"); }

void transpose_r2c(fft_float *xin, fft_float *xout, int N) {
  check(ct2g_transpose_r2c(ctx(), xin, xout, N), "transpose_r2c");
}

void transpose_c2r(fft_float *xin, fft_float *xout, int N) {
  check(ct2g_transpose_c2r(ctx(), xin, xout, N), "transpose_c2r");
}

// twiddle tables, cached per N like the reference's (src/fft/twiddles.cpp);
// the references stay valid for the life of the process
namespace {
const std::vector<fft_float> &twiddle_table(int which, int N) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, std::vector<fft_float>> tables;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_pair(which, N);
  auto it = tables.find(key);
  if (it == tables.end()) {
    std::vector<fft_float> w((size_t)std::max(N, 0));
    if (N > 0) check(ct2g_twiddles(ctx(), which, N, w.data()), "twiddles");
    it = tables.emplace(key, std::move(w)).first;
  }
  return it->second;
}
}  // namespace

const std::vector<fft_float> &cos_twiddles(int N) { return twiddle_table(0, N); }
const std::vector<fft_float> &sin_twiddles(int N) { return twiddle_table(1, N); }
const std::vector<fft_float> &inv_sin_twiddles(int N) { return twiddle_table(2, N); }

// ---------------------------------------------------------------- cosmology --
// src/cosmology.cpp restated: Friedmann expansion rate, an SSP-RK3 update of
// (a, adot) in 128 substeps, and trapezoid integrals in log a.
namespace {
double hubble_code() {
  const options &o = get_options();
  return 1e7 / 3.086e24 * o.code_to_s * o.hubble;
}
double accel(double a) {
  const options &o = get_options();
  const double H = hubble_code();
  return a * H * H * (-o.omega_r / (a * a * a * a) - 0.5 * o.omega_m / (a * a * a) + o.omega_lam);
}
}  // namespace

double cosmos_dadt(double a) {
  const options &o = get_options();
  return hubble_code() * a *
         std::sqrt(o.omega_r / (a * a * a * a) + o.omega_m / (a * a * a) + o.omega_lam);
}

void cosmos_update(double &adotdot, double &adot, double &a, double dt0) {
  const int N = 128;
  const double dt = dt0 / N;
  for (int i = 0; i < N; i++) {
    // y = (a, adot), y' = (adot a, accel(a) a)
    const double a0 = a, v0 = adot;
    adotdot = accel(a0);
    const double ka1 = v0 * a0 * dt, kv1 = adotdot * a0 * dt;
    const double a1 = a0 + ka1, v1 = v0 + kv1;
    adotdot = accel(a1);
    const double ka2 = v1 * a1 * dt, kv2 = adotdot * a1 * dt;
    const double a2 = a0 + 0.25 * (ka1 + ka2), v2 = v0 + 0.25 * (kv1 + kv2);
    adotdot = accel(a2);
    const double ka3 = v2 * a2 * dt, kv3 = adotdot * a2 * dt;
    a = a0 + (ka1 + ka2 + 4.0 * ka3) / 6.0;
    adot = v0 + (kv1 + kv2 + 4.0 * kv3) / 6.0;
  }
}

double cosmos_conformal_time(double a0, double a1) {
  // integral over log a of 1/(a dadt(a)) * a, refined by doubling to 1e-9
  auto f = [](double a) { return a / (a * cosmos_dadt(a)); };
  const double l0 = std::log(a0), l1 = std::log(a1);
  double prev = 0.0, t = 0.0;
  for (int N = 2; N < (1 << 26); N *= 2) {
    const double h = (l1 - l0) / N;
    double s = 0.5 * (f(a0) + f(a1));
    for (int i = 1; i < N; i++) s += f(std::exp(l0 + h * i));
    t = s * h;
    if (N > 2 && std::fabs(t - prev) <= 1e-9 * std::fabs(t)) break;
    prev = t;
  }
  return t;
}

double cosmos_time(double a0, double a1) {
  const int N = 1 << 20;
  const double l0 = std::log(a0), l1 = std::log(a1), h = (l1 - l0) / N;
  auto f = [](double a) { return a / cosmos_dadt(a); };
  double s = 0.5 * (f(a0) + f(a1));
  for (int i = 1; i < N; i++) s += f(std::exp(l0 + h * i));
  return s * h;
}
