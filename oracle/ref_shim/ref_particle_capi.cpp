// C entry points over the reference's own particle store, binning, rung
// bookkeeping and rung-level step driver (test infrastructure; built into
// oracle/_ref only).
//
// src/particle.cpp and src/main.cpp are compiled unchanged by including them
// into this translation unit, which gives these entry points access to their
// file-static store (particle_pos_ptr, particle_cnt, rung_begin, cells).  The
// store is pointed at caller-owned arrays instead of particle_allocate's
// buffer, whose array offsets overlap (particle.cpp:273-288).  get_options(),
// kick() and drift() -- defined in src/options.cpp, src/kick.cpp and
// src/drift.cpp, which need HPX program options and the sfmm operators -- are
// supplied here: options come from ref_set_options, and kick/drift call back
// into the test harness, which applies them to the same arrays.
#include <cosmictiger/options.hpp>

static options g_ref_opts;
const options &get_options() { return g_ref_opts; }
bool process_options(int, char **) { return true; }

#include "src/particle.cpp"

#define main ct2ref_unused_main
#include "src/main.cpp"
#undef main

#include <cosmictiger/cosmology.hpp>
#include <cosmictiger/drift.hpp>

typedef int (*ref_kick_fn)(int ascending, int descending, int top, int first, int rung, float t0,
                           float eta, float max_dt, float scale, size_t begin, size_t end);
typedef void (*ref_drift_fn)(float dt, float scale);
static ref_kick_fn g_kick = nullptr;
static ref_drift_fn g_drift = nullptr;

int kick(const kick_params &p) {
  const auto r = particle_current_range();
  return g_kick(p.ascending, p.descending, p.top, p.first, p.rung, p.t0, p.eta, p.max_dt, p.scale,
                r.first, r.second);
}

void drift(float dt, float scale) { g_drift(dt, scale); }

extern "C" {

void ref_set_options(float eta, int ppcell, size_t Ngrid, float bwidth, float hsoft) {
  g_ref_opts.eta = eta;
  g_ref_opts.ppcell = ppcell;
  g_ref_opts.Ngrid = Ngrid;
  g_ref_opts.nparts = Ngrid * Ngrid * Ngrid;
  g_ref_opts.bwidth = bwidth;
  g_ref_opts.hsoft = hsoft;
  g_ref_opts.GM = 1.0 / (double)(Ngrid * Ngrid * Ngrid);
}

void ref_set_cosmology(float omega_m, float omega_r, float omega_lam, float hubble,
                       float code_to_s) {
  g_ref_opts.omega_m = omega_m;
  g_ref_opts.omega_r = omega_r;
  g_ref_opts.omega_lam = omega_lam;
  g_ref_opts.hubble = hubble;
  g_ref_opts.code_to_s = code_to_s;
}

// Point the reference's store at caller arrays (positions as fixed32 bit
// patterns), keeping the current range and the rung stack.
void ref_set_arrays(uint32_t *x, uint32_t *y, uint32_t *z, float *vx, float *vy, float *vz,
                    int8_t *rung, size_t n) {
  particle_x_ptr = reinterpret_cast<pos_fixed *>(x);
  particle_y_ptr = reinterpret_cast<pos_fixed *>(y);
  particle_z_ptr = reinterpret_cast<pos_fixed *>(z);
  particle_vx_ptr = vx;
  particle_vy_ptr = vy;
  particle_vz_ptr = vz;
  particle_rung_ptr = reinterpret_cast<char *>(rung);
  particle_pos_ptr[0] = particle_x_ptr;
  particle_pos_ptr[1] = particle_y_ptr;
  particle_pos_ptr[2] = particle_z_ptr;
  particle_cnt = n;
}

// ref_set_arrays, then the current range becomes [0, n) with an empty rung
// stack.
void ref_set_store(uint32_t *x, uint32_t *y, uint32_t *z, float *vx, float *vy, float *vz,
                   int8_t *rung, size_t n) {
  ref_set_arrays(x, y, z, vx, vy, vz, rung, n);
  rung_begin = 0;
  while (!rung_begins.empty()) rung_begins.pop();
}

size_t ref_stack_depth() { return rung_begins.size(); }

// particle_to_grid() (particle.cpp:349-362) on the current range; returns the
// Ncell it chose.  The cell table is emptied first: the reference only ever
// grows it (particle.cpp:355-356), which breaks when Ncell changes.
int ref_particle_to_grid() {
  cells.clear();
  particle_to_grid();
  return Ncell;
}

void ref_sort_by_rung(int minrung) { particle_sort_by_rung(minrung); }
void ref_push_rungs() { particle_push_rungs(); }
void ref_pop_rungs() { particle_pop_rungs(); }
void ref_set_minrung(int minrung) { particle_set_minrung(minrung); }
void ref_current_range(size_t *begin, size_t *end) {
  const auto r = particle_current_range();
  *begin = r.first;
  *end = r.second;
}
// particle_rung_counts (particle.cpp:40-50): returns the vector's size and
// copies up to cap counts
int ref_rung_counts(size_t *counts, int cap) {
  const auto c = particle_rung_counts();
  for (int i = 0; i < (int)c.size() && i < cap; i++) counts[i] = c[i];
  return (int)c.size();
}

// kick_step (main.cpp:8-92) with kick() and drift() routed to the callbacks;
// *minrung is updated as the reference's reference argument.
int ref_kick_step(int *minrung, int max_rung, double scale, double adot, double tau, double t0,
                  int minrung0, int nocrop, ref_kick_fn k, ref_drift_fn d) {
  g_kick = k;
  g_drift = d;
  return kick_step(*minrung, max_rung, scale, adot, tau, t0, minrung0, nocrop != 0);
}

// src/cosmology.cpp
double ref_cosmos_dadt(double a) { return cosmos_dadt(a); }
double ref_cosmos_time(double a0, double a1) { return cosmos_time(a0, a1); }
double ref_cosmos_conformal_time(double a0, double a1) { return cosmos_conformal_time(a0, a1); }
void ref_cosmos_update(double *adotdot, double *adot, double *a, double dt0) {
  cosmos_update(*adotdot, *adot, *a, dt0);
}
}
