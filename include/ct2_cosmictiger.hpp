/*
 * ct2_cosmictiger.hpp -- the reference's C++ interface for the gravity step,
 * served by the B200 library (libct2g.so).  A program written against the
 * reference's cosmictiger headers links this library in place of
 * src/kick.cpp, src/drift.cpp, src/fft/fft_{r2c,c2r}_3d.cpp, src/options.cpp,
 * src/cosmology.cpp and the particle half of src/particle.cpp.
 *
 * Names, argument meaning and return values follow the reference
 * (dmarce1/ct2, file:line within that project).  Differences, all forced by
 * the reference depending on absent libraries:
 *   - pos_fixed is a plain uint32_t holding x * 2^32 (the reference's
 *     sfmm::fixed32, cosmictiger/cosmictiger.hpp:22, same bit pattern);
 *   - particle_get_expansion returns the Cartesian Taylor coefficients as a
 *     std::vector<double> (the reference returns sfmm::expansion);
 *   - the mesh is an explicit power of two (options::mesh) instead of
 *     cbrt(count/ppcell)+4 (src/particle.cpp:355), and the expansion order is
 *     options::order instead of the compile-time PORDER.
 * Errors: the reference has no error reporting (it aborts on allocation
 * failure, src/memory.cpp:8-9); these functions throw ct2_error.
 */
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

using fft_float = double;    // cosmictiger/cosmictiger.hpp:18
using force_float = float;   // cosmictiger/cosmictiger.hpp:20
using pos_fixed = uint32_t;  // cosmictiger/cosmictiger.hpp:22 (fixed32 bit pattern)

struct ct2_error : std::runtime_error {
  int status;
  ct2_error(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

// cosmictiger/options.hpp:14-32, plus mesh / order / kernel
struct options {
  float bwidth;
  std::string config_file;
  float code_to_cm;
  float code_to_g;
  float code_to_s;
  float eta;
  float GM;
  float hsoft;
  float hubble;
  float omega_lam;
  float omega_m;
  float omega_r;
  float mass_res;
  size_t Ngrid;
  size_t nparts;
  int ppcell;
  float Theta;
  int mesh;    // cells per dimension (power of two)
  int order;   // multipole expansion order
  int kernel;  // 0 Plummer, 1 the reference's uniform-sphere kernel
};

const options &get_options();                         // options.hpp:34
bool process_options(int argc, char *argv[]);         // options.hpp:35
void set_options(const options &opts);                // (library users without argv)

// cosmictiger/kick.hpp:10-20
struct kick_params {
  bool ascending;
  bool descending;
  bool top;
  bool first;
  int rung;
  float t0;
  float eta;
  float max_dt;
  float scale;
};

// returns its max_rung argument, as the reference does (the max_rung its
// loop body declares, main.cpp:68, shadows the parameter returned at :90)
int kick_step(int &minrung, int max_rung, double scale, double adot, double tau, double t0,
              int minrung0, bool nocrop);             // kick.hpp:23, main.cpp:8-92
int kick(const kick_params &params);                  // kick.hpp:24, kick.cpp:105-125
void drift(float dt, float scale);                    // drift.hpp:12, drift.cpp:4-18

void fft_r2c_3d(fft_float *xin, fft_float *xout, int N);  // fft.hpp:28
void fft_c2r_3d(fft_float *xin, fft_float *xout, int N);  // fft.hpp:29

// The 1D FFT surface, cosmictiger/fft.hpp:18-27.  The reference's fft_simd is
// sfmm::simd_f64 with FFT_SIMD_SIZE = 4 lanes (cosmictiger/cosmictiger.hpp:12,19)
// and its complex type sfmm::complex<T>; sfmm is not part of the reference
// tree, so these are layout-compatible stand-ins: fft_simd is four doubles,
// ct2::complex<fft_simd> the four real lanes followed by the four imaginary
// lanes (an sfmm array of the same shape can be passed by reinterpret_cast).
// Inputs of fft_real / fft_complex are in bit-reversed order (scramble
// first); dir = -1 is the transform with exp(+2 pi i n k / N).  Computed on
// the GPU in FP64 (ct2g_fft1d_real / ct2g_fft1d_complex).
namespace ct2 {
struct simd_f64 {
  double v[4];
  double &operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
};
template <class T>
struct complex {
  T re, im;
  T &real() { return re; }
  T &imag() { return im; }
  const T &real() const { return re; }
  const T &imag() const { return im; }
};
}  // namespace ct2
using fft_simd = ct2::simd_f64;                                       // cosmictiger.hpp:19
void transpose_yz(fft_float *X, int N);                               // fft.hpp:18
void transpose_r2c(fft_float *xin, fft_float *xout, int N);           // fft.hpp:19
void transpose_c2r(fft_float *xin, fft_float *xout, int N);           // fft.hpp:20
void scramble(fft_float *X, int N1, int N2, int N3);                  // fft.hpp:21
const std::vector<fft_float> &cos_twiddles(int N);                    // fft.hpp:22
const std::vector<fft_float> &sin_twiddles(int N);                    // fft.hpp:23
const std::vector<fft_float> &inv_sin_twiddles(int N);                // fft.hpp:24
void fft_real(fft_float *X, int N, int dir = 1);                      // fft.hpp:25
void fft_real(fft_simd *X, int N, int dir = 1);                       // fft.hpp:26
void fft_complex(ct2::complex<fft_simd> *X, int N, int dir = 1);      // fft.hpp:27

// cosmictiger/particle.hpp:22-73 and src/particle.cpp
void particle_allocate(size_t count);                 // particle.cpp:273
void particles_init();                                // particle.cpp:364
size_t particle_count();                              // particle.hpp:58
pos_fixed &particle_x(int i);                         // particle.hpp:30-56
pos_fixed &particle_y(int i);
pos_fixed &particle_z(int i);
force_float &particle_vx(int i);
force_float &particle_vy(int i);
force_float &particle_vz(int i);
char &particle_rung(int i);
void particle_sort_by_rung(int minrung);              // particle.hpp:60
std::vector<size_t> particle_rung_counts();           // particle.hpp:61
void particle_to_grid();                              // particle.hpp:62
std::pair<size_t, size_t> particle_current_range();   // particle.hpp:63
void particle_pop_rungs();                            // particle.hpp:65
void particle_push_rungs();                           // particle.hpp:66
void particle_set_minrung(int minrung);               // particle.hpp:67
std::vector<std::pair<size_t, size_t>> particle_cell_neighbors(int i, int j, int k);  // :68
int particle_cell_dim();                              // particle.hpp:69
std::pair<size_t, size_t> particle_get_cell(int i, int j, int k);  // particle.hpp:70
std::vector<double> particle_get_expansion(int i, int j, int k);   // particle.hpp:71
// Raw SoA particle files: no counterpart in the reference (its only initial
// conditions come from particles_init).  Magic "CT2SOA1\0", uint64 count,
// then x, y, z (uint32), vx, vy, vz (float), rung (int8) arrays.
void particles_save(const std::string &path);
void particles_load(const std::string &path);

// cosmictiger/cosmology.hpp:13-16
double cosmos_conformal_time(double a0, double a1);
double cosmos_dadt(double a);
double cosmos_time(double a0, double a1);
void cosmos_update(double &adotdot, double &adot, double &a, double dt0);

// util.hpp:13-34 rung-time helpers are header-only in the reference and are
// not part of this library.
