// Minimal stand-in for the un-vendored sfmm header (test infrastructure).
// It is just enough for these reference sources to compile unchanged:
//   * the 1D FFT (src/fft/fft_real_scalar.cpp, fft_real_vector.cpp,
//     fft_complex_vector.cpp, twiddles.cpp, scramble.cpp): a complex<T> whose
//     real()/imag() return references and a 4-lane FP64 SIMD type
//     (FFT_SIMD_SIZE = 4);
//   * the particle store, binning and rung bookkeeping (src/particle.cpp)
//     and the step driver (src/main.cpp): a fixed32 position type and
//     declarations of the multipole types and operators.  Only the binning
//     and rung functions are ever called; the multipole operators
//     (P2M, MG2L, greens, greens_ewald) are inert stubs here, since their
//     arithmetic lives in sfmm itself.
// fixed32 holds x * 2^32 in a uint32_t (the bit pattern the reference's
// pos_fixed carries); a double in [0, 1) converts by truncation.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <utility>

namespace sfmm {

template <class T>
struct complex {
  T re, im;
  complex() = default;
  complex(T r, T i) : re(r), im(i) {}
  T &real() { return re; }
  T &imag() { return im; }
  const T &real() const { return re; }
  const T &imag() const { return im; }
  complex operator+(const complex &o) const { return complex(re + o.re, im + o.im); }
  complex operator-(const complex &o) const { return complex(re - o.re, im - o.im); }
  complex operator*(const complex &o) const {
    return complex(re * o.re - im * o.im, re * o.im + im * o.re);
  }
  complex &operator+=(const complex &o) { re = re + o.re; im = im + o.im; return *this; }
  complex &operator-=(const complex &o) { re = re - o.re; im = im - o.im; return *this; }
  complex operator*(const T &s) const { return complex(re * s, im * s); }
};

struct simd_f64 {
  double v[4];
  simd_f64() = default;
  simd_f64(double a) { for (int i = 0; i < 4; i++) v[i] = a; }
  double &operator[](int i) { return v[i]; }
  double operator[](int i) const { return v[i]; }
#define SIMD_OP(op)                                                      \
  simd_f64 operator op(const simd_f64 &o) const {                        \
    simd_f64 r;                                                          \
    for (int i = 0; i < 4; i++) r.v[i] = v[i] op o.v[i];                 \
    return r;                                                            \
  }                                                                      \
  simd_f64 &operator op##=(const simd_f64 &o) {                          \
    for (int i = 0; i < 4; i++) v[i] = v[i] op o.v[i];                   \
    return *this;                                                        \
  }
  SIMD_OP(+)
  SIMD_OP(-)
  SIMD_OP(*)
#undef SIMD_OP
  simd_f64 operator-() const {
    simd_f64 r;
    for (int i = 0; i < 4; i++) r.v[i] = -v[i];
    return r;
  }
};
inline simd_f64 operator*(double a, const simd_f64 &b) { return simd_f64(a) * b; }

struct simd_f32 {
  float v[8];
  simd_f32() = default;
  simd_f32(double a) { for (int i = 0; i < 8; i++) v[i] = (float)a; }
  static simd_f32 mask(size_t n) {
    simd_f32 r;
    for (int i = 0; i < 8; i++) r.v[i] = i < (int)n ? 1.f : 0.f;
    return r;
  }
};

struct fixed32 {
  uint32_t i;
  fixed32() = default;
  fixed32(double d) : i((uint32_t)(int64_t)(d * 4294967296.0)) {}
  bool operator<(const fixed32 &o) const { return i < o.i; }
  bool operator>=(const fixed32 &o) const { return i >= o.i; }
  bool operator==(const fixed32 &o) const { return i == o.i; }
};
struct simd_fixed32 {
  uint32_t v[8];
  simd_fixed32() = default;
  simd_fixed32 &operator=(const fixed32 &f) {
    for (int k = 0; k < 8; k++) v[k] = f.i;
    return *this;
  }
};

template <class T>
struct vec3 {
  T x[3];
  T &operator[](int i) { return x[i]; }
  const T &operator[](int i) const { return x[i]; }
};

template <class T, int P>
struct multipole {
  static constexpr int size() { return (P + 1) * (P + 2) * (P + 3) / 6; }
  T m[(P + 1) * (P + 2) * (P + 3) / 6];
  multipole() = default;
  multipole(double) {}
  T &operator[](int i) { return m[i]; }
  const T &operator[](int i) const { return m[i]; }
};

template <class T, int P>
struct expansion {
  static constexpr int size() { return (P + 1) * (P + 2) * (P + 3) / 6; }
  T l[(P + 1) * (P + 2) * (P + 3) / 6];
  T &operator[](int i) { return l[i]; }
  const T &operator[](int i) const { return l[i]; }
  expansion &operator+=(const expansion &) { return *this; }
};

template <class T, int P>
void greens(expansion<T, P> &, const vec3<T> &) {}
template <class T, int P>
void greens_ewald(expansion<T, P> &, const vec3<T> &) {}
template <class M, class W, class D>
void P2M(M &, const W &, const D &) {}
template <class L, class M, class G>
void MG2L(L &, const M &, const G &) {}
inline vec3<simd_f32> distance(const vec3<simd_fixed32> &, const vec3<simd_fixed32> &) {
  return vec3<simd_f32>();
}
template <int P>
multipole<double, P> reduce_sum(const multipole<simd_f32, P> &) {
  return multipole<double, P>();
}

}  // namespace sfmm

namespace simd {}
