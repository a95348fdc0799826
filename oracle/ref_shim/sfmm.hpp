// Minimal stand-in for the un-vendored sfmm header, just enough for the
// reference's 1D FFT sources (src/fft/fft_real_scalar.cpp,
// fft_complex_vector.cpp, twiddles.cpp, scramble.cpp) to compile unchanged:
// a complex<T> whose real()/imag() return references, a 4-lane FP64 SIMD
// type (FFT_SIMD_SIZE = 4), and placeholder position/force types.
#pragma once
#include <cmath>
#include <cstdint>
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

struct simd_f32 { float v[8]; };
struct fixed32 { uint32_t i; };
struct simd_fixed32 { uint32_t v[8]; };

}  // namespace sfmm

namespace simd {}
