// C entry points over the reference's own 1D FFT routines and layout helpers,
// compiled from the reference tree (oracle/_ref only; test infrastructure).
#include <cosmictiger/fft.hpp>

extern "C" {
void ref_fft_real(double *X, int N, int dir) { fft_real(X, N, dir); }
void ref_scramble(double *X, int N1, int N2, int N3) { scramble(X, N1, N2, N3); }
// X: N elements of simd_f64 = 4 lanes
void ref_fft_real4(double *X, int N, int dir) {
  fft_real(reinterpret_cast<fft_simd *>(X), N, dir);
}
// X: N elements of complex<simd_f64> = [re lane0..3, im lane0..3]
void ref_fft_complex4(double *X, int N, int dir) {
  fft_complex(reinterpret_cast<sfmm::complex<fft_simd> *>(X), N, dir);
}
void ref_transpose_yz(double *X, int N) { transpose_yz(X, N); }
void ref_transpose_r2c(double *xin, double *xout, int N) { transpose_r2c(xin, xout, N); }
void ref_transpose_c2r(double *xin, double *xout, int N) { transpose_c2r(xin, xout, N); }
// twiddle tables: which = 0 cos, 1 sin, 2 inv_sin; copies N values
void ref_twiddles(int which, int N, double *out) {
  const auto &w = which == 0 ? cos_twiddles(N) : which == 1 ? sin_twiddles(N) : inv_sin_twiddles(N);
  for (int i = 0; i < N; i++) out[i] = w[i];
}
}
