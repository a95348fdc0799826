// C entry points over the reference's own 1D FFT routines, compiled from the
// reference tree (oracle/_ref only; test infrastructure).
#include <cosmictiger/fft.hpp>

extern "C" {
void ref_fft_real(double *X, int N, int dir) { fft_real(X, N, dir); }
void ref_scramble(double *X, int N1, int N2, int N3) { scramble(X, N1, N2, N3); }
// X: N elements of complex<simd_f64> = [re lane0..3, im lane0..3]
void ref_fft_complex4(double *X, int N, int dir) {
  fft_complex(reinterpret_cast<sfmm::complex<fft_simd> *>(X), N, dir);
}
}
