// The reference's 1D FFT and layout surface (cosmictiger/fft.hpp:18-27) on the
// GPU: fft_real, fft_complex, scramble, transpose_yz / r2c / c2r and the
// twiddle tables.  The reference runs these on the CPU
// (src/fft/fft_real_scalar.cpp, fft_real_vector.cpp, fft_complex_vector.cpp,
// scramble.cpp, transpose.cpp, twiddles.cpp); here each call stages the host
// array through device memory and runs one kernel.  They keep the reference's
// layouts and conventions:
//   * fft_real / fft_complex take their input in bit-reversed order (the
//     caller scrambles first, as src/fft/fft_test.cpp:81-159 does) and leave
//     the forward DFT X(k) = sum_n x(n) exp(-2 pi i n k / N): fft_real in
//     halfcomplex order (X[0], Re X1 .. Re X(N/2), Im X(N/2-1) .. Im X1),
//     fft_complex in natural order;
//   * several independent sequences ("lanes") interleave element by element,
//     as the reference's 4-lane SIMD type does: real element n of lane l at
//     n*lanes + l, complex element n at (2n)*lanes + l (real) and
//     (2n+1)*lanes + l (imaginary).
// dir = -1 is the transform with the opposite sign, exp(+2 pi i n k / N) (the
// reference's dir = -1 path does not compute an inverse; the restatement
// follows the twiddle tables it selects, twiddles.cpp:44-56).
#include "ct2g_internal.cuh"

namespace {

constexpr int kFft1dMaxN = 8192;

bool pow2(int n) { return n >= 1 && (n & (n - 1)) == 0; }
int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

// One block per lane: the sequence is loaded in the order it arrives (bit
// reversed), which is the order an in-place decimation-in-time transform
// starts from, and log2(N) radix-2 stages run in shared memory.
template <bool COMPLEX>
__global__ void fft1d_lanes_kernel(double *__restrict__ X, int N, int logN, int lanes, int dir) {
  extern __shared__ double2 a[];
  const int l = blockIdx.x;
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    const double re = COMPLEX ? X[(size_t)(2 * n) * lanes + l] : X[(size_t)n * lanes + l];
    const double im = COMPLEX ? X[(size_t)(2 * n + 1) * lanes + l] : 0.0;
    a[n] = make_double2(re, im);
  }
  __syncthreads();
  for (int s = 1; s <= logN; s++) {
    const int half = 1 << (s - 1);
    for (int k = threadIdx.x; k < N / 2; k += blockDim.x) {
      const int j = k & (half - 1);
      const int i0 = ((k >> (s - 1)) << s) + j;
      const int i1 = i0 + half;
      double sn, cs;
      // exp(-dir 2 pi i j / (2 half))
      sincospi(-(double)dir * (double)j / (double)half, &sn, &cs);
      const double2 b = a[i1], c = a[i0];
      const double tr = cs * b.x - sn * b.y, ti = cs * b.y + sn * b.x;
      a[i0] = make_double2(c.x + tr, c.y + ti);
      a[i1] = make_double2(c.x - tr, c.y - ti);
    }
    __syncthreads();
  }
  for (int n = threadIdx.x; n < N; n += blockDim.x) {
    if (COMPLEX) {
      X[(size_t)(2 * n) * lanes + l] = a[n].x;
      X[(size_t)(2 * n + 1) * lanes + l] = a[n].y;
    } else if (n <= N / 2) {
      // halfcomplex: Re X(n) at n, Im X(n) at N - n (0 < n < N/2)
      X[(size_t)n * lanes + l] = a[n].x;
      if (n > 0 && n < N / 2) X[(size_t)(N - n) * lanes + l] = a[n].y;
    }
  }
}

// scramble (scramble.cpp:26-43): row j of every block of N2 rows (rows of N3
// values) trades places with row bitrev(j)
__global__ void scramble_kernel(const double *__restrict__ in, double *__restrict__ out,
                                size_t total, int N2, int bits, int N3) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t k = t % N3, r = t / N3;
    const int j = (int)(r % N2);
    const size_t i = r / N2;
    const int jr = bits ? (int)(__brev((unsigned)j) >> (32 - bits)) : j;
    out[(i * N2 + jr) * N3 + k] = in[t];
  }
}

// transpose_yz: X[ix][iy][iz] -> X[ix][iz][iy]
__global__ void transpose_yz_kernel(const double *__restrict__ in, double *__restrict__ out,
                                    int N) {
  const size_t total = (size_t)N * N * N;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(t % N), iy = (int)((t / N) % N);
    const size_t ix = t / ((size_t)N * N);
    out[(ix * N + iz) * N + iy] = in[t];
  }
}

// transpose_r2c (transpose.cpp:33-72): y halfcomplex rows in, split planes
// out: re[(ix*N + iz)*(N/2+1) + iy] = in[ix][iy][iz] and
// im[...] = in[ix][N-iy][iz] (0 for iy = 0 and N/2), iy in [0, N/2]
__global__ void transpose_r2c_kernel(const double *__restrict__ in, double *__restrict__ out,
                                     int N) {
  const int h = N / 2 + 1;
  const size_t dimag = (size_t)N * N * h;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < dimag;
       t += (size_t)gridDim.x * blockDim.x) {
    const int iy = (int)(t % h);
    const int iz = (int)((t / h) % N);
    const size_t ix = t / ((size_t)h * N);
    out[t] = in[(ix * N + iy) * N + iz];
    out[dimag + t] = (iy == 0 || iy == N / 2) ? 0.0 : in[(ix * N + (N - iy)) * N + iz];
  }
}

// transpose_c2r: the inverse of transpose_r2c (split planes in, y halfcomplex
// rows out)
__global__ void transpose_c2r_kernel(const double *__restrict__ in, double *__restrict__ out,
                                     int N) {
  const int h = N / 2 + 1;
  const size_t dimag = (size_t)N * N * h;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < dimag;
       t += (size_t)gridDim.x * blockDim.x) {
    const int iy = (int)(t % h);
    const int iz = (int)((t / h) % N);
    const size_t ix = t / ((size_t)h * N);
    out[(ix * N + iy) * N + iz] = in[t];
    if (iy > 0 && iy < N / 2) out[(ix * N + (N - iy)) * N + iz] = in[dimag + t];
  }
}

// twiddles.cpp:5-56: 0 cos(-2 pi n/N), 1 sin(-2 pi n/N), 2 sin(2 pi n/N)
__global__ void twiddle_kernel(double *__restrict__ out, int N, int which) {
  for (int n = blockIdx.x * blockDim.x + threadIdx.x; n < N; n += gridDim.x * blockDim.x) {
    const double a = 2.0 * (double)n / (double)N;
    out[n] = which == 0 ? cospi(-a) : which == 1 ? sinpi(-a) : sinpi(a);
  }
}

unsigned grid_for(size_t total) {
  return (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
}

// device staging: copy `nin` doubles from host `hin` to a device buffer of
// max(nin, nout) doubles plus a second buffer of nout doubles, run `body`,
// copy `nout` doubles back to `hout`
template <class F>
int staged(ct2g_ctx *ctx, const double *hin, size_t nin, double *hout, size_t nout, bool two,
           const char *what, F body) {
  double *d0 = nullptr, *d1 = nullptr;
  const size_t n0 = std::max(nin, nout);
  CT2G_CUDA(ctx, cudaMalloc(&d0, sizeof(double) * std::max<size_t>(n0, 1)));
  if (two) {
    cudaError_t e = cudaMalloc(&d1, sizeof(double) * std::max<size_t>(nout, 1));
    if (e != cudaSuccess) {
      cudaFree(d0);
      return ct2g_cuda_fail(ctx, e, what);
    }
  }
  cudaStream_t st = ctx->stream;
  int rc = CT2G_OK;
  cudaError_t e = cudaMemcpyAsync(d0, hin, sizeof(double) * nin, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    body(d0, d1);
    ctx->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hout, two ? d1 : d0, sizeof(double) * nout, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(d0);
  if (d1) cudaFree(d1);
  if (e != cudaSuccess) rc = ct2g_cuda_fail(ctx, e, what);
  return rc;
}

int fft1d(ct2g_ctx *ctx, double *X, int N, int lanes, int dir, bool cplx) {
  CT2G_TRY(ct2g_check(ctx));
  if (!X || !pow2(N) || N < 2 || N > kFft1dMaxN || lanes < 1 || lanes > 65535 ||
      (dir != 1 && dir != -1))
    return ct2g_fail(ctx, CT2G_EINVAL,
                     "fft1d: N must be a power of two in [2, 8192], lanes in [1, 65535], dir +-1");
  const size_t nd = (size_t)N * lanes * (cplx ? 2 : 1);
  const int smem = (int)sizeof(double2) * N;
  auto kern = cplx ? fft1d_lanes_kernel<true> : fft1d_lanes_kernel<false>;
  CT2G_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  const int logN = ilog2(N);
  const int threads = std::min(256, std::max(32, N / 2));
  return staged(ctx, X, nd, X, nd, false, "fft1d", [&](double *d0, double *) {
    kern<<<lanes, threads, smem, ctx->stream>>>(d0, N, logN, lanes, dir);
  });
}

}  // namespace

int ct2g_fft1d_real(ct2g_ctx *ctx, double *X, int N, int lanes, int dir) {
  return fft1d(ctx, X, N, lanes, dir, false);
}

int ct2g_fft1d_complex(ct2g_ctx *ctx, double *X, int N, int lanes, int dir) {
  return fft1d(ctx, X, N, lanes, dir, true);
}

int ct2g_scramble(ct2g_ctx *ctx, double *X, int N1, int N2, int N3) {
  CT2G_TRY(ct2g_check(ctx));
  if (!X || N1 < 0 || N3 < 0 || !pow2(N2))
    return ct2g_fail(ctx, CT2G_EINVAL, "scramble: N2 must be a power of two, N1, N3 >= 0");
  const size_t total = (size_t)N1 * N2 * N3;
  if (total == 0) return CT2G_OK;
  const int bits = ilog2(N2);
  return staged(ctx, X, total, X, total, true, "scramble", [&](double *d0, double *d1) {
    scramble_kernel<<<grid_for(total), 256, 0, ctx->stream>>>(d0, d1, total, N2, bits, N3);
  });
}

int ct2g_transpose_yz(ct2g_ctx *ctx, double *X, int N) {
  CT2G_TRY(ct2g_check(ctx));
  if (!X || N < 1 || N > 512) return ct2g_fail(ctx, CT2G_EINVAL, "transpose_yz: N in [1, 512]");
  const size_t total = (size_t)N * N * N;
  return staged(ctx, X, total, X, total, true, "transpose_yz", [&](double *d0, double *d1) {
    transpose_yz_kernel<<<grid_for(total), 256, 0, ctx->stream>>>(d0, d1, N);
  });
}

int ct2g_transpose_r2c(ct2g_ctx *ctx, const double *xin, double *xout, int N) {
  CT2G_TRY(ct2g_check(ctx));
  if (!xin || !xout || N < 2 || (N & 1) || N > 512)
    return ct2g_fail(ctx, CT2G_EINVAL, "transpose_r2c: N even in [2, 512]");
  const size_t nin = (size_t)N * N * N, dimag = (size_t)N * N * (N / 2 + 1);
  return staged(ctx, xin, nin, xout, 2 * dimag, true, "transpose_r2c",
                [&](double *d0, double *d1) {
                  transpose_r2c_kernel<<<grid_for(dimag), 256, 0, ctx->stream>>>(d0, d1, N);
                });
}

int ct2g_transpose_c2r(ct2g_ctx *ctx, const double *xin, double *xout, int N) {
  CT2G_TRY(ct2g_check(ctx));
  if (!xin || !xout || N < 2 || (N & 1) || N > 512)
    return ct2g_fail(ctx, CT2G_EINVAL, "transpose_c2r: N even in [2, 512]");
  const size_t nout = (size_t)N * N * N, dimag = (size_t)N * N * (N / 2 + 1);
  return staged(ctx, xin, 2 * dimag, xout, nout, true, "transpose_c2r",
                [&](double *d0, double *d1) {
                  transpose_c2r_kernel<<<grid_for(dimag), 256, 0, ctx->stream>>>(d0, d1, N);
                });
}

int ct2g_twiddles(ct2g_ctx *ctx, int which, int N, double *out) {
  CT2G_TRY(ct2g_check(ctx));
  if (!out || N < 1 || which < 0 || which > 2)
    return ct2g_fail(ctx, CT2G_EINVAL, "twiddles: which in {0,1,2}, N >= 1");
  return staged(ctx, out, 0, out, (size_t)N, false, "twiddles", [&](double *d0, double *) {
    twiddle_kernel<<<grid_for((size_t)N), 256, 0, ctx->stream>>>(d0, N, which);
  });
}
