// Batched 3D real-to-complex / complex-to-real FFTs (FP32 and FP64).
//
// Replaces the reference's FP64 radix-2/4 FFT family (src/fft/*.cpp,
// cosmictiger/fft.hpp:18-29) and its 3D drivers fft_r2c_3d / fft_c2r_3d,
// whose bodies are empty or commented out in the reference
// (src/fft/fft_r2c_3d.cpp:4-31, src/fft/fft_c2r_3d.cpp:4-40).
//
// Layout: real grid x[b][i][j][k] (k contiguous), spectrum
// X[b][qi][qj][qk] with qk in [0, N/2] (k is the halved axis).  Forward sign
// exp(-2 pi i q.r/N) (the reference's twiddles cos(-2 pi n/N), sin(-2 pi n/N),
// src/fft/twiddles.cpp:6-38); c2r is the unnormalised inverse.
//
// Three passes, each one read and one write of the array:
//   Z: r2c along the contiguous axis, two real lines packed as one complex line
//   Y: complex FFT along j, tiles of W contiguous qk columns staged in smem
//   X: complex FFT along i, tiles of W contiguous (qj,qk) columns
// Each 1D transform is radix-2 decimation in time on bit-reversed input, the
// order the reference's scramble() produces (src/fft/scramble.cpp:26-43),
// computed in shared memory.
#include "ct2g_internal.cuh"

namespace {

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

template <typename C2>
__device__ __forceinline__ C2 cmul(C2 a, C2 b) {
  C2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}

// In-place radix-2 DIT on `nlines` lines of length N=2^logN held in smem,
// element (l, r) at s[l*ls + r*es], input in bit-reversed order.  The
// twiddles tw[k] = exp(-2 pi i k/N), k < N/2, are in smem.
template <typename C2>
__device__ __forceinline__ void smem_fft(C2 *s, int logN, int nlines, int ls, int es,
                                         const C2 *tw, bool inv) {
  const int N = 1 << logN, half = N >> 1;
  const int total = nlines * half;
  for (int lh = 0; lh < logN; lh++) {
    const int h = 1 << lh;
    const int tstep = logN - 1 - lh;  // twiddle index = pos << tstep
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
      int j = b & (half - 1);
      int l = b >> (logN - 1);
      int pos = j & (h - 1);
      int i0 = ((j >> lh) << (lh + 1)) + pos;
      int i1 = i0 + h;
      C2 w = tw[pos << tstep];
      if (inv) w.y = -w.y;
      C2 *p0 = s + l * ls + i0 * es;
      C2 *p1 = s + l * ls + i1 * es;
      C2 a = *p0;
      C2 m = cmul(w, *p1);
      C2 r0, r1;
      r0.x = a.x + m.x;
      r0.y = a.y + m.y;
      r1.x = a.x - m.x;
      r1.y = a.y - m.y;
      *p0 = r0;
      *p1 = r1;
    }
    __syncthreads();
  }
}

template <typename C2>
__device__ __forceinline__ void load_twiddles(C2 *stw, const C2 *tw, int half) {
  for (int k = threadIdx.x; k < half; k += blockDim.x) stw[k] = tw[k];
}

__device__ __forceinline__ int bitrev(int j, int logN) {
  return (int)(__brev((unsigned)j) >> (32 - logN));
}

// ---- pass Z forward: pairs of real lines -> half spectra -------------------
// lines: total number of real lines (even); LP complex (packed) lines per block
template <typename T>
__global__ void fftz_r2c_kernel(const T *__restrict__ in, typename Cplx<T>::type *__restrict__ out,
                                int logN, size_t npairs, int LP,
                                const typename Cplx<T>::type *__restrict__ tw) {
  using C2 = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  const int N = 1 << logN, NH = N / 2 + 1;
  C2 *stw = reinterpret_cast<C2 *>(smraw);
  C2 *s = stw + N / 2;
  const int ls = N + 1;  // padded line stride
  load_twiddles(stw, tw, N / 2);
  const size_t pair0 = (size_t)blockIdx.x * LP;
  const int np = (int)min((size_t)LP, npairs - pair0);
  for (int e = threadIdx.x; e < np * N; e += blockDim.x) {
    int l = e >> logN, j = e & (N - 1);
    size_t line = 2 * (pair0 + l);
    C2 v;
    v.x = in[line * N + j];
    v.y = in[(line + 1) * N + j];
    s[l * ls + bitrev(j, logN)] = v;
  }
  __syncthreads();
  smem_fft(s, logN, np, ls, 1, stw, false);
  for (int e = threadIdx.x; e < np * NH; e += blockDim.x) {
    int l = e / NH, k = e - l * NH;
    size_t line = 2 * (pair0 + l);
    C2 zk = s[l * ls + (k & (N - 1))];
    C2 zc = s[l * ls + ((N - k) & (N - 1))];
    // A_k = (Z_k + conj Z_{N-k})/2, B_k = (Z_k - conj Z_{N-k})/(2i)
    C2 a, b;
    a.x = (T)0.5 * (zk.x + zc.x);
    a.y = (T)0.5 * (zk.y - zc.y);
    b.x = (T)0.5 * (zk.y + zc.y);
    b.y = (T)0.5 * (zc.x - zk.x);
    out[line * NH + k] = a;
    out[(line + 1) * NH + k] = b;
  }
}

// ---- pass Z inverse: pairs of half spectra -> real lines --------------------
template <typename T>
__global__ void fftz_c2r_kernel(const typename Cplx<T>::type *__restrict__ in, T *__restrict__ out,
                                int logN, size_t npairs, int LP,
                                const typename Cplx<T>::type *__restrict__ tw) {
  using C2 = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  const int N = 1 << logN, NH = N / 2 + 1;
  C2 *stw = reinterpret_cast<C2 *>(smraw);
  C2 *s = stw + N / 2;
  const int ls = N + 1;
  load_twiddles(stw, tw, N / 2);
  const size_t pair0 = (size_t)blockIdx.x * LP;
  const int np = (int)min((size_t)LP, npairs - pair0);
  for (int e = threadIdx.x; e < np * N; e += blockDim.x) {
    int l = e >> logN, k = e & (N - 1);
    size_t line = 2 * (pair0 + l);
    // Z_k = A_k + i B_k, with A_{N-k} = conj(A_k) for the upper half
    C2 a, b, z;
    if (k < NH) {
      a = in[line * NH + k];
      b = in[(line + 1) * NH + k];
    } else {
      a = in[line * NH + (N - k)];
      b = in[(line + 1) * NH + (N - k)];
      a.y = -a.y;
      b.y = -b.y;
    }
    z.x = a.x - b.y;
    z.y = a.y + b.x;
    s[l * ls + bitrev(k, logN)] = z;
  }
  __syncthreads();
  smem_fft(s, logN, np, ls, 1, stw, true);
  for (int e = threadIdx.x; e < np * N; e += blockDim.x) {
    int l = e >> logN, j = e & (N - 1);
    size_t line = 2 * (pair0 + l);
    C2 z = s[l * ls + j];
    out[line * N + j] = z.x;
    out[(line + 1) * N + j] = z.y;
  }
}

// ---- strided passes: FFT along rows for tiles of W contiguous columns -------
// array: outer blocks of `ostride` elements; inside, rows of `rstride`; ncols
// valid columns per row.  grid.x = nouter * ntiles.
template <typename C2>
__global__ void fft_cols_kernel(C2 *__restrict__ a, int logN, size_t nouter, size_t ostride,
                                size_t rstride, size_t ncols, int W, int ntiles, bool inv,
                                const C2 *__restrict__ tw) {
  extern __shared__ unsigned char smraw[];
  const int N = 1 << logN;
  C2 *stw = reinterpret_cast<C2 *>(smraw);
  C2 *s = stw + N / 2;
  load_twiddles(stw, tw, N / 2);
  const size_t outer = blockIdx.x / ntiles;
  const size_t col0 = (size_t)(blockIdx.x % ntiles) * W;
  const int wv = (int)min((size_t)W, ncols - col0);
  C2 *base = a + outer * ostride + col0;
  const int logW = __ffs(W) - 1;
  for (int e = threadIdx.x; e < N * W; e += blockDim.x) {
    int r = e >> logW, w = e & (W - 1);
    if (w < wv) s[bitrev(r, logN) * W + w] = base[(size_t)r * rstride + w];
  }
  __syncthreads();
  smem_fft(s, logN, W, 1, W, stw, inv);
  for (int e = threadIdx.x; e < N * W; e += blockDim.x) {
    int r = e >> logW, w = e & (W - 1);
    if (w < wv) base[(size_t)r * rstride + w] = s[r * W + w];
  }
}

int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

template <typename C2>
const C2 *twiddle_ptr(ct2g_ctx *ctx);
template <>
const float2 *twiddle_ptr<float2>(ct2g_ctx *ctx) { return ctx->tw32; }
template <>
const double2 *twiddle_ptr<double2>(ct2g_ctx *ctx) { return ctx->tw64; }

template <typename T>
int run_cols(ct2g_ctx *ctx, typename Cplx<T>::type *spec, int N, int batch, bool inv) {
  using C2 = typename Cplx<T>::type;
  const int logN = ilog2(N);
  const size_t NH = N / 2 + 1;
  const int W = 16;
  const size_t smem = sizeof(C2) * ((size_t)N / 2 + (size_t)N * W);
  auto kern = fft_cols_kernel<C2>;
  CT2G_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  const C2 *tw = twiddle_ptr<C2>(ctx);
  // X pass first on inverse, Y first on forward (order does not matter)
  for (int pass = 0; pass < 2; pass++) {
    bool ypass = (pass == 0) != inv;
    size_t nouter, ostride, rstride, ncols;
    if (ypass) {
      nouter = (size_t)batch * N;
      ostride = (size_t)N * NH;
      rstride = NH;
      ncols = NH;
    } else {
      nouter = (size_t)batch;
      ostride = (size_t)N * N * NH;
      rstride = (size_t)N * NH;
      ncols = (size_t)N * NH;
    }
    int ntiles = (int)((ncols + W - 1) / W);
    size_t nblocks = nouter * ntiles;
    kern<<<(unsigned)nblocks, 256, smem, ctx->stream>>>(spec, logN, nouter, ostride, rstride,
                                                         ncols, W, ntiles, inv, tw);
    CT2G_LAUNCHED(ctx);
  }
  return CT2G_OK;
}

template <typename T>
int fft_r2c(ct2g_ctx *ctx, const T *in, typename Cplx<T>::type *out, int N, int batch) {
  using C2 = typename Cplx<T>::type;
  CT2G_TRY(ct2g_twiddles(ctx, N));
  const int logN = ilog2(N);
  const size_t npairs = (size_t)batch * N * N / 2;
  const int LP = (int)std::max<size_t>(1, (size_t)8192 / N);
  const size_t smem = sizeof(C2) * ((size_t)N / 2 + (size_t)LP * (N + 1));
  auto kern = fftz_r2c_kernel<T>;
  CT2G_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  kern<<<ct2g_div_up(npairs, LP), 256, smem, ctx->stream>>>(in, out, logN, npairs, LP,
                                                            twiddle_ptr<C2>(ctx));
  CT2G_LAUNCHED(ctx);
  return run_cols<T>(ctx, out, N, batch, false);
}

template <typename T>
int fft_c2r(ct2g_ctx *ctx, typename Cplx<T>::type *in, T *out, int N, int batch) {
  using C2 = typename Cplx<T>::type;
  CT2G_TRY(ct2g_twiddles(ctx, N));
  CT2G_TRY(run_cols<T>(ctx, in, N, batch, true));
  const int logN = ilog2(N);
  const size_t npairs = (size_t)batch * N * N / 2;
  const int LP = (int)std::max<size_t>(1, (size_t)8192 / N);
  const size_t smem = sizeof(C2) * ((size_t)N / 2 + (size_t)LP * (N + 1));
  auto kern = fftz_c2r_kernel<T>;
  CT2G_CUDA(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
  kern<<<ct2g_div_up(npairs, LP), 256, smem, ctx->stream>>>(in, out, logN, npairs, LP,
                                                            twiddle_ptr<C2>(ctx));
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

}  // namespace

// twiddles exp(-2 pi i k/N), k < N/2, computed on the host in FP64
int ct2g_twiddles(ct2g_ctx *ctx, int N) {
  if (ctx->tw_n == N) return CT2G_OK;
  if (ctx->tw32) cudaFree(ctx->tw32);
  if (ctx->tw64) cudaFree(ctx->tw64);
  ctx->tw32 = nullptr;
  ctx->tw64 = nullptr;
  ctx->tw_n = 0;
  const int h = N / 2;
  std::vector<float2> t32(h);
  std::vector<double2> t64(h);
  const double twopi = 6.283185307179586476925286766559;
  for (int k = 0; k < h; k++) {
    double a = -twopi * (double)k / (double)N;
    t64[k] = make_double2(std::cos(a), std::sin(a));
    t32[k] = make_float2((float)t64[k].x, (float)t64[k].y);
  }
  CT2G_CUDA(ctx, cudaMalloc(&ctx->tw32, sizeof(float2) * h));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->tw64, sizeof(double2) * h));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->tw32, t32.data(), sizeof(float2) * h,
                                 cudaMemcpyHostToDevice, ctx->stream));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->tw64, t64.data(), sizeof(double2) * h,
                                 cudaMemcpyHostToDevice, ctx->stream));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->tw_n = N;
  return CT2G_OK;
}

int ct2g_fft_r2c_f32(ct2g_ctx *ctx, const float *in, float2 *out, int N, int batch) {
  return fft_r2c<float>(ctx, in, out, N, batch);
}
int ct2g_fft_c2r_f32(ct2g_ctx *ctx, float2 *in, float *out, int N, int batch) {
  return fft_c2r<float>(ctx, in, out, N, batch);
}
int ct2g_fft_r2c_f64(ct2g_ctx *ctx, const double *in, double2 *out, int N, int batch) {
  return fft_r2c<double>(ctx, in, out, N, batch);
}
int ct2g_fft_c2r_f64(ct2g_ctx *ctx, double2 *in, double *out, int N, int batch) {
  return fft_c2r<double>(ctx, in, out, N, batch);
}
