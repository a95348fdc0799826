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
//   Y: complex FFT along j, tiles of W contiguous qk columns
//   X: complex FFT along i, tiles of W contiguous (qj,qk) columns
// A tile is staged in shared memory with coalesced loads.  Each line of
// N = R1*R2 points is transformed in two register stages (the "four-step"
// factorisation): R1 threads each do an R2-point DFT in registers over a
// stride-R1 subsequence, multiply by exp(-2 pi i n1 k2/N), and exchange
// through shared memory; R2 threads each then do an R1-point DFT.  The
// in-register DFTs are radix-2 decimation-in-frequency butterflies with
// compile-time twiddles.  Row tiles pad one word pair every R1 points so both
// exchange patterns are free of bank conflicts.
#include <type_traits>

#include <cuda.h>  // CUtensorMap and the cuTensorMapEncodeTiled signature (called through the runtime's entry point)

#include "ct2g_internal.cuh"
#include "ct2g_tc.cuh"

namespace {

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

// exp(-2 pi i k/32), k < 32, set at context creation from host FP64 cos/sin
__constant__ float2 c_w32f[32];
__constant__ double2 c_w32d[32];

template <typename C2> __device__ __forceinline__ C2 w32(int k);
template <> __device__ __forceinline__ float2 w32<float2>(int k) { return c_w32f[k]; }
template <> __device__ __forceinline__ double2 w32<double2>(int k) { return c_w32d[k]; }

template <typename C2>
__device__ __forceinline__ C2 cmul(C2 a, C2 b) {
  C2 r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
template <typename C2>
__device__ __forceinline__ C2 cadd(C2 a, C2 b) {
  C2 r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  return r;
}
template <typename C2>
__device__ __forceinline__ C2 csub(C2 a, C2 b) {
  C2 r;
  r.x = a.x - b.x;
  r.y = a.y - b.y;
  return r;
}
// FP32 complex sums as one packed f32x2 instruction (two round-to-nearest
// FP32 operations, the same results as the scalar pair)
template <>
__device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) {
  unsigned long long pa, pb, pr;
  asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b.x), "f"(b.y));
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(pr) : "l"(pa), "l"(pb));
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(pr));
  return r;
}
template <>
__device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  unsigned long long pa, pb, pr;
  asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a.x), "f"(a.y));
  asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b.x), "f"(b.y));
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(pr) : "l"(pa), "l"(pb));
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(pr));
  return r;
}

constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }
constexpr int brevc(int v, int bits) {
  int r = 0;
  for (int i = 0; i < bits; i++) r |= ((v >> i) & 1) << (bits - 1 - i);
  return r;
}

// In-register R-point DFT (R <= 32), natural order in and out.
// Radix-2 DIF: span h from R/2 down to 1, butterfly (a, b) ->
// (a + b, (a - b) W_{2h}^j); the result lands in bit-reversed order and is
// permuted back at compile time.  W = -i (a quarter turn) is a swap and a
// sign, not a complex product.
template <int R, typename C2, bool INV>
__device__ __forceinline__ void reg_dft(C2 (&v)[R]) {
#pragma unroll
  for (int h = R / 2; h >= 1; h >>= 1) {
#pragma unroll
    for (int blk = 0; blk < R; blk += 2 * h) {
#pragma unroll
      for (int j = 0; j < h; j++) {
        const C2 a = v[blk + j], b = v[blk + j + h];
        v[blk + j] = cadd(a, b);
        C2 d = csub(a, b);
        if (j * (32 / (2 * h)) == 8) {  // W = -i (forward), +i (inverse): a swap
          const C2 e = d;
          d.x = INV ? -e.y : e.y;
          d.y = INV ? e.x : -e.x;
        } else if (j != 0) {
          C2 w = w32<C2>(j * (32 / (2 * h)));
          if (INV) w.y = -w.y;
          d = cmul(d, w);
        }
        v[blk + j + h] = d;
      }
    }
  }
  C2 t[R];
#pragma unroll
  for (int k = 0; k < R; k++) t[k] = v[brevc(k, ilog2c(R))];
#pragma unroll
  for (int k = 0; k < R; k++) v[k] = t[k];
}

// Line FFTs on smem lines.  Layout ROWS: element (l, r) at
// l*(N + N/R1 + 1) + r + r/R1 (one pad every R1 points); layout COLS: element
// (l, r) at r*W + l.
template <int N, bool ROWS>
struct LineLayout {
  static constexpr int R2 = N >= 4 ? (1 << (ilog2c(N) / 2)) : 1;
  static constexpr int R1 = N / R2;  // R1 >= R2
  // odd in complex units, so that the same point of consecutive lines falls
  // in different banks
  static constexpr int LS = N + N / R1 + 1;
  __device__ __forceinline__ static int at(int l, int r, int W) {
    return ROWS ? l * LS + r + r / R1 : r * W + l;
  }
};

// Transform `nlines` lines (nlines*R1 and nlines*R2 jobs spread over the block).
// stw: N twiddles exp(-2 pi i k/N) in smem.
template <int N, bool ROWS, typename C2, bool INV>
__device__ __forceinline__ void tile_fft(C2 *s, int nlines, int W, const C2 *stw) {
  using LL = LineLayout<N, ROWS>;
  constexpr int R1 = LL::R1, R2 = LL::R2;
  // step 1: job (line, n1): R2-point DFT over r = n1 + R1*n2, twiddle.  The
  // block has 256 threads.
  for (int job = threadIdx.x; job < nlines * R1; job += blockDim.x) {
    int l, n1;
    if (ROWS) {
      n1 = job % R1;
      l = job / R1;
    } else {
      l = job % nlines;
      n1 = job / nlines;
    }
    C2 v[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; n2++) v[n2] = s[LL::at(l, n1 + R1 * n2, W)];
    reg_dft<R2, C2, INV>(v);
#pragma unroll
    for (int k2 = 1; k2 < R2; k2++) {
      C2 w = stw[(n1 * k2) & (N - 1)];
      if (INV) w.y = -w.y;
      v[k2] = cmul(v[k2], w);
    }
    // Y[n1][k2] back into the slots just read (slot n1 + R1*k2)
#pragma unroll
    for (int k2 = 0; k2 < R2; k2++) s[LL::at(l, n1 + R1 * k2, W)] = v[k2];
  }
  __syncthreads();
  // step 2: job (line, k2): R1-point DFT over n1 -> X[k2 + R2*k1].  Jobs go
  // in rounds of whole lines (LW lines per round), so a round's writes never
  // touch slots that a later round still has to read.
  constexpr int LW = 256 / R2;
  for (int l0 = 0; l0 < nlines; l0 += LW) {
    int l, k2;
    if (ROWS) {
      k2 = threadIdx.x % R2;
      l = l0 + threadIdx.x / R2;
    } else {
      l = l0 + threadIdx.x % LW;
      k2 = threadIdx.x / LW;
    }
    const bool on = l < nlines;
    C2 v[R1];
    if (on) {
#pragma unroll
      for (int n1 = 0; n1 < R1; n1++) v[n1] = s[LL::at(l, n1 + R1 * k2, W)];
      reg_dft<R1, C2, INV>(v);
    }
    __syncthreads();  // all reads of this round before any write
    if (on) {
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) s[LL::at(l, k2 + R2 * k1, W)] = v[k1];
    }
    __syncthreads();
  }
}

template <typename C2>
__device__ __forceinline__ void load_twiddles(C2 *stw, const C2 *tw, int n) {
  for (int k = threadIdx.x; k < n; k += blockDim.x) stw[k] = tw[k];
}

// ---- pass Z forward: pairs of real lines -> half spectra -------------------
// LP complex (packed) lines per block; npairs = number of real-line pairs;
// output rows hold ld >= N/2+1 complex (the rest is written as zero).  VEC:
// ld*sizeof(complex) is a multiple of 16 bytes.
template <typename T, int N, bool VEC>
__global__ void __launch_bounds__(256, 3) fftz_r2c_kernel(const T *__restrict__ in,
                                                          typename Cplx<T>::type *__restrict__ out,
                                                          size_t npairs, int LP, int ld,
                                                          const typename Cplx<T>::type *__restrict__ tw) {
  using C2 = typename Cplx<T>::type;
  using LL = LineLayout<N, true>;
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int NH = N / 2 + 1;
  constexpr int RC = 16 / sizeof(T);  // reals per 16-byte chunk
  using RV = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  C2 *stw = reinterpret_cast<C2 *>(smraw);
  C2 *s = stw + N;
  T *sr = reinterpret_cast<T *>(s);
  load_twiddles(stw, tw, N);
  const size_t pair0 = (size_t)blockIdx.x * LP;
  const int np = (int)min((size_t)LP, npairs - pair0);
  const T *src = in + pair0 * 2 * N;
  // real line 2l -> .x of complex line l, real line 2l+1 -> .y
  for (int c = threadIdx.x; c < np * 2 * N / RC; c += 256) {
    const int e = c * RC, rl = e / N, r = e % N;
    const RV v = *reinterpret_cast<const RV *>(src + e);
    const T *vv = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int q = 0; q < RC; q++) sr[2 * LL::at(rl >> 1, r + q, 0) + (rl & 1)] = vv[q];
  }
  __syncthreads();
  tile_fft<N, true, C2, false>(s, np, 0, stw);
  C2 *dst = out + pair0 * 2 * (size_t)ld;
  constexpr int CC = (VEC && sizeof(C2) == 8) ? 2 : 1;  // complex per store
  const int nchunk = ld / CC;
  for (int c = threadIdx.x; c < np * nchunk; c += 256) {
    const int l = c / nchunk, k0 = (c % nchunk) * CC;
    C2 a[CC], b[CC];
#pragma unroll
    for (int q = 0; q < CC; q++) {
      const int k = k0 + q;
      if (k < NH) {
        const C2 zk = s[LL::at(l, k & (N - 1), 0)];
        const C2 zc = s[LL::at(l, (N - k) & (N - 1), 0)];
        // A_k = (Z_k + conj Z_{N-k})/2, B_k = (Z_k - conj Z_{N-k})/(2i)
        a[q].x = (T)0.5 * (zk.x + zc.x);
        a[q].y = (T)0.5 * (zk.y - zc.y);
        b[q].x = (T)0.5 * (zk.y + zc.y);
        b[q].y = (T)0.5 * (zc.x - zk.x);
      } else {
        a[q].x = a[q].y = b[q].x = b[q].y = (T)0;
      }
    }
    if (CC == 2) {
      *reinterpret_cast<float4 *>(dst + (size_t)(2 * l) * ld + k0) = *reinterpret_cast<float4 *>(a);
      *reinterpret_cast<float4 *>(dst + (size_t)(2 * l + 1) * ld + k0) = *reinterpret_cast<float4 *>(b);
    } else {
      dst[(size_t)(2 * l) * ld + k0] = a[0];
      dst[(size_t)(2 * l + 1) * ld + k0] = b[0];
    }
  }
}

// ---- pass Z inverse: pairs of half spectra -> real lines --------------------
template <typename T, int N, bool VEC>
__global__ void __launch_bounds__(256, 3) fftz_c2r_kernel(const typename Cplx<T>::type *__restrict__ in,
                                                          T *__restrict__ out, size_t npairs, int LP,
                                                          int ld,
                                                          const typename Cplx<T>::type *__restrict__ tw) {
  using C2 = typename Cplx<T>::type;
  using LL = LineLayout<N, true>;
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int NH = N / 2 + 1;
  constexpr int RC = 16 / sizeof(T);
  using RV = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
  C2 *stw = reinterpret_cast<C2 *>(smraw);
  C2 *s = stw + N;
  const T *sr = reinterpret_cast<const T *>(s);
  load_twiddles(stw, tw, N);
  const size_t pair0 = (size_t)blockIdx.x * LP;
  const int np = (int)min((size_t)LP, npairs - pair0);
  const C2 *src = in + pair0 * 2 * (size_t)ld;
  constexpr int CC = (VEC && sizeof(C2) == 8) ? 2 : 1;
  constexpr int NCH = (NH + CC - 1) / CC;  // chunks covering k = 0..N/2
  for (int c = threadIdx.x; c < np * NCH; c += 256) {
    const int l = c / NCH, k0 = (c % NCH) * CC;
    C2 a[CC], b[CC];
    if (CC == 2) {
      *reinterpret_cast<float4 *>(a) = *reinterpret_cast<const float4 *>(src + (size_t)(2 * l) * ld + k0);
      *reinterpret_cast<float4 *>(b) = *reinterpret_cast<const float4 *>(src + (size_t)(2 * l + 1) * ld + k0);
    } else {
      a[0] = src[(size_t)(2 * l) * ld + k0];
      b[0] = src[(size_t)(2 * l + 1) * ld + k0];
    }
#pragma unroll
    for (int q = 0; q < CC; q++) {
      const int k = k0 + q;
      if (k >= NH) continue;
      // Z_k = A_k + i B_k; Z_{N-k} = conj(A_k) + i conj(B_k)
      C2 z;
      z.x = a[q].x - b[q].y;
      z.y = a[q].y + b[q].x;
      s[LL::at(l, k, 0)] = z;
      if (k > 0 && k < N / 2) {
        C2 w;
        w.x = a[q].x + b[q].y;
        w.y = -a[q].y + b[q].x;
        s[LL::at(l, N - k, 0)] = w;
      }
    }
  }
  __syncthreads();
  tile_fft<N, true, C2, true>(s, np, 0, stw);
  T *dst = out + pair0 * 2 * N;
  for (int c = threadIdx.x; c < np * 2 * N / RC; c += 256) {
    const int e = c * RC, rl = e / N, r = e % N;
    RV v;
    T *vv = reinterpret_cast<T *>(&v);
#pragma unroll
    for (int q = 0; q < RC; q++) vv[q] = sr[2 * LL::at(rl >> 1, r + q, 0) + (rl & 1)];
    *reinterpret_cast<RV *>(dst + e) = v;
  }
}

// ---- strided passes: FFT along rows for tiles of W contiguous columns -------
// array: outer blocks of `ostride` elements; inside, rows of `rstride`; ncols
// valid columns per row.  grid.x = nouter * ntiles.  VEC: rows start on
// 16-byte boundaries, so the tile moves in 16-byte chunks.
template <typename C2, int N, int W, bool INV, bool VEC>
__global__ void __launch_bounds__(256, 3) fft_cols_kernel(C2 *__restrict__ a, size_t ostride,
                                                          size_t rstride, size_t ncols,
                                                          int ntiles, const C2 *__restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C2 *stw = reinterpret_cast<C2 *>(smraw);
  C2 *s = stw + N;
  load_twiddles(stw, tw, N);
  const size_t outer = blockIdx.x / ntiles;
  const size_t col0 = (size_t)(blockIdx.x % ntiles) * W;
  const int wv = (int)min((size_t)W, ncols - col0);
  C2 *base = a + outer * ostride + col0;
  // complex elements per 16-byte chunk
  constexpr int CPC = (VEC && sizeof(C2) == 8) ? 2 : 1;
  constexpr int CH = W / CPC;  // chunks per row
  using V = typename std::conditional<CPC == 2, float4, C2>::type;
#pragma unroll 4
  for (int e = threadIdx.x; e < N * CH; e += 256) {
    const int r = e / CH, c = (e % CH) * CPC;
    if (c < wv) *reinterpret_cast<V *>(s + r * W + c) = *reinterpret_cast<const V *>(base + (size_t)r * rstride + c);
  }
  __syncthreads();
  tile_fft<N, false, C2, INV>(s, W, W, stw);
#pragma unroll 4
  for (int e = threadIdx.x; e < N * CH; e += 256) {
    const int r = e / CH, c = (e % CH) * CPC;
    if (c < wv) *reinterpret_cast<V *>(base + (size_t)r * rstride + c) = *reinterpret_cast<const V *>(s + r * W + c);
  }
}

// Persistent, double-buffered form of the column pass for 16-byte aligned
// rows: each block walks tiles blockIdx.x, blockIdx.x + gridDim.x, ...; the
// next tile is copied into the second smem buffer with cp.async while the
// current one is transformed and written back.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}

template <typename C2, int N, int W, bool INV>
__global__ void __launch_bounds__(256, 2) fft_cols_pipe_kernel(C2 *__restrict__ a, size_t ostride,
                                                               size_t rstride, size_t ncols,
                                                               int ntiles, size_t ntot,
                                                               const C2 *__restrict__ tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C2 *stw = reinterpret_cast<C2 *>(smraw);
  C2 *buf[2] = {stw + N, stw + N + N * W};
  load_twiddles(stw, tw, N);
  constexpr int CPC = 16 / sizeof(C2);  // complex per 16-byte chunk
  constexpr int CH = W / CPC;           // chunks per row
  auto issue = [&](size_t tile, C2 *s) {
    const size_t outer = tile / ntiles;
    const size_t col0 = (size_t)(tile % ntiles) * W;
    const int wv = (int)min((size_t)W, ncols - col0);
    const C2 *base = a + outer * ostride + col0;
#pragma unroll 4
    for (int e = threadIdx.x; e < N * CH; e += 256) {
      const int r = e / CH, c = (e % CH) * CPC;
      if (c < wv) cp_async16(s + r * W + c, base + (size_t)r * rstride + c);
    }
  };
  size_t tile = blockIdx.x;
  if (tile < ntot) issue(tile, buf[0]);
  cp_async_commit();
  for (int it = 0; tile < ntot; it++, tile += gridDim.x) {
    C2 *s = buf[it & 1];
    const size_t next = tile + gridDim.x;
    if (next < ntot) issue(next, buf[(it + 1) & 1]);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    tile_fft<N, false, C2, INV>(s, W, W, stw);
    const size_t outer = tile / ntiles;
    const size_t col0 = (size_t)(tile % ntiles) * W;
    const int wv = (int)min((size_t)W, ncols - col0);
    C2 *base = a + outer * ostride + col0;
#pragma unroll 4
    for (int e = threadIdx.x; e < N * CH; e += 256) {
      const int r = e / CH, c = (e % CH) * CPC;
      if (c < wv) *reinterpret_cast<float4 *>(base + (size_t)r * rstride + c) = *reinterpret_cast<const float4 *>(s + r * W + c);
    }
    __syncthreads();  // this buffer is refilled two tiles later
  }
  cp_async_wait<0>();
}

template <typename C2>
const C2 *twiddle_ptr(ct2g_ctx *ctx);
template <>
const float2 *twiddle_ptr<float2>(ct2g_ctx *ctx) { return ctx->tw32; }
template <>
const double2 *twiddle_ptr<double2>(ct2g_ctx *ctx) { return ctx->tw64; }

template <typename C2, int N, int W, bool INV>
int launch_pipe(ct2g_ctx *ctx, C2 *spec, size_t nouter, size_t ostride, size_t rstride,
                size_t ncols) {
  const size_t smem = sizeof(C2) * ((size_t)N + 2 * (size_t)N * W);
  auto k = fft_cols_pipe_kernel<C2, N, W, INV>;
  CT2G_TRY(ct2g_smem_attrs(ctx, k, smem));
  int per_sm = 0;
  CT2G_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, smem));
  // the query can miss the maximum carveout the attributes ask for: count
  // from the kernel's registers and shared memory as well, keep the larger
  per_sm = std::max(per_sm, ct2g_blocks_per_sm(ctx, (const void *)k, 256, smem));
  const int ntiles = (int)((ncols + W - 1) / W);
  const size_t ntot = nouter * ntiles;
  const size_t grid = std::min(ntot, (size_t)std::max(1, per_sm) * ctx->num_sms);
  k<<<(unsigned)grid, 256, smem, ctx->stream>>>(spec, ostride, rstride, ncols, ntiles, ntot,
                                                twiddle_ptr<C2>(ctx));
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// ---- y pass with tiles moved by TMA --------------------------------------------
// The same column transform as fft_cols_pipe_kernel on the spectrum's y pass,
// with each tile (N rows x W complex columns of one plane) brought into shared
// memory by one tiled bulk tensor copy and written back by another: a
// persistent block keeps S tiles in flight (S - 1 loading while one is
// transformed), completion through one mbarrier per stage (bounded waits), and
// no thread spends issue slots on addresses or copies.  The tensor map views
// the spectrum as floats [plane][y][2 * ldk * NC]; x coordinates are
// multiples of 2W floats (16-byte aligned), and the last tile of a row reads
// zeros past its end and stores nothing there.
constexpr uint32_t kTmaWaitLimit = 1u << 22;

template <int N, int W, bool INV, int S>
__global__ void __launch_bounds__(256, 1) fft_cols_tma_kernel(
    const __grid_constant__ CUtensorMap map, uint32_t ntiles, uint32_t ntot,
    const float2 *__restrict__ tw, uint32_t *__restrict__ status) {
  // the tensor copies need 128-byte aligned shared memory: the tiles start at
  // the first 128-byte boundary of the dynamic region (128 bytes reserved for
  // it), whatever offset the static variables leave that region at
  extern __shared__ __align__(128) unsigned char smraw[];
  const uint32_t pad = (128u - (tc::smem_addr(smraw) & 127u)) & 127u;
  float2 *buf = reinterpret_cast<float2 *>(smraw + pad);  // S tiles of N * W
  float2 *stw = buf + S * N * W;
  __shared__ uint64_t bar[S];
  const int tid = threadIdx.x;
  if (tc::smem_addr(buf) & 127u) {  // not reached: checked before any copy
    if (tid == 0) atomicExch(status, (uint32_t)CT2G_ECUDA);
    return;
  }
  load_twiddles(stw, tw, N);
  if (tid == 0)
    for (int k = 0; k < S; k++) tc::mbar_init(&bar[k], 1);
  __syncthreads();
  // a tensor copy's box holds at most 256 rows: N = 512 moves as two boxes
  constexpr int NB = (N + 255) / 256, BR = N / NB;
  auto issue = [&](uint32_t t, int k) {  // thread 0
    tc::mbar_arrive_expect_tx(&bar[k], (uint32_t)(N * W * sizeof(float2)));
#pragma unroll
    for (int b = 0; b < NB; b++)
      tc::tma_load_3d(buf + k * N * W + b * BR * W, &map, (int)(2 * W * (t % ntiles)), b * BR,
                      (int)(t / ntiles), &bar[k]);
  };
  uint32_t t = blockIdx.x;
  if (tid == 0)
    for (int k = 0; k < S - 1; k++)
      if (t + k * gridDim.x < ntot) issue(t + k * gridDim.x, k);
  uint32_t parity = 0;
  bool ok = true;
  for (int it = 0; t < ntot; t += gridDim.x, it++) {
    const int k = it % S;
    if (tid == 0) {
      // the next tile goes into the previous tile's stage once its store has
      // read it
      const uint32_t tn = t + (S - 1) * gridDim.x;
      if (tn < ntot) {
        tc::bulk_wait_read();
        issue(tn, (it + S - 1) % S);
      }
    }
    ok = tc::mbar_wait(&bar[k], (parity >> k) & 1u, kTmaWaitLimit);
    parity ^= 1u << k;
    if (!__syncthreads_and(ok)) break;
    float2 *s = buf + k * N * W;
    tile_fft<N, false, float2, INV>(s, W, W, stw);
    tc::fence_async_smem();  // this thread's writes, before the bulk store reads them
    __syncthreads();
    if (tid == 0) {
#pragma unroll
      for (int b = 0; b < NB; b++)
        tc::tma_store_3d(&map, (int)(2 * W * (t % ntiles)), b * BR, (int)(t / ntiles),
                         s + b * BR * W);
      tc::bulk_commit();
    }
  }
  if (tid == 0) {
    if (!ok) {
      atomicExch(status, (uint32_t)CT2G_ETIMEOUT);
      // loads still in flight land before the block's shared memory goes away
      for (int k = 0; k < S; k++) tc::mbar_wait(&bar[k], (parity >> k) & 1u, kTmaWaitLimit);
    }
    tc::bulk_wait_all();
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// the driver's tensor-map encoder, looked up once through the runtime
int tensor_map_encoder(ct2g_ctx *ctx, EncodeTiledFn *out) {
  static EncodeTiledFn encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
      cudaGetLastError();
      return ct2g_fail(ctx, CT2G_ECUDA, "cuTensorMapEncodeTiled not available");
    }
    encode = reinterpret_cast<EncodeTiledFn>(fn);
  }
  *out = encode;
  return CT2G_OK;
}

// The tensor map of a column pass over complex FP32 data: `nouter` blocks
// (ostride complex apart) of N rows (rstride complex apart), seen as floats
// [outer][row][2 * rstride]; a box is W complex columns x N / NB rows.
int cols_map(ct2g_ctx *ctx, void *base, size_t nouter, size_t ostride, size_t rstride, int N,
             int W, CUtensorMap *m) {
  EncodeTiledFn encode = nullptr;
  CT2G_TRY(tensor_map_encoder(ctx, &encode));
  const cuuint64_t dims[3] = {2 * (cuuint64_t)rstride, (cuuint64_t)N, (cuuint64_t)nouter};
  const cuuint64_t strides[2] = {rstride * sizeof(float2), ostride * sizeof(float2)};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * W), (cuuint32_t)(N > 256 ? 256 : N), 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  if (encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return ct2g_fail(ctx, CT2G_ECUDA, "column-pass tensor map");
  return CT2G_OK;
}

// a column pass (y pass, or an x pass over whole planes) with its tiles moved
// by TMA: N rows x W columns per tile (W 32, or 16 with fft_tile 16 and at
// N = 512), three tiles in flight per block; the data 16-byte aligned with
// rstride and ostride even (the callers' vector condition)
template <int N, bool INV>
int launch_cols_tma(ct2g_ctx *ctx, float2 *data, size_t nouter, size_t ostride, size_t rstride,
                    size_t ncols) {
  if constexpr (N < 64 || N > 512) {
    return ct2g_fail(ctx, CT2G_EINVAL, "TMA column pass: sizes 64-512");
  } else {
    const bool narrow = N > 256 || ctx->fft_tile == 16;
    const int W = narrow ? 16 : 32;
    alignas(64) CUtensorMap map;
    CT2G_TRY(cols_map(ctx, data, nouter, ostride, rstride, N, W, &map));
    const uint32_t ntiles = (uint32_t)((ncols + W - 1) / W), ntot = ntiles * (uint32_t)nouter;
    auto k = fft_cols_tma_kernel<N, 16, INV, 3>;
    if constexpr (N <= 256)
      if (!narrow) k = fft_cols_tma_kernel<N, 32, INV, 3>;
    const size_t smem = sizeof(float2) * (3 * (size_t)N * W + N) + 128;
    CT2G_TRY(ct2g_smem_attrs(ctx, k, smem));
    const int per_sm = ct2g_blocks_per_sm(ctx, (const void *)k, 256, smem);
    const uint32_t grid = std::min(ntot, (uint32_t)(per_sm * ctx->num_sms));
    k<<<grid, 256, smem, ctx->stream>>>(map, ntiles, ntot, twiddle_ptr<float2>(ctx),
                                        ctx->d_counts + 6);
    CT2G_LAUNCHED(ctx);
    return CT2G_OK;
  }
}

// column tile widths: the default W, and W/2 or 2W (FP32 only) when the
// context's tuning asks for them and the double buffer fits in shared memory
template <typename T, int N, bool INV, bool VEC>
int launch_cols(ct2g_ctx *ctx, typename Cplx<T>::type *spec, size_t nouter, size_t ostride,
                size_t rstride, size_t ncols) {
  using C2 = typename Cplx<T>::type;
  if constexpr (sizeof(C2) == 8 && N >= 64 && N <= 512) {
    // FP32 columns with 16-byte aligned rows: tiles moved by TMA (tuning cols_tma)
    if (VEC && ctx->cols_tma)
      return launch_cols_tma<N, INV>(ctx, spec, nouter, ostride, rstride, ncols);
  }
  // 16-column tiles from N = 256 on; FP64 at N = 512 takes 8 so that the
  // double-buffered tile fits in shared memory
  constexpr int W = N >= 256 ? (sizeof(C2) == 16 && N >= 512 ? 8 : 16) : 4096 / N;
  if (VEC && N >= 64) {
    if constexpr (sizeof(C2) == 8) {
      if (ctx->fft_tile == W / 2)
        return launch_pipe<C2, N, W / 2, INV>(ctx, spec, nouter, ostride, rstride, ncols);
      if constexpr (sizeof(C2) * ((size_t)N + 4 * (size_t)N * W) <= 200 * 1024)
        if (ctx->fft_tile == 2 * W)
          return launch_pipe<C2, N, 2 * W, INV>(ctx, spec, nouter, ostride, rstride, ncols);
    }
    return launch_pipe<C2, N, W, INV>(ctx, spec, nouter, ostride, rstride, ncols);
  }
  const size_t smem = sizeof(C2) * ((size_t)N + (size_t)N * W);
  auto k = fft_cols_kernel<C2, N, W, INV, VEC>;
  CT2G_TRY(ct2g_smem_attrs(ctx, k, smem));
  const int ntiles = (int)((ncols + W - 1) / W);
  k<<<(unsigned)(nouter * ntiles), 256, smem, ctx->stream>>>(spec, ostride, rstride, ncols, ntiles,
                                                             twiddle_ptr<C2>(ctx));
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// Y and X passes over a spectrum whose qk rows hold ld >= N/2+1 elements (a
// half spectrum: the Y pass transforms its first N/2+1 columns) or, `full`,
// N elements (a complex grid: every column)
template <typename T, int N>
int run_cols(ct2g_ctx *ctx, typename Cplx<T>::type *spec, int batch, bool inv, size_t ld,
             bool full = false) {
  using C2 = typename Cplx<T>::type;
  const size_t NH = full ? (size_t)N : (size_t)N / 2 + 1;
  const bool vec = (ld * sizeof(C2)) % 16 == 0;
  for (int pass = 0; pass < 2; pass++) {
    const bool ypass = (pass == 0) != inv;
    size_t nouter, ostride, rstride, ncols;
    if (ypass) {
      nouter = (size_t)batch * N;
      ostride = (size_t)N * ld;
      rstride = ld;
      ncols = NH;
    } else {
      nouter = (size_t)batch;
      ostride = (size_t)N * N * ld;
      rstride = (size_t)N * ld;
      ncols = (size_t)N * ld;
    }
    if constexpr (sizeof(C2) == 8 && (N == 256 || N == 512)) {
      if (ctx->fft_tc) {
        CT2G_TRY(ct2g_fft_cols_tc(ctx, spec, N, nouter, ostride, rstride, ncols, inv));
        continue;
      }
    }
    if (inv) {
      if (vec) CT2G_TRY((launch_cols<T, N, true, true>(ctx, spec, nouter, ostride, rstride, ncols)));
      else CT2G_TRY((launch_cols<T, N, true, false>(ctx, spec, nouter, ostride, rstride, ncols)));
    } else {
      if (vec) CT2G_TRY((launch_cols<T, N, false, true>(ctx, spec, nouter, ostride, rstride, ncols)));
      else CT2G_TRY((launch_cols<T, N, false, false>(ctx, spec, nouter, ostride, rstride, ncols)));
    }
  }
  return CT2G_OK;
}

template <typename T, int N>
int fft_r2c_n(ct2g_ctx *ctx, const T *in, typename Cplx<T>::type *out, int batch, int ld) {
  using C2 = typename Cplx<T>::type;
  const size_t npairs = (size_t)batch * N * N / 2;
  const int LP = std::max(1, 4096 / N);
  const size_t smem = sizeof(C2) * ((size_t)N + (size_t)LP * LineLayout<N, true>::LS);
  const bool vec = ((size_t)ld * sizeof(C2)) % 16 == 0;
  auto kern = vec ? fftz_r2c_kernel<T, N, true> : fftz_r2c_kernel<T, N, false>;
  CT2G_TRY(ct2g_smem_attrs(ctx, kern, smem));
  kern<<<ct2g_div_up(npairs, LP), 256, smem, ctx->stream>>>(in, out, npairs, LP, ld,
                                                            twiddle_ptr<C2>(ctx));
  CT2G_LAUNCHED(ctx);
  return run_cols<T, N>(ctx, out, batch, false, ld);
}

template <typename T, int N>
int fft_c2r_n(ct2g_ctx *ctx, typename Cplx<T>::type *in, T *out, int batch, int ld) {
  using C2 = typename Cplx<T>::type;
  CT2G_TRY((run_cols<T, N>(ctx, in, batch, true, ld)));
  const size_t npairs = (size_t)batch * N * N / 2;
  const int LP = std::max(1, 4096 / N);
  const size_t smem = sizeof(C2) * ((size_t)N + (size_t)LP * LineLayout<N, true>::LS);
  const bool vec = ((size_t)ld * sizeof(C2)) % 16 == 0;
  auto kern = vec ? fftz_c2r_kernel<T, N, true> : fftz_c2r_kernel<T, N, false>;
  CT2G_TRY(ct2g_smem_attrs(ctx, kern, smem));
  kern<<<ct2g_div_up(npairs, LP), 256, smem, ctx->stream>>>(in, out, npairs, LP, ld,
                                                            twiddle_ptr<C2>(ctx));
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

template <typename T>
int fft_r2c(ct2g_ctx *ctx, const T *in, typename Cplx<T>::type *out, int N, int batch, int ld) {
  CT2G_TRY(ct2g_twiddles(ctx, N));
  switch (N) {
    case 4: return fft_r2c_n<T, 4>(ctx, in, out, batch, ld);
    case 8: return fft_r2c_n<T, 8>(ctx, in, out, batch, ld);
    case 16: return fft_r2c_n<T, 16>(ctx, in, out, batch, ld);
    case 32: return fft_r2c_n<T, 32>(ctx, in, out, batch, ld);
    case 64: return fft_r2c_n<T, 64>(ctx, in, out, batch, ld);
    case 128: return fft_r2c_n<T, 128>(ctx, in, out, batch, ld);
    case 256: return fft_r2c_n<T, 256>(ctx, in, out, batch, ld);
    case 512: return fft_r2c_n<T, 512>(ctx, in, out, batch, ld);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "FFT size must be a power of two in [4, 512]");
}

template <typename T>
int fft_c2r(ct2g_ctx *ctx, typename Cplx<T>::type *in, T *out, int N, int batch, int ld) {
  CT2G_TRY(ct2g_twiddles(ctx, N));
  switch (N) {
    case 4: return fft_c2r_n<T, 4>(ctx, in, out, batch, ld);
    case 8: return fft_c2r_n<T, 8>(ctx, in, out, batch, ld);
    case 16: return fft_c2r_n<T, 16>(ctx, in, out, batch, ld);
    case 32: return fft_c2r_n<T, 32>(ctx, in, out, batch, ld);
    case 64: return fft_c2r_n<T, 64>(ctx, in, out, batch, ld);
    case 128: return fft_c2r_n<T, 128>(ctx, in, out, batch, ld);
    case 256: return fft_c2r_n<T, 256>(ctx, in, out, batch, ld);
    case 512: return fft_c2r_n<T, 512>(ctx, in, out, batch, ld);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "FFT size must be a power of two in [4, 512]");
}

// ---- complex-to-complex 3D FFT ------------------------------------------------
// Pass Z of a complex grid a[b][i][j][k] (k contiguous, N per row): LP rows
// per block through shared memory, moved in 16-byte chunks (two complex
// values); the Y and X passes are the column passes of the real transforms
// over every column (run_cols, `full`).
template <int N, bool INV>
__global__ void __launch_bounds__(256, 3) fftz_c2c_kernel(float2 *__restrict__ a, size_t nrows,
                                                          int LP, const float2 *__restrict__ tw) {
  using LL = LineLayout<N, true>;
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *stw = reinterpret_cast<float2 *>(smraw);
  float2 *s = stw + N;
  load_twiddles(stw, tw, N);
  const size_t row0 = (size_t)blockIdx.x * LP;
  const int nr = (int)min((size_t)LP, nrows - row0);
  float2 *g = a + row0 * N;
  for (int c = threadIdx.x; c < nr * N / 2; c += 256) {
    const int e = 2 * c, l = e / N, r = e % N;
    const float4 v = *reinterpret_cast<const float4 *>(g + e);
    s[LL::at(l, r, 0)] = make_float2(v.x, v.y);
    s[LL::at(l, r + 1, 0)] = make_float2(v.z, v.w);
  }
  __syncthreads();
  tile_fft<N, true, float2, INV>(s, nr, 0, stw);
  for (int c = threadIdx.x; c < nr * N / 2; c += 256) {
    const int e = 2 * c, l = e / N, r = e % N;
    const float2 u = s[LL::at(l, r, 0)], w = s[LL::at(l, r + 1, 0)];
    *reinterpret_cast<float4 *>(g + e) = make_float4(u.x, u.y, w.x, w.y);
  }
}

template <int N>
int fft_c2c_n(ct2g_ctx *ctx, float2 *a, int batch, bool inv) {
  const size_t nrows = (size_t)batch * N * N;
  const int LP = std::max(1, 4096 / N);
  const size_t smem = sizeof(float2) * ((size_t)N + (size_t)LP * LineLayout<N, true>::LS);
  auto kern = inv ? fftz_c2c_kernel<N, true> : fftz_c2c_kernel<N, false>;
  if (inv) CT2G_TRY((run_cols<float, N>(ctx, a, batch, true, N, true)));
  CT2G_TRY(ct2g_smem_attrs(ctx, kern, smem));
  kern<<<ct2g_div_up(nrows, LP), 256, smem, ctx->stream>>>(a, nrows, LP, twiddle_ptr<float2>(ctx));
  CT2G_LAUNCHED(ctx);
  if (!inv) CT2G_TRY((run_cols<float, N>(ctx, a, batch, false, N, true)));
  return CT2G_OK;
}

int fft_c2c(ct2g_ctx *ctx, float2 *a, int N, int batch, bool inv) {
  CT2G_TRY(ct2g_twiddles(ctx, N));
  switch (N) {
    case 4: return fft_c2c_n<4>(ctx, a, batch, inv);
    case 8: return fft_c2c_n<8>(ctx, a, batch, inv);
    case 16: return fft_c2c_n<16>(ctx, a, batch, inv);
    case 32: return fft_c2c_n<32>(ctx, a, batch, inv);
    case 64: return fft_c2c_n<64>(ctx, a, batch, inv);
    case 128: return fft_c2c_n<128>(ctx, a, batch, inv);
    case 256: return fft_c2c_n<256>(ctx, a, batch, inv);
    case 512: return fft_c2c_n<512>(ctx, a, batch, inv);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "FFT size must be a power of two in [4, 512]");
}

// ---- the mesh solve's spectrum ------------------------------------------------
// ctx->spec keeps the NC components of a k-point side by side,
// [box][qi][qj][qk][NC] with qk < ldk, so that a (qi, qj) row is RS = ldk*NC
// complex values (16-byte aligned rows: ldk is even; slots qk > N/2 hold
// zeros).  The z passes write and read whole rows; the Y pass transforms tiles
// of W contiguous (qk, c) columns; the X pass runs inside the MG2L kernel,
// whose block holds every component of one (qj, qk) column.

// (x, y) lines per block of a z pass that reads or writes the moment grid:
// enough packed lines for a block's transform to fill its threads (one line
// when the components alone give 16 packed lines or more)
template <int P>
constexpr int z_lines() {
  constexpr int NL = (ct2g_ncomp(P) + 1) / 2;
  return NL >= 8 ? 1 : NL >= 4 ? 2 : NL >= 2 ? 4 : 8;
}

// ---- forward z pass fused with P2M -----------------------------------------
// One block per (x, y) line of one box: the moments of the line's N cells
// (FP64 sums about the cell centres, as p2m_kernel) go straight into shared
// memory as FP32, components paired into complex lines (2l -> .x, 2l+1 ->
// .y), are transformed along z and split into the half spectra of the two
// components.  The moment grid is never written to HBM.  A thread sums a
// cell of up to kWarpCell particles; bigger cells are summed by a warp
// (lanes stride over the particles, partial moments reduced by shuffles), so
// no block waits on one thread's long loop: a thread's FP64 sums are a serial
// chain, and a block's transform waits for its slowest cell.  GRID: the moments are read from
// the moment grid (component k of box b at grid + (k * nbox + b) * N^3).
constexpr uint32_t kWarpCell = 6;

// components [K0, K1) of one particle's moments about the cell centre u
template <int P, int K0, int K1>
__device__ __forceinline__ void p2m_accumulate(const uint32_t *__restrict__ px,
                                               const uint32_t *__restrict__ py,
                                               const uint32_t *__restrict__ pz, uint32_t i,
                                               uint32_t ux, uint32_t uy, uint32_t uz,
                                               double *acc) {
  constexpr MiTable<P> T{};
  const double sx = -(double)(int32_t)(px[i] - ux) * CT2G_TWO_M32;
  const double sy = -(double)(int32_t)(py[i] - uy) * CT2G_TWO_M32;
  const double sz = -(double)(int32_t)(pz[i] - uz) * CT2G_TWO_M32;
  double qx[P + 1], qy[P + 1], qz[P + 1];
  qx[0] = qy[0] = qz[0] = 1.0;
#pragma unroll
  for (int q = 1; q <= P; q++) {
    qx[q] = qx[q - 1] * sx * (1.0 / q);
    qy[q] = qy[q - 1] * sy * (1.0 / q);
    qz[q] = qz[q - 1] * sz * (1.0 / q);
  }
#pragma unroll
  for (int k = K0; k < K1; k++) acc[k - K0] += qx[T.nx[k]] * qy[T.ny[k]] * qz[T.nz[k]];
}

// the moments of cell particles b, b + step, ... < e (a thread: step 1; a
// warp: lane offset, step 32, then summed over the warp) into the packed smem
// lines at z, for components [K0, K1): the components go in two halves so
// that only half of the FP64 sums are live at once
template <int P, int K0, int K1, typename ST>
__device__ __forceinline__ void p2m_group(const uint32_t *__restrict__ px,
                                          const uint32_t *__restrict__ py,
                                          const uint32_t *__restrict__ pz, uint32_t b, uint32_t e,
                                          uint32_t step, bool warp_sum, uint32_t ux, uint32_t uy,
                                          uint32_t uz, bool write, ST st) {
  double acc[K1 - K0];
#pragma unroll
  for (int k = 0; k < K1 - K0; k++) acc[k] = 0.0;
  for (uint32_t i = b; i < e; i += step) p2m_accumulate<P, K0, K1>(px, py, pz, i, ux, uy, uz, acc);
  if (warp_sum) {
#pragma unroll
    for (int k = 0; k < K1 - K0; k++) {
      double v = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      acc[k] = v;
    }
  }
  if (write) {
#pragma unroll
    for (int k = K0; k < K1; k++) st(k, (float)acc[k - K0]);
  }
}

// the same sums into the packed smem lines at z
template <int P, int N, int K0, int K1>
__device__ __forceinline__ void p2m_half(const uint32_t *__restrict__ px,
                                         const uint32_t *__restrict__ py,
                                         const uint32_t *__restrict__ pz, uint32_t b, uint32_t e,
                                         uint32_t step, bool warp_sum, uint32_t ux, uint32_t uy,
                                         uint32_t uz, int z, float *sr, bool write) {
  using LL = LineLayout<N, true>;
  p2m_group<P, K0, K1>(px, py, pz, b, e, step, warp_sum, ux, uy, uz, write,
                       [&](int k, float v) { sr[2 * LL::at(k >> 1, z, 0) + (k & 1)] = v; });
}

// ---- P2M into compact per-cell records ---------------------------------------
// The moments of every occupied cell (the same FP64 sums about the cell
// centre as the fused z pass, term for term, stored FP32) as NC floats at
// cmom + rank * NC, where rank is the cell's index among the occupied cells
// in key order: blk_rank[block] (an exclusive scan of the occupancy words'
// populations) plus the occupied cells before it in its 4x4x4 block's word.
// A thread per particle of the binned range: the first particle of each
// cell's run (in the sorted keys) sums the cell; cells of more than
// kWarpCell particles are listed (by key) for p2m_compact_big_kernel, a warp
// each.  The z pass then reads the records instead of summing particles, so
// its blocks no longer wait on the slowest cell of a line.
__device__ __forceinline__ uint32_t occ_rank(const unsigned long long *__restrict__ occ,
                                             const uint32_t *__restrict__ blk_rank, uint32_t key,
                                             bool &on) {
  const unsigned long long w = occ[key >> 6];
  on = (w >> (key & 63u)) & 1ull;
  return blk_rank[key >> 6] + (uint32_t)__popcll(w & ((1ull << (key & 63u)) - 1ull));
}

__global__ void occ_popc_kernel(const unsigned long long *__restrict__ occ, size_t nw,
                                uint32_t *__restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nw) out[i] = (uint32_t)__popcll(occ[i]);
}

// the cell coordinates of a Morton key's low 3 * mbits bits (the inverse of
// ct2g_morton: bit 3b + 2 is x's bit b, 3b + 1 y's, 3b z's)
__device__ __forceinline__ void demorton(uint32_t key, int mbits, uint32_t &x, uint32_t &y,
                                         uint32_t &z) {
  x = y = z = 0;
  for (int b = 0; b < mbits; b++) {
    z |= ((key >> (3 * b)) & 1u) << b;
    y |= ((key >> (3 * b + 1)) & 1u) << b;
    x |= ((key >> (3 * b + 2)) & 1u) << b;
  }
}

// the moments of the cell `key` (particles b .. e) into out (a thread: step
// 1; a warp: lanes strided, summed over the warp, lane 0 writes)
template <int P>
__device__ __forceinline__ void p2m_cell(const uint32_t *__restrict__ px,
                                         const uint32_t *__restrict__ py,
                                         const uint32_t *__restrict__ pz, uint32_t key, int mbits,
                                         uint32_t b, uint32_t e, bool warp, int lane,
                                         float *out) {
  constexpr int NC = ct2g_ncomp(P);
  uint32_t cx, cy, cz;
  demorton(key, mbits, cx, cy, cz);
  const int sh = 32 - mbits;
  const uint32_t halfc = 1u << (sh - 1);
  const uint32_t ux = (cx << sh) + halfc, uy = (cy << sh) + halfc, uz = (cz << sh) + halfc;
  const uint32_t b0 = warp ? b + (uint32_t)lane : b, step = warp ? 32u : 1u;
  const bool write = !warp || lane == 0;
  auto st = [&](int k, float v) { out[k] = v; };
  p2m_group<P, 0, NC / 3>(px, py, pz, b0, e, step, warp, ux, uy, uz, write, st);
  p2m_group<P, NC / 3, 2 * NC / 3>(px, py, pz, b0, e, step, warp, ux, uy, uz, write, st);
  p2m_group<P, 2 * NC / 3, NC>(px, py, pz, b0, e, step, warp, ux, uy, uz, write, st);
}

// a thread per particle j of the range (absolute index rbegin + j, key
// skeys[j]); the first of its cell's run sums the cell
template <int P>
__global__ void __launch_bounds__(256) p2m_compact_kernel(
    const uint32_t *__restrict__ px, const uint32_t *__restrict__ py,
    const uint32_t *__restrict__ pz, const uint32_t *__restrict__ cs,
    const unsigned long long *__restrict__ occ, const uint32_t *__restrict__ blk_rank, int mbits,
    const uint32_t *__restrict__ skeys, uint32_t rbegin, uint32_t nr, float *__restrict__ cmom,
    uint32_t *__restrict__ big) {
  const uint32_t j = blockIdx.x * 256 + threadIdx.x;
  if (j >= nr) return;
  const uint32_t key = skeys[j];
  if (j > 0 && skeys[j - 1] == key) return;  // not the first of its cell
  const uint32_t b = rbegin + j, e = cs[key + 1];
  if (e - b > kWarpCell) {
    big[1 + atomicAdd(big, 1u)] = key;
    return;
  }
  bool on;
  float *out = cmom + (size_t)occ_rank(occ, blk_rank, key, on) * ct2g_ncomp(P);
  p2m_cell<P>(px, py, pz, key, mbits, b, e, false, 0, out);
}

template <int P>
__global__ void __launch_bounds__(256) p2m_compact_big_kernel(
    const uint32_t *__restrict__ px, const uint32_t *__restrict__ py,
    const uint32_t *__restrict__ pz, const uint32_t *__restrict__ cs,
    const unsigned long long *__restrict__ occ, const uint32_t *__restrict__ blk_rank, int mbits,
    float *__restrict__ cmom, const uint32_t *__restrict__ big) {
  const uint32_t nbig = big[0];
  const int lane = threadIdx.x & 31;
  for (uint32_t q = (blockIdx.x * 256 + threadIdx.x) >> 5; q < nbig; q += gridDim.x * 8) {
    const uint32_t key = big[1 + q];
    bool on;
    float *out = cmom + (size_t)occ_rank(occ, blk_rank, key, on) * ct2g_ncomp(P);
    p2m_cell<P>(px, py, pz, key, mbits, cs[key], cs[key + 1], true, lane, out);
  }
}

// The moments of the N cells of line `line` (x * N + y) of box `box`, from
// the particles, into the packed smem lines sr (line l = components 2l, 2l+1
// as .x, .y).  big / nbig: smem list of the cells summed by a warp.  Ends
// with the block synchronised.
template <int P, int N>
__device__ __forceinline__ void p2m_line(const uint32_t *__restrict__ px,
                                         const uint32_t *__restrict__ py,
                                         const uint32_t *__restrict__ pz,
                                         const uint32_t *__restrict__ cs, int mbits, uint32_t box,
                                         size_t line, float *sr, uint32_t *big, uint32_t &nbig) {
  using LL = LineLayout<N, true>;
  constexpr int NC = ct2g_ncomp(P), NL = (NC + 1) / 2;
  const uint32_t cx = (uint32_t)(line / N), cy = (uint32_t)(line % N);
  const int sh = 32 - mbits;
  const uint32_t halfc = 1u << (sh - 1);
  const uint32_t ux = (cx << sh) + halfc, uy = (cy << sh) + halfc;
  for (int zc = threadIdx.x; zc < N; zc += 256) {
    const uint32_t key = (box << (3 * mbits)) | ct2g_morton(cx, cy, (uint32_t)zc);
    const uint32_t b = cs[key], e = cs[key + 1];
    if (e - b > kWarpCell) {
      big[atomicAdd(&nbig, 1u)] = (uint32_t)zc;
      continue;
    }
    const uint32_t uz = ((uint32_t)zc << sh) + halfc;
    p2m_half<P, N, 0, NC / 3>(px, py, pz, b, e, 1, false, ux, uy, uz, zc, sr, true);
    p2m_half<P, N, NC / 3, 2 * NC / 3>(px, py, pz, b, e, 1, false, ux, uy, uz, zc, sr, true);
    p2m_half<P, N, 2 * NC / 3, NC>(px, py, pz, b, e, 1, false, ux, uy, uz, zc, sr, true);
    if (NC & 1) sr[2 * LL::at(NL - 1, zc, 0) + 1] = 0.f;
  }
  __syncthreads();
  {  // the big cells, a warp each
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t q = warp; q < nbig; q += 8) {
      const uint32_t zc = big[q];
      const uint32_t key = (box << (3 * mbits)) | ct2g_morton(cx, cy, zc);
      const uint32_t b = cs[key], e = cs[key + 1];
      const uint32_t uz = (zc << sh) + halfc;
      p2m_half<P, N, 0, NC / 3>(px, py, pz, b + lane, e, 32, true, ux, uy, uz, (int)zc, sr,
                                lane == 0);
      p2m_half<P, N, NC / 3, 2 * NC / 3>(px, py, pz, b + lane, e, 32, true, ux, uy, uz,
                                         (int)zc, sr, lane == 0);
      p2m_half<P, N, 2 * NC / 3, NC>(px, py, pz, b + lane, e, 32, true, ux, uy, uz, (int)zc,
                                     sr, lane == 0);
      if ((NC & 1) && lane == 0) sr[2 * LL::at(NL - 1, (int)zc, 0) + 1] = 0.f;
    }
  }
  __syncthreads();
}

// The moments of the N cells of line `line` of box `box` from the compact
// per-cell records (zeros for empty cells) into the packed smem lines sr.
// Ends with the block synchronised.
template <int P, int N>
__device__ __forceinline__ void cmom_line(const float *__restrict__ cmom,
                                          const unsigned long long *__restrict__ occ,
                                          const uint32_t *__restrict__ blk_rank, int mbits,
                                          uint32_t box, size_t line, float *sr) {
  using LL = LineLayout<N, true>;
  constexpr int NC = ct2g_ncomp(P), NL = (NC + 1) / 2;
  const uint32_t cx = (uint32_t)(line / N), cy = (uint32_t)(line % N);
  for (int zc = threadIdx.x; zc < N; zc += 256) {
    const uint32_t key = (box << (3 * mbits)) | ct2g_morton(cx, cy, (uint32_t)zc);
    bool on;
    const uint32_t rank = occ_rank(occ, blk_rank, key, on);
    float v[NC];
    if (on) {
      const float *m = cmom + (size_t)rank * NC;
#pragma unroll
      for (int k = 0; k < NC; k++) v[k] = __ldg(m + k);
    } else {
#pragma unroll
      for (int k = 0; k < NC; k++) v[k] = 0.f;
    }
#pragma unroll
    for (int k = 0; k < NC; k++) sr[2 * LL::at(k >> 1, zc, 0) + (k & 1)] = v[k];
    if (NC & 1) sr[2 * LL::at(NL - 1, zc, 0) + 1] = 0.f;
  }
  __syncthreads();
}

// The transformed packed lines of LB mesh lines, split into the half spectra
// of their two components, written as LB spectrum rows from `rows` on (row
// lb at rows + lb * ldk * NC; k-point k's components at k * NC; the slots
// k > N/2 get zeros).
template <int P, int N, int LB>
__device__ __forceinline__ void store_half_spectra(const float2 *s, float2 *rows, int ldk) {
  using LL = LineLayout<N, true>;
  constexpr int NC = ct2g_ncomp(P), NL = (NC + 1) / 2, NH = N / 2 + 1;
  const int64_t RS = (int64_t)ldk * NC;
  for (int e = threadIdx.x; e < LB * ldk * NL; e += 256) {
    const int lb = LB == 1 ? 0 : e / (ldk * NL), r = e - lb * ldk * NL;
    const int k = r / NL, l = r - k * NL;
    float2 *row = rows + lb * RS;
    float2 a = make_float2(0.f, 0.f), bb = make_float2(0.f, 0.f);
    if (k < NH) {
      const float2 zk = s[LL::at(lb * NL + l, k & (N - 1), 0)];
      const float2 zn = s[LL::at(lb * NL + l, (N - k) & (N - 1), 0)];
      // A_k = (Z_k + conj Z_{N-k})/2, B_k = (Z_k - conj Z_{N-k})/(2i)
      a = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
      bb = make_float2(0.5f * (zk.y + zn.y), 0.5f * (zn.x - zk.x));
    }
    row[k * NC + 2 * l] = a;
    if (2 * l + 1 < NC) row[k * NC + 2 * l + 1] = bb;
  }
}

// occupancy: 4 blocks per SM up to order 4 (64 registers); at N = 512 the
// 32-point in-register DFTs need more registers than that, so 2
template <int P, int N, int SRC>
__global__ void __launch_bounds__(256, N >= 512 ? 2 : P <= 4 ? 4 : 2) fftz_p2m_r2c_kernel(
    const uint32_t *__restrict__ px, const uint32_t *__restrict__ py,
    const uint32_t *__restrict__ pz, const uint32_t *__restrict__ cs, int mbits,
    float *__restrict__ grid, int64_t CB, float2 *__restrict__ spec, int ldk,
    const float2 *__restrict__ tw, const float *__restrict__ cmom,
    const unsigned long long *__restrict__ occ, const uint32_t *__restrict__ blk_rank) {
  using LL = LineLayout<N, true>;
  constexpr int NC = ct2g_ncomp(P), NL = (NC + 1) / 2, NH = N / 2 + 1;
  constexpr bool GRID = SRC == CT2G_P2M_GRID;
  constexpr int LB = GRID ? z_lines<P>() : 1;  // lines of this block
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *stw = reinterpret_cast<float2 *>(smraw);
  float2 *s = stw + N;
  float *sr = reinterpret_cast<float *>(s);
  __shared__ uint32_t big[GRID ? 1 : N], nbig;
  if (threadIdx.x == 0) nbig = 0;
  load_twiddles(stw, tw, N);
  __syncthreads();
  const size_t L0 = (size_t)blockIdx.x * LB;  // first line (box * N^2 + line)
  const size_t line = L0 % ((size_t)N * N);
  const uint32_t box = (uint32_t)(L0 / ((size_t)N * N));
  if constexpr (GRID) {
    // line lb of the block: packed lines lb * NL ...; its grid rows follow
    const float *g = grid + ((int64_t)box * N * N + (int64_t)line) * N;
    for (int e = threadIdx.x; e < LB * NC * N; e += 256) {
      const int lb = LB == 1 ? 0 : e / (NC * N), r = e - lb * NC * N;
      const int k = r / N, z = r % N;
      sr[2 * LL::at(lb * NL + (k >> 1), z, 0) + (k & 1)] = g[(int64_t)k * CB + lb * N + z];
    }
    if (NC & 1)
      for (int e = threadIdx.x; e < LB * N; e += 256)
        sr[2 * LL::at((e / N) * NL + NL - 1, e % N, 0) + 1] = 0.f;
  } else if constexpr (SRC == CT2G_P2M_COMPACT) {
    cmom_line<P, N>(cmom, occ, blk_rank, mbits, box, line, sr);
  } else {
    p2m_line<P, N>(px, py, pz, cs, mbits, box, line, sr, big, nbig);
  }
  __syncthreads();
  if constexpr (SRC == CT2G_P2M_FUSED_STORE) {
    // the moments also go to the moment grid (for passes that read it)
    float *g = grid + ((int64_t)box * N * N + (int64_t)line) * N;
    for (int e = threadIdx.x; e < NC * N; e += 256) {
      const int k = e / N, z = e % N;
      g[(int64_t)k * CB + z] = sr[2 * LL::at(k >> 1, z, 0) + (k & 1)];
    }
    __syncthreads();
  }
  tile_fft<N, true, float2, false>(s, LB * NL, 0, stw);
  store_half_spectra<P, N, LB>(s, spec + (int64_t)L0 * ldk * NC, ldk);
}

// the compact per-cell moment records of the current binning: the occupied
// cells' ranks, then a thread per small cell and a warp per listed big cell
template <int P>
int launch_p2m_compact(ct2g_ctx *ctx) {
  const size_t nw = (size_t)ctx->CB / 64;
  occ_popc_kernel<<<ct2g_div_up(nw, 256), 256, 0, ctx->stream>>>(ctx->occ, nw, ctx->blk_rank);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, ctx->blk_rank, ctx->blk_rank, nw, nullptr, 0));
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->p2m_big, 0, sizeof(uint32_t), ctx->stream));
  const size_t nr = ctx->n - ctx->rung_begin;  // the binned range, as ct2g_bin_range sorted it
  p2m_compact_kernel<P><<<(unsigned)std::max<size_t>(1, ct2g_div_up(nr, 256)), 256, 0,
                          ctx->stream>>>(ctx->x, ctx->y, ctx->z, ctx->cell_start, ctx->occ,
                                         ctx->blk_rank, ctx->mbits, ctx->keys,
                                         (uint32_t)ctx->rung_begin, (uint32_t)nr, ctx->cmom,
                                         ctx->p2m_big);
  CT2G_LAUNCHED(ctx);
  p2m_compact_big_kernel<P><<<(unsigned)(4 * ctx->num_sms), 256, 0, ctx->stream>>>(
      ctx->x, ctx->y, ctx->z, ctx->cell_start, ctx->occ, ctx->blk_rank, ctx->mbits, ctx->cmom,
      ctx->p2m_big);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

template <int P, int N>
int launch_p2m_r2c(ct2g_ctx *ctx, int src) {
  constexpr int NL = (ct2g_ncomp(P) + 1) / 2;
  const int LB = src == CT2G_P2M_GRID ? z_lines<P>() : 1;
  const size_t smem = sizeof(float2) * ((size_t)N + (size_t)LB * NL * LineLayout<N, true>::LS);
  auto k = src == CT2G_P2M_GRID      ? fftz_p2m_r2c_kernel<P, N, CT2G_P2M_GRID>
           : src == CT2G_P2M_FUSED   ? fftz_p2m_r2c_kernel<P, N, CT2G_P2M_FUSED>
           : src == CT2G_P2M_COMPACT ? fftz_p2m_r2c_kernel<P, N, CT2G_P2M_COMPACT>
                                     : fftz_p2m_r2c_kernel<P, N, CT2G_P2M_FUSED_STORE>;
  CT2G_TRY(ct2g_smem_attrs(ctx, k, smem));
  k<<<(unsigned)((size_t)N * N * ctx->nbox / LB), 256, smem, ctx->stream>>>(
      ctx->x, ctx->y, ctx->z, ctx->cell_start, ctx->mbits, ctx->grid, ctx->CB, ctx->spec,
      ctx->ldk, twiddle_ptr<float2>(ctx), ctx->cmom, ctx->occ, ctx->blk_rank);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// ---- inverse z pass fused with L2P ------------------------------------------
// LB spectrum rows from `rows` on (layout as store_half_spectra) unpacked
// into packed complex lines in smem: Z = A + iB for the components 2l, 2l+1,
// both halves of the line from the k <= N/2 slots.  ld(q) loads one value
// (a plain load, or one that bypasses L1).  The row's loads go out in batches
// of RB per thread before any of them is used, so that their latencies
// overlap.
template <int P, int N, int LB, typename LD>
__device__ __forceinline__ void load_half_spectra(const float2 *rows, int ldk, float2 *s, LD ld) {
  using LL = LineLayout<N, true>;
  constexpr int NC = ct2g_ncomp(P), NL = (NC + 1) / 2, NH = N / 2 + 1;
  const int64_t RS = (int64_t)ldk * NC;
  constexpr int RB = 5;
  for (int e0 = threadIdx.x; e0 < LB * NH * NL; e0 += RB * 256) {
    float2 a[RB], b[RB];
#pragma unroll
    for (int u = 0; u < RB; u++) {
      const int e = e0 + 256 * u;
      const int lb = LB == 1 ? 0 : e / (NH * NL), r = e - lb * NH * NL;
      const int k = r / NL, l = r - k * NL;
      a[u] = b[u] = make_float2(0.f, 0.f);
      if (e < LB * NH * NL) {
        a[u] = ld(rows + lb * RS + k * NC + 2 * l);
        if (2 * l + 1 < NC) b[u] = ld(rows + lb * RS + k * NC + 2 * l + 1);
      }
    }
#pragma unroll
    for (int u = 0; u < RB; u++) {
      const int e = e0 + 256 * u;
      const int lb = LB == 1 ? 0 : e / (NH * NL), r = e - lb * NH * NL;
      const int k = r / NL, l = r - k * NL;
      if (e < LB * NH * NL) {
        // Z_k = A_k + i B_k; Z_{N-k} = conj(A_k) + i conj(B_k)
        s[LL::at(lb * NL + l, k, 0)] = make_float2(a[u].x - b[u].y, a[u].y + b[u].x);
        if (k > 0 && k < N / 2)
          s[LL::at(lb * NL + l, N - k, 0)] = make_float2(a[u].x + b[u].y, b[u].x - a[u].y);
      }
    }
  }
}

// Inverse transform of one line's packed expansion lines in smem (s, loaded
// and synchronised), then the far field of every particle of the line's
// cells: cb / ce hold the cells' particle ranges (smem, written before the
// caller's last barrier), off is smem scratch of N + 1 words.
template <int P, int N, bool POT>
__device__ __forceinline__ void l2p_line(float2 *s, const float2 *stw, const uint32_t *cb,
                                         const uint32_t *ce, uint32_t *off,
                                         const float4 *__restrict__ src, float GM,
                                         float *__restrict__ ofx, float *__restrict__ ofy,
                                         float *__restrict__ ofz, float *__restrict__ opot) {
  using LL = LineLayout<N, true>;
  constexpr int NL = (ct2g_ncomp(P) + 1) / 2;
  // offsets of the cells' particles in the line's particle list (inclusive
  // scan of the counts, off[0] = 0): thread t holds cells [t ZT, t ZT + ZT),
  // scans its sum across its warp by shuffles before the transform and
  // across the block's warps after it (one barrier of its own)
  constexpr int ZT = (N + 255) / 256;  // cells per thread
  static_assert(N % 256 == 0 || N < 256, "cells per thread");
  __shared__ uint32_t wsum[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t c[ZT], tsum = 0;
#pragma unroll
  for (int q = 0; q < ZT; q++) {
    const int z = threadIdx.x * ZT + q;
    c[q] = z < N ? ce[z] - cb[z] : 0u;
    tsum += c[q];
  }
  uint32_t inc = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) wsum[warp] = inc;
  tile_fft<N, true, float2, true>(s, NL, 0, stw);
  __syncthreads();
  {
    uint32_t run = inc - tsum;
    for (int w = 0; w < warp; w++) run += wsum[w];
#pragma unroll
    for (int q = 0; q < ZT; q++) {
      const int z = threadIdx.x * ZT + q;
      run += c[q];
      if (z < N) off[z + 1] = run;
    }
    if (threadIdx.x == 0) off[0] = 0;
  }
  __syncthreads();
  // every particle of the line, one per thread: its cell is the last z with
  // off[z] <= q (that cell holds it: off[z] <= q < off[z + 1])
  const uint32_t total = off[N];
  for (uint32_t q = threadIdx.x; q < total; q += 256) {
    int lo = 0, hi = N;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (off[mid] <= q) lo = mid; else hi = mid;
    }
    const int z = lo;
    const uint32_t i = cb[z] + (q - off[z]);
    const auto acc = [&](int k) {
      const float2 v = s[LL::at(k >> 1, z, 0)];
      return (k & 1) ? v.y : v.x;
    };
    const float4 t = src[i];
    float fx, fy, fz, ph;
    ct2g_l2p<P>(acc, t.x, t.y, t.z, fx, fy, fz, ph);
    ofx[i] = GM * fx;
    ofy[i] = GM * fy;
    ofz[i] = GM * fz;
    if (POT) opot[i] = GM * ph;
  }
}


// One block per (x, y) line of the mesh, all NC expansion components: pairs of
// components are packed into complex lines (A + iB), transformed back along z
// in shared memory, and the block then evaluates the far field of every
// particle of the line's cells from the expansions in shared memory.  The
// expansion grid itself is never written to HBM.  Block b is line b % N^2
// of box b / N^2.  MODE 0: forces, 1: forces and potentials, 2: no L2P, the
// expansions go to the expansion grid (layout as the moment grid).
// occupancy: 5 blocks per SM (48 registers) below N = 512, whose 32-point
// in-register DFTs need more
template <int P, int N, int MODE>
__global__ void __launch_bounds__(256, N >= 512 ? 1 : 5) fftz_c2r_l2p_kernel(
    const float2 *__restrict__ spec, int ldk, const uint32_t *__restrict__ cs,
    const float4 *__restrict__ src, int mbits, const float *__restrict__ box_gm,
    float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, float *__restrict__ grid, int64_t CB,
    const float2 *__restrict__ tw) {
  using LL = LineLayout<N, true>;
  constexpr int NC = ct2g_ncomp(P), NL = (NC + 1) / 2, NH = N / 2 + 1;
  constexpr bool L2P = MODE < 2;
  constexpr int LB = L2P ? 1 : z_lines<P>();  // lines of this block
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *stw = reinterpret_cast<float2 *>(smraw);
  float2 *s = stw + N;
  __shared__ uint32_t cb[L2P ? N + 1 : 1], ce[L2P ? N : 1];  // particle ranges of the line's cells
  load_twiddles(stw, tw, N);
  const size_t L0 = (size_t)blockIdx.x * LB;  // first line (box * N^2 + line)
  const size_t line = L0 % ((size_t)N * N);
  const uint32_t box = (uint32_t)(L0 / ((size_t)N * N));
  const uint32_t x = (uint32_t)(line / N), y = (uint32_t)(line % N);
  if constexpr (L2P) {
    // issue the range loads first: their latency hides behind the transform
    for (int z = threadIdx.x; z < N; z += 256) {
      const uint32_t key = (box << (3 * mbits)) | ct2g_morton(x, y, (uint32_t)z);
      cb[z] = cs[key];
      ce[z] = cs[key + 1];
    }
  }
  load_half_spectra<P, N, LB>(spec + (int64_t)L0 * ldk * NC, ldk, s,
                              [](const float2 *q) { return *q; });
  __syncthreads();
  if constexpr (!L2P) {
    tile_fft<N, true, float2, true>(s, LB * NL, 0, stw);
    float *g = grid + ((int64_t)box * N * N + (int64_t)line) * N;
    for (int e = threadIdx.x; e < LB * NC * N; e += 256) {
      const int lb = LB == 1 ? 0 : e / (NC * N), r = e - lb * NC * N;
      const int k = r / N, z = r % N;
      const float2 v = s[LL::at(lb * NL + (k >> 1), z, 0)];
      g[(int64_t)k * CB + lb * N + z] = (k & 1) ? v.y : v.x;
    }
    return;
  } else {
    __shared__ uint32_t off[N + 1];
    l2p_line<P, N, MODE == 1>(s, stw, cb, ce, off, src, __ldg(box_gm + box), ofx, ofy, ofz,
                              opot);
  }
}

template <int P, int N>
int launch_c2r_l2p(ct2g_ctx *ctx, int mode) {
  constexpr int NL = (ct2g_ncomp(P) + 1) / 2;
  const int LB = mode == 2 ? z_lines<P>() : 1;
  const size_t smem = sizeof(float2) * ((size_t)N + (size_t)LB * NL * LineLayout<N, true>::LS);
  auto k = mode == 0 ? fftz_c2r_l2p_kernel<P, N, 0>
           : mode == 1 ? fftz_c2r_l2p_kernel<P, N, 1> : fftz_c2r_l2p_kernel<P, N, 2>;
  CT2G_TRY(ct2g_smem_attrs(ctx, k, smem));
  k<<<(unsigned)((size_t)N * N * ctx->nbox / LB), 256, smem, ctx->stream>>>(
      ctx->spec, ctx->ldk, ctx->cell_start, ctx->src, ctx->mbits, ctx->box_gm, ctx->fx, ctx->fy,
      ctx->fz, ctx->pot, ctx->grid, ctx->CB, twiddle_ptr<float2>(ctx));
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// ---- z and y passes plane by plane: one persistent kernel per direction -----
// The z pass and the y pass both work plane by plane (an x plane of a box is
// N spectrum rows, N * ldk * NC complex values: 9.3 MB at N = 256, order 4),
// so the y pass of a plane can start as soon as the z pass has written the
// plane, while it is still in L2.  One persistent kernel hands out the items
// of both passes in plane order from a device counter: the z lines of plane
// t, then the y tiles of plane t - 1, then the z lines of plane t + 1, ...;
// a y tile first waits (bounded) for the count of finished z lines of its
// plane.  The spectrum then crosses HBM once per direction instead of three
// times: forward, the y tiles read the rows from L2 and overwrite them in
// place, so only the final values are written back; inverse, the z lines
// read the y pass's output from L2 and (`discard`) drop the lines they have
// read, which nothing reads again, without writing them back.
//
// Waiting is deadlock free whatever the number of resident blocks: a block
// takes an item only while it runs, items are taken in order, and a waiting
// item waits only for items of the other pass taken before it, which never
// wait themselves.

// Item order of a plane pipeline over T planes with a lag of D planes: A(t),
// the first pass's NA items of plane t, and B(t), the second pass's NB items,
// in the order A(0) ... A(D-1), then A(t) B(t-D) for t = D ... T-1, then
// B(T-D) ... B(T-1).  The lag is how long a plane's first-pass items have
// to finish before its second-pass items are handed out; D + 1 planes are in
// flight at a time.
struct PipeOrder {
  uint32_t NA, NB, T, D;  // 1 <= D <= T
  __device__ __forceinline__ uint32_t total() const { return T * (NA + NB); }
  // true for an item of the first pass
  __device__ __forceinline__ bool decode(uint32_t i, uint32_t &plane, uint32_t &sub) const {
    if (i < D * NA) {
      plane = i / NA;
      sub = i - plane * NA;
      return true;
    }
    i -= D * NA;
    const uint32_t R = NA + NB;
    if (i < (T - D) * R) {
      const uint32_t t = i / R, o = i - t * R;
      plane = o < NA ? t + D : t;
      sub = o < NA ? o : o - NA;
      return o < NA;
    }
    i -= (T - D) * R;
    plane = T - D + i / NB;
    sub = i - (plane - (T - D)) * NB;
    return false;
  }
};

constexpr uint32_t kPipeWaitLimit = 1u << 21;  // polls of a plane count (about a second)
constexpr int kPipeW = 16;                     // y tile width (complex columns)

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Thread 0 waits until *count reaches target (the producers' row stores are
// then visible to the block); false for every thread when the wait gave up,
// after the status word was set to CT2G_ETIMEOUT.
__device__ __forceinline__ bool pipe_wait(const uint32_t *count, uint32_t target,
                                          uint32_t *status) {
  int good = 1;
  if (threadIdx.x == 0) {
    uint32_t polls = 0;
    while (ld_acquire(count) < target) {
      if (++polls > kPipeWaitLimit) {
        atomicExch(status, (uint32_t)CT2G_ETIMEOUT);
        good = 0;
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
  }
  return __syncthreads_and(good) != 0;
}

// After the block's stores: the item is counted as finished in *count.
__device__ __forceinline__ void pipe_done(uint32_t *count) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(count, 1u);
  }
}

// One y tile: columns [c0, c0 + wv) of the N rows of a plane (row r at
// plane + r * RS), copied into smem by cp.async past L1 (other blocks of the
// kernel wrote them; the whole tile is in flight at once, without staging
// registers), transformed along y in smem (column layout, W columns) and
// written back.  Columns go in 16-byte pairs; a pair that starts below wv
// moves whole (its second column, when past the last one, is a zero slot of
// the row); the smem columns of pairs past wv are left as they are (columns
// transform independently).
template <int N, int W, bool INV>
__device__ __forceinline__ void y_tile(float2 *plane, int64_t RS, int c0, int wv, float2 *s,
                                       const float2 *stw) {
  constexpr int CH = W / 2;  // 16-byte chunks per tile row
  static_assert(N * CH % 256 == 0, "tile chunks per thread");
#pragma unroll 4
  for (int e = threadIdx.x; e < N * CH; e += 256) {
    const int r = e / CH, c = (e % CH) * 2;
    if (c < wv) cp_async16(s + r * W + c, plane + r * RS + c0 + c);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  tile_fft<N, false, float2, INV>(s, W, W, stw);
#pragma unroll 4
  for (int e = threadIdx.x; e < N * CH; e += 256) {
    const int r = e / CH, c = (e % CH) * 2;
    if (c < wv)
      *reinterpret_cast<float4 *>(plane + r * RS + c0 + c) =
          *reinterpret_cast<const float4 *>(s + r * W + c);
  }
}

template <int P, int N>
struct PipeShape {
  static constexpr int NC = ct2g_ncomp(P), NL = (NC + 1) / 2, NH = N / 2 + 1;
  static constexpr size_t ZS = (size_t)NL * LineLayout<N, true>::LS;  // a z line's packed lines
  static constexpr size_t YS = (size_t)N * kPipeW;                    // a y tile
  static constexpr size_t SMEM = sizeof(float2) * ((size_t)N + (ZS > YS ? ZS : YS));
  // the z kernels' register budgets: 64 per thread up to order 4
  static constexpr int MINB = P <= 4 ? 4 : 2;
  static constexpr bool OK = N >= 64 && N <= 256;
};

// Forward: z lines (P2M from the particles + r2c along z, store_half_spectra)
// and y tiles.  sync[0]: item counter; sync[2 + t]: finished z lines of plane t.
template <int P, int N>
__global__ void __launch_bounds__(256, PipeShape<P, N>::MINB) zy_forward_kernel(
    const uint32_t *__restrict__ px, const uint32_t *__restrict__ py,
    const uint32_t *__restrict__ pz, const uint32_t *__restrict__ cs, int mbits,
    float2 *__restrict__ spec, int ldk, const float2 *__restrict__ tw, uint32_t nplanes,
    uint32_t lag, uint32_t *__restrict__ sync, uint32_t *__restrict__ status) {
  using S = PipeShape<P, N>;
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *stw = reinterpret_cast<float2 *>(smraw);
  float2 *s = stw + N;
  __shared__ uint32_t big[N], nbig, item_s;
  load_twiddles(stw, tw, N);
  const int64_t RS = (int64_t)ldk * S::NC;
  const uint32_t ncols = (uint32_t)(S::NH * S::NC);
  const PipeOrder ord{(uint32_t)N, (ncols + kPipeW - 1) / kPipeW, nplanes, min(lag, nplanes)};
  if (threadIdx.x == 0) item_s = atomicAdd(sync, 1u);
  __syncthreads();
  for (;;) {
    const uint32_t item = item_s;
    if (item >= ord.total()) break;
    uint32_t next = 0;
    if (threadIdx.x == 0) {
      next = atomicAdd(sync, 1u);  // the next item, asked for early
      nbig = 0;
    }
    __syncthreads();
    uint32_t plane, sub;
    if (ord.decode(item, plane, sub)) {
      const size_t L0 = (size_t)plane * N + sub;  // box * N^2 + x * N + y
      p2m_line<P, N>(px, py, pz, cs, mbits, plane / N, L0 % ((size_t)N * N),
                     reinterpret_cast<float *>(s), big, nbig);
      tile_fft<N, true, float2, false>(s, S::NL, 0, stw);
      store_half_spectra<P, N, 1>(s, spec + (int64_t)L0 * RS, ldk);
      pipe_done(sync + 2 + plane);
    } else {
      if (!pipe_wait(sync + 2 + plane, (uint32_t)N, status)) break;
      const int c0 = (int)sub * kPipeW;
      y_tile<N, kPipeW, false>(spec + (int64_t)plane * N * RS, RS, c0,
                               (int)min((uint32_t)kPipeW, ncols - (uint32_t)c0), s, stw);
    }
    if (threadIdx.x == 0) item_s = next;
    __syncthreads();
  }
}

// Inverse: y tiles and z lines (c2r along z + L2P); with `discard` a z line
// drops the L2 lines that lie wholly inside the row it has read.  sync[0]:
// item counter; sync[2 + t]: finished y tiles of plane t.
template <int P, int N, bool POT>
__global__ void __launch_bounds__(256, PipeShape<P, N>::MINB) yz_inverse_kernel(
    float2 *__restrict__ spec, int ldk, const uint32_t *__restrict__ cs,
    const float4 *__restrict__ src, int mbits, const float *__restrict__ box_gm,
    float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, const float2 *__restrict__ tw, uint32_t nplanes, uint32_t lag,
    int discard, uint32_t *__restrict__ sync, uint32_t *__restrict__ status) {
  using S = PipeShape<P, N>;
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *stw = reinterpret_cast<float2 *>(smraw);
  float2 *s = stw + N;
  __shared__ uint32_t cb[N + 1], ce[N], off[N + 1], item_s;
  load_twiddles(stw, tw, N);
  const int64_t RS = (int64_t)ldk * S::NC;
  const uint32_t ncols = (uint32_t)(S::NH * S::NC), NT = (ncols + kPipeW - 1) / kPipeW;
  const PipeOrder ord{NT, (uint32_t)N, nplanes, min(lag, nplanes)};
  if (threadIdx.x == 0) item_s = atomicAdd(sync, 1u);
  __syncthreads();
  for (;;) {
    const uint32_t item = item_s;
    if (item >= ord.total()) break;
    uint32_t next = 0;
    if (threadIdx.x == 0) next = atomicAdd(sync, 1u);
    uint32_t plane, sub;
    if (ord.decode(item, plane, sub)) {
      const int c0 = (int)sub * kPipeW;
      y_tile<N, kPipeW, true>(spec + (int64_t)plane * N * RS, RS, c0,
                              (int)min((uint32_t)kPipeW, ncols - (uint32_t)c0), s, stw);
      pipe_done(sync + 2 + plane);
    } else {
      const size_t L0 = (size_t)plane * N + sub;
      const uint32_t box = plane / N, x = plane % N, y = sub;
      // the cells' particle ranges first: their latency hides behind the wait
      for (int z = threadIdx.x; z < N; z += 256) {
        const uint32_t key = (box << (3 * mbits)) | ct2g_morton(x, y, (uint32_t)z);
        cb[z] = cs[key];
        ce[z] = cs[key + 1];
      }
      if (!pipe_wait(sync + 2 + plane, NT, status)) break;
      const float2 *row = spec + (int64_t)L0 * RS;
      load_half_spectra<P, N, 1>(row, ldk, s, [](const float2 *q) { return __ldcg(q); });
      __syncthreads();
      if (discard) {
        // the row's own 128-byte lines: every value of them is in smem now
        const uintptr_t a = reinterpret_cast<uintptr_t>(row), e = a + (uintptr_t)RS * 8;
        for (uintptr_t q = ((a + 127) & ~(uintptr_t)127) + 128 * threadIdx.x; q + 128 <= e;
             q += 128 * 256)
          asm volatile("discard.global.L2 [%0], 128;" ::"l"(q) : "memory");
      }
      l2p_line<P, N, POT>(s, stw, cb, ce, off, src, __ldg(box_gm + box), ofx, ofy, ofz, opot);
    }
    if (threadIdx.x == 0) item_s = next;
    __syncthreads();
  }
}

// the plane pipeline of one direction, when the configuration has one
// (FP32 passes, the meshes it is built for, P2M from the particles or L2P
// into the forces); *done = false otherwise, nothing launched
template <int P, int N>
int launch_plane_pipe(ct2g_ctx *ctx, bool inverse, int mode, bool *done) {
  using S = PipeShape<P, N>;
  *done = false;
  if constexpr (!S::OK) {
    return CT2G_OK;
  } else {
    if (!ctx->plane_pipe || ctx->fft_tc || !ctx->pipe_sync) return CT2G_OK;
    if (inverse ? mode > 1 : mode != CT2G_P2M_FUSED) return CT2G_OK;
    const uint32_t nplanes = (uint32_t)(ctx->nbox * N);
    const void *kf = inverse ? (mode == 1 ? (const void *)yz_inverse_kernel<P, N, true>
                                          : (const void *)yz_inverse_kernel<P, N, false>)
                             : (const void *)zy_forward_kernel<P, N>;
    CT2G_TRY(ct2g_smem_attrs(ctx, kf, S::SMEM));
    const unsigned grid = (unsigned)(ct2g_blocks_per_sm(ctx, kf, 256, S::SMEM) * ctx->num_sms);
    uint32_t *sync = ctx->pipe_sync + (inverse ? 2 + nplanes : 0);
    CT2G_CUDA(ctx, cudaMemsetAsync(sync, 0, sizeof(uint32_t) * (2 + nplanes), ctx->stream));
    if (inverse) {
      auto k = mode == 1 ? yz_inverse_kernel<P, N, true> : yz_inverse_kernel<P, N, false>;
      k<<<grid, 256, S::SMEM, ctx->stream>>>(ctx->spec, ctx->ldk, ctx->cell_start, ctx->src,
                                             ctx->mbits, ctx->box_gm, ctx->fx, ctx->fy, ctx->fz,
                                             ctx->pot, twiddle_ptr<float2>(ctx), nplanes,
                                             (uint32_t)ctx->plane_pipe, ctx->pipe_discard, sync,
                                             ctx->d_counts + 6);
    } else {
      zy_forward_kernel<P, N><<<grid, 256, S::SMEM, ctx->stream>>>(
          ctx->x, ctx->y, ctx->z, ctx->cell_start, ctx->mbits, ctx->spec, ctx->ldk,
          twiddle_ptr<float2>(ctx), nplanes, (uint32_t)ctx->plane_pipe, sync, ctx->d_counts + 6);
    }
    CT2G_LAUNCHED(ctx);
    *done = true;
    return CT2G_OK;
  }
}

// ---- X pass + MG2L + inverse X pass ------------------------------------------
// One block per spectrum column (box, qj, qk): the column's N k-points with all
// NC components, s[qi * NC + c], are transformed along x, contracted with the
// Green's tensor (L_a = sum_b G_{a+b} M_b, src/particle.cpp:244-250) and
// transformed back, so neither the transformed moments nor the expansions
// make a round trip through HBM between the three steps.  The first transform
// step reads the column's moments from HBM into registers, the last one
// writes the expansions back from registers; the Green's values ([c][qi], one
// contiguous run of the column-ordered table) arrive by cp.async meanwhile.
// GD: the Green's values are read straight from HBM by the contraction (no
// shared-memory copy of the Green's column, so one more block fits per SM)
template <int P, int N, bool GD = false>
struct FxShape {
  static constexpr int NC = ct2g_ncomp(P), NH = N / 2 + 1;
  static constexpr int GCOL = NC * N;  // floats per Green's column (a multiple of 8)
  static constexpr size_t SMEM = sizeof(float2) * (size_t)N + sizeof(float2) * (size_t)N * NC +
                                 (GD ? 0 : sizeof(float) * (size_t)GCOL);
  static constexpr bool FITS = SMEM <= 227 * 1024;
  // three blocks per SM only where the contraction fits 85 registers
  // (orders up to 4 with the Green's values read directly)
  static constexpr int MINB = (GD && NC <= 35 && SMEM <= 75 * 1024) ? 3
                              : SMEM <= 112 * 1024                  ? 2
                                                                    : 1;
  static constexpr bool GREG = !GD && NC <= 35;  // Green's values in registers
  // (a persistent form with one 512-thread block per SM and the next
  // column's data arriving by cp.async in a second buffer measured slower:
  // 2.45 against 1.90 ms at N = 256, order 4)
};

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}

// The two steps of tile_fft for NL lines in the COLS layout s[r * NL + l],
// with the first step's input and the second step's output going through
// functors, so that a line can come straight from HBM or go straight back
// without a pass through shared memory.  cols_step1: jobs (l, n1), input
// ld(l, r), Y[n1][k2] to smem.  cols_step2: jobs (l, k2), X[k2 + R2*k1] to
// st(l, r, v); INPLACE when st writes the smem slots the step reads.
template <int N, int NL, bool INV, int NT, int PITCH = NL, typename LD>
__device__ __forceinline__ void cols_step1(float2 *s, const float2 *stw, LD ld, int off = 0) {
  using LL = LineLayout<N, false>;
  constexpr int R1 = LL::R1, R2 = LL::R2;
  for (int job = threadIdx.x; job < NL * R1; job += NT) {
    const int l = job % NL, n1 = job / NL;
    float2 v[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; n2++) v[n2] = ld(l, n1 + R1 * n2);
    reg_dft<R2, float2, INV>(v);
#pragma unroll
    for (int k2 = 1; k2 < R2; k2++) {
      float2 w = stw[(n1 * k2) & (N - 1)];
      if (INV) w.y = -w.y;
      v[k2] = cmul(v[k2], w);
    }
#pragma unroll
    for (int k2 = 0; k2 < R2; k2++) s[(n1 + R1 * k2) * PITCH + off + l] = v[k2];
  }
}

template <int N, int NL, bool INV, bool INPLACE, int NT, int PITCH = NL, typename ST>
__device__ __forceinline__ void cols_step2(const float2 *s, ST st, int off = 0) {
  using LL = LineLayout<N, false>;
  constexpr int R1 = LL::R1, R2 = LL::R2;
  static_assert(NT % R2 == 0, "block size must be a multiple of R2");
  constexpr int LW = NT / R2;
  for (int l0 = 0; l0 < NL; l0 += LW) {
    const int l = l0 + threadIdx.x % LW, k2 = threadIdx.x / LW;
    const bool on = l < NL;
    float2 v[R1];
    if (on) {
#pragma unroll
      for (int n1 = 0; n1 < R1; n1++) v[n1] = s[(n1 + R1 * k2) * PITCH + off + l];
      reg_dft<R1, float2, INV>(v);
    }
    if (INPLACE) __syncthreads();  // all reads of this round before any write
    if (on) {
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) st(l, k2 + R2 * k1, v[k1]);
    }
    if (INPLACE) __syncthreads();
  }
}

template <int P, int N, bool GD>
__global__ void __launch_bounds__(256, FxShape<P, N, GD>::MINB) fftx_mg2l_kernel(
    float2 *__restrict__ spec, int ldk, const float *__restrict__ gx,
    const float2 *__restrict__ tw) {
  using S = FxShape<P, N, GD>;
  constexpr int NC = S::NC, NH = S::NH;
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *stw = reinterpret_cast<float2 *>(smraw);
  float2 *s = stw + N;
  float *sg = reinterpret_cast<float *>(s + N * NC);
  const int qk = (int)(blockIdx.x % NH);
  const int qj = (int)((blockIdx.x / NH) % N);
  const int box = (int)(blockIdx.x / ((unsigned)NH * N));
  const int64_t RS = (int64_t)ldk * NC, XS = (int64_t)N * RS;
  float2 *col = spec + (int64_t)box * N * XS + (int64_t)qj * RS + (int64_t)qk * NC;
  // the Green's values arrive while the forward transform runs (or, GD, are
  // read by the contraction itself)
  const float *gcol = gx + ((int64_t)qj * NH + qk) * S::GCOL;
  if constexpr (!GD) {
    for (int e = threadIdx.x; e < S::GCOL / 4; e += 256) cp_async16(sg + 4 * e, gcol + 4 * e);
    cp_async_commit();
  }
  load_twiddles(stw, tw, N);
  __syncthreads();
  // forward: the first step reads the column from HBM
  cols_step1<N, NC, false, 256>(s, stw, [&](int l, int r) { return col[r * XS + l]; });
  __syncthreads();
  cols_step2<N, NC, false, true, 256>(s, [&](int l, int r, float2 v) { s[r * NC + l] = v; });
  if constexpr (!GD) cp_async_wait<0>();
  __syncthreads();
  for (int qi = threadIdx.x; qi < N; qi += 256) {
    float2 m[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) m[k] = s[qi * NC + k];
    if constexpr (GD) {
      ct2g_mg2l_all<P, N>(m, gcol + qi, s + qi * NC,
                          std::make_integer_sequence<int, Mg2lPairs<P>::NP>{});
    } else if constexpr (S::GREG) {
      float g[NC];
#pragma unroll
      for (int k = 0; k < NC; k++) g[k] = sg[k * N + qi];
      ct2g_mg2l_all<P, 1>(m, g, s + qi * NC, std::make_integer_sequence<int, Mg2lPairs<P>::NP>{});
    } else {
      ct2g_mg2l_all<P, N>(m, sg + qi, s + qi * NC,
                          std::make_integer_sequence<int, Mg2lPairs<P>::NP>{});
    }
  }
  __syncthreads();
  // inverse: the second step writes the column back to HBM
  cols_step1<N, NC, true, 256>(s, stw, [&](int l, int r) { return s[r * NC + l]; });
  __syncthreads();
  cols_step2<N, NC, true, false, 256>(s, [&](int l, int r, float2 v) { col[r * XS + l] = v; });
}

// The fused x pass + MG2L with its inputs brought in by bulk copies: the
// column (every qi row's NC components) by one tiled tensor copy, its rows
// PITCH complex apart (the copy starts on the 16-byte boundary at or below
// the column: `off` = 0 or 1 complex into each row), and, unless GD, the
// Green's column (contiguous) by one bulk copy, completing on one mbarrier
// (bounded wait) while the twiddles load; GD: the contraction reads the
// Green's values from HBM, and the smaller block (no Green's column, no
// static shared memory, so the dynamic region starts 128-byte aligned) fits
// three to an SM.  CPA: the column arrives instead by per-thread 8-byte
// cp.async copies, all in flight at once, into rows NC complex apart: the
// tensor copy's rows are a 16-byte multiple apart (36 complex at order 4),
// which puts the rows that the contraction's threads read (a k-point each,
// all NC components) into only four bank groups (an 8-way conflict on every
// component); NC apart (odd at order 4) they spread over all banks.  The
// transforms run in place in the copied tile; the inverse's last step
// writes the column back from registers (a tensor store would also write the
// neighbouring column's element that the tile carries, which another block
// owns).
template <int P, int N, bool GD, bool CPA = false>
struct FxTma {
  static constexpr int NC = ct2g_ncomp(P), NH = N / 2 + 1;
  static constexpr int BW = (2 * NC + 3) / 4 * 4;    // floats per tensor-copy row (16-byte multiple)
  static constexpr int PITCH = CPA ? NC : BW / 2;    // complex per tile row
  static constexpr int GCOL = NC * N;
  // GD: tile, twiddles, the mbarrier; else 128 bytes of alignment slack,
  // tile, Green's column, twiddles, the mbarrier
  static constexpr size_t SMEM = (GD ? 0 : 128) + sizeof(float2) * (size_t)N * PITCH +
                                 (GD ? 0 : sizeof(float) * (size_t)GCOL) +
                                 sizeof(float2) * (size_t)N + 16;
  static constexpr bool OK = N >= 64 && N <= 256 && SMEM <= 227 * 1024;
  // three blocks per SM where the contraction fits 85 registers (GD, orders
  // up to 4) and three blocks' shared memory fit
  static constexpr int MINB = (GD && NC <= 35 && 3 * (SMEM + 1024) <= 228 * 1024) ? 3
                              : 2 * (SMEM + 1024) <= 228 * 1024               ? 2
                                                                              : 1;
};

template <int P, int N, bool GD, bool CPA>
__global__ void __launch_bounds__(256, FxTma<P, N, GD, CPA>::MINB) fftx_mg2l_tma_kernel(
    const __grid_constant__ CUtensorMap xmap, float2 *__restrict__ spec, int ldk,
    const float *__restrict__ gx, const float2 *__restrict__ tw, uint32_t *__restrict__ status) {
  using S = FxTma<P, N, GD, CPA>;
  constexpr int NC = S::NC, NH = S::NH, PITCH = S::PITCH;
  // the tensor copy needs a 128-byte aligned destination
  extern __shared__ __align__(128) unsigned char smraw[];
  const uint32_t pad = GD ? 0u : (128u - (tc::smem_addr(smraw) & 127u)) & 127u;
  float2 *s = reinterpret_cast<float2 *>(smraw + pad);  // N rows of PITCH
  float *sg = reinterpret_cast<float *>(s + N * PITCH);
  float2 *stw = reinterpret_cast<float2 *>(sg + (GD ? 0 : S::GCOL));
  uint64_t *bar = reinterpret_cast<uint64_t *>(stw + N);
  const int qk = (int)(blockIdx.x % NH);
  const int qj = (int)((blockIdx.x / NH) % N);
  const int box = (int)(blockIdx.x / ((unsigned)NH * N));
  const int64_t RS = (int64_t)ldk * NC, XS = (int64_t)N * RS;
  const int f0 = 2 * qk * NC, x0 = f0 & ~3, off = CPA ? 0 : (f0 - x0) / 2;
  const float *gcol = gx + ((int64_t)qj * NH + qk) * S::GCOL;
  float2 *col = spec + (int64_t)box * N * XS + (int64_t)qj * RS + (int64_t)qk * NC;
  if (!CPA && (tc::smem_addr(s) & 127u)) {  // checked before any tensor copy
    if (threadIdx.x == 0) atomicExch(status, (uint32_t)CT2G_ECUDA);
    return;
  }
  if (threadIdx.x == 0) tc::mbar_init(bar, 1);
  __syncthreads();  // the barrier is initialised before any thread polls it
  if (threadIdx.x == 0) {
    tc::mbar_arrive_expect_tx(bar, (uint32_t)((CPA ? 0 : sizeof(float2) * N * PITCH) +
                                              (GD ? 0 : sizeof(float) * S::GCOL)));
    if constexpr (!CPA) tc::tma_load_4d(s, &xmap, x0, qj, 0, box, bar);
    if constexpr (!GD) tc::bulk_load(sg, gcol, (uint32_t)(sizeof(float) * S::GCOL), bar);
  }
  if constexpr (CPA) {
    for (int e = threadIdx.x; e < N * NC; e += 256) {
      const int r = e / NC, l = e - r * NC;
      const unsigned sa = tc::smem_addr(s + e);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(col + r * XS + l)
                   : "memory");
    }
    cp_async_commit();
  }
  load_twiddles(stw, tw, N);
  if constexpr (CPA) cp_async_wait<0>();
  const bool ok = tc::mbar_wait(bar, 0, kTmaWaitLimit);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) {
      atomicExch(status, (uint32_t)CT2G_ETIMEOUT);
      tc::mbar_wait(bar, 0, kTmaWaitLimit);  // copies in flight land before the block exits
    }
    return;
  }
  // forward transform in place in the tile
  cols_step1<N, NC, false, 256, PITCH>(
      s, stw, [&](int l, int r) { return s[r * PITCH + off + l]; }, off);
  __syncthreads();
  cols_step2<N, NC, false, true, 256, PITCH>(
      s, [&](int l, int r, float2 v) { s[r * PITCH + off + l] = v; }, off);
  __syncthreads();
  for (int qi = threadIdx.x; qi < N; qi += 256) {
    float2 *row = s + qi * PITCH + off;
    float2 m[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) m[k] = row[k];
    if constexpr (GD) {
      ct2g_mg2l_all<P, N>(m, gcol + qi, row, std::make_integer_sequence<int, Mg2lPairs<P>::NP>{});
    } else if constexpr (FxShape<P, N>::GREG) {
      float g[NC];
#pragma unroll
      for (int k = 0; k < NC; k++) g[k] = sg[k * N + qi];
      ct2g_mg2l_all<P, 1>(m, g, row, std::make_integer_sequence<int, Mg2lPairs<P>::NP>{});
    } else {
      ct2g_mg2l_all<P, N>(m, sg + qi, row, std::make_integer_sequence<int, Mg2lPairs<P>::NP>{});
    }
  }
  __syncthreads();
  // inverse: the second step writes the column back to HBM
  cols_step1<N, NC, true, 256, PITCH>(
      s, stw, [&](int l, int r) { return s[r * PITCH + off + l]; }, off);
  __syncthreads();
  cols_step2<N, NC, true, false, 256, PITCH>(
      s, [&](int l, int r, float2 v) { col[r * XS + l] = v; }, off);
}

template <int P, int N, bool GD>
int launch_fx_mg2l_g(ct2g_ctx *ctx) {
  using S = FxShape<P, N, GD>;
  if constexpr (!S::FITS) {
    return ct2g_fail(ctx, CT2G_EINVAL, "fused X pass + MG2L does not fit in shared memory");
  } else {
    const size_t ncol = (size_t)ctx->nbox * N * S::NH;
    auto k = fftx_mg2l_kernel<P, N, GD>;
    CT2G_TRY(ct2g_smem_attrs(ctx, k, S::SMEM));
    k<<<(unsigned)ncol, 256, S::SMEM, ctx->stream>>>(ctx->spec, ctx->ldk, ctx->greens_x,
                                                     twiddle_ptr<float2>(ctx));
    CT2G_LAUNCHED(ctx);
    return CT2G_OK;
  }
}

// the x-pass tensor map: the spectrum as floats [box][qi][qj][2 * ldk * NC],
// a box of BW floats x all N rows qi of one (qj, box)
int xmap_build(ct2g_ctx *ctx, int BW) {
  if (ctx->xmap_bw == BW) return CT2G_OK;
  EncodeTiledFn encode = nullptr;
  CT2G_TRY(tensor_map_encoder(ctx, &encode));
  const cuuint64_t RS = (cuuint64_t)ctx->ldk * ctx->nc, N = (cuuint64_t)ctx->M;
  const cuuint64_t dims[4] = {2 * RS, N, N, (cuuint64_t)ctx->nbox};
  const cuuint64_t strides[3] = {RS * sizeof(float2), N * RS * sizeof(float2),
                                 N * N * RS * sizeof(float2)};
  const cuuint32_t box[4] = {(cuuint32_t)BW, 1, (cuuint32_t)N, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUtensorMap *m = reinterpret_cast<CUtensorMap *>(ctx->xmap);
  if (encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, ctx->spec, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return ct2g_fail(ctx, CT2G_ECUDA, "x-pass tensor map");
  ctx->xmap_bw = BW;
  return CT2G_OK;
}

template <int P, int N, bool GD, bool CPA>
int launch_fx_mg2l_tma(ct2g_ctx *ctx) {
  using S = FxTma<P, N, GD, CPA>;
  if constexpr (!S::OK) {
    return ct2g_fail(ctx, CT2G_EINVAL, "TMA x pass: meshes 64-256");
  } else {
    CT2G_TRY(xmap_build(ctx, S::BW));
    const size_t ncol = (size_t)ctx->nbox * N * S::NH;
    auto k = fftx_mg2l_tma_kernel<P, N, GD, CPA>;
    CT2G_TRY(ct2g_smem_attrs(ctx, k, S::SMEM));
    const CUtensorMap *m = reinterpret_cast<const CUtensorMap *>(ctx->xmap);
    k<<<(unsigned)ncol, 256, S::SMEM, ctx->stream>>>(*m, ctx->spec, ctx->ldk, ctx->greens_x,
                                                     twiddle_ptr<float2>(ctx), ctx->d_counts + 6);
    CT2G_LAUNCHED(ctx);
    return CT2G_OK;
  }
}

template <int P, int N>
int launch_fx_mg2l(ct2g_ctx *ctx) {
  if (ctx->x_tma == 1) {
    if constexpr (FxTma<P, N, true>::OK) {
      if (ctx->mg2l_greens_direct) return launch_fx_mg2l_tma<P, N, true, false>(ctx);
    }
    if constexpr (FxTma<P, N, false>::OK) return launch_fx_mg2l_tma<P, N, false, false>(ctx);
  }
  if (ctx->x_tma == 2) {
    if constexpr (FxTma<P, N, true, true>::OK) {
      if (ctx->mg2l_greens_direct) return launch_fx_mg2l_tma<P, N, true, true>(ctx);
    }
    if constexpr (FxTma<P, N, false, true>::OK) return launch_fx_mg2l_tma<P, N, false, true>(ctx);
  }
  return ctx->mg2l_greens_direct ? launch_fx_mg2l_g<P, N, true>(ctx)
                                 : launch_fx_mg2l_g<P, N, false>(ctx);
}

// the Y pass (tiles of the (qk, c) columns of each (box, qi) plane) or the
// split X pass (tiles of the (qj, qk, c) columns of each box)
template <int N>
int spec_cols(ct2g_ctx *ctx, bool inv, bool xpass) {
  const size_t RS = (size_t)ctx->ldk * ctx->nc, nb = (size_t)ctx->nbox;
  size_t nouter, ostride, rstride, ncols;
  if (!xpass) {
    nouter = nb * N;
    ostride = (size_t)N * RS;
    rstride = RS;
    ncols = (size_t)(N / 2 + 1) * ctx->nc;
  } else {
    nouter = nb;
    ostride = (size_t)N * N * RS;
    rstride = (size_t)N * RS;
    ncols = (size_t)N * RS;
  }
  if constexpr (N == 256 || N == 512) {
    if (ctx->fft_tc)
      return ct2g_fft_cols_tc(ctx, ctx->spec, N, nouter, ostride, rstride, ncols, inv);
  }
  if (inv) return launch_cols<float, N, true, true>(ctx, ctx->spec, nouter, ostride, rstride, ncols);
  return launch_cols<float, N, false, true>(ctx, ctx->spec, nouter, ostride, rstride, ncols);
}

template <int P>
bool fx_fits(int N) {
  switch (N) {
    case 8: return FxShape<P, 8>::FITS;
    case 16: return FxShape<P, 16>::FITS;
    case 32: return FxShape<P, 32>::FITS;
    case 64: return FxShape<P, 64>::FITS;
    case 128: return FxShape<P, 128>::FITS;
    case 256: return FxShape<P, 256>::FITS;
    case 512: return FxShape<P, 512>::FITS;
  }
  return false;
}

// order x mesh dispatch of the mesh-solve kernels
template <int P>
int spec_stage(ct2g_ctx *ctx, int stage, bool flag, int mode) {
  switch (ctx->M) {
#define CT2G_SPEC_CASE(NN)                                                  \
  case NN:                                                                  \
    if (stage == 0 && mode == CT2G_P2M_COMPACT)                             \
      CT2G_TRY(launch_p2m_compact<P>(ctx));                                 \
    if (stage == 0) return launch_p2m_r2c<P, NN>(ctx, mode);                \
    if (stage == 1) return launch_fx_mg2l<P, NN>(ctx);                      \
    if (stage == 2) return launch_c2r_l2p<P, NN>(ctx, mode);                \
    return spec_cols<NN>(ctx, flag, mode != 0);
    CT2G_SPEC_CASE(8)
    CT2G_SPEC_CASE(16)
    CT2G_SPEC_CASE(32)
    CT2G_SPEC_CASE(64)
    CT2G_SPEC_CASE(128)
    CT2G_SPEC_CASE(256)
    CT2G_SPEC_CASE(512)
#undef CT2G_SPEC_CASE
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "mesh must be a power of two in [8, 512]");
}

// stage 0: z pass (mode: CT2G_P2M_*); 1: fused X + MG2L; 2: inverse
// z pass (mode 0/1/2 as fftz_c2r_l2p_kernel); 3: Y pass (mode 0) or X pass
// (mode 1), inverse when flag
int spec_run(ct2g_ctx *ctx, int stage, bool flag, int mode) {
  switch (ctx->p) {
    case 1: return spec_stage<1>(ctx, stage, flag, mode);
    case 2: return spec_stage<2>(ctx, stage, flag, mode);
    case 3: return spec_stage<3>(ctx, stage, flag, mode);
    case 4: return spec_stage<4>(ctx, stage, flag, mode);
    case 5: return spec_stage<5>(ctx, stage, flag, mode);
    case 6: return spec_stage<6>(ctx, stage, flag, mode);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "unsupported order");
}

template <int P>
int spec_pipe_p(ct2g_ctx *ctx, bool inverse, int mode, bool *done) {
  switch (ctx->M) {
    case 64: return launch_plane_pipe<P, 64>(ctx, inverse, mode, done);
    case 128: return launch_plane_pipe<P, 128>(ctx, inverse, mode, done);
    case 256: return launch_plane_pipe<P, 256>(ctx, inverse, mode, done);
  }
  *done = false;
  return CT2G_OK;
}

// the z and y passes of one direction as the plane pipeline, when the
// context's configuration has one (*done tells)
int spec_pipe(ct2g_ctx *ctx, bool inverse, int mode, bool *done) {
  switch (ctx->p) {
    case 1: return spec_pipe_p<1>(ctx, inverse, mode, done);
    case 2: return spec_pipe_p<2>(ctx, inverse, mode, done);
    case 3: return spec_pipe_p<3>(ctx, inverse, mode, done);
    case 4: return spec_pipe_p<4>(ctx, inverse, mode, done);
    case 5: return spec_pipe_p<5>(ctx, inverse, mode, done);
    case 6: return spec_pipe_p<6>(ctx, inverse, mode, done);
  }
  *done = false;
  return CT2G_OK;
}

}  // namespace

// constant twiddles of the in-register DFTs, once per context (device)
int ct2g_fft_init(ct2g_ctx *ctx) {
  float2 wf[32];
  double2 wd[32];
  const double twopi = 6.283185307179586476925286766559;
  for (int k = 0; k < 32; k++) {
    const double a = -twopi * (double)k / 32.0;
    wd[k] = make_double2(std::cos(a), std::sin(a));
    wf[k] = make_float2((float)wd[k].x, (float)wd[k].y);
  }
  CT2G_CUDA(ctx, cudaMemcpyToSymbol(c_w32f, wf, sizeof(wf)));
  CT2G_CUDA(ctx, cudaMemcpyToSymbol(c_w32d, wd, sizeof(wd)));
  return CT2G_OK;
}

// twiddles exp(-2 pi i k/N), k < N, computed on the host in FP64
int ct2g_twiddles(ct2g_ctx *ctx, int N) {
  if (ctx->tw_n == N) return CT2G_OK;
  if (ctx->capturing) return ct2g_fail(ctx, CT2G_ESTATE, "FFT twiddles not set up before recording");
  ctx->epoch++;  // twiddle pointers are part of a recorded graph
  if (ctx->tw32) cudaFree(ctx->tw32);
  if (ctx->tw64) cudaFree(ctx->tw64);
  ctx->tw32 = nullptr;
  ctx->tw64 = nullptr;
  ctx->tw_n = 0;
  std::vector<float2> t32(N);
  std::vector<double2> t64(N);
  const double twopi = 6.283185307179586476925286766559;
  for (int k = 0; k < N; k++) {
    const double a = -twopi * (double)k / (double)N;
    t64[k] = make_double2(std::cos(a), std::sin(a));
    t32[k] = make_float2((float)t64[k].x, (float)t64[k].y);
  }
  CT2G_CUDA(ctx, cudaMalloc(&ctx->tw32, sizeof(float2) * N));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->tw64, sizeof(double2) * N));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->tw32, t32.data(), sizeof(float2) * N,
                                 cudaMemcpyHostToDevice, ctx->stream));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->tw64, t64.data(), sizeof(double2) * N,
                                 cudaMemcpyHostToDevice, ctx->stream));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->tw_n = N;
  return CT2G_OK;
}

int ct2g_fft_r2c_f32(ct2g_ctx *ctx, const float *in, float2 *out, int N, int batch, int ld) {
  return fft_r2c<float>(ctx, in, out, N, batch, ld);
}
int ct2g_fft_c2r_f32(ct2g_ctx *ctx, float2 *in, float *out, int N, int batch, int ld) {
  return fft_c2r<float>(ctx, in, out, N, batch, ld);
}
int ct2g_fft_c2c_f32(ct2g_ctx *ctx, float2 *a, int N, int batch, bool inv) {
  return fft_c2c(ctx, a, N, batch, inv);
}
int ct2g_fft_r2c_f64(ct2g_ctx *ctx, const double *in, double2 *out, int N, int batch, int ld) {
  return fft_r2c<double>(ctx, in, out, N, batch, ld);
}
int ct2g_fft_c2r_f64(ct2g_ctx *ctx, double2 *in, double *out, int N, int batch, int ld) {
  return fft_c2r<double>(ctx, in, out, N, batch, ld);
}

bool ct2g_mg2l_fused(const ct2g_ctx *ctx) {
  if (ctx->fft_tc || ctx->split_mg2l || !ctx->greens_x) return false;
  switch (ctx->p) {
    case 1: return fx_fits<1>(ctx->M);
    case 2: return fx_fits<2>(ctx->M);
    case 3: return fx_fits<3>(ctx->M);
    case 4: return fx_fits<4>(ctx->M);
    case 5: return fx_fits<5>(ctx->M);
    case 6: return fx_fits<6>(ctx->M);
  }
  return false;
}

// z pass (P2M inside it, or from the moment grid), Y pass, X pass when split
int ct2g_spec_forward(ct2g_ctx *ctx, int src) {
  CT2G_TRY(ct2g_twiddles(ctx, ctx->M));
  bool piped = false;
  CT2G_TRY(spec_pipe(ctx, false, src, &piped));
  if (!piped) {
    // P2M into compact per-cell records first, read by the z pass
    if (src == CT2G_P2M_FUSED && ctx->p2m_compact && ctx->cmom) src = CT2G_P2M_COMPACT;
    CT2G_TRY(spec_run(ctx, 0, false, src));
    CT2G_TRY(spec_run(ctx, 3, false, 0));
  }
  if (!ct2g_mg2l_fused(ctx)) CT2G_TRY(spec_run(ctx, 3, false, 1));
  return CT2G_OK;
}

int ct2g_spec_mg2l(ct2g_ctx *ctx) {
  if (ct2g_mg2l_fused(ctx)) return spec_run(ctx, 1, false, 0);
  return ct2g_mg2l_split(ctx);
}

// inverse X pass when split, Y pass, z pass (L2P inside it, or into the
// expansion grid)
int ct2g_spec_inverse(ct2g_ctx *ctx, bool l2p, bool pot) {
  CT2G_TRY(ct2g_twiddles(ctx, ctx->M));
  if (!ct2g_mg2l_fused(ctx)) CT2G_TRY(spec_run(ctx, 3, true, 1));
  const int mode = l2p ? (pot ? 1 : 0) : 2;
  bool piped = false;
  CT2G_TRY(spec_pipe(ctx, true, mode, &piped));
  if (piped) return CT2G_OK;
  CT2G_TRY(spec_run(ctx, 3, true, 0));
  return spec_run(ctx, 2, false, mode);
}
