// Precision form of the mesh FFT: the strided (y and x) passes as DFT matrix
// products on the tensor cores (tcgen05, BF16 operands, FP32 accumulation in
// tensor memory), with every operand split into BF16 hi + lo parts.
//
// A pass transforms lines of N = 16 * R2 points (N = 256: R2 = 16; N = 512:
// R2 = 32) by the four-step factorisation n = n1 + 16 n2, k = k2 + R2 k1:
//   stage 1  Y[n1][k2] = sum_n2 x[n1 + 16 n2] w_R2^(n2 k2)      (radix R2)
//   twiddle  Y[n1][k2] *= w_N^(n1 k2)                           (FP32)
//   stage 2  X[k2 + R2 k1] = sum_n1 Y[n1][k2] w_16^(n1 k1)      (radix 16)
// A CTA takes a tile of 8 lines.  Each stage is one GEMM D = A B^T: rows of
// A are (line, n1) for stage 1 and (line, k2) for stage 2; a complex radix-R
// DFT is the real 2R x 2R matrix [[Re F, -Im F], [Im F, Re F]] acting on
// (Re, Im), and the split products x_hi F_hi + x_lo F_hi + x_hi F_lo are one
// accumulation over K = 3 * 2R: B = [F_hi | F_hi | F_lo] in shared memory,
// A = [x_hi | x_lo] with the third K block read from x_hi again (its
// descriptor points back at the first block).  The DFT matrices are split on
// the host from FP64 values.
#include <cstring>

#include "ct2g_internal.cuh"
#include "ct2g_tc.cuh"

namespace {

constexpr int TW = 8;   // lines per tile
constexpr int TP = 9;   // tile buffer size per row (complex; the row view uses 8 of them)

// Row view of the tile buffer: element (row r, line c) at r * 8 + (c ^
// ((r >> 1) & 7)).  The XOR spreads the accesses of a half-warp over all 16
// complex-wide bank slots in the three patterns that use this view: a row
// run of (line pairs x 4 rows) when the tile moves in and out, 16 rows of one
// line for the stage-1 operand, and 16 rows of one line for the stage-2
// result (a plain pitch of 9 left 2-way conflicts on the first, of 8 made
// the second 8-way).
__device__ __forceinline__ int tidx(int r, int c) { return r * 8 + (c ^ ((r >> 1) & 7)); }
constexpr int R1 = 16;  // radix of stage 2
constexpr uint32_t kWaitLimit = 1u << 22;

template <int N>
struct TcShape {
  static constexpr int R2 = N / R1;
  static constexpr int K1 = 6 * R2, N1 = 2 * R2;  // stage 1 GEMM (B's K extent)
  static constexpr int K2 = 6 * R1, N2 = 2 * R1;  // stage 2 GEMM
  static constexpr int KA1 = 4 * R2, KA2 = 4 * R1; // A's stored K extent: [hi | lo]
  static constexpr int MT2 = TW * R2 / 128;        // 128-row tiles in stage 2
  static constexpr uint32_t KA = 16 * 128;         // K step of a 128-row A tile
  static constexpr uint32_t KB1 = (N1 / 8) * 128, KB2 = (N2 / 8) * 128;
  static constexpr uint32_t SZ_A1 = (KA1 / 8) * KA, SZ_A2 = MT2 * (KA2 / 8) * KA;
  static constexpr uint32_t SZ_A = SZ_A1 > SZ_A2 ? SZ_A1 : SZ_A2;
  static constexpr uint32_t SZ_B1 = (K1 / 8) * KB1, SZ_B2 = (K2 / 8) * KB2;
  static constexpr uint32_t SZ_TW = N * 8, SZ_T = N * TP * 8;
  static constexpr uint32_t OFF_B1 = SZ_A, OFF_B2 = OFF_B1 + SZ_B1, OFF_TW = OFF_B2 + SZ_B2,
                            OFF_T = OFF_TW + SZ_TW, SMEM = OFF_T + SZ_T;
  static constexpr uint32_t TABLE = SZ_B1 + SZ_B2 + SZ_TW;  // bytes of one direction's tables
  static constexpr uint32_t TCOLS = (N1 + MT2 * N2) <= 64 ? 64 : 128;
  static_assert(TW * R1 == 128, "stage 1 rows");
  static_assert(TW * R2 * 17 * 8 <= SZ_T, "transposed stage-1 results fit the tile buffer");
  static_assert(SMEM <= 200 * 1024, "shared memory");
};

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat16 x = __float2bfloat16_rn(a), y = __float2bfloat16_rn(b);
  return (uint32_t)__bfloat16_as_ushort(x) | ((uint32_t)__bfloat16_as_ushort(y) << 16);
}

// value v -> (hi, lo) with hi = bf16(v), lo = bf16(v - hi)
__device__ __forceinline__ void split_bf16(float v, float &hi, float &lo) {
  hi = __bfloat162float(__float2bfloat16_rn(v));
  lo = v - hi;
}

// VEC: rows start on 16-byte boundaries (tile rows move as float4 pairs);
// otherwise element by element
template <int N, bool VEC>
__global__ void __launch_bounds__(128) fft_cols_tc_kernel(float2 *__restrict__ a, size_t ostride,
                                                          size_t rstride, size_t ncols,
                                                          uint32_t ntiles, size_t ntot,
                                                          const uint4 *__restrict__ tables,
                                                          uint32_t *__restrict__ status) {
  using S = TcShape<N>;
  constexpr int R2 = S::R2;
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (uint32_t i = tid; i < S::TABLE / 16; i += 128)
    reinterpret_cast<uint4 *>(sm + S::OFF_B1)[i] = tables[i];
  if (warp == 0) tc::tmem_alloc(&slot, S::TCOLS);
  if (tid == 0) tc::mbar_init(&bar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = slot;
  const uint32_t lane_base = (uint32_t)(32 * warp) << 16;
  unsigned char *A = sm;
  const float2 *tw = reinterpret_cast<const float2 *>(sm + S::OFF_TW);
  float2 *T = reinterpret_cast<float2 *>(sm + S::OFF_T);  // rows of TW lines (tidx)
  const uint32_t sA = tc::smem_addr(A), sB1 = tc::smem_addr(sm + S::OFF_B1),
                 sB2 = tc::smem_addr(sm + S::OFF_B2);
  uint32_t phase = 0;
  bool ok = true;
  // a tile is N rows of TW complex, 4 chunks of 16 bytes per row; every
  // thread holds its chunks of the next tile in registers while the current
  // one is transformed
  constexpr int CH = N * 4 / 128;
  float4 pre[CH];
  auto fetch = [&](size_t t) {
    const size_t outer = t / ntiles, c0 = (size_t)(t % ntiles) * TW;
    const int nv = (int)min((size_t)TW, ncols - c0);
    const float2 *b = a + outer * ostride + c0;
#pragma unroll
    for (int j = 0; j < CH; j++) {
      const int e = tid + 128 * j, r = e >> 2, c = (e & 3) * 2;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (VEC && c + 1 < nv) {
        v = __ldg(reinterpret_cast<const float4 *>(b + (size_t)r * rstride + c));
      } else {
        if (c < nv) {
          const float2 u = b[(size_t)r * rstride + c];
          v.x = u.x;
          v.y = u.y;
        }
        if (c + 1 < nv) {
          const float2 u = b[(size_t)r * rstride + c + 1];
          v.z = u.x;
          v.w = u.y;
        }
      }
      pre[j] = v;
    }
  };
  if ((size_t)blockIdx.x < ntot) fetch(blockIdx.x);
  for (size_t tile = blockIdx.x; tile < ntot; tile += gridDim.x) {
    const size_t outer = tile / ntiles;
    const size_t col0 = (size_t)(tile % ntiles) * TW;
    const int wv = (int)min((size_t)TW, ncols - col0);
    float2 *base = a + outer * ostride + col0;
#pragma unroll
    for (int j = 0; j < CH; j++) {
      const int e = tid + 128 * j, r = e >> 2, c = (e & 3) * 2;
      T[tidx(r, c)] = make_float2(pre[j].x, pre[j].y);
      T[tidx(r, c + 1)] = make_float2(pre[j].z, pre[j].w);
    }
    if (tile + gridDim.x < ntot) fetch(tile + gridDim.x);
    __syncthreads();
    // stage 1 operand: row tid = (w, n1); K = [hi | lo | hi] x (Re, Im) x n2
    {
      const int w = tid / R1, n1 = tid % R1;
      float hr[R2], lr[R2], hi_[R2], li[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; n2++) {
        const float2 x = T[tidx(n1 + R1 * n2, w)];
        split_bf16(x.x, hr[n2], lr[n2]);
        split_bf16(x.y, hi_[n2], li[n2]);
      }
#pragma unroll
      for (int kg = 0; kg < S::KA1 / 8; kg++) {
        const int blk = (8 * kg) / (2 * R2), kk = (8 * kg) % (2 * R2);
        const bool im = kk >= R2;
        const int m0 = im ? kk - R2 : kk;
        const float *src = blk == 1 ? (im ? li : lr) : (im ? hi_ : hr);
        uint4 q;
        q.x = pack_bf16(src[m0 + 0], src[m0 + 1]);
        q.y = pack_bf16(src[m0 + 2], src[m0 + 3]);
        q.z = pack_bf16(src[m0 + 4], src[m0 + 5]);
        q.w = pack_bf16(src[m0 + 6], src[m0 + 7]);
        *reinterpret_cast<uint4 *>(A + tc::kmajor_offset(tid, 8 * kg, S::KA, 128)) = q;
      }
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(128, S::N1);
#pragma unroll
      for (int kk = 0; kk < S::K1 / 16; kk++) {
        const int ka = kk < S::KA1 / 16 ? kk : kk - S::KA1 / 16;  // third block: x_hi again
        tc::mma_bf16(tmem, tc::sdesc(sA + ka * 2 * S::KA, S::KA, 128),
                     tc::sdesc(sB1 + kk * 2 * S::KB1, S::KB1, 128), idesc, kk > 0);
      }
      tc::mma_commit(&bar);
    }
    ok = __syncthreads_and(tc::mbar_wait(&bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    // stage 1 result of row (w, n1): Re Y[n1][k2] in columns k2, Im in R2 + k2
    {
      const int w = tid / R1, n1 = tid % R1;
      float y[S::N1];
#pragma unroll
      for (int c = 0; c < S::N1; c += 32) tc::tmem_ld32(tmem + lane_base + (uint32_t)c, y + c);
      // twiddle; the results go through the tile buffer (free now) transposed
      // to rows (w, k2) of 16 complex n1 values (pitch 17)
#pragma unroll
      for (int k2 = 0; k2 < R2; k2++) {
        const float2 t = tw[n1 * k2];
        const float re = y[k2] * t.x - y[R2 + k2] * t.y;
        const float im = y[k2] * t.y + y[R2 + k2] * t.x;
        T[(w * R2 + k2) * 17 + n1] = make_float2(re, im);
      }
    }
    __syncthreads();
    // stage 2 operand: row r2 = (w, k2); K = [hi | lo | hi] x (Re, Im) x n1
#pragma unroll
    for (int mt = 0; mt < S::MT2; mt++) {
      const int r2 = mt * 128 + tid;
      float hr[R1], lr[R1], hi_[R1], li[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; n1++) {
        const float2 x = T[r2 * 17 + n1];
        split_bf16(x.x, hr[n1], lr[n1]);
        split_bf16(x.y, hi_[n1], li[n1]);
      }
      unsigned char *At = A + mt * (S::KA2 / 8) * S::KA;
#pragma unroll
      for (int kg = 0; kg < S::KA2 / 8; kg++) {
        const int blk = (8 * kg) / (2 * R1), kk = (8 * kg) % (2 * R1);
        const bool im = kk >= R1;
        const int m0 = im ? kk - R1 : kk;
        const float *src = blk == 1 ? (im ? li : lr) : (im ? hi_ : hr);
        uint4 q;
        q.x = pack_bf16(src[m0 + 0], src[m0 + 1]);
        q.y = pack_bf16(src[m0 + 2], src[m0 + 3]);
        q.z = pack_bf16(src[m0 + 4], src[m0 + 5]);
        q.w = pack_bf16(src[m0 + 6], src[m0 + 7]);
        *reinterpret_cast<uint4 *>(At + tc::kmajor_offset(tid, 8 * kg, S::KA, 128)) = q;
      }
    }
    tc::fence_before_sync();
    tc::fence_async_smem();
    __syncthreads();
    tc::fence_after_sync();
    if (tid == 0) {
      constexpr uint32_t idesc = tc::idesc_bf16_f32(128, S::N2);
#pragma unroll
      for (int mt = 0; mt < S::MT2; mt++)
#pragma unroll
        for (int kk = 0; kk < S::K2 / 16; kk++) {
          const int ka = kk < S::KA2 / 16 ? kk : kk - S::KA2 / 16;
          tc::mma_bf16(tmem + (uint32_t)(S::N1 + mt * S::N2),
                       tc::sdesc(sA + mt * (S::KA2 / 8) * S::KA + ka * 2 * S::KA, S::KA, 128),
                       tc::sdesc(sB2 + kk * 2 * S::KB2, S::KB2, 128), idesc, kk > 0);
        }
      tc::mma_commit(&bar);
    }
    ok = __syncthreads_and(tc::mbar_wait(&bar, phase, kWaitLimit));
    phase ^= 1;
    if (!ok) break;
    tc::fence_after_sync();
    // stage 2 result of row (w, k2): Re X[k2 + R2 k1] in columns k1, Im in 16 + k1
#pragma unroll
    for (int mt = 0; mt < S::MT2; mt++) {
      const int r2 = mt * 128 + tid, w = r2 / R2, k2 = r2 % R2;
      float v[32];
      tc::tmem_ld32(tmem + lane_base + (uint32_t)(S::N1 + mt * S::N2), v);
#pragma unroll
      for (int k1 = 0; k1 < R1; k1++) T[tidx(k2 + R2 * k1, w)] = make_float2(v[k1], v[R1 + k1]);
    }
    __syncthreads();
    for (int e = tid; e < N * 4; e += 128) {
      const int r = e >> 2, c = (e & 3) * 2;
      const float2 u0 = T[tidx(r, c)], u1 = T[tidx(r, c + 1)];
      const float4 v = make_float4(u0.x, u0.y, u1.x, u1.y);
      if (VEC && c + 1 < wv) {
        *reinterpret_cast<float4 *>(base + (size_t)r * rstride + c) = v;
      } else {
        if (c < wv) base[(size_t)r * rstride + c] = make_float2(v.x, v.y);
        if (c + 1 < wv) base[(size_t)r * rstride + c + 1] = make_float2(v.z, v.w);
      }
    }
    // the next tile rewrites the tile buffer and tensor memory
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  if (!ok) {
    if (tid == 0) atomicExch(status, (uint32_t)CT2G_ETIMEOUT);
    tc::mbar_wait(&bar, phase ^ 1, kWaitLimit);  // the MMAs still in flight
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, S::TCOLS);
}

// host image of one direction's tables: B1 (radix R2), B2 (radix 16) in the
// K-major layout, then the twiddles w_N^p, p < N (sign -1 forward, +1 inverse)
template <int N>
std::vector<unsigned char> make_tables(bool inv) {
  using S = TcShape<N>;
  std::vector<unsigned char> img(S::TABLE, 0);
  const double twopi = 6.283185307179586476925286766559;
  const double sgn = inv ? 1.0 : -1.0;
  auto bf16 = [](double v, float &hi, float &lo) {
    // round to nearest even on the FP32 value's top 16 bits
    auto rnd = [](float f) {
      uint32_t u;
      std::memcpy(&u, &f, 4);
      u = (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
      float r;
      std::memcpy(&r, &u, 4);
      return r;
    };
    hi = rnd((float)v);
    lo = rnd((float)(v - (double)hi));
  };
  auto put = [&](size_t off, float bf) {
    uint32_t u;
    std::memcpy(&u, &bf, 4);
    const uint16_t h = (uint16_t)(u >> 16);
    std::memcpy(img.data() + off, &h, 2);
  };
  auto fill = [&](size_t base, int R, uint32_t kstep) {
    for (int n = 0; n < 2 * R; n++)
      for (int k = 0; k < 6 * R; k++) {
        const int blk = k / (2 * R), kk = k % (2 * R);
        const int j = n % R, m = kk % R;
        const bool out_im = n >= R, in_im = kk >= R;
        const double th = twopi * (double)((j * m) % R) / (double)R;
        const double fr = std::cos(th), fi = sgn * std::sin(th);
        const double v = out_im ? (in_im ? fr : fi) : (in_im ? -fi : fr);
        float hi, lo;
        bf16(v, hi, lo);
        put(base + tc::kmajor_offset((uint32_t)n, (uint32_t)k, kstep, 128), blk == 2 ? lo : hi);
      }
  };
  fill(0, S::R2, S::KB1);
  fill(S::SZ_B1, R1, S::KB2);
  float2 *t = reinterpret_cast<float2 *>(img.data() + S::SZ_B1 + S::SZ_B2);
  for (int p = 0; p < N; p++) {
    const double th = twopi * (double)p / (double)N;
    t[p] = make_float2((float)std::cos(th), (float)(sgn * std::sin(th)));
  }
  return img;
}

template <int N>
int launch_tc(ct2g_ctx *ctx, float2 *spec, size_t nouter, size_t ostride, size_t rstride,
              size_t ncols, bool inv) {
  using S = TcShape<N>;
  // float4 tile rows need 16-byte aligned rows and outer blocks
  const bool vec = (rstride % 2 == 0) && (ostride % 2 == 0) &&
                   (reinterpret_cast<uintptr_t>(spec) % 16 == 0);
  auto k = vec ? fft_cols_tc_kernel<N, true> : fft_cols_tc_kernel<N, false>;
  CT2G_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM));
  // all of the unified L1 as shared memory, so that several CTAs fit per SM
  CT2G_CUDA(ctx, cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
  // CTAs per SM from the kernel's own limits -- registers, shared memory at
  // the maximum carveout, tensor-memory columns -- rather than from the
  // occupancy query, which reported one CTA per SM here (it does not apply
  // the carveout preference set above)
  int per_sm = std::min(ct2g_blocks_per_sm(ctx, (const void *)k, 128, S::SMEM),
                        (int)(512 / S::TCOLS));
  per_sm = std::max(1, per_sm);
  const uint32_t ntiles = (uint32_t)((ncols + TW - 1) / TW);
  const size_t ntot = nouter * ntiles;
  const size_t grid = std::min(ntot, (size_t)per_sm * ctx->num_sms);
  const uint4 *tab = reinterpret_cast<const uint4 *>(ctx->tc_tables + (inv ? S::TABLE : 0));
  k<<<(unsigned)grid, 128, S::SMEM, ctx->stream>>>(spec, ostride, rstride, ncols, ntiles, ntot,
                                                    tab, ctx->d_counts + 6);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

}  // namespace

bool ct2g_fft_tc_supported(int N) { return N == 256 || N == 512; }

// both directions' tables for the context's mesh, built once (not while a
// graph is recorded)
int ct2g_fft_tc_prepare(ct2g_ctx *ctx) {
  if (ctx->tc_tables) return CT2G_OK;
  if (ctx->capturing) return ct2g_fail(ctx, CT2G_ESTATE, "tensor-core FFT tables not built before recording");
  std::vector<unsigned char> f, b;
  if (ctx->M == 256) {
    f = make_tables<256>(false);
    b = make_tables<256>(true);
  } else if (ctx->M == 512) {
    f = make_tables<512>(false);
    b = make_tables<512>(true);
  } else {
    return ct2g_fail(ctx, CT2G_EINVAL, "the tensor-core FFT supports meshes 256 and 512");
  }
  unsigned char *d = nullptr;
  CT2G_CUDA(ctx, cudaMalloc(&d, f.size() + b.size()));
  cudaError_t e = cudaMemcpy(d, f.data(), f.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + f.size(), b.data(), b.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return ct2g_cuda_fail(ctx, e, "tensor-core FFT tables");
  }
  ctx->tc_tables = d;
  ctx->epoch++;
  return CT2G_OK;
}

int ct2g_fft_cols_tc(ct2g_ctx *ctx, float2 *spec, int N, size_t nouter, size_t ostride,
                     size_t rstride, size_t ncols, bool inv) {
  if (!ctx->tc_tables || N != ctx->M) return ct2g_fail(ctx, CT2G_ESTATE, "tensor-core FFT not prepared for this size");
  if (N == 256) return launch_tc<256>(ctx, spec, nouter, ostride, rstride, ncols, inv);
  if (N == 512) return launch_tc<512>(ctx, spec, nouter, ostride, rstride, ncols, inv);
  return ct2g_fail(ctx, CT2G_EINVAL, "the tensor-core FFT supports sizes 256 and 512");
}
