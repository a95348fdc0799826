// Self-test of the tcgen05 building blocks (ct2g_tc.cuh): one CTA computes
// D[128][N] = A[128][K] * B[N][K]^T with BF16 operands staged in shared
// memory (K-major, no swizzle) and the FP32 accumulator in tensor memory.
#include "ct2g_internal.cuh"
#include "ct2g_tc.cuh"

namespace {

constexpr uint32_t kWaitLimit = 1u << 22;  // mbarrier polls (~0.3 s) before giving up

template <int N, int K>
__global__ void __launch_bounds__(128) tc_gemm_test_kernel(const float *__restrict__ A,
                                                           const float *__restrict__ B,
                                                           float *__restrict__ D,
                                                           int *__restrict__ status) {
  // A: 128 rows, K step 2048 B (16 row groups of 128 B), row step 128 B;
  // B: N rows, K step N/8 * 128 B, row step 128 B.  The dynamic allocation
  // (64 KB) covers every address either operand could reach.
  constexpr uint32_t KA = 16 * 128, KB = (N / 8) * 128;
  constexpr uint32_t SA = (K / 8) * KA;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *sa = sm, *sb = sm + SA;
  __shared__ uint64_t bar;
  __shared__ uint32_t slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < 128 * K; i += 128) {
    const int r = i / K, k = i % K;
    *reinterpret_cast<__nv_bfloat16 *>(sa + tc::kmajor_offset(r, k, KA, 128)) =
        __float2bfloat16_rn(A[i]);
  }
  for (int i = tid; i < N * K; i += 128) {
    const int r = i / K, k = i % K;
    *reinterpret_cast<__nv_bfloat16 *>(sb + tc::kmajor_offset(r, k, KB, 128)) =
        __float2bfloat16_rn(B[i]);
  }
  tc::fence_async_smem();
  if (warp == 0) tc::tmem_alloc(&slot, N < 32 ? 32 : N);
  if (tid == 0) tc::mbar_init(&bar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = slot;
  if (tid == 0) {
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, N);
#pragma unroll
    for (int kk = 0; kk < K / 16; kk++)
      tc::mma_bf16(taddr, tc::sdesc(tc::smem_addr(sa + kk * 2 * KA), KA, 128),
                   tc::sdesc(tc::smem_addr(sb + kk * 2 * KB), KB, 128), idesc, kk > 0);
    tc::mma_commit(&bar);
  }
  bool ok = tc::mbar_wait(&bar, 0, kWaitLimit);
  if (!ok) {
    if (tid == 0) status[0] = CT2G_ETIMEOUT;
    ok = tc::mbar_wait(&bar, 0, kWaitLimit);  // the MMA may still be running
  }
  tc::fence_after_sync();
  if (ok) {
    const int row = 32 * warp + (tid & 31);
#pragma unroll
    for (int c = 0; c < N; c += 32) {
      float v[32];
      tc::tmem_ld32(taddr + ((uint32_t)(32 * warp) << 16) + (uint32_t)c, v);
#pragma unroll
      for (int j = 0; j < 32; j++)
        if (c + j < N) D[row * N + c + j] = v[j];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, N < 32 ? 32 : N);
}

template <int N, int K>
int run_test(ct2g_ctx *ctx, const float *dA, const float *dB, float *dD, int *dS,
             cudaStream_t st) {
  auto k = tc_gemm_test_kernel<N, K>;
  const int smem = 64 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return CT2G_ECUDA;
  k<<<1, 128, smem, st>>>(dA, dB, dD, dS);
  (void)ctx;
  return cudaGetLastError() == cudaSuccess ? CT2G_OK : CT2G_ECUDA;
}

// The bounded wait and its error report, with nothing to wait for: an
// mbarrier that expects one arrival and never gets it.  Each thread polls it
// `polls` times (tc::mbar_wait), then the first thread records CT2G_ETIMEOUT
// in the context's device error word, exactly as the tensor-core passes do
// when their MMA completion does not arrive, and the kernel returns.
__global__ void __launch_bounds__(128) wait_selftest_kernel(uint32_t polls,
                                                            uint32_t *__restrict__ status) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  __syncthreads();
  const bool ok = tc::mbar_wait(&bar, 0, polls);
  if (!ok && threadIdx.x == 0) atomicExch(status, (uint32_t)CT2G_ETIMEOUT);
}

}  // namespace

extern "C" int ct2g_wait_selftest(ct2g_ctx *ctx, uint32_t polls) {
  CT2G_TRY(ct2g_check(ctx));
  if (polls < 1 || polls > (1u << 22))
    return ct2g_fail(ctx, CT2G_EINVAL, "wait_selftest: polls in [1, 2^22]");
  if (!ctx->d_counts) return ct2g_fail(ctx, CT2G_ESTATE, "wait_selftest: context has no device state");
  wait_selftest_kernel<<<1, 128, 0, ctx->stream>>>(polls, ctx->d_counts + 6);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

extern "C" int ct2g_tc_selftest(int device, const float *A, const float *B, int N, int K,
                                float *D) {
  if (!A || !B || !D) return CT2G_EINVAL;
  if (!((N == 32 || N == 64) && (K == 16 || K == 32 || K == 64 || K == 96))) return CT2G_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return CT2G_ENODEV;
  }
  if (cudaSetDevice(device) != cudaSuccess) return CT2G_ENODEV;
  float *dA = nullptr, *dB = nullptr, *dD = nullptr;
  int *dS = nullptr;
  int rc = CT2G_OK;
  cudaError_t e = cudaMalloc(&dA, sizeof(float) * 128 * K);
  if (e == cudaSuccess) e = cudaMalloc(&dB, sizeof(float) * N * K);
  if (e == cudaSuccess) e = cudaMalloc(&dD, sizeof(float) * 128 * N);
  if (e == cudaSuccess) e = cudaMalloc(&dS, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(dA, A, sizeof(float) * 128 * K, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dB, B, sizeof(float) * N * K, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dS, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(dD, 0, sizeof(float) * 128 * N);
  if (e != cudaSuccess) rc = CT2G_ECUDA;
  if (rc == CT2G_OK) {
    const int key = N * 1000 + K;
    switch (key) {
      case 32016: rc = run_test<32, 16>(nullptr, dA, dB, dD, dS, 0); break;
      case 32032: rc = run_test<32, 32>(nullptr, dA, dB, dD, dS, 0); break;
      case 32064: rc = run_test<32, 64>(nullptr, dA, dB, dD, dS, 0); break;
      case 32096: rc = run_test<32, 96>(nullptr, dA, dB, dD, dS, 0); break;
      case 64016: rc = run_test<64, 16>(nullptr, dA, dB, dD, dS, 0); break;
      case 64032: rc = run_test<64, 32>(nullptr, dA, dB, dD, dS, 0); break;
      case 64064: rc = run_test<64, 64>(nullptr, dA, dB, dD, dS, 0); break;
      case 64096: rc = run_test<64, 96>(nullptr, dA, dB, dD, dS, 0); break;
    }
  }
  int st = 0;
  if (rc == CT2G_OK && cudaDeviceSynchronize() != cudaSuccess) rc = CT2G_ECUDA;
  if (rc == CT2G_OK && cudaMemcpy(&st, dS, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = CT2G_ECUDA;
  if (rc == CT2G_OK && st) rc = st;
  if (rc == CT2G_OK && cudaMemcpy(D, dD, sizeof(float) * 128 * N, cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = CT2G_ECUDA;
  if (dA) cudaFree(dA);
  if (dB) cudaFree(dB);
  if (dD) cudaFree(dD);
  if (dS) cudaFree(dS);
  return rc;
}
