// Cloud-in-cell deposit of the particle store onto a complex mesh, and the
// complex-to-complex 3D FFT over device grids.  No counterpart in the
// reference (its mesh quantities are per-cell multipoles, src/particle.cpp:
// 180-209); these serve callers that want a plain density mesh and its
// spectrum, in FP32 on the CUDA cores or with the y and x passes on the
// tensor cores (ct2g_set_fft_mode).
//
// Deposit: a particle at x (box units) sits between mesh points
// m = floor(x N - 1/2) and m + 1 along each axis, at fraction
// f = x N - 1/2 - m; it adds weight w = prod_d (f_d or 1 - f_d) to the 8
// surrounding points (periodic), and the four grids receive, at every point,
//   grid 0: sum_p w            (the CIC mass, unit particle mass)
//   grid 1..3: sum_p w * s_d   (the first moment about the point, s_d the
//                                particle's offset from it, in mesh units)
// as the real parts of complex values (imaginary parts zero), so that a
// batch of four complex transforms of N^3 points follows.
#include "ct2g_internal.cuh"

namespace {

__global__ void cic_deposit_kernel(const uint32_t *__restrict__ x, const uint32_t *__restrict__ y,
                                   const uint32_t *__restrict__ z, size_t n, int N,
                                   float2 *__restrict__ grid) {
  const size_t N3 = (size_t)N * N * N;
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < n;
       p += (size_t)gridDim.x * blockDim.x) {
    const uint32_t c[3] = {x[p], y[p], z[p]};
    int m[3];
    float f[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      // x N - 1/2 in mesh units, exact in FP64 for N <= 2^20
      const double u = (double)c[d] * CT2G_TWO_M32 * (double)N - 0.5;
      const double fl = floor(u);
      m[d] = (int)fl;
      f[d] = (float)(u - fl);
    }
#pragma unroll
    for (int corner = 0; corner < 8; corner++) {
      float w = 1.f, s[3];
      int idx[3];
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const int b = (corner >> (2 - d)) & 1;
        w *= b ? f[d] : 1.f - f[d];
        s[d] = b ? f[d] - 1.f : f[d];
        idx[d] = (m[d] + b) & (N - 1);
      }
      const size_t q = ((size_t)idx[0] * N + idx[1]) * N + idx[2];
      atomicAdd(&grid[q].x, w);
      atomicAdd(&grid[N3 + q].x, w * s[0]);
      atomicAdd(&grid[2 * N3 + q].x, w * s[1]);
      atomicAdd(&grid[3 * N3 + q].x, w * s[2]);
    }
  }
}

bool pow2(int n) { return n >= 1 && (n & (n - 1)) == 0; }

}  // namespace

extern "C" int ct2g_cic_deposit(ct2g_ctx *ctx, int N, void *d_grid) {
  CT2G_TRY(ct2g_check(ctx));
  if (!d_grid || !pow2(N) || N < 4 || N > 512)
    return ct2g_fail(ctx, CT2G_EINVAL, "cic_deposit: N a power of two in [4, 512], grid non-null");
  if (!ctx->has_particles) return ct2g_fail(ctx, CT2G_ESTATE, "no particles uploaded");
  const size_t N3 = (size_t)N * N * N;
  float2 *g = reinterpret_cast<float2 *>(d_grid);
  CT2G_CUDA(ctx, cudaMemsetAsync(g, 0, sizeof(float2) * 4 * N3, ctx->stream));
  if (ctx->n == 0) return CT2G_OK;
  const unsigned blocks = (unsigned)std::min<size_t>((ctx->n + 255) / 256, (size_t)ctx->num_sms * 8);
  cic_deposit_kernel<<<blocks, 256, 0, ctx->stream>>>(ctx->x, ctx->y, ctx->z, ctx->n, N, g);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

extern "C" int ct2g_fft3d_c2c_f32_dev(ct2g_ctx *ctx, int dir, void *d_data, int N, int batch) {
  CT2G_TRY(ct2g_check(ctx));
  if (!d_data || batch < 1 || !pow2(N) || N < 4 || N > 512 || (dir != 1 && dir != -1))
    return ct2g_fail(ctx, CT2G_EINVAL, "fft3d_c2c_f32_dev: bad arguments");
  if ((reinterpret_cast<uintptr_t>(d_data) & 15) != 0)
    return ct2g_fail(ctx, CT2G_EINVAL, "fft3d_c2c_f32_dev: the grid must be 16-byte aligned");
  if (ctx->fft_tc && N != ctx->M)
    return ct2g_fail(ctx, CT2G_EINVAL,
                     "fft3d_c2c_f32_dev: the tensor-core passes are prepared for the context's mesh");
  return ct2g_fft_c2c_f32(ctx, reinterpret_cast<float2 *>(d_data), N, batch, dir < 0);
}
