// Velocity + rung update of kick_cell (src/kick.cpp:75-99) and drift
// (src/drift.cpp:4-18).  Kept in their own translation unit, built with IEEE
// single precision (no flush-to-zero), because both must match the CPU
// restatement bit for bit: the update in FP64 arithmetic with explicit
// round-to-nearest operations, ceil(log2(t0/dt)) from the exponent bits, the
// drift as a truncating fixed32 conversion of v * (dt/scale).
#include "ct2g_internal.cuh"

namespace {

__device__ __forceinline__ int ceil_log2_exact(float v) {
  // exact ceil(log2(v)) for finite normal v > 0
  const uint32_t u = __float_as_uint(v);
  const int e = (int)((u >> 23) & 255u) - 127;
  return (u & 0x7fffffu) ? e + 1 : e;
}

__global__ void update_kernel(size_t begin, size_t end, const float *__restrict__ fx,
                              const float *__restrict__ fy, const float *__restrict__ fz,
                              float *__restrict__ vx, float *__restrict__ vy,
                              float *__restrict__ vz, int8_t *__restrict__ rung,
                              ct2g_kick_params p, float hsoft, int *__restrict__ maxrung) {
  const size_t i = begin + (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  int mr = 0;
  if (i < end) {
    const float f[3] = {fx[i], fy[i], fz[i]};
    double v[3] = {vx[i], vy[i], vz[i]};
    const double sgn = p.top ? 1.0 : -1.0;
    const float dth = __fdiv_rn(__fmul_rn(0.5f, p.t0), (float)(1 << p.rung));
    if (p.ascending && !p.first) {
#pragma unroll
      for (int d = 0; d < 3; d++) v[d] = __dadd_rn(v[d], __dmul_rn(__dmul_rn(sgn, (double)f[d]), (double)dth));
    }
    if (p.descending) {
      float g2 = __fmul_rn(f[0], f[0]);
      g2 = __fadd_rn(g2, __fmul_rn(f[1], f[1]));
      g2 = __fadd_rn(g2, __fmul_rn(f[2], f[2]));
      float dt = fminf(__fmul_rn(p.eta, __fsqrt_rn(__fdiv_rn(__fmul_rn(p.scale, hsoft),
                                                              __fsqrt_rn(g2)))),
                       p.t0);
      dt = fminf(p.max_dt, dt);
      int r = rung[i];
      int up = (ceil_log2_exact(__fdiv_rn(p.t0, dt)) > p.rung) ? 1 : 0;
      int nr = max(p.rung + up, r - 1);
      rung[i] = (int8_t)nr;
      mr = nr;
#pragma unroll
      for (int d = 0; d < 3; d++) v[d] = __dadd_rn(v[d], __dmul_rn(__dmul_rn(sgn, (double)f[d]), (double)dth));
    }
    vx[i] = (float)v[0];
    vy[i] = (float)v[1];
    vz[i] = (float)v[2];
  }
  // block max -> global
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mr = max(mr, __shfl_xor_sync(0xffffffffu, mr, o));
  if ((threadIdx.x & 31) == 0 && mr > 0) atomicMax(maxrung, mr);
}

__global__ void drift_kernel(size_t n, uint32_t *__restrict__ x, uint32_t *__restrict__ y,
                             uint32_t *__restrict__ z, const float *__restrict__ vx,
                             const float *__restrict__ vy, const float *__restrict__ vz,
                             float lambda) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float two32 = 4294967296.0f;
  x[i] += (uint32_t)__float2ll_rz(__fmul_rn(__fmul_rn(vx[i], lambda), two32));
  y[i] += (uint32_t)__float2ll_rz(__fmul_rn(__fmul_rn(vy[i], lambda), two32));
  z[i] += (uint32_t)__float2ll_rz(__fmul_rn(__fmul_rn(vz[i], lambda), two32));
}

}  // namespace

int ct2g_update(ct2g_ctx *ctx, const ct2g_kick_params *p, int *max_rung, bool fuse_drift,
                float drift_dt, float drift_scale) {
  const size_t b = ctx->rung_begin, e = ctx->n;
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->d_maxrung, 0, sizeof(int), ctx->stream));
  if (e > b) {
    update_kernel<<<ct2g_div_up(e - b, 256), 256, 0, ctx->stream>>>(
        b, e, ctx->fx, ctx->fy, ctx->fz, ctx->vx, ctx->vy, ctx->vz, ctx->rung, *p,
        ctx->opt.hsoft, ctx->d_maxrung);
    CT2G_LAUNCHED(ctx);
  }
  if (fuse_drift) CT2G_TRY(ct2g_drift_all(ctx, drift_dt, drift_scale));
  if (max_rung) {
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, ctx->d_maxrung, sizeof(int),
                                   cudaMemcpyDeviceToHost, ctx->stream));
    CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    *max_rung = (int)ctx->h_pinned[0];
  }
  return CT2G_OK;
}

int ct2g_drift_all(ct2g_ctx *ctx, float dt, float scale) {
  if (ctx->n == 0) return CT2G_OK;
  const float lambda = dt / scale;
  drift_kernel<<<ct2g_div_up(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->n, ctx->x, ctx->y, ctx->z,
                                                                   ctx->vx, ctx->vy, ctx->vz,
                                                                   lambda);
  CT2G_LAUNCHED(ctx);
  // positions changed: the cell structure is stale
  ctx->grid_valid = false;
  ctx->moments_valid = false;
  ctx->expansions_valid = false;
  ctx->forces_valid = false;
  return CT2G_OK;
}
