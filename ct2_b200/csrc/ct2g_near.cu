// Forces, kick update and drift.
//
//   forces  L2P far field + direct-sum near field per sink chunk
//           (kick_cell, src/kick.cpp:3-74): one warp per chunk of <= 32
//           sinks of one cell; every source of each stencil cell is a
//           warp-uniform (broadcast) load of a float4 offset from its cell
//           centre, so the inner loop is 3 FADD + 3 FFMA + RSQRT + 2 FMUL +
//           3 FFMA per interaction in FP32.
//   update  velocity + rung update (src/kick.cpp:75-99), FP64 arithmetic,
//           stored FP32; ceil(log2(t0/dt)) taken exactly from the exponent bits
//   drift   x += fixed32(v * dt/scale) (src/drift.cpp:4-18)
//
// Defects of the reference fixed here: the source loop advanced by one but
// loaded eight sources (kick.cpp:38-43), the near-field force was reduced
// from the far-field accumulator (kick.cpp:72), and the update indexed the
// SIMD lane with the absolute particle index (kick.cpp:82-98).
#include "ct2g_internal.cuh"

namespace {

__constant__ int c_stencil[4 * 729];  // (ox, oy, oz, unused) per offset

template <int P>
__device__ __forceinline__ void l2p(const float *__restrict__ grid, int64_t C, int64_t cell,
                                    float tx, float ty, float tz, float &fx, float &fy,
                                    float &fz, float &pot) {
  constexpr MiTable<P> T{};
  constexpr int NC = MiTable<P>::NC;
  float L[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) L[k] = __ldg(grid + (int64_t)k * C + cell);
  float px[P + 1], py[P + 1], pz[P + 1];
  px[0] = py[0] = pz[0] = 1.f;
#pragma unroll
  for (int q = 1; q <= P; q++) {
    px[q] = px[q - 1] * tx * (1.f / q);
    py[q] = py[q - 1] * ty * (1.f / q);
    pz[q] = pz[q - 1] * tz * (1.f / q);
  }
  float ax = 0.f, ay = 0.f, az = 0.f, ph = 0.f;
#pragma unroll
  for (int k = 0; k < NC; k++) {
    const float mono = px[T.nx[k]] * py[T.ny[k]] * pz[T.nz[k]];
    ph = fmaf(-L[k], mono, ph);
    if (T.deg[k] < P) {
      ax = fmaf(L[ct2g_mi_index(T.nx[k] + 1, T.ny[k], T.nz[k])], mono, ax);
      ay = fmaf(L[ct2g_mi_index(T.nx[k], T.ny[k] + 1, T.nz[k])], mono, ay);
      az = fmaf(L[ct2g_mi_index(T.nx[k], T.ny[k], T.nz[k] + 1)], mono, az);
    }
  }
  fx = ax;
  fy = ay;
  fz = az;
  pot = ph;
}

template <int P, int KERNEL, bool POT>
__global__ void __launch_bounds__(256) forces_kernel(
    const uint32_t *__restrict__ chunk_begin, uint32_t nchunks, const uint32_t *__restrict__ cs,
    const uint32_t *__restrict__ skeys, uint32_t rbegin, const float4 *__restrict__ src,
    const float *__restrict__ grid, int mbits, int nstencil, float soft, float GM,
    float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, unsigned long long *__restrict__ inter) {
  __shared__ float4 sbuf[8][32];  // one batch of 32 sources per warp
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t ch = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (ch >= nchunks) return;
  const int M = 1 << mbits;
  const int64_t C = (int64_t)M * M * M;
  const uint32_t b = chunk_begin[ch];
  const uint32_t key = skeys[b - rbegin];  // Morton key of the sink cell
  const uint32_t cend = min(cs[key + 1], b + 32u);
  const uint32_t i = b + lane;
  const bool act = i < cend;
  const float4 si = src[act ? i : b];
  const int cx = (int)ct2g_compact3(key >> 2), cy = (int)ct2g_compact3(key >> 1),
            cz = (int)ct2g_compact3(key);
  const int64_t cell = ((int64_t)cx * M + cy) * M + cz;  // row-major grid index
  float fx = 0.f, fy = 0.f, fz = 0.f, ph = 0.f;
  l2p<P>(grid, C, cell, si.x, si.y, si.z, fx, fy, fz, ph);
  const float hc = 1.0f / (float)M;
  const float h2 = soft * soft, hinv = 1.f / soft, hinv3 = hinv * hinv * hinv;
  float nx = 0.f, ny = 0.f, nz = 0.f, np = 0.f;
  uint32_t nsrc = 0;
  float4 *sb = sbuf[wib];
  for (int s0 = 0; s0 < nstencil; s0 += 32) {
    // 32 neighbour ranges fetched at once, one per lane
    uint32_t jb = 0, je = 0;
    const int sl = s0 + lane;
    if (sl < nstencil) {
      const uint32_t nb = ct2g_morton((uint32_t)((cx + c_stencil[4 * sl]) & (M - 1)),
                                      (uint32_t)((cy + c_stencil[4 * sl + 1]) & (M - 1)),
                                      (uint32_t)((cz + c_stencil[4 * sl + 2]) & (M - 1)));
      jb = cs[nb];
      je = cs[nb + 1];
    }
    const int nt = min(32, nstencil - s0);
    for (int t = 0; t < nt; t++) {
      const uint32_t j0 = __shfl_sync(0xffffffffu, jb, t), j1 = __shfl_sync(0xffffffffu, je, t);
      if (j0 == j1) continue;
      nsrc += j1 - j0;
      const int st = s0 + t;
      // sink position relative to the neighbour cell's centre
      const float xs = si.x - (float)c_stencil[4 * st] * hc;
      const float ys = si.y - (float)c_stencil[4 * st + 1] * hc;
      const float zs = si.z - (float)c_stencil[4 * st + 2] * hc;
      for (uint32_t jj = j0; jj < j1; jj += 32) {
        const int cnt = (int)min(32u, j1 - jj);
        __syncwarp();
        if (lane < cnt) sb[lane] = __ldg(src + jj + lane);
        __syncwarp();
#pragma unroll 8
        for (int u = 0; u < cnt; u++) {
          const float4 q = sb[u];
          const float dx = xs - q.x, dy = ys - q.y, dz = zs - q.z;
          const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          float g;
          if (KERNEL == CT2G_SOFT_PLUMMER) {
            const float ri = rsqrtf(r2 + h2);
            g = ri * ri * ri;
            if (POT) np -= ri;
          } else {
            if (r2 < h2) {
              g = hinv3;
              if (POT) np -= 1.5f * hinv - 0.5f * r2 * hinv3;
            } else {
              const float ri = rsqrtf(r2);
              g = ri * ri * ri;
              if (POT) np -= ri;
            }
          }
          nx = fmaf(-dx, g, nx);
          ny = fmaf(-dy, g, ny);
          nz = fmaf(-dz, g, nz);
        }
      }
    }
  }
  if (act) {
    ofx[i] = GM * (fx + nx);
    ofy[i] = GM * (fy + ny);
    ofz[i] = GM * (fz + nz);
    if (POT) opot[i] = GM * (ph + np);
  }
  if (lane == 0 && inter) atomicAdd(inter, (unsigned long long)(cend - b) * nsrc);
}

// Thread-per-sink near field for sinks of sparse cells (fewer than 16
// particles).  Every lane walks its own stencil (neighbouring lanes are
// neighbouring sinks, so source loads mostly hit L1).  A neighbour cell with
// fewer than kLight sources is consumed by the lane alone; a heavier one (a
// cluster core next to a halo sink) is consumed by the whole warp: lanes take
// 32 sources at a time against the owning lane's sink, and a warp reduction
// hands the sum to the owner, so no lane idles through a long private loop.
constexpr uint32_t kLight = 24;

template <int KERNEL, bool POT>
__device__ __forceinline__ void pair_term(float dx, float dy, float dz, float h2, float hinv,
                                          float hinv3, float &ax, float &ay, float &az,
                                          float &ap, bool on) {
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  float g, pp;
  if (KERNEL == CT2G_SOFT_PLUMMER) {
    const float ri = rsqrtf(r2 + h2);
    g = ri * ri * ri;
    pp = ri;
  } else {
    if (r2 < h2) {
      g = hinv3;
      pp = 1.5f * hinv - 0.5f * r2 * hinv3;
    } else {
      const float ri = rsqrtf(r2);
      g = ri * ri * ri;
      pp = ri;
    }
  }
  if (!on) g = pp = 0.f;
  ax = fmaf(-dx, g, ax);
  ay = fmaf(-dy, g, ay);
  az = fmaf(-dz, g, az);
  if (POT) ap -= pp;
}

template <int P, int KERNEL, bool POT>
__global__ void __launch_bounds__(128) forces_sparse_kernel(
    const uint32_t *__restrict__ sinks, uint32_t nsinks, const uint32_t *__restrict__ cs,
    const uint32_t *__restrict__ skeys, uint32_t rbegin, const float4 *__restrict__ src,
    const float *__restrict__ grid, int mbits, int nstencil, float soft, float GM,
    float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, unsigned long long *__restrict__ inter) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  if ((t & ~31u) >= nsinks) return;  // whole warps only: the loop below shuffles
  const bool act = t < nsinks;
  const int M = 1 << mbits;
  const int64_t C = (int64_t)M * M * M;
  const uint32_t i = sinks[act ? t : nsinks - 1];
  const uint32_t key = skeys[i - rbegin];
  const float4 si = src[i];
  const int cx = (int)ct2g_compact3(key >> 2), cy = (int)ct2g_compact3(key >> 1),
            cz = (int)ct2g_compact3(key);
  const float hc = 1.0f / (float)M;
  const float h2 = soft * soft, hinv = 1.f / soft, hinv3 = hinv * hinv * hinv;
  float nx = 0.f, ny = 0.f, nz = 0.f, np = 0.f;
  uint32_t nsrc = 0;
  for (int s0 = 0; s0 < nstencil; s0 += 4) {
    uint32_t jb[4], je[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int s = min(s0 + u, nstencil - 1);
      const uint32_t nb = ct2g_morton((uint32_t)((cx + c_stencil[4 * s]) & (M - 1)),
                                      (uint32_t)((cy + c_stencil[4 * s + 1]) & (M - 1)),
                                      (uint32_t)((cz + c_stencil[4 * s + 2]) & (M - 1)));
      jb[u] = cs[nb];
      je[u] = (act && s0 + u < nstencil) ? cs[nb + 1] : jb[u];
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const int s = min(s0 + u, nstencil - 1);
      const uint32_t k = je[u] - jb[u];
      nsrc += k;
      const float xs = si.x - (float)c_stencil[4 * s] * hc;
      const float ys = si.y - (float)c_stencil[4 * s + 1] * hc;
      const float zs = si.z - (float)c_stencil[4 * s + 2] * hc;
      if (k < kLight) {
        for (uint32_t j = jb[u]; j < je[u]; j++) {
          const float4 q = __ldg(src + j);
          pair_term<KERNEL, POT>(xs - q.x, ys - q.y, zs - q.z, h2, hinv, hinv3, nx, ny, nz, np,
                                 true);
        }
      }
      unsigned heavy = __ballot_sync(0xffffffffu, k >= kLight);
      while (heavy) {
        const int L = __ffs(heavy) - 1;
        heavy &= heavy - 1;
        const float bx = __shfl_sync(0xffffffffu, xs, L), by = __shfl_sync(0xffffffffu, ys, L),
                    bz = __shfl_sync(0xffffffffu, zs, L);
        const uint32_t b0 = __shfl_sync(0xffffffffu, jb[u], L),
                       b1 = __shfl_sync(0xffffffffu, je[u], L);
        float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
        for (uint32_t jj = b0; jj < b1; jj += 32) {
          const bool on = jj + lane < b1;
          const float4 q = __ldg(src + (on ? jj + lane : b0));
          pair_term<KERNEL, POT>(bx - q.x, by - q.y, bz - q.z, h2, hinv, hinv3, ax, ay, az, ap,
                                 on);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          ax += __shfl_xor_sync(0xffffffffu, ax, o);
          ay += __shfl_xor_sync(0xffffffffu, ay, o);
          az += __shfl_xor_sync(0xffffffffu, az, o);
          if (POT) ap += __shfl_xor_sync(0xffffffffu, ap, o);
        }
        if (lane == L) {
          nx += ax;
          ny += ay;
          nz += az;
          np += ap;
        }
      }
    }
  }
  if (act) {
    float fx = 0.f, fy = 0.f, fz = 0.f, ph = 0.f;
    l2p<P>(grid, C, ((int64_t)cx * M + cy) * M + cz, si.x, si.y, si.z, fx, fy, fz, ph);
    ofx[i] = GM * (fx + nx);
    ofy[i] = GM * (fy + ny);
    ofz[i] = GM * (fz + nz);
    if (POT) opot[i] = GM * (ph + np);
  }
  // warp-summed interaction count
  unsigned long long c = act ? nsrc : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0 && c && inter) atomicAdd(inter, c);
}

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

template <int P, int K, bool POT>
int launch_forces_t(ct2g_ctx *ctx) {
  if (ctx->nchunks) {
    const unsigned T = 256;
    const size_t threads = (size_t)ctx->nchunks * 32;
    forces_kernel<P, K, POT><<<ct2g_div_up(threads, T), T, 0, ctx->stream>>>(
        ctx->chunk_begin, ctx->nchunks, ctx->cell_start, ctx->keys, (uint32_t)ctx->rung_begin,
        ctx->src, ctx->grid, ctx->mbits, ctx->nstencil, ctx->opt.hsoft, ctx->opt.GM, ctx->fx,
        ctx->fy, ctx->fz, ctx->pot, ctx->d_inter);
    CT2G_LAUNCHED(ctx);
  }
  if (ctx->nsparse) {
    const unsigned T = 128;
    forces_sparse_kernel<P, K, POT><<<ct2g_div_up(ctx->nsparse, T), T, 0, ctx->stream>>>(
        ctx->sparse_list, ctx->nsparse, ctx->cell_start, ctx->keys, (uint32_t)ctx->rung_begin,
        ctx->src, ctx->grid, ctx->mbits, ctx->nstencil, ctx->opt.hsoft, ctx->opt.GM, ctx->fx,
        ctx->fy, ctx->fz, ctx->pot, ctx->d_inter);
    CT2G_LAUNCHED(ctx);
  }
  return CT2G_OK;
}

template <int P>
int launch_forces_p(ct2g_ctx *ctx, bool pot) {
  if (ctx->opt.kernel == CT2G_SOFT_SPHERE)
    return pot ? launch_forces_t<P, CT2G_SOFT_SPHERE, true>(ctx)
               : launch_forces_t<P, CT2G_SOFT_SPHERE, false>(ctx);
  return pot ? launch_forces_t<P, CT2G_SOFT_PLUMMER, true>(ctx)
             : launch_forces_t<P, CT2G_SOFT_PLUMMER, false>(ctx);
}

}  // namespace

int ct2g_upload_stencil(ct2g_ctx *ctx, const std::vector<int> &st4) {
  CT2G_CUDA(ctx, cudaMemcpyToSymbolAsync(c_stencil, st4.data(), sizeof(int) * st4.size(), 0,
                                         cudaMemcpyHostToDevice, ctx->stream));
  return CT2G_OK;
}

int ct2g_forces(ct2g_ctx *ctx, bool pot) {
  const size_t n = ctx->n;
  // entries outside the range read as zero
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->fx, 0, n * 4, ctx->stream));
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->fy, 0, n * 4, ctx->stream));
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->fz, 0, n * 4, ctx->stream));
  if (pot) CT2G_CUDA(ctx, cudaMemsetAsync(ctx->pot, 0, n * 4, ctx->stream));
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->d_inter, 0, sizeof(unsigned long long), ctx->stream));
  if (ctx->nchunks == 0 && ctx->nsparse == 0) return CT2G_OK;
  switch (ctx->p) {
    case 1: return launch_forces_p<1>(ctx, pot);
    case 2: return launch_forces_p<2>(ctx, pot);
    case 3: return launch_forces_p<3>(ctx, pot);
    case 4: return launch_forces_p<4>(ctx, pot);
    case 5: return launch_forces_p<5>(ctx, pot);
    case 6: return launch_forces_p<6>(ctx, pot);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "unsupported order");
}

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
