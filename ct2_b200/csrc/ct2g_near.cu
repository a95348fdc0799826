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

// ---------------------------------------------------------------------------
// Near-field neighbour walk.  The stencil (offsets |o|^2 <= bwidth^2, bwidth
// <= 4) of a cell touches the 27 4x4x4 cell blocks around its own; a block
// is 64 consecutive Morton keys, so its occupancy is one 64-bit word.  For
// the cell at in-block position p and block offset o, stmask[p*27+o] holds
// the stencil cells of that block; occ & stmask lists exactly the occupied
// stencil cells.  Neighbour block keys come from dilated (bit-interleaved)
// addition, which wraps periodically by itself.
// ---------------------------------------------------------------------------
__constant__ uint32_t c_doff[27 * 3];  // dilated block offsets, x/y/z lanes of the key

struct Walk {
  uint32_t mx, my, mz;  // block-key masks of the x, y, z bits
  __device__ __forceinline__ uint32_t add(uint32_t sb, int o) const {
    const uint32_t x = ((sb | ~mx) + c_doff[3 * o]) & mx;
    const uint32_t y = ((sb | ~my) + c_doff[3 * o + 1]) & my;
    const uint32_t z = ((sb | ~mz) + c_doff[3 * o + 2]) & mz;
    return x | y | z;
  }
};

// minimum-image offset (in cells) from cell c to cell n along one axis
__device__ __forceinline__ int wrap_off(int n, int c, int M) { return ((n - c + M / 2) & (M - 1)) - M / 2; }

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

// Dense cells: one warp per chunk of <= 32 sinks of one cell; every occupied
// stencil cell is a warp-uniform range whose sources are staged 32 at a time
// in shared memory and read back as broadcasts.
template <int P, int KERNEL, bool POT>
__global__ void __launch_bounds__(256) forces_kernel(
    const uint32_t *__restrict__ chunk_begin, uint32_t nchunks, const uint32_t *__restrict__ cs,
    const unsigned long long *__restrict__ occ, const unsigned long long *__restrict__ stmask,
    Walk walk, const uint32_t *__restrict__ skeys, uint32_t rbegin,
    const float4 *__restrict__ src, const float *__restrict__ grid, int mbits, float soft,
    float GM, float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, unsigned long long *__restrict__ inter) {
  __shared__ float4 sbuf[8][32];    // one batch of 32 sources per warp
  __shared__ uint32_t cells[8][736];  // occupied stencil cells per warp (<= 729)
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
  const float hc = 1.0f / (float)M;
  const float h2 = soft * soft, hinv = 1.f / soft, hinv3 = hinv * hinv * hinv;
  float nx = 0.f, ny = 0.f, nz = 0.f, np = 0.f;
  uint32_t nsrc = 0;
  float4 *sb = sbuf[wib];
  // the 27 neighbour-block words, one per lane; their set bits are compacted
  // into a list of occupied stencil cells (exclusive popc prefix over lanes)
  uint32_t *list = cells[wib];
  const uint32_t p = key & 63u, blk = key >> 6;
  unsigned long long word = 0;
  uint32_t nblk = 0;
  if (lane < 27) {
    nblk = walk.add(blk, lane);
    word = occ[nblk] & __ldg(stmask + p * 27 + lane);
  }
  const int cnt_mine = __popcll(word);
  int incl = cnt_mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const int ncell = __shfl_sync(0xffffffffu, incl, 31);
  {
    int at = incl - cnt_mine;
    unsigned long long w = word;
    while (w) {
      const int bb = __ffsll((long long)w) - 1;
      w &= w - 1;
      list[at++] = (nblk << 6) | (uint32_t)bb;
    }
  }
  __syncwarp();
  for (int s0 = 0; s0 < ncell; s0 += 32) {
    // 32 occupied neighbours at a time: ranges and offsets fetched per lane
    uint32_t jb = 0, je = 0;
    int ox = 0, oy = 0, oz = 0;
    if (s0 + lane < ncell) {
      const uint32_t ck = list[s0 + lane];
      jb = cs[ck];
      je = cs[ck + 1];
      ox = wrap_off((int)ct2g_compact3(ck >> 2), cx, M);
      oy = wrap_off((int)ct2g_compact3(ck >> 1), cy, M);
      oz = wrap_off((int)ct2g_compact3(ck), cz, M);
    }
    const int nt = min(32, ncell - s0);
    for (int t = 0; t < nt; t++) {
      const uint32_t j0 = __shfl_sync(0xffffffffu, jb, t), j1 = __shfl_sync(0xffffffffu, je, t);
      nsrc += j1 - j0;
      // sink position relative to the neighbour cell's centre
      const float xs = si.x - (float)__shfl_sync(0xffffffffu, ox, t) * hc;
      const float ys = si.y - (float)__shfl_sync(0xffffffffu, oy, t) * hc;
      const float zs = si.z - (float)__shfl_sync(0xffffffffu, oz, t) * hc;
      for (uint32_t jj = j0; jj < j1; jj += 32) {
        const int cnt = (int)min(32u, j1 - jj);
        __syncwarp();
        if (lane < cnt) sb[lane] = __ldg(src + jj + lane);
        __syncwarp();
#pragma unroll 8
        for (int u = 0; u < cnt; u++) {
          const float4 q = sb[u];
          pair_term<KERNEL, POT>(xs - q.x, ys - q.y, zs - q.z, h2, hinv, hinv3, nx, ny, nz, np,
                                 true);
        }
      }
    }
  }
  // the far field (L2P, with GM) is already in the force buffers
  if (act) {
    ofx[i] += GM * nx;
    ofy[i] += GM * ny;
    ofz[i] += GM * nz;
    if (POT) opot[i] += GM * np;
  }
  if (lane == 0 && inter) atomicAdd(inter, (unsigned long long)(cend - b) * nsrc);
}

// Sparse cells (fewer than 16 particles): one thread per sink, each walking
// its own occupied stencil cells.  A neighbour with fewer than kLight
// sources is consumed by the lane alone; heavier ones (a cluster core beside
// a halo sink) are queued in shared memory and consumed afterwards by the
// whole warp -- lanes take 32 sources at a time against the owning lane's
// sink, and a warp reduction hands the sum back -- so no lane idles through
// a long private loop.
constexpr uint32_t kLight = 24;
constexpr int kQueue = 16;

template <int P, int KERNEL, bool POT>
__global__ void __launch_bounds__(128) forces_sparse_kernel(
    const uint32_t *__restrict__ sinks, uint32_t nsinks, const uint32_t *__restrict__ cs,
    const unsigned long long *__restrict__ occ, const unsigned long long *__restrict__ stmask,
    Walk walk, const uint32_t *__restrict__ skeys, uint32_t rbegin,
    const float4 *__restrict__ src, const float *__restrict__ grid, int mbits, float soft,
    float GM, float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, unsigned long long *__restrict__ inter) {
  __shared__ uint32_t queue[kQueue][128];  // queued heavy cells: key
  __shared__ uint2 qrange[kQueue][128];    // and source range
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  if ((t & ~31u) >= nsinks) return;  // whole warps only: the queue phase shuffles
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
  int nq = 0;
  const uint32_t p = key & 63u, blk = key >> 6;
  if (act) {
    for (int o = 0; o < 27; o++) {
      const uint32_t nb = walk.add(blk, o);
      unsigned long long bits = occ[nb] & __ldg(stmask + p * 27 + o);
      while (bits) {
        const int bb = __ffsll((long long)bits) - 1;
        bits &= bits - 1;
        const uint32_t ck = (nb << 6) | (uint32_t)bb;
        const uint32_t j0 = cs[ck], j1 = cs[ck + 1];
        nsrc += j1 - j0;
        if (j1 - j0 >= kLight && nq < kQueue) {
          queue[nq][threadIdx.x] = ck;
          qrange[nq++][threadIdx.x] = make_uint2(j0, j1);
          continue;
        }
        const float xs = si.x - (float)wrap_off((int)ct2g_compact3(ck >> 2), cx, M) * hc;
        const float ys = si.y - (float)wrap_off((int)ct2g_compact3(ck >> 1), cy, M) * hc;
        const float zs = si.z - (float)wrap_off((int)ct2g_compact3(ck), cz, M) * hc;
        for (uint32_t j = j0; j < j1; j++) {
          const float4 q = __ldg(src + j);
          pair_term<KERNEL, POT>(xs - q.x, ys - q.y, zs - q.z, h2, hinv, hinv3, nx, ny, nz, np,
                                 true);
        }
      }
    }
  }
  // queued heavy cells, one per lane per round, each consumed by the warp
  for (;;) {
    const unsigned pending = __ballot_sync(0xffffffffu, nq > 0);
    if (!pending) break;
    uint32_t mine = 0;
    uint2 mr = make_uint2(0u, 0u);
    float mx = 0.f, my = 0.f, mz = 0.f;
    if (nq > 0) {
      --nq;
      mine = queue[nq][threadIdx.x];
      mr = qrange[nq][threadIdx.x];
      mx = si.x - (float)wrap_off((int)ct2g_compact3(mine >> 2), cx, M) * hc;
      my = si.y - (float)wrap_off((int)ct2g_compact3(mine >> 1), cy, M) * hc;
      mz = si.z - (float)wrap_off((int)ct2g_compact3(mine), cz, M) * hc;
    }
    unsigned todo = pending;
    while (todo) {
      const int L = __ffs(todo) - 1;
      todo &= todo - 1;
      const float bx = __shfl_sync(0xffffffffu, mx, L), by = __shfl_sync(0xffffffffu, my, L),
                  bz = __shfl_sync(0xffffffffu, mz, L);
      const uint32_t b0 = __shfl_sync(0xffffffffu, mr.x, L), b1 = __shfl_sync(0xffffffffu, mr.y, L);
      float ax = 0.f, ay = 0.f, az = 0.f, ap = 0.f;
      for (uint32_t jj = b0; jj < b1; jj += 32) {
        const bool on = jj + lane < b1;
        const float4 q = __ldg(src + (on ? jj + lane : b0));
        pair_term<KERNEL, POT>(bx - q.x, by - q.y, bz - q.z, h2, hinv, hinv3, ax, ay, az, ap, on);
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
  if (act) {  // the far field (L2P, with GM) is already in the force buffers
    ofx[i] += GM * nx;
    ofy[i] += GM * ny;
    ofz[i] += GM * nz;
    if (POT) opot[i] += GM * np;
  }
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

Walk make_walk(int mbits) {
  Walk w{0u, 0u, 0u};
  for (int i = 0; i < mbits - 2; i++) {
    w.mx |= 1u << (3 * i + 2);
    w.my |= 1u << (3 * i + 1);
    w.mz |= 1u << (3 * i);
  }
  return w;
}

template <int P, int K, bool POT>
int launch_forces_t(ct2g_ctx *ctx) {
  const Walk walk = make_walk(ctx->mbits);
  if (ctx->nchunks) {
    const unsigned T = 256;
    const size_t threads = (size_t)ctx->nchunks * 32;
    forces_kernel<P, K, POT><<<ct2g_div_up(threads, T), T, 0, ctx->stream>>>(
        ctx->chunk_begin, ctx->nchunks, ctx->cell_start, ctx->occ, ctx->stmask, walk, ctx->keys,
        (uint32_t)ctx->rung_begin, ctx->src, ctx->grid, ctx->mbits, ctx->opt.hsoft, ctx->opt.GM,
        ctx->fx, ctx->fy, ctx->fz, ctx->pot, ctx->d_inter);
    CT2G_LAUNCHED(ctx);
  }
  if (ctx->nsparse) {
    const unsigned T = 128;
    forces_sparse_kernel<P, K, POT><<<ct2g_div_up(ctx->nsparse, T), T, 0, ctx->stream>>>(
        ctx->sparse_list, ctx->nsparse, ctx->cell_start, ctx->occ, ctx->stmask, walk, ctx->keys,
        (uint32_t)ctx->rung_begin, ctx->src, ctx->grid, ctx->mbits, ctx->opt.hsoft, ctx->opt.GM,
        ctx->fx, ctx->fy, ctx->fz, ctx->pot, ctx->d_inter);
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
  // dilated block offsets for the 27 neighbouring 4x4x4 blocks
  const int nb = ctx->mbits - 2;
  uint32_t d[27 * 3];
  for (int o = 0; o < 27; o++) {
    const int dd[3] = {o / 9 - 1, (o / 3) % 3 - 1, o % 3 - 1};
    for (int a = 0; a < 3; a++) {
      const uint32_t v = (uint32_t)dd[a] & ((1u << nb) - 1u);
      d[3 * o + a] = ct2g_spread3(v) << (2 - a);
    }
  }
  CT2G_CUDA(ctx, cudaMemcpyToSymbolAsync(c_doff, d, sizeof(d), 0, cudaMemcpyHostToDevice,
                                         ctx->stream));
  return CT2G_OK;
}

int ct2g_forces(ct2g_ctx *ctx, bool pot) {
  const size_t n = ctx->n;
  // the far-field pass (ct2g_fft_c2r_l2p) has written the range's entries
  (void)n;
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
