// Particle binning (particle_to_grid, src/particle.cpp:69-114,349-362):
// Morton cell keys from the top mesh bits of the fixed-point positions, a
// stable LSD radix sort of (key, index) pairs, cell ranges, the gather of the
// SoA into cell order, per-particle float offsets from the cell centre for
// the direct sum, and the sink-chunk list.
//
// The reference partitions recursively (a Hoare partition per level,
// dimension depth%3); for a power-of-two mesh every particle lands in the
// same leaf as here, because the split point fixed32((I+N/2)/Ncell) equals
// (I+N/2) << (32-mbits), and the leaves come out in the same (Morton) order.
// Only the order inside a cell differs: the reference's partition leaves it
// arbitrary, here it is the stable (previous) order, so the sort is
// deterministic.
#include "ct2g_internal.cuh"

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;  // per thread
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// block-wide exclusive scan of one value per thread; returns block total
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *smem32,
                                                    uint32_t &total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t inc = warp_incl_scan(v);
  if (lane == 31) smem32[w] = inc;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < nw ? smem32[lane] : 0;
    uint32_t si = warp_incl_scan(s);
    if (lane < nw) smem32[lane] = si - s;
    if (lane == nw - 1) smem32[32] = si;
  }
  __syncthreads();
  uint32_t res = inc - v + smem32[w];
  total = smem32[32];
  __syncthreads();
  return res;
}

__global__ void scan_reduce_kernel(const uint32_t *__restrict__ in, size_t n,
                                   uint32_t *__restrict__ bsum) {
  __shared__ uint32_t sm[33];
  size_t base = (size_t)blockIdx.x * kScanTile;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
    if (i < n) s += in[i];
  }
  uint32_t tot;
  block_excl_scan(s, sm, tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

// single block: exclusive scan of bsum[nb] in place (nb arbitrary)
__global__ void scan_single_kernel(uint32_t *__restrict__ a, size_t nb, uint32_t *total) {
  __shared__ uint32_t sm[33];
  uint32_t carry = 0;
  for (size_t base = 0; base < nb; base += blockDim.x) {
    size_t i = base + threadIdx.x;
    uint32_t v = i < nb ? a[i] : 0;
    uint32_t tot;
    uint32_t ex = block_excl_scan(v, sm, tot);
    if (i < nb) a[i] = ex + carry;
    carry += tot;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void scan_apply_kernel(const uint32_t *__restrict__ in, size_t n,
                                  const uint32_t *__restrict__ boff, uint32_t offset,
                                  uint32_t *__restrict__ out) {
  __shared__ uint32_t sm[33];
  size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  uint32_t tot;
  uint32_t ex = block_excl_scan(s, sm, tot) + boff[blockIdx.x] + offset;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
}

// ---------------------------------------------------------------------------
// radix sort, 8-bit digits, tiles of 256 threads x 16 items (striped per warp)
// ---------------------------------------------------------------------------
constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;
constexpr int kRadixWarps = kRadixThreads / 32;

__device__ __forceinline__ size_t radix_item(int slot) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  return (size_t)blockIdx.x * kRadixTile + (size_t)w * 32 * kRadixItems + slot * 32 + lane;
}

__global__ void radix_hist_kernel(const uint32_t *__restrict__ keys, size_t n, int shift,
                                  uint32_t ntiles, uint32_t *__restrict__ hist) {
  __shared__ uint32_t cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kRadixItems; k++) {
    size_t i = radix_item(k);
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void radix_scatter_kernel(const uint32_t *__restrict__ keys,
                                     const uint32_t *__restrict__ vals, size_t n, int shift,
                                     uint32_t ntiles, const uint32_t *__restrict__ hscan,
                                     uint32_t *__restrict__ okeys, uint32_t *__restrict__ ovals) {
  __shared__ uint32_t wcnt[kRadixWarps][256];
  __shared__ uint32_t base[256];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kRadixWarps * 256; i += kRadixThreads) (&wcnt[0][0])[i] = 0;
  base[threadIdx.x] = hscan[(size_t)threadIdx.x * ntiles + blockIdx.x];
  __syncthreads();
  uint32_t k_[kRadixItems], v_[kRadixItems], r_[kRadixItems];
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int k = 0; k < kRadixItems; k++) {
    size_t i = radix_item(k);
    bool valid = i < n;
    uint32_t key = valid ? keys[i] : 0u;
    uint32_t d = (key >> shift) & 255u;
    k_[k] = key;
    v_[k] = valid ? vals[i] : 0u;
    unsigned act = __ballot_sync(0xffffffffu, valid);
    unsigned peers = __match_any_sync(0xffffffffu, valid ? d : 256u + lane) & act;
    uint32_t before = valid ? wcnt[w][d] : 0u;
    __syncwarp();
    if (valid) {
      r_[k] = before + __popc(peers & lt);
      if ((peers & lt) == 0) wcnt[w][d] = before + __popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  {  // exclusive prefix over warps for digit threadIdx.x
    uint32_t run = 0;
    for (int ww = 0; ww < kRadixWarps; ww++) {
      uint32_t t = wcnt[ww][threadIdx.x];
      wcnt[ww][threadIdx.x] = run;
      run += t;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < kRadixItems; k++) {
    size_t i = radix_item(k);
    if (i < n) {
      uint32_t d = (k_[k] >> shift) & 255u;
      uint32_t pos = base[d] + wcnt[w][d] + r_[k];
      okeys[pos] = k_[k];
      ovals[pos] = v_[k];
    }
  }
}

// ---------------------------------------------------------------------------
// key = (box << 3*mbits) | Morton index of the cell; the box of a particle
// is found by bisection of the box offsets (boxes never exchange particles)
__global__ void keys_kernel(const uint32_t *__restrict__ x, const uint32_t *__restrict__ y,
                            const uint32_t *__restrict__ z, size_t begin, size_t nr, int mbits,
                            const uint32_t *__restrict__ box_off, int nbox,
                            uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  const int sh = 32 - mbits;
  size_t g = begin + i;
  uint32_t box = 0;
  if (nbox > 1) {
    uint32_t lo = 0, hi = (uint32_t)nbox;  // box_off[lo] <= g < box_off[hi]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (__ldg(box_off + mid) <= (uint32_t)g) lo = mid; else hi = mid;
    }
    box = lo << (3 * mbits);
  }
  keys[i] = box | ct2g_morton(x[g] >> sh, y[g] >> sh, z[g] >> sh);
  vals[i] = (uint32_t)i;
}

// per-cell particle counts of the sorted range (cell_start = begin + their
// exclusive scan)
// particles per cell (counts, zero on entry) and the occupancy bit of every
// occupied cell (occ, zero on entry), from the sorted keys: the first
// particle of a run of equal keys subtracts its index, the last adds its
// index + 1 (two atomics per occupied cell, none per particle, so a crowded
// cell costs no more than an empty one)
__global__ void cell_count_kernel(const uint32_t *__restrict__ skeys, size_t nr,
                                  uint32_t *__restrict__ counts,
                                  unsigned long long *__restrict__ occ) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  const uint32_t k = skeys[i];
  if (i == 0 || skeys[i - 1] != k) {
    atomicAdd(counts + k, 0u - (uint32_t)i);
    atomicOr(occ + (k >> 6), 1ull << (k & 63u));
  }
  if (i + 1 == nr || skeys[i + 1] != k) atomicAdd(counts + k, (uint32_t)(i + 1));
}

// gather the active range into cell order; write the direct-sum source records
__global__ void gather_kernel(const uint32_t *__restrict__ perm, size_t begin, size_t nr,
                              int mbits, const uint32_t *__restrict__ x,
                              const uint32_t *__restrict__ y, const uint32_t *__restrict__ z,
                              const float *__restrict__ vx, const float *__restrict__ vy,
                              const float *__restrict__ vz, const int8_t *__restrict__ rung,
                              const uint32_t *__restrict__ id, uint32_t *__restrict__ x2,
                              uint32_t *__restrict__ y2, uint32_t *__restrict__ z2,
                              float *__restrict__ vx2, float *__restrict__ vy2,
                              float *__restrict__ vz2, int8_t *__restrict__ rung2,
                              uint32_t *__restrict__ id2, float4 *__restrict__ src,
                              bool vel) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  size_t s = begin + perm[i], d = begin + i;
  uint32_t px = x[s], py = y[s], pz = z[s];
  x2[d] = px;
  y2[d] = py;
  z2[d] = pz;
  if (vel) {
    vx2[d] = vx[s];
    vy2[d] = vy[s];
    vz2[d] = vz[s];
    rung2[d] = rung[s];
  } else {
    // velocities and rungs follow later (gather_vel_kernel): keep the source
    // index in their gather target
    reinterpret_cast<uint32_t *>(vx2)[d] = (uint32_t)s;
  }
  id2[d] = id[s];
  // offset from the cell centre: low (32-mbits) bits minus half a cell,
  // exact in float (|value| < 2^(31-mbits) <= 2^24)
  const int sh = 32 - mbits;
  const uint32_t mask = (sh == 32) ? 0xffffffffu : ((1u << sh) - 1u);
  const int32_t half = (int32_t)(1u << (sh - 1));
  const float sc = (float)CT2G_TWO_M32;
  src[d] = make_float4((float)((int32_t)(px & mask) - half) * sc,
                       (float)((int32_t)(py & mask) - half) * sc,
                       (float)((int32_t)(pz & mask) - half) * sc, 0.f);
}

// Sink work lists for the near field, all in warp chunks of <= 32 sinks:
// cells with at least kDenseCell particles are split into chunks of one cell
// (every 32nd particle of the cell starts one); the particles of sparser
// cells are listed (sparse_list) and chunked per 4x4x4 cell block (a block is
// 64 consecutive Morton keys), every 32nd sparse particle of a block starting
// a chunk.
constexpr uint32_t kSparseChunk = 32;  // sinks per sparse chunk (near_kernel)

__global__ void chunk_flag_kernel(const uint32_t *__restrict__ skeys,
                                  const uint32_t *__restrict__ cs, size_t begin, size_t nr,
                                  uint32_t dense_cell, uint32_t *__restrict__ flags,
                                  uint32_t *__restrict__ sflags) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  const uint32_t k = skeys[i];
  const uint32_t c0 = cs[k], n = cs[k + 1] - c0;
  const bool dense = n >= dense_cell;
  flags[i] = (dense && ((((uint32_t)(begin + i) - c0) & 31u) == 0)) ? 1u : 0u;
  sflags[i] = dense ? 0u : 1u;
}

// sparse chunk starts, indexed by sparse rank r (rank = exclusive scan of sflags)
__global__ void sparse_chunk_flag_kernel(const uint32_t *__restrict__ skeys,
                                         const uint32_t *__restrict__ cs,
                                         const uint32_t *__restrict__ sflags,
                                         const uint32_t *__restrict__ rank, size_t begin, size_t nr,
                                         const uint32_t *__restrict__ nsparse_dev,
                                         uint32_t *__restrict__ scflag) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr || !sflags[i]) return;
  const uint32_t nsparse = *nsparse_dev;
  const uint32_t r = rank[i];
  const uint32_t f = cs[skeys[i] & ~63u] - (uint32_t)begin;  // first particle of the block
  const uint32_t rf = f < nr ? rank[f] : nsparse;
  scflag[r] = ((r - rf) % kSparseChunk) == 0 ? 1u : 0u;
}

// (start, count) of dense chunks: particle index, sinks
__global__ void dense_chunk_fill_kernel(const uint32_t *__restrict__ flags,
                                        const uint32_t *__restrict__ fscan,
                                        const uint32_t *__restrict__ skeys,
                                        const uint32_t *__restrict__ cs, size_t begin, size_t nr,
                                        uint2 *__restrict__ list) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr || !flags[i]) return;
  const uint32_t g = (uint32_t)(begin + i);
  list[fscan[i]] = make_uint2(g, min(32u, cs[skeys[i] + 1] - g));
}

// (start, count) of sparse chunks: index into sparse_list, sinks
__global__ void sparse_chunk_fill_kernel(const uint32_t *__restrict__ scflag,
                                         const uint32_t *__restrict__ scscan,
                                         const uint32_t *__restrict__ sparse_list,
                                         const uint32_t *__restrict__ skeys,
                                         const uint32_t *__restrict__ cs,
                                         const uint32_t *__restrict__ rank, size_t begin, size_t nr,
                                         const uint32_t *__restrict__ counts,
                                         uint2 *__restrict__ list) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nsparse = counts[1];
  if (r >= nsparse || !scflag[r]) return;
  const uint32_t i = sparse_list[r] - (uint32_t)begin;
  const uint32_t e = cs[(skeys[i] | 63u) + 1] - (uint32_t)begin;  // past the block
  const uint32_t re = e < nr ? rank[e] : nsparse;
  list[counts[0] + scscan[r]] = make_uint2(r, min(kSparseChunk, re - r));
}

__global__ void chunk_fill_kernel(const uint32_t *__restrict__ flags,
                                  const uint32_t *__restrict__ fscan, size_t begin, size_t nr,
                                  uint32_t *__restrict__ list) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  if (flags[i]) list[fscan[i]] = (uint32_t)(begin + i);
}


// the gathered (cell-ordered) store goes back into the primary buffers, so
// that every step reads and writes the same addresses (a recorded graph
// replays with fixed pointers)
__global__ void copy_back_kernel(size_t begin, size_t nr, const uint32_t *__restrict__ x2,
                                 const uint32_t *__restrict__ y2, const uint32_t *__restrict__ z2,
                                 const float *__restrict__ vx2, const float *__restrict__ vy2,
                                 const float *__restrict__ vz2, const int8_t *__restrict__ rung2,
                                 const uint32_t *__restrict__ id2, uint32_t *__restrict__ x,
                                 uint32_t *__restrict__ y, uint32_t *__restrict__ z,
                                 float *__restrict__ vx, float *__restrict__ vy,
                                 float *__restrict__ vz, int8_t *__restrict__ rung,
                                 uint32_t *__restrict__ id, bool vel) {
  const size_t i = begin + (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= begin + nr) return;
  x[i] = x2[i];
  y[i] = y2[i];
  z[i] = z2[i];
  if (vel) {
    vx[i] = vx2[i];
    vy[i] = vy2[i];
    vz[i] = vz2[i];
    rung[i] = rung2[i];
  }
  id[i] = id2[i];
}

// the deferred half of the gather: velocities and rungs into cell order,
// from the source indices the position gather left in vx2
__global__ void gather_vel_kernel(size_t begin, size_t nr, const float *__restrict__ vx,
                                  const float *__restrict__ vy, const float *__restrict__ vz,
                                  const int8_t *__restrict__ rung, float *__restrict__ vx2,
                                  float *__restrict__ vy2, float *__restrict__ vz2,
                                  int8_t *__restrict__ rung2) {
  const size_t d = begin + (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (d >= begin + nr) return;
  const uint32_t s = reinterpret_cast<const uint32_t *>(vx2)[d];
  if (s < begin || s >= begin + nr) return;  // the position gather wrote every index in range
  vx2[d] = vx[s];
  vy2[d] = vy[s];
  vz2[d] = vz[s];
  rung2[d] = rung[s];
}

__global__ void copy_back_vel_kernel(size_t begin, size_t nr, const float *__restrict__ vx2,
                                     const float *__restrict__ vy2,
                                     const float *__restrict__ vz2,
                                     const int8_t *__restrict__ rung2, float *__restrict__ vx,
                                     float *__restrict__ vy, float *__restrict__ vz,
                                     int8_t *__restrict__ rung) {
  const size_t i = begin + (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= begin + nr) return;
  vx[i] = vx2[i];
  vy[i] = vy2[i];
  vz[i] = vz2[i];
  rung[i] = rung2[i];
}

__global__ void fill_kernel(uint32_t *__restrict__ a, size_t n, uint32_t v) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

}  // namespace

size_t ct2g_scan_scratch_words(size_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

// exclusive scan of n uint32 values (in may equal out); the sum optionally
// goes to the device word total_dev
int ct2g_scan_exclusive(ct2g_ctx *ctx, const uint32_t *in, uint32_t *out, size_t n,
                        uint32_t *total_dev, uint32_t offset) {
  if (n == 0) {
    if (total_dev) CT2G_CUDA(ctx, cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), ctx->stream));
    return CT2G_OK;
  }
  unsigned nb = ct2g_div_up(n, kScanTile);
  if (ctx->scan_tmp_words < (size_t)nb + 1) {
    if (ctx->capturing) return ct2g_fail(ctx, CT2G_ESTATE, "scan scratch too small while recording");
    ctx->epoch++;
    if (ctx->scan_tmp) cudaFree(ctx->scan_tmp);
    ctx->scan_tmp = nullptr;
    ctx->scan_tmp_words = 0;
    CT2G_CUDA(ctx, cudaMalloc(&ctx->scan_tmp, sizeof(uint32_t) * ((size_t)nb + 1)));
    ctx->scan_tmp_words = (size_t)nb + 1;
  }
  uint32_t *bsum = ctx->scan_tmp;
  scan_reduce_kernel<<<nb, kScanThreads, 0, ctx->stream>>>(in, n, bsum);
  CT2G_LAUNCHED(ctx);
  scan_single_kernel<<<1, 1024, 0, ctx->stream>>>(bsum, nb, total_dev ? total_dev : bsum + nb);
  CT2G_LAUNCHED(ctx);
  scan_apply_kernel<<<nb, kScanThreads, 0, ctx->stream>>>(in, n, bsum, offset, out);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// Sort the current range [rung_begin, n) by cell; build cell ranges, source
// records and sink chunks.  Every size a later kernel needs stays on the
// device (ctx->d_counts), so the sequence can be recorded into a graph.
int ct2g_bin_range(ct2g_ctx *ctx) {
  const size_t begin = ctx->rung_begin, nr = ctx->n - ctx->rung_begin;
  const int mbits = ctx->mbits;
  cudaStream_t st = ctx->stream;
  const unsigned T = 256;
  if (!ctx->boxes_set) return ct2g_fail(ctx, CT2G_ESTATE, "box sizes not set since the upload");
  uint32_t *counts = ctx->d_counts;
  CT2G_CUDA(ctx, cudaMemsetAsync(counts, 0, sizeof(uint32_t) * 6, st));
  if (nr > 0) {
    keys_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(ctx->x, ctx->y, ctx->z, begin, nr, mbits,
                                                    ctx->box_off, ctx->nbox, ctx->keys, ctx->vals);
    CT2G_LAUNCHED(ctx);
    const int bits = 3 * mbits + ctx->boxbits;
    const uint32_t ntiles = ct2g_div_up(nr, kRadixTile);
    uint32_t *ka = ctx->keys, *va = ctx->vals, *kb = ctx->keys2, *vb = ctx->vals2;
    for (int shift = 0; shift < bits; shift += 8) {
      radix_hist_kernel<<<ntiles, kRadixThreads, 0, st>>>(ka, nr, shift, ntiles, ctx->hist);
      CT2G_LAUNCHED(ctx);
      CT2G_TRY(ct2g_scan_exclusive(ctx, ctx->hist, ctx->hist, (size_t)256 * ntiles, nullptr, 0));
      radix_scatter_kernel<<<ntiles, kRadixThreads, 0, st>>>(ka, va, nr, shift, ntiles,
                                                             ctx->hist, kb, vb);
      CT2G_LAUNCHED(ctx);
      uint32_t *t = ka;
      ka = kb;
      kb = t;
      t = va;
      va = vb;
      vb = t;
    }
    // sorted keys/perm now in (ka, va); keep them addressable as keys/vals
    // (the number of passes is fixed per context, so a replay ends in the
    // same buffers)
    if (ka != ctx->keys) {
      uint32_t *t = ctx->keys;
      ctx->keys = ka;
      ctx->keys2 = t;
      t = ctx->vals;
      ctx->vals = va;
      ctx->vals2 = t;
    }
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->cell_start, 0, sizeof(uint32_t) * (ctx->CB + 1), st));
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->occ, 0, sizeof(unsigned long long) * (ctx->CB / 64), st));
    cell_count_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(ctx->keys, nr, ctx->cell_start, ctx->occ);
    CT2G_LAUNCHED(ctx);
    CT2G_TRY(ct2g_scan_exclusive(ctx, ctx->cell_start, ctx->cell_start, (size_t)ctx->CB + 1,
                                 nullptr, (uint32_t)begin));
    gather_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(
        ctx->vals, begin, nr, mbits, ctx->x, ctx->y, ctx->z, ctx->vx, ctx->vy, ctx->vz,
        ctx->rung, ctx->id, ctx->x2, ctx->y2, ctx->z2, ctx->vx2, ctx->vy2, ctx->vz2, ctx->rung2,
        ctx->id2, ctx->src, !ctx->defer_vel);
    CT2G_LAUNCHED(ctx);
    copy_back_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(
        begin, nr, ctx->x2, ctx->y2, ctx->z2, ctx->vx2, ctx->vy2, ctx->vz2, ctx->rung2, ctx->id2,
        ctx->x, ctx->y, ctx->z, ctx->vx, ctx->vy, ctx->vz, ctx->rung, ctx->id, !ctx->defer_vel);
    CT2G_LAUNCHED(ctx);
    ctx->vel_pending = ctx->defer_vel;
    // near-field work lists (scratch: flags, vals, vals2, x2, y2 are free here)
    chunk_flag_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(ctx->keys, ctx->cell_start, begin, nr,
                                                        ctx->dense_cell, ctx->flags, ctx->vals);
    CT2G_LAUNCHED(ctx);
    CT2G_TRY(ct2g_scan_exclusive(ctx, ctx->flags, ctx->vals2, nr, counts + 0, 0));
    dense_chunk_fill_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(
        ctx->flags, ctx->vals2, ctx->keys, ctx->cell_start, begin, nr, ctx->chunks);
    CT2G_LAUNCHED(ctx);
    uint32_t *rank = ctx->x2, *scflag = ctx->y2;
    CT2G_TRY(ct2g_scan_exclusive(ctx, ctx->vals, rank, nr, counts + 1, 0));
    chunk_fill_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(ctx->vals, rank, begin, nr,
                                                        ctx->sparse_list);
    CT2G_LAUNCHED(ctx);
    // sparse chunk starts, indexed by sparse rank (entries past the sparse
    // count stay zero)
    CT2G_CUDA(ctx, cudaMemsetAsync(scflag, 0, sizeof(uint32_t) * nr, st));
    sparse_chunk_flag_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(
        ctx->keys, ctx->cell_start, ctx->vals, rank, begin, nr, counts + 1, scflag);
    CT2G_LAUNCHED(ctx);
    CT2G_TRY(ct2g_scan_exclusive(ctx, scflag, ctx->vals2, nr, counts + 2, 0));
    sparse_chunk_fill_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(
        scflag, ctx->vals2, ctx->sparse_list, ctx->keys, ctx->cell_start, rank, begin, nr, counts,
        ctx->chunks);
    CT2G_LAUNCHED(ctx);
  } else {
    // empty range: every cell empty
    fill_kernel<<<ct2g_div_up(ctx->CB + 1, T), T, 0, st>>>(ctx->cell_start, ctx->CB + 1,
                                                          (uint32_t)begin);
    CT2G_LAUNCHED(ctx);
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->occ, 0, sizeof(unsigned long long) * (ctx->CB / 64), st));
  }
  ctx->grid_valid = true;
  ctx->moments_valid = false;
  ctx->expansions_valid = false;
  ctx->forces_valid = false;
  return CT2G_OK;
}

// The second half of a deferred gather (ctx->defer_vel at binning): the
// velocities and rungs of the binned range into cell order, after `stream`
// has waited for ctx->ev_vel (the host-state step's velocity upload; a no-op
// wait otherwise).  Bitwise the same store as the one-pass gather.
int ct2g_gather_velocities(ct2g_ctx *ctx) {
  if (!ctx->vel_pending) return CT2G_OK;
  ctx->vel_pending = false;
  const size_t begin = ctx->rung_begin, nr = ctx->n - ctx->rung_begin;
  cudaStream_t st = ctx->stream;
  CT2G_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev_vel,
                                     ctx->capturing ? cudaEventWaitExternal : 0));
  if (nr == 0) return CT2G_OK;
  const unsigned T = 256;
  gather_vel_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(begin, nr, ctx->vx, ctx->vy, ctx->vz,
                                                      ctx->rung, ctx->vx2, ctx->vy2, ctx->vz2,
                                                      ctx->rung2);
  CT2G_LAUNCHED(ctx);
  copy_back_vel_kernel<<<ct2g_div_up(nr, T), T, 0, st>>>(begin, nr, ctx->vx2, ctx->vy2,
                                                         ctx->vz2, ctx->rung2, ctx->vx, ctx->vy,
                                                         ctx->vz, ctx->rung);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}
