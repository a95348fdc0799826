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
  uint32_t mx, my, mz;  // block-key masks of the x, y, z bits; the bits above
                        // them are the box index, which the walk keeps
  __device__ __forceinline__ uint32_t add(uint32_t sb, int o) const {
    const uint32_t x = ((sb | ~mx) + c_doff[3 * o]) & mx;
    const uint32_t y = ((sb | ~my) + c_doff[3 * o + 1]) & my;
    const uint32_t z = ((sb | ~mz) + c_doff[3 * o + 2]) & mz;
    return x | y | z | (sb & ~(mx | my | mz));
  }
};

// minimum-image offset (in cells) from cell c to cell n along one axis
__device__ __forceinline__ int wrap_off(int n, int c, int M) { return ((n - c + M / 2) & (M - 1)) - M / 2; }

// Near field, one warp per chunk of <= 32 sinks; the grid is persistent and
// warps take chunks from a device work counter until the device-held chunk
// count is reached.  A dense chunk is sinks of
// one cell; a sparse chunk is sinks of sparse cells of one 4x4x4 block.  The
// warp walks the union of its sinks' stencils (per neighbouring block:
// occupancy & the OR of the sinks' stencil masks), fetching the ranges of 32
// candidate cells at a time; each source batch is staged in shared memory and
// read back as broadcasts.  A lane takes part in a source cell only if the
// cell lies in its own stencil (always true in a dense chunk), so every sink
// sees exactly its own near zone.

// ---------------------------------------------------------------------------
// Packed pairs: Blackwell's f32x2 add/mul/fma do two FP32 operations per
// issued instruction.  For the Plummer kernel the warp's source batch is
// staged as pair records -- (x0, x1, y0, y1) in one 16-byte slot and (z0, z1)
// in an 8-byte slot -- so one broadcast load of each feeds two interactions.
// ---------------------------------------------------------------------------
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2_pack(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void f2_unpack(f32x2 v, float &a, float &b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}

// two Plummer interactions of a sink at (X, Y, Z) (both halves equal) with
// the sources of pair record pr; accumulates +d g (the caller negates) and
// the potential +1/r; MASK (sparse chunks) is 1 or 0 per lane
template <bool POT, bool MASKED>
__device__ __forceinline__ void plummer_pair(const float *sbf, int pr, f32x2 X, f32x2 Y, f32x2 Z,
                                             f32x2 H2, f32x2 MASK, f32x2 &ax, f32x2 &ay,
                                             f32x2 &az, f32x2 &ap) {
  const float4 a = reinterpret_cast<const float4 *>(sbf)[pr];       // x0 x1 y0 y1
  const float2 b = reinterpret_cast<const float2 *>(sbf + 64)[pr];  // z0 z1
  const f32x2 dx = f2_sub(X, f2_pack(a.x, a.y));
  const f32x2 dy = f2_sub(Y, f2_pack(a.z, a.w));
  const f32x2 dz = f2_sub(Z, f2_pack(b.x, b.y));
  const f32x2 r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_fma(dx, dx, H2)));
  float r0, r1;
  f2_unpack(r2, r0, r1);
  f32x2 ri = f2_pack(rsqrtf(r0), rsqrtf(r1));
  if (MASKED) ri = f2_mul(ri, MASK);
  const f32x2 g = f2_mul(f2_mul(ri, ri), ri);
  ax = f2_fma(dx, g, ax);
  ay = f2_fma(dy, g, ay);
  az = f2_fma(dz, g, az);
  if (POT) ap = f2_sub(ap, ri);
}

__device__ __forceinline__ void inblock(int b, int &x, int &y, int &z) {
  x = ((b >> 2) & 1) | ((b >> 4) & 2);
  y = ((b >> 1) & 1) | ((b >> 3) & 2);
  z = (b & 1) | ((b >> 2) & 2);
}

// index of the r-th set bit (r < popcount) of w
__device__ __forceinline__ int nth_set_bit(unsigned long long w, uint32_t r) {
  int base = 0;
  uint32_t c = __popc((uint32_t)w);
  if (r >= c) {
    r -= c;
    w >>= 32;
    base = 32;
  }
  uint32_t v = (uint32_t)w;
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    c = __popc(v & ((1u << h) - 1u));
    if (r >= c) {
      r -= c;
      v >>= h;
      base += h;
    }
  }
  return base;
}

// two masked Plummer interactions from a streamed pair record: (x0 x1 y0 y1)
// at sbf[4 pr], (z0 z1 t0 t1) at sbf[64 + 4 pr], t the source's window cell
// (its bits as a float) and tb[t] this lane's 1 / 0 for that cell
template <bool POT>
__device__ __forceinline__ void plummer_pair_window(const float *sbf, const float *tb, int pr,
                                                    f32x2 X, f32x2 Y, f32x2 Z, f32x2 H2,
                                                    f32x2 &ax, f32x2 &ay, f32x2 &az,
                                                    f32x2 &ap) {
  const float4 a = reinterpret_cast<const float4 *>(sbf)[pr];
  const float4 b = reinterpret_cast<const float4 *>(sbf + 64)[pr];
  const f32x2 MASK = f2_pack(tb[__float_as_int(b.z)], tb[__float_as_int(b.w)]);
  const f32x2 dx = f2_sub(X, f2_pack(a.x, a.y));
  const f32x2 dy = f2_sub(Y, f2_pack(a.z, a.w));
  const f32x2 dz = f2_sub(Z, f2_pack(b.x, b.y));
  const f32x2 r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_fma(dx, dx, H2)));
  float r0, r1;
  f2_unpack(r2, r0, r1);
  const f32x2 ri = f2_mul(f2_pack(rsqrtf(r0), rsqrtf(r1)), MASK);
  const f32x2 g = f2_mul(f2_mul(ri, ri), ri);
  ax = f2_fma(dx, g, ax);
  ay = f2_fma(dy, g, ay);
  az = f2_fma(dz, g, az);
  if (POT) ap = f2_sub(ap, ri);
}

// Sparse chunk, streamed (Plummer): the candidate cells of the chunk (the set
// bits of `word`, lane o < 27 holding neighbouring block o's) go in windows of
// 32, a cell per lane; every lane first tabulates, for each cell of the
// window, whether it lies in its own sink's stencil window (lo2 < |o|^2 <=
// bw2: tb[t] = 1 or 0, slot 32 always 0); the sources of the window's cells
// then form one stream, staged in full batches of 32 in the chunk block's
// frame with the cell slot of each source, and every lane evaluates every
// staged source, multiplied by its table entry.  Unlike the cell-by-cell walk
// this keeps the batches full where the candidate cells hold a few particles
// each.
template <bool POT>
__device__ __forceinline__ void sparse_stream(
    unsigned long long word, uint32_t nblk, const uint32_t *__restrict__ cs,
    const float4 *__restrict__ src, int px, int py, int pz, float hc, float lo2, float bw2,
    bool act, f32x2 SX, f32x2 SY, f32x2 SZ, f32x2 H2, float *sbf, float *tb, int lane,
    f32x2 &pax, f32x2 &pay, f32x2 &paz, f32x2 &pap, uint32_t &nsrc) {
  const uint32_t c1 = (uint32_t)__popcll(word);
  uint32_t in1 = c1;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, in1, d);
    if (lane >= d) in1 += t;
  }
  const uint32_t ex1 = in1 - c1, C = __shfl_sync(0xffffffffu, in1, 31);
  tb[32] = 0.f;
  const int rec = 4 * (lane >> 1) + (lane & 1);
  for (uint32_t w0 = 0; w0 < C; w0 += 32) {
    const uint32_t nw = min(32u, C - w0);
    // window cell of this lane: the (g - ex1[o])-th candidate cell of block o
    const uint32_t g = min(w0 + (uint32_t)lane, C - 1);
    int o = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const uint32_t e = __shfl_sync(0xffffffffu, ex1, o + step);
      if (e <= g) o += step;
    }
    const unsigned long long wo = __shfl_sync(0xffffffffu, word, o);
    const uint32_t nbo = __shfl_sync(0xffffffffu, nblk, o);
    const uint32_t exo = __shfl_sync(0xffffffffu, ex1, o);
    const int q = nth_set_bit(wo, g - exo);
    int bx, by, bz;
    inblock(q, bx, by, bz);
    // cell offset from the chunk block's cell (0,0,0), biased by 8 per axis
    const int cpk = (4 * (o / 9 - 1) + bx + 8) | ((4 * ((o / 3) % 3 - 1) + by + 8) << 8) |
                    ((4 * (o % 3 - 1) + bz + 8) << 16);
    uint32_t jb = 0, je = 0;
    if ((uint32_t)lane < nw) {
      const uint32_t ck = (nbo << 6) | (uint32_t)q;
      jb = cs[ck];
      je = cs[ck + 1];
    }
    const uint32_t c = je - jb;
    // this lane's stencil entries for the window's cells
    for (uint32_t t = 0; t < nw; t++) {
      const int ct = __shfl_sync(0xffffffffu, cpk, (int)t);
      const uint32_t nt = __shfl_sync(0xffffffffu, c, (int)t);
      const int ox = (ct & 255) - 8 - px, oy = ((ct >> 8) & 255) - 8 - py,
                oz = (ct >> 16) - 8 - pz;
      const float d2 = (float)(ox * ox + oy * oy + oz * oz);
      const bool in = d2 > lo2 && d2 <= bw2;
      tb[t] = in ? 1.f : 0.f;
      if (in && act) nsrc += nt;
    }
    // the window's sources as one stream (lane order)
    uint32_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    const uint32_t excl = incl - c;
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    // source gs of the stream in the block frame, and its window slot (32
    // past the end of the stream: masked for every lane)
    auto fetch = [&](uint32_t gs, float4 &v) {
      const uint32_t gg = min(gs, max(total, 1u) - 1);
      int t = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        const uint32_t e = __shfl_sync(0xffffffffu, excl, t + step);
        if (e <= gg) t += step;
      }
      const uint32_t jt = __shfl_sync(0xffffffffu, jb, t), et = __shfl_sync(0xffffffffu, je, t);
      const int ct = __shfl_sync(0xffffffffu, cpk, t);
      const uint32_t j = min(jt + (gg - __shfl_sync(0xffffffffu, excl, t)), max(et, 1u) - 1u);
      const float4 s = __ldg(src + j);
      v = make_float4(fmaf((float)((ct & 255) - 8), hc, s.x),
                      fmaf((float)(((ct >> 8) & 255) - 8), hc, s.y),
                      fmaf((float)((ct >> 16) - 8), hc, s.z), __int_as_float(gs < total ? t : 32));
    };
    if (total == 0) continue;
    float4 nq;
    fetch((uint32_t)lane, nq);
    for (uint32_t b0 = 0; b0 < total; b0 += 32) {
      __syncwarp();
      sbf[rec] = nq.x;
      sbf[rec + 2] = nq.y;
      sbf[64 + rec] = nq.z;
      sbf[64 + rec + 2] = nq.w;
      __syncwarp();
      if (b0 + 32 < total) fetch(b0 + 32 + (uint32_t)lane, nq);
      const int npair = (int)((min(32u, total - b0) + 1) >> 1);
      if (npair == 16) {
#pragma unroll 8
        for (int pr = 0; pr < 16; pr++)
          plummer_pair_window<POT>(sbf, tb, pr, SX, SY, SZ, H2, pax, pay, paz, pap);
      } else {
#pragma unroll 2
        for (int pr = 0; pr < npair; pr++)
          plummer_pair_window<POT>(sbf, tb, pr, SX, SY, SZ, H2, pax, pay, paz, pap);
      }
    }
  }
}

template <int KERNEL, bool POT, bool SPARSE, bool STREAM>
__device__ __forceinline__ void near_chunk(
    const uint2 cd, const uint32_t *__restrict__ sparse_list,
    const uint32_t *__restrict__ cs, const unsigned long long *__restrict__ occ,
    const unsigned long long *__restrict__ stmask, const Walk &walk,
    const uint32_t *__restrict__ skeys, uint32_t rbegin, const float4 *__restrict__ src,
    int mbits, float soft, float lo2, float bw2, const float *__restrict__ box_gm,
    float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, bool store, unsigned long long *__restrict__ inter, float4 *sb,
    float *tbl, int lane) {
  const int M = 1 << mbits;
  const bool act = (uint32_t)lane < cd.y;
  const uint32_t slot = cd.x + (act ? (uint32_t)lane : 0u);
  const uint32_t i = SPARSE ? sparse_list[slot] : slot;
  const uint32_t key = skeys[i - rbegin];
  const float4 si = src[i];
  const uint32_t p = key & 63u, blk = key >> 6;  // blk is the same for the whole chunk
  const float GM = __ldg(box_gm + (key >> (3 * mbits)));
  int px, py, pz;
  inblock((int)p, px, py, pz);
  // cells of the block present in the chunk
  unsigned long long pm = 1ull << p;
  if (SPARSE) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) pm |= __shfl_xor_sync(0xffffffffu, pm, o);
  }
  unsigned long long word = 0;
  uint32_t nblk = 0;
  if (lane < 27) {
    nblk = walk.add(blk, lane);
    unsigned long long m = 0, q = pm;
    while (q) {
      const int pp = __ffsll((long long)q) - 1;
      q &= q - 1;
      m |= __ldg(stmask + pp * 27 + lane);
    }
    word = occ[nblk] & m;
  }
  const float hc = 1.0f / (float)M;
  const float h2 = soft * soft, hinv = 1.f / soft, hinv3 = hinv * hinv * hinv;
  float nx = 0.f, ny = 0.f, nz = 0.f, np = 0.f;
  // packed accumulators of the Plummer path (+d g and +1/r per pair half)
  f32x2 pax = 0ull, pay = 0ull, paz = 0ull, pap = 0ull;
  const f32x2 H2 = f2_pack(h2, h2);
  // dense chunks: the sink in its own cell's frame (sources are shifted there)
  const f32x2 SX = f2_pack(si.x, si.x), SY = f2_pack(si.y, si.y), SZ = f2_pack(si.z, si.z);
  const f32x2 ONE = f2_pack(1.f, 1.f);
  uint32_t nsrc = 0;
  if constexpr (STREAM) {
    static_assert(SPARSE && KERNEL == CT2G_SOFT_PLUMMER, "streamed sparse chunks: Plummer only");
    // the sink in the chunk block's frame (from the centre of its cell (0,0,0))
    const float sx = fmaf((float)px, hc, si.x), sy = fmaf((float)py, hc, si.y),
                sz = fmaf((float)pz, hc, si.z);
    sparse_stream<POT>(word, nblk, cs, src, px, py, pz, hc, lo2, bw2, act,
                       f2_pack(sx, sx), f2_pack(sy, sy), f2_pack(sz, sz), H2,
                       reinterpret_cast<float *>(sb), tbl + 33 * lane, lane, pax, pay, paz, pap,
                       nsrc);
  } else {
  for (int o = 0; o < 27; o++) {
    const unsigned long long bits = __shfl_sync(0xffffffffu, word, o);
    if (!bits) continue;
    const uint32_t nb = __shfl_sync(0xffffffffu, nblk, o);
    const int dX = 4 * (o / 9 - 1) - px, dY = 4 * ((o / 3) % 3 - 1) - py, dZ = 4 * (o % 3 - 1) - pz;
#pragma unroll 1
    for (int half = 0; half < 2; half++) {
      unsigned hb = (unsigned)(bits >> (32 * half));
      if (!hb) continue;
      // the ranges of up to 32 candidate cells, one per lane
      uint32_t jb = 0, je = 0;
      if ((hb >> lane) & 1u) {
        const uint32_t ck = (nb << 6) | (uint32_t)(32 * half + lane);
        jb = cs[ck];
        je = cs[ck + 1];
      }
      if constexpr (KERNEL == CT2G_SOFT_PLUMMER && !SPARSE) {
        // Every candidate cell is in the stencil of every lane: the cells'
        // sources form one stream (lane order), staged in full batches of 32,
        // each source shifted into the sink cell's frame.
        const uint32_t c = je - jb;
        uint32_t incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
          if (lane >= d) incl += t;
        }
        const uint32_t excl = incl - c;
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        if (act) nsrc += total;
        // source g of the stream, in the sink cell's frame
        auto fetch = [&](uint32_t g) {
          const uint32_t gg = min(g, total - 1);
          int t = 0;  // owner: the last lane whose stream offset is <= gg
#pragma unroll
          for (int step = 16; step > 0; step >>= 1) {
            const uint32_t e = __shfl_sync(0xffffffffu, excl, t + step);
            if (e <= gg) t += step;
          }
          const uint32_t jt = __shfl_sync(0xffffffffu, jb, t), et = __shfl_sync(0xffffffffu, je, t);
          // j < et by the scan; the clamp keeps the load inside the owner cell regardless
          const uint32_t j = min(jt + (gg - __shfl_sync(0xffffffffu, excl, t)), max(et, 1u) - 1u);
          int bx, by, bz;
          inblock(32 * half + t, bx, by, bz);
          const float4 q = __ldg(src + j);
          return make_float3(fmaf((float)(dX + bx), hc, q.x), fmaf((float)(dY + by), hc, q.y),
                             fmaf((float)(dZ + bz), hc, q.z));
        };
        float *sbf = reinterpret_cast<float *>(sb);
        const int rec = 4 * (lane >> 1) + (lane & 1);
        float3 nq = fetch((uint32_t)lane);
        for (uint32_t b0 = 0; b0 < total; b0 += 32) {
          const int cnt = (int)min(32u, total - b0);
          __syncwarp();
          sbf[rec] = nq.x;
          sbf[rec + 2] = nq.y;
          sbf[64 + 2 * (lane >> 1) + (lane & 1)] = nq.z;
          __syncwarp();
          if (b0 + 32 < total) nq = fetch(b0 + 32 + (uint32_t)lane);
          if (cnt == 32) {
#pragma unroll 8
            for (int pr = 0; pr < 16; pr++)
              plummer_pair<POT, false>(sbf, pr, SX, SY, SZ, H2, ONE, pax, pay, paz, pap);
          } else {
#pragma unroll 2
            for (int pr = 0; pr < (cnt >> 1); pr++)
              plummer_pair<POT, false>(sbf, pr, SX, SY, SZ, H2, ONE, pax, pay, paz, pap);
            if (cnt & 1) {  // the odd last source
              const int pr = cnt >> 1;
              const float qx = sbf[4 * pr], qy = sbf[4 * pr + 2], qz = sbf[64 + 2 * pr];
              ct2g_pair_term<KERNEL, POT>(si.x - qx, si.y - qy, si.z - qz, h2, hinv, hinv3, nx,
                                          ny, nz, np, true);
            }
          }
        }
        continue;
      }
      while (hb) {
        const int t = __ffs(hb) - 1;
        hb &= hb - 1;
        const uint32_t j0 = __shfl_sync(0xffffffffu, jb, t), j1 = __shfl_sync(0xffffffffu, je, t);
        int bx, by, bz;
        inblock(32 * half + t, bx, by, bz);
        const int ox = dX + bx, oy = dY + by, oz = dZ + bz;  // cells, from this lane's cell
        bool in = act;
        if (SPARSE) {
          const float d2 = (float)(ox * ox + oy * oy + oz * oz);
          in = in && d2 > lo2 && d2 <= bw2;
        }
        if (in) nsrc += j1 - j0;
        // sink position relative to the neighbour cell's centre
        const float xs = si.x - (float)ox * hc, ys = si.y - (float)oy * hc, zs = si.z - (float)oz * hc;
        float4 nxt = __ldg(src + min(j0 + lane, j1 - 1));
        if constexpr (KERNEL == CT2G_SOFT_PLUMMER) {
          const f32x2 X = f2_pack(xs, xs), Y = f2_pack(ys, ys), Z = f2_pack(zs, zs);
          const float mk = (!SPARSE || in) ? 1.f : 0.f;
          const f32x2 MASK = f2_pack(mk, mk);
          float *sbf = reinterpret_cast<float *>(sb);
          const int rec = 4 * (lane >> 1) + (lane & 1);
          for (uint32_t jj = j0; jj < j1; jj += 32) {
            const int cnt = (int)min(32u, j1 - jj);
            __syncwarp();
            sbf[rec] = nxt.x;
            sbf[rec + 2] = nxt.y;
            sbf[64 + 2 * (lane >> 1) + (lane & 1)] = nxt.z;
            __syncwarp();
            if (jj + 32 < j1) nxt = __ldg(src + min(jj + 32 + lane, j1 - 1));
            if (cnt == 32) {
#pragma unroll 8
              for (int pr = 0; pr < 16; pr++)
                plummer_pair<POT, SPARSE>(sbf, pr, X, Y, Z, H2, MASK, pax, pay, paz, pap);
            } else {
#pragma unroll 2
              for (int pr = 0; pr < (cnt >> 1); pr++)
                plummer_pair<POT, SPARSE>(sbf, pr, X, Y, Z, H2, MASK, pax, pay, paz, pap);
              if (cnt & 1) {  // the odd last source
                const int pr = cnt >> 1;
                const float qx = sbf[4 * pr], qy = sbf[4 * pr + 2], qz = sbf[64 + 2 * pr];
                ct2g_pair_term<KERNEL, POT>(xs - qx, ys - qy, zs - qz, h2, hinv, hinv3, nx, ny,
                                            nz, np, !SPARSE || in);
              }
            }
          }
          continue;
        }
        for (uint32_t jj = j0; jj < j1; jj += 32) {
          const int cnt = (int)min(32u, j1 - jj);
          __syncwarp();
          sb[lane] = nxt;
          __syncwarp();
          if (jj + 32 < j1) nxt = __ldg(src + min(jj + 32 + lane, j1 - 1));
          if (cnt == 32) {
#pragma unroll 16
            for (int u = 0; u < 32; u++) {
              const float4 q = sb[u];
              ct2g_pair_term<KERNEL, POT>(xs - q.x, ys - q.y, zs - q.z, h2, hinv, hinv3, nx, ny, nz,
                                     np, !SPARSE || in);
            }
          } else {
#pragma unroll 4
            for (int u = 0; u < cnt; u++) {
              const float4 q = sb[u];
              ct2g_pair_term<KERNEL, POT>(xs - q.x, ys - q.y, zs - q.z, h2, hinv, hinv3, nx, ny, nz,
                                     np, !SPARSE || in);
            }
          }
        }
      }
    }
  }
  }  // not STREAM
  if constexpr (KERNEL == CT2G_SOFT_PLUMMER) {
    float a0, a1;
    f2_unpack(pax, a0, a1);
    nx -= a0 + a1;
    f2_unpack(pay, a0, a1);
    ny -= a0 + a1;
    f2_unpack(paz, a0, a1);
    nz -= a0 + a1;
    if (POT) {
      f2_unpack(pap, a0, a1);
      np += a0 + a1;
    }
  }
  // added to the far field (L2P, with GM) already in the force buffers, or
  // stored into the near-field buffers when the two run side by side; the
  // product is rounded on its own (no fused multiply-add into the far
  // field), so that both forms add the same two values
  if (act) {
    const float gx = __fmul_rn(GM, nx), gy = __fmul_rn(GM, ny), gz = __fmul_rn(GM, nz);
    if (store) {
      ofx[i] = gx;
      ofy[i] = gy;
      ofz[i] = gz;
      if (POT) opot[i] = __fmul_rn(GM, np);
    } else {
      ofx[i] += gx;
      ofy[i] += gy;
      ofz[i] += gz;
      if (POT) opot[i] += __fmul_rn(GM, np);
    }
  }
  unsigned long long c = nsrc;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0 && c && inter) atomicAdd(inter, c);
}

// The chunk count is *nch_ptr, the chunks start at chunks + *off_ptr (none:
// at chunks), warps take them from the work counter *work (zero at launch).
// Sparse-style chunks (SPARSE) list sinks through slist and take only the
// source cells with lo2 < |o|^2 <= bw2 of each lane's own cell; the stencil
// masks stm must cover that window.
template <int KERNEL, bool POT, bool SPARSE, bool STREAM = false>
__global__ void __launch_bounds__(256, 4) near_kernel(
    const uint2 *__restrict__ chunks, const uint32_t *__restrict__ nch_ptr,
    const uint32_t *__restrict__ off_ptr, uint32_t *__restrict__ work,
    const uint32_t *__restrict__ sparse_list, const uint32_t *__restrict__ cs,
    const unsigned long long *__restrict__ occ, const unsigned long long *__restrict__ stmask,
    Walk walk, const uint32_t *__restrict__ skeys, uint32_t rbegin,
    const float4 *__restrict__ src, int mbits, float soft, float lo2, float bw2,
    const float *__restrict__ box_gm, float *__restrict__ ofx, float *__restrict__ ofy,
    float *__restrict__ ofz, float *__restrict__ opot, bool store, uint32_t maxch,
    unsigned long long *__restrict__ inter) {
  __shared__ float4 sbuf[8][32];  // one batch of 32 sources per warp
  // streamed sparse chunks: per warp, per lane a row of 33 window-cell entries
  __shared__ float tbl[STREAM ? 8 * 32 * 33 : 1];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t nch = *nch_ptr;
  const uint2 *list = off_ptr ? chunks + *off_ptr : chunks;
  // maxch > 0: a warp takes at most maxch chunks and the block then exits,
  // so that blocks of kernels on other streams get the SM in between
  for (uint32_t taken = 0; maxch == 0 || taken < maxch; taken++) {
    uint32_t ch = 0;
    if (lane == 0) ch = atomicAdd(work, 1u);
    ch = __shfl_sync(0xffffffffu, ch, 0);
    if (ch >= nch) break;
    near_chunk<KERNEL, POT, SPARSE, STREAM>(list[ch], sparse_list, cs, occ, stmask, walk, skeys,
                                            rbegin, src, mbits, soft, lo2, bw2, box_gm, ofx, ofy,
                                            ofz, opot, store, inter, sbuf[wib],
                                            tbl + (STREAM ? wib * 32 * 33 : 0), lane);
  }
}

// Sparse sinks, one per lane: the warp takes 32 consecutive entries of the
// sparse sink list (cell order, so the lanes are neighbours) and every lane
// walks the stencil of its own cell -- the 27 neighbouring 4x4x4 blocks,
// occupancy & its own stencil mask, the ranges of the occupied cells -- and
// sums its own sources, read through the read-only cache, two at a time with
// the packed f32x2 arithmetic.  No lane evaluates a source outside its
// stencil, and a warp is not bound to one cell block, so sparse regions fill
// whole warps.  The work counter hands out groups of 32 sinks until the
// device-held sparse count is covered.
template <int KERNEL, bool POT>
__global__ void __launch_bounds__(256, 4) near_lane_kernel(
    const uint32_t *__restrict__ nsparse_ptr, uint32_t *__restrict__ work,
    const uint32_t *__restrict__ sparse_list, const uint32_t *__restrict__ cs,
    const unsigned long long *__restrict__ occ, const unsigned long long *__restrict__ stmask,
    Walk walk, const uint32_t *__restrict__ skeys, uint32_t rbegin,
    const float4 *__restrict__ src, int mbits, float soft, const float *__restrict__ box_gm,
    float *__restrict__ ofx, float *__restrict__ ofy, float *__restrict__ ofz,
    float *__restrict__ opot, bool store, unsigned long long *__restrict__ inter) {
  const int lane = threadIdx.x & 31;
  const uint32_t ns = *nsparse_ptr;
  const int M = 1 << mbits;
  const float hc = 1.0f / (float)M;
  const float h2 = soft * soft, hinv = 1.f / soft, hinv3 = hinv * hinv * hinv;
  const f32x2 H2 = f2_pack(h2, h2);
  for (;;) {
    uint32_t ch = 0;
    if (lane == 0) ch = atomicAdd(work, 1u);
    ch = __shfl_sync(0xffffffffu, ch, 0);
    if ((size_t)ch * 32 >= ns) break;
    const uint32_t r = ch * 32 + (uint32_t)lane;
    const bool act = r < ns;
    uint32_t nsrc = 0;
    if (act) {
      const uint32_t i = sparse_list[r];
      const uint32_t key = skeys[i - rbegin];
      const float4 si = src[i];
      const uint32_t p = key & 63u, blk = key >> 6;
      const float GM = __ldg(box_gm + (key >> (3 * mbits)));
      int px, py, pz;
      inblock((int)p, px, py, pz);
      float nx = 0.f, ny = 0.f, nz = 0.f, np = 0.f;
      f32x2 pax = 0ull, pay = 0ull, paz = 0ull, pap = 0ull;
      const unsigned long long *sm = stmask + p * 27;
#pragma unroll 1
      for (int o = 0; o < 27; o++) {
        const unsigned long long m = __ldg(sm + o);
        if (!m) continue;
        const uint32_t nb = walk.add(blk, o);
        unsigned long long word = __ldg(occ + nb) & m;
        const int dX = 4 * (o / 9 - 1) - px, dY = 4 * ((o / 3) % 3 - 1) - py,
                  dZ = 4 * (o % 3 - 1) - pz;
        while (word) {
          const int c = __ffsll((long long)word) - 1;
          word &= word - 1;
          const uint32_t ck = (nb << 6) | (uint32_t)c;
          const uint32_t j0 = __ldg(cs + ck), j1 = __ldg(cs + ck + 1);
          nsrc += j1 - j0;
          int bx, by, bz;
          inblock(c, bx, by, bz);
          // the sink relative to the source cell's centre
          const float xs = si.x - (float)(dX + bx) * hc, ys = si.y - (float)(dY + by) * hc,
                      zs = si.z - (float)(dZ + bz) * hc;
          uint32_t j = j0;
          if constexpr (KERNEL == CT2G_SOFT_PLUMMER) {
            const f32x2 X = f2_pack(xs, xs), Y = f2_pack(ys, ys), Z = f2_pack(zs, zs);
            for (; j + 1 < j1; j += 2) {
              const float4 a = __ldg(src + j), b = __ldg(src + j + 1);
              const f32x2 dx = f2_sub(X, f2_pack(a.x, b.x));
              const f32x2 dy = f2_sub(Y, f2_pack(a.y, b.y));
              const f32x2 dz = f2_sub(Z, f2_pack(a.z, b.z));
              const f32x2 r2 = f2_fma(dz, dz, f2_fma(dy, dy, f2_fma(dx, dx, H2)));
              float r0, r1;
              f2_unpack(r2, r0, r1);
              const f32x2 ri = f2_pack(rsqrtf(r0), rsqrtf(r1));
              const f32x2 g = f2_mul(f2_mul(ri, ri), ri);
              pax = f2_fma(dx, g, pax);
              pay = f2_fma(dy, g, pay);
              paz = f2_fma(dz, g, paz);
              if (POT) pap = f2_sub(pap, ri);
            }
          }
          for (; j < j1; j++) {
            const float4 q = __ldg(src + j);
            ct2g_pair_term<KERNEL, POT>(xs - q.x, ys - q.y, zs - q.z, h2, hinv, hinv3, nx, ny,
                                        nz, np, true);
          }
        }
      }
      if constexpr (KERNEL == CT2G_SOFT_PLUMMER) {
        float a0, a1;
        f2_unpack(pax, a0, a1);
        nx -= a0 + a1;
        f2_unpack(pay, a0, a1);
        ny -= a0 + a1;
        f2_unpack(paz, a0, a1);
        nz -= a0 + a1;
        if (POT) {
          f2_unpack(pap, a0, a1);
          np += a0 + a1;
        }
      }
      // added to the far field already in the force buffers, or stored (the
      // product rounded on its own, as in near_chunk)
      const float gx = __fmul_rn(GM, nx), gy = __fmul_rn(GM, ny), gz = __fmul_rn(GM, nz);
      if (store) {
        ofx[i] = gx;
        ofy[i] = gy;
        ofz[i] = gz;
        if (POT) opot[i] = __fmul_rn(GM, np);
      } else {
        ofx[i] += gx;
        ofy[i] += gy;
        ofz[i] += gz;
        if (POT) opot[i] += __fmul_rn(GM, np);
      }
    }
    unsigned long long c = nsrc;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0 && c && inter) atomicAdd(inter, c);
  }
}

template <int K, bool POT>
int launch_near_lanes(ct2g_ctx *ctx, const Walk &walk, cudaStream_t st, float *fx, float *fy,
                      float *fz, float *pot, bool store) {
  auto k = near_lane_kernel<K, POT>;
  int per_sm = 0;
  CT2G_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, 0));
  const size_t nr = ctx->n - ctx->rung_begin;
  if (ctx->near_blocks_per_sm > 0) per_sm = std::min(per_sm, ctx->near_blocks_per_sm);
  size_t blocks = (size_t)std::max(1, per_sm) * ctx->num_sms;
  blocks = std::max<size_t>(1, std::min(blocks, (nr + 255) / 256));
  uint32_t *c = ctx->d_counts;
  k<<<(unsigned)blocks, 256, 0, st>>>(
      c + 1, c + 4, ctx->sparse_list, ctx->cell_start, ctx->occ, ctx->stmask, walk, ctx->keys,
      (uint32_t)ctx->rung_begin, ctx->src, ctx->mbits, ctx->opt.hsoft, ctx->box_gm, fx, fy, fz,
      pot, store, ctx->d_inter);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
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

// persistent grid: the resident blocks of every SM (or the tuned count), and
// no more than one block per 256 sinks of the range
template <int K, bool POT, bool SPARSE, bool STREAM = false>
int launch_near1(ct2g_ctx *ctx, const Walk &walk, const uint2 *chunks, const uint32_t *nch,
                 const uint32_t *off, uint32_t *work, const uint32_t *slist,
                 const unsigned long long *stm, float lo2, float bw2, float *fx, float *fy,
                 float *fz, float *pot, unsigned long long *inter, cudaStream_t st = nullptr,
                 bool store = false, uint32_t maxch = 0) {
  auto k = near_kernel<K, POT, SPARSE, STREAM>;
  if (!st) st = ctx->stream;
  int per_sm = 0;
  if constexpr (STREAM) {
    // 38 KB of static shared memory a block: the whole L1 as shared memory,
    // and the resident blocks counted from the kernel's own limits
    CT2G_TRY(ct2g_smem_attrs(ctx, k, 0));
    per_sm = ct2g_blocks_per_sm(ctx, (const void *)k, 256, 0);
  } else {
    CT2G_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, 0));
  }
  const size_t nr = ctx->n - ctx->rung_begin;
  if (ctx->near_blocks_per_sm > 0) per_sm = std::min(per_sm, ctx->near_blocks_per_sm);
  size_t blocks = (size_t)std::max(1, per_sm) * ctx->num_sms;
  blocks = std::max<size_t>(1, std::min(blocks, (nr + 255) / 256));
  // capped warps: enough blocks for every chunk the range can have (one per
  // sink at most); blocks past the device-held chunk count exit at once
  if (maxch) blocks = std::max<size_t>(1, (nr + 8 * (size_t)maxch - 1) / (8 * (size_t)maxch));
  k<<<(unsigned)blocks, 256, 0, st>>>(
      chunks, nch, off, work, slist, ctx->cell_start, ctx->occ, stm, walk, ctx->keys,
      (uint32_t)ctx->rung_begin, ctx->src, ctx->mbits, ctx->opt.hsoft, lo2, bw2, ctx->box_gm, fx,
      fy, fz, pot, store, maxch, inter);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// dense chunks (counts[0], work counter counts[3]), then the sparse sinks
// (counts[1] of them; work counter counts[4]): one per lane (sparse_path 0) or
// as the per-block chunks stored after the dense ones (counts[2], sparse_path 1)
template <int K, bool POT>
int launch_near(ct2g_ctx *ctx, cudaStream_t st, float *fx, float *fy, float *fz, float *pot,
                bool store) {
  const Walk walk = make_walk(ctx->mbits);
  const float bw2 = ctx->opt.bwidth * ctx->opt.bwidth;
  uint32_t *c = ctx->d_counts;
  // capped warps only beside the mesh solve (overlap), where they let the
  // mesh kernels' blocks in
  const uint32_t maxch = store ? (uint32_t)ctx->near_chunks_per_warp : 0u;
  CT2G_TRY((launch_near1<K, POT, false>(ctx, walk, ctx->chunks, c + 0, nullptr, c + 3,
                                        ctx->sparse_list, ctx->stmask, -1.f, bw2, fx, fy, fz, pot,
                                        ctx->d_inter, st, store, maxch)));
  if (ctx->sparse_path == 0) return launch_near_lanes<K, POT>(ctx, walk, st, fx, fy, fz, pot, store);
  if constexpr (K == CT2G_SOFT_PLUMMER) {
    if (ctx->sparse_path == 2)
      return launch_near1<K, POT, true, true>(ctx, walk, ctx->chunks, c + 2, c + 0, c + 4,
                                              ctx->sparse_list, ctx->stmask, -1.f, bw2, fx, fy,
                                              fz, pot, ctx->d_inter, st, store, maxch);
  }
  return launch_near1<K, POT, true>(ctx, walk, ctx->chunks, c + 2, c + 0, c + 4,
                                    ctx->sparse_list, ctx->stmask, -1.f, bw2, fx, fy, fz, pot,
                                    ctx->d_inter, st, store, maxch);
}

int near_all(ct2g_ctx *ctx, bool pot, cudaStream_t st, float *fx, float *fy, float *fz,
             float *po, bool store) {
  if (ctx->opt.kernel == CT2G_SOFT_SPHERE)
    return pot ? launch_near<CT2G_SOFT_SPHERE, true>(ctx, st, fx, fy, fz, po, store)
               : launch_near<CT2G_SOFT_SPHERE, false>(ctx, st, fx, fy, fz, po, store);
  return pot ? launch_near<CT2G_SOFT_PLUMMER, true>(ctx, st, fx, fy, fz, po, store)
             : launch_near<CT2G_SOFT_PLUMMER, false>(ctx, st, fx, fy, fz, po, store);
}

// far field + near field, added in that order: f = far + GM * near
__global__ void combine_kernel(size_t b, size_t n, float *__restrict__ fx, float *__restrict__ fy,
                               float *__restrict__ fz, const float *__restrict__ nfx,
                               const float *__restrict__ nfy, const float *__restrict__ nfz,
                               float *__restrict__ po, const float *__restrict__ npo) {
  for (size_t i = b + blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    fx[i] += nfx[i];
    fy[i] += nfy[i];
    fz[i] += nfz[i];
    if (po) po[i] += npo[i];
  }
}

}  // namespace

// direct sum over a window lo2 < |o|^2 <= hi2 of cells for listed sinks
// (sparse-style chunks), added into the given force buffers
int ct2g_near_window(ct2g_ctx *ctx, const uint2 *chunks, const uint32_t *nch, uint32_t *work,
                     const uint32_t *slist, const unsigned long long *stm, float lo2, float hi2,
                     bool pot, float *fx, float *fy, float *fz, float *po) {
  const Walk walk = make_walk(ctx->mbits);
  if (ctx->opt.kernel == CT2G_SOFT_SPHERE)
    return pot ? launch_near1<CT2G_SOFT_SPHERE, true, true>(ctx, walk, chunks, nch, nullptr, work,
                                                            slist, stm, lo2, hi2, fx, fy, fz, po,
                                                            nullptr)
               : launch_near1<CT2G_SOFT_SPHERE, false, true>(ctx, walk, chunks, nch, nullptr,
                                                             work, slist, stm, lo2, hi2, fx, fy,
                                                             fz, po, nullptr);
  if (ctx->sparse_path == 2)
    return pot ? launch_near1<CT2G_SOFT_PLUMMER, true, true, true>(
                     ctx, walk, chunks, nch, nullptr, work, slist, stm, lo2, hi2, fx, fy, fz, po,
                     nullptr)
               : launch_near1<CT2G_SOFT_PLUMMER, false, true, true>(
                     ctx, walk, chunks, nch, nullptr, work, slist, stm, lo2, hi2, fx, fy, fz, po,
                     nullptr);
  return pot ? launch_near1<CT2G_SOFT_PLUMMER, true, true>(ctx, walk, chunks, nch, nullptr, work,
                                                           slist, stm, lo2, hi2, fx, fy, fz, po,
                                                           nullptr)
             : launch_near1<CT2G_SOFT_PLUMMER, false, true>(ctx, walk, chunks, nch, nullptr, work,
                                                            slist, stm, lo2, hi2, fx, fy, fz, po,
                                                            nullptr);
}

// direct sum over the cells of the stencil masks stm for dense-style chunks
// (<= 32 consecutive sinks of one cell), added into the given force buffers
int ct2g_near_dense_window(ct2g_ctx *ctx, const uint2 *chunks, const uint32_t *nch,
                           uint32_t *work, const unsigned long long *stm, bool pot, float *fx,
                           float *fy, float *fz, float *po) {
  const Walk walk = make_walk(ctx->mbits);
  if (ctx->opt.kernel == CT2G_SOFT_SPHERE)
    return pot ? launch_near1<CT2G_SOFT_SPHERE, true, false>(ctx, walk, chunks, nch, nullptr, work,
                                                             nullptr, stm, -1.f, 0.f, fx, fy, fz,
                                                             po, nullptr)
               : launch_near1<CT2G_SOFT_SPHERE, false, false>(ctx, walk, chunks, nch, nullptr,
                                                              work, nullptr, stm, -1.f, 0.f, fx,
                                                              fy, fz, po, nullptr);
  return pot ? launch_near1<CT2G_SOFT_PLUMMER, true, false>(ctx, walk, chunks, nch, nullptr, work,
                                                            nullptr, stm, -1.f, 0.f, fx, fy, fz,
                                                            po, nullptr)
             : launch_near1<CT2G_SOFT_PLUMMER, false, false>(ctx, walk, chunks, nch, nullptr,
                                                             work, nullptr, stm, -1.f, 0.f, fx, fy,
                                                             fz, po, nullptr);
}

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
  // the far-field pass (the inverse z pass with L2P) has written the range's entries
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->d_inter, 0, sizeof(unsigned long long), ctx->stream));
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + 3, 0, 2 * sizeof(uint32_t), ctx->stream));
  if (ctx->n == ctx->rung_begin) return CT2G_OK;
  CT2G_TRY(near_all(ctx, pot, ctx->stream, ctx->fx, ctx->fy, ctx->fz, ctx->pot, false));
  return ct2g_learned_apply(ctx, pot);
}

// Far field and near field of the current range.  Serial (ctx->overlap 0):
// the mesh solve writes the far field, then the near field adds to it.
// Overlapped: the near field forks onto stream2 as soon as binning is done
// and stores into its own buffers while the mesh solve runs on the context
// stream (the near kernels are issue-bound, the mesh passes bound by memory
// latency, so the two fill each other's idle cycles); the context stream then
// joins it and adds the two, in the serial order (far + GM near), so both
// forms give the same forces bit for bit.
int ct2g_all_forces(ct2g_ctx *ctx, bool pot) {
  if (!ctx->overlap || ctx->n == ctx->rung_begin) {
    CT2G_TRY(ct2g_far_field(ctx, pot));
    return ct2g_forces(ctx, pot);
  }
  cudaStream_t st = ctx->stream;
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->d_inter, 0, sizeof(unsigned long long), st));
  CT2G_CUDA(ctx, cudaMemsetAsync(ctx->d_counts + 3, 0, 2 * sizeof(uint32_t), st));
  CT2G_CUDA(ctx, cudaEventRecord(ctx->ev_fork, st));
  CT2G_CUDA(ctx, cudaStreamWaitEvent(ctx->stream2, ctx->ev_fork, 0));
  CT2G_TRY(near_all(ctx, pot, ctx->stream2, ctx->nfx, ctx->nfy, ctx->nfz, ctx->npot, true));
  CT2G_CUDA(ctx, cudaEventRecord(ctx->ev_join, ctx->stream2));
  const int rc = ct2g_far_field(ctx, pot);
  // join before any return, so that stream2 never outlives a recording
  CT2G_CUDA(ctx, cudaStreamWaitEvent(st, ctx->ev_join, 0));
  CT2G_TRY(rc);
  const size_t b = ctx->rung_begin, nr = ctx->n - b;
  combine_kernel<<<(unsigned)std::min<size_t>((nr + 255) / 256, (size_t)ctx->num_sms * 16), 256, 0,
                   st>>>(b, ctx->n, ctx->fx, ctx->fy, ctx->fz, ctx->nfx, ctx->nfy, ctx->nfz,
                         pot ? ctx->pot : nullptr, ctx->npot);
  CT2G_LAUNCHED(ctx);
  return ct2g_learned_apply(ctx, pot);
}

