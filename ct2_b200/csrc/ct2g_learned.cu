// Learned near-field correction.
//
// The plain step sums directly over the stencil |o|^2 <= bwidth^2 and takes
// every other cell from the mesh (order-p Taylor expansions).  For a chosen
// set of sink cells the correction widens the direct sum to the shell
// bwidth^2 < |o|^2 <= bwidth_ext^2: it adds the exact pair forces of the
// shell's particles and subtracts what the mesh holds for those cells, the
// primary-image Taylor term
//     L_a = sum_{o in shell} sum_b D^{a+b} phi_eps(-o h) M_b(c + o),
// evaluated by L2P at each sink.  A corrected cell therefore gets exactly the
// forces of the method run with bwidth_ext (the Green's table excludes the
// near zone's primary images and nothing else).
//
// Which cells: a fixed criterion (the shell's monopole pull relative to the
// sink's force above a threshold), or a small MLP (24 per-cell moment and
// density features -> 64 -> 64 -> 1, BF16 weights, FP32 accumulation) that
// predicts log10 of the cell's rms relative force residual.  The MLP is
// trained on the GPU by the kernels below (forward, backward, Adam) on
// residuals the method generates itself: widened minus plain forces, with
// every cell corrected.
//
// Everything a step needs stays on the device (cell counts, chunk lists), so
// the correction records into the step's CUDA graph.
#include <cuda_bf16.h>

#include <array>
#include <cstring>
#include <random>

#include "ct2g_internal.cuh"

namespace {

constexpr int NIN = CT2G_MLP_NIN, NH = CT2G_MLP_NHID, NP = CT2G_MLP_NPARAM;
constexpr int OW1 = 0, OB1 = OW1 + NH * NIN, OW2 = OB1 + NH, OB2 = OW2 + NH * NH,
              OW3 = OB2 + NH, OB3 = OW3 + NH;
static_assert(OB3 + 1 == NP, "parameter layout");
// per-sample values kept for the weight gradients: h1 | dz1 | h2 | dz2 | dy
constexpr int kStash = 4 * NH + 4;

}  // namespace

struct ct2g_learn {
  float bw_ext = 0.f;
  int nshell = 0;
  int *d_shell = nullptr;     // [nshell][4]: ox, oy, oz, distance bin
  float *d_shellG = nullptr;  // [nshell][nc]
  float bin_d2[2] = {0.f, 0.f};
  int mode = CT2G_SELECT_NONE;
  float threshold = 0.f;
  // per-cell work arrays, capacity = particle capacity
  size_t cap = 0;
  uint32_t *cells = nullptr;   // occupied cell keys
  uint32_t *flags = nullptr;   // scratch
  uint32_t *scan = nullptr;    // scratch
  uint32_t *d_cnt = nullptr;   // [0] cells [1] selected cells [2] chunks [3] work counter
                               // [4] sinks of the selected cells; widening: [5] dense
                               // chunks [6] their work counter [7] sparse sinks
                               // [4] selected sinks [5] scan total scratch
  // block-walk form of the widening (bwidth_ext <= 4): stencil masks of the
  // shell per (in-block cell, neighbouring block), selected cells and sinks
  unsigned long long *d_stm = nullptr;  // [64][27]
  uint32_t *sel_cells = nullptr;        // [nsel] index into cells
  uint32_t *pflag = nullptr, *pscan = nullptr;  // per particle of the range
  uint32_t *ssink = nullptr, *scell = nullptr;  // [nsink] particle, selected-cell rank
  uint32_t *cflag = nullptr, *cscan = nullptr;  // chunk starts over the sink list
  float *lsub = nullptr;                        // [nsel][nc] mesh terms of the shell
  // compact moments of the occupied cells ([ncell][nc], components
  // contiguous) and the cell key -> record index (~0u: empty cell)
  float *mc = nullptr;
  uint32_t *idx = nullptr;
  size_t idx_cap = 0;
  float *X = nullptr;          // [cap][NIN] features
  float *score = nullptr;      // fixed criterion
  float *pred = nullptr;       // MLP output
  uint8_t *sel = nullptr;      // selected
  uint2 *chunks = nullptr;     // (cell index, first sink << 8 | count)
  uint2 *dchunks = nullptr;    // widening: dense-style chunks of selected dense cells
  uint32_t *ssink2 = nullptr;  // widening: sinks of the selected sparse cells
  float *ex = nullptr, *ey = nullptr, *ez = nullptr;  // widened forces (training)
  // MLP
  float *params = nullptr, *grad = nullptr, *am = nullptr, *av = nullptr;
  __nv_bfloat16 *wbf = nullptr;
  float *fmean = nullptr, *fstd = nullptr;
  bool have_mlp = false;
  int adam_t = 0;
  // training set
  float *tX = nullptr, *tT = nullptr;
  size_t tn = 0, tcap = 0;
  float *stash = nullptr;      // [batch][kStash]
  float *sloss = nullptr;      // [batch]
  uint32_t *tidx = nullptr;    // [tcap] sample order
  size_t stash_cap = 0;
};

namespace {

// ---------------------------------------------------------------------------
// occupied cells of the range: runs of equal sorted keys
// ---------------------------------------------------------------------------
__global__ void run_flag_kernel(const uint32_t *__restrict__ keys, size_t nr,
                                uint32_t *__restrict__ flag) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nr) flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

__global__ void run_list_kernel(const uint32_t *__restrict__ keys, size_t nr,
                                const uint32_t *__restrict__ flag,
                                const uint32_t *__restrict__ scan, uint32_t *__restrict__ cells) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nr && flag[i]) cells[scan[i]] = keys[i];
}

__global__ void cell_index_kernel(const uint32_t *__restrict__ cells,
                                  const uint32_t *__restrict__ cnt, uint32_t *__restrict__ idx) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < cnt[0]) idx[cells[c]] = c;
}

struct CellGeo {
  int mbits;
  uint32_t cmask;  // C - 1
  __device__ __forceinline__ void decode(uint32_t key, uint32_t &box, int &i, int &j, int &k) const {
    box = key >> (3 * mbits);
    const uint32_t m = key & cmask;
    i = (int)ct2g_compact3(m >> 2);
    j = (int)ct2g_compact3(m >> 1);
    k = (int)ct2g_compact3(m);
  }
  __device__ __forceinline__ uint32_t key(uint32_t box, int i, int j, int k) const {
    const int M1 = (1 << mbits) - 1;
    return (box << (3 * mbits)) | ct2g_morton((uint32_t)(i & M1), (uint32_t)(j & M1), (uint32_t)(k & M1));
  }
  __device__ __forceinline__ int64_t rowmajor(uint32_t box, int i, int j, int k) const {
    const int M1 = (1 << mbits) - 1;
    return ((int64_t)box << (3 * mbits)) +
           (((int64_t)(i & M1) << (2 * mbits)) | ((int64_t)(j & M1) << mbits) | (k & M1));
  }
};

// all components of an occupied cell's moments, contiguous
__global__ void compact_moments_kernel(const uint32_t *__restrict__ cells,
                                       const uint32_t *__restrict__ cnt,
                                       const float *__restrict__ grid, int64_t CB, CellGeo geo,
                                       int nc, float *__restrict__ mc) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cnt[0]) return;
  uint32_t box;
  int i, j, k;
  geo.decode(cells[c], box, i, j, k);
  const int64_t r = geo.rowmajor(box, i, j, k);
  for (int q = 0; q < nc; q++) mc[(size_t)c * nc + q] = grid[(int64_t)q * CB + r];
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// features: one warp per occupied cell, lanes over the shell offsets
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(256) features_kernel(
    const uint32_t *__restrict__ cells, const uint32_t *__restrict__ cnt,
    const uint32_t *__restrict__ cs, const float *__restrict__ mc,
    const uint32_t *__restrict__ idx, CellGeo geo, const int *__restrict__ shell, int nshell,
    const float *__restrict__ fx, const float *__restrict__ fy, const float *__restrict__ fz,
    const uint32_t *__restrict__ box_off, const float *__restrict__ box_gm,
    float *__restrict__ X, float *__restrict__ score) {
  constexpr int NC = ct2g_ncomp(P);
  const int lane = threadIdx.x & 31;
  const uint32_t ncell = cnt[0];
  const int M = 1 << geo.mbits;
  const float h = 1.0f / (float)M;
  constexpr int i200 = ct2g_mi_index(2, 0, 0), i020 = ct2g_mi_index(0, 2, 0),
                i002 = ct2g_mi_index(0, 0, 2);
  constexpr int i100 = ct2g_mi_index(1, 0, 0), i010 = ct2g_mi_index(0, 1, 0),
                i001 = ct2g_mi_index(0, 0, 1);
  for (uint32_t ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < ncell;
       ci += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t key = cells[ci];
    uint32_t box;
    int ix, iy, iz;
    geo.decode(key, box, ix, iy, iz);
    const uint32_t c0 = cs[key], c1 = cs[key + 1];
    const float nc = (float)(c1 - c0);
    const float GM = box_gm[box];
    const float nbox = (float)(box_off[box + 1] - box_off[box]);
    // sink force magnitudes
    float s1 = 0.f, s2 = 0.f;
    for (uint32_t i = c0 + lane; i < c1; i += 32) {
      const float f = sqrtf(fx[i] * fx[i] + fy[i] * fy[i] + fz[i] * fz[i]);
      s1 += f;
      s2 += f * f;
    }
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    const float fmean = fmaxf(s1 / nc, 1e-30f);
    const float fstdv = sqrtf(fmaxf(s2 / nc - fmean * fmean, 0.f));
    const float *mo = mc + (size_t)ci * NC;
    const float sig_c = sqrtf(fmaxf(2.f * (mo[i200] + mo[i020] + mo[i002]) / nc, 0.f));
    const float dip = sqrtf(mo[i100] * mo[i100] + mo[i010] * mo[i010] + mo[i001] * mo[i001]) / nc;
    // shell sums per distance bin
    float cntb[3] = {0.f, 0.f, 0.f}, mono[3] = {0.f, 0.f, 0.f}, quad[3] = {0.f, 0.f, 0.f},
          trunc[3] = {0.f, 0.f, 0.f};
    float monop = 0.f, maxn = 0.f, px = 0.f, py = 0.f, pz = 0.f;
    for (int s = lane; s < nshell; s += 32) {
      const int4 o = reinterpret_cast<const int4 *>(shell)[s];
      const uint32_t k2 = geo.key(box, ix + o.x, iy + o.y, iz + o.z);
      const uint32_t c2 = idx[k2];
      if (c2 == ~0u) continue;
      const float ns = (float)(cs[k2 + 1] - cs[k2]);
      const float *m2 = mc + (size_t)c2 * NC;
      const float sig2 = fmaxf(2.f * (m2[i200] + m2[i020] + m2[i002]) / ns, 0.f);
      const float R2 = (float)(o.x * o.x + o.y * o.y + o.z * o.z) * h * h;
      const float R = sqrtf(R2);
      const float m = ns / R2;
      float tr = m;
      const float q = sqrtf(sig2) / R;
#pragma unroll
      for (int e = 0; e <= P; e++) tr *= q;  // n sigma^(p+1) / R^(p+3)
      float tp = ns / R2;
#pragma unroll
      for (int e = 0; e <= P; e++) tp /= R;  // n / R^(p+3)
      const int b = o.w;
      cntb[b] += ns;
      mono[b] += m;
      quad[b] += m * sig2 / R2;
      trunc[b] += tr;
      monop += tp;
      maxn = fmaxf(maxn, ns);
      const float w = m * h / R;  // monopole pull along the unit vector o / |o|
      px = fmaf(w, (float)o.x, px);
      py = fmaf(w, (float)o.y, py);
      pz = fmaf(w, (float)o.z, pz);
    }
#pragma unroll
    for (int b = 0; b < 3; b++) {
      cntb[b] = warp_sum(cntb[b]);
      mono[b] = warp_sum(mono[b]);
      quad[b] = warp_sum(quad[b]);
      trunc[b] = warp_sum(trunc[b]);
    }
    monop = warp_sum(monop);
    px = warp_sum(px);
    py = warp_sum(py);
    pz = warp_sum(pz);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxn = fmaxf(maxn, __shfl_xor_sync(0xffffffffu, maxn, o));
    if (lane == 0) {
      float *x = X + (size_t)ci * NIN;
      const float inv = GM / fmean;
      const float mono_all = mono[0] + mono[1] + mono[2];
      const float cnt_all = cntb[0] + cntb[1] + cntb[2];
      float sp = sig_c;
#pragma unroll
      for (int e = 0; e < P; e++) sp *= sig_c;  // sigma_c^(p+1)
      x[0] = log2f(1.f + nc);
      x[1] = log10f(fmean / (GM * nbox * (float)M * (float)M) + 1e-30f);
      x[2] = fstdv / fmean;
      x[3] = sig_c / h;
      x[4] = dip / h;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        x[5 + b] = log2f(1.f + cntb[b]);
        x[8 + b] = log10f(inv * mono[b] + 1e-12f);
        x[11 + b] = log10f(inv * quad[b] + 1e-14f);
        x[14 + b] = log10f(inv * trunc[b] + 1e-16f);
      }
      x[17] = log10f(inv * sp * monop + 1e-16f);
      x[18] = log2f(1.f + maxn);
      // one-sidedness of the shell's pull: |sum n o/|o| / R^2| / sum n / R^2
      x[19] = mono_all > 0.f ? fminf(sqrtf(px * px + py * py + pz * pz) / mono_all, 1.f) : 0.f;
      x[20] = log10f(inv * mono_all + 1e-12f);
      x[21] = (float)geo.mbits / 10.f;
      x[22] = (c1 - c0 == 1) ? 1.f : 0.f;
      x[23] = cntb[0] / (cnt_all + 1.f);
      score[ci] = inv * mono_all;
    }
  }
}

// ---------------------------------------------------------------------------
// MLP
// ---------------------------------------------------------------------------
// forward of one normalised sample with weights w (FP32 values of BF16s).
// Every loop is unrolled, so the activations stay in registers.
__device__ __forceinline__ float mlp_forward(const float *__restrict__ w, const float *x) {
  float h1[NH];
#pragma unroll
  for (int j = 0; j < NH; j++) {
    float a = w[OB1 + j];
#pragma unroll
    for (int i = 0; i < NIN; i++) a = fmaf(w[OW1 + j * NIN + i], x[i], a);
    h1[j] = fmaxf(a, 0.f);
  }
  float y = w[OB3];
#pragma unroll 1
  for (int j = 0; j < NH; j++) {
    float a = w[OB2 + j];
#pragma unroll
    for (int k = 0; k < NH; k++) a = fmaf(w[OW2 + j * NH + k], h1[k], a);
    y = fmaf(w[OW3 + j], fmaxf(a, 0.f), y);
  }
  return y;
}

__device__ __forceinline__ void load_weights(float *ws, const __nv_bfloat16 *__restrict__ wbf) {
  for (int i = threadIdx.x; i < NP; i += blockDim.x) ws[i] = __bfloat162float(wbf[i]);
  __syncthreads();
}

__global__ void __launch_bounds__(256) mlp_infer_kernel(
    const __nv_bfloat16 *__restrict__ wbf, const float *__restrict__ fmean,
    const float *__restrict__ fstd, const float *__restrict__ X,
    const uint32_t *__restrict__ cnt, float *__restrict__ pred) {
  extern __shared__ float ws[];
  load_weights(ws, wbf);
  const uint32_t n = cnt[0];
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    // keeps the weight loads inside the loop (hoisted, they would not fit
    // in registers)
    asm volatile("" ::: "memory");
    float x[NIN];
#pragma unroll
    for (int i = 0; i < NIN; i++) x[i] = (X[(size_t)c * NIN + i] - fmean[i]) / fstd[i];
    pred[c] = mlp_forward(ws, x);
  }
}

// forward + backward of samples idx[start .. start+count): per sample the
// hidden activations and the errors go to the stash (h1 | dz1 | h2 | dz2 |
// dy), the squared error to sloss.  dL/dy = 2 (y - t) / count (mean squared
// error); the ReLU derivatives are kept as bit masks.
__global__ void __launch_bounds__(128) mlp_fwdbwd_kernel(
    const __nv_bfloat16 *__restrict__ wbf, const float *__restrict__ fmean,
    const float *__restrict__ fstd, const float *__restrict__ X, const float *__restrict__ T,
    const uint32_t *__restrict__ idx, size_t start, int count, float *__restrict__ stash,
    float *__restrict__ sloss) {
  extern __shared__ float ws[];
  load_weights(ws, wbf);
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count) return;
  const uint32_t q = idx[start + s];
  float x[NIN];
#pragma unroll
  for (int i = 0; i < NIN; i++) x[i] = (X[(size_t)q * NIN + i] - fmean[i]) / fstd[i];
  float *st = stash + (size_t)s * kStash;
  float h1[NH];
  unsigned long long m1 = 0ull, m2 = 0ull;
#pragma unroll
  for (int j = 0; j < NH; j++) {
    float a = ws[OB1 + j];
#pragma unroll
    for (int i = 0; i < NIN; i++) a = fmaf(ws[OW1 + j * NIN + i], x[i], a);
    h1[j] = fmaxf(a, 0.f);
    if (a > 0.f) m1 |= 1ull << j;
    st[j] = h1[j];
  }
  float y = ws[OB3];
#pragma unroll 1
  for (int j = 0; j < NH; j++) {
    float a = ws[OB2 + j];
#pragma unroll
    for (int k = 0; k < NH; k++) a = fmaf(ws[OW2 + j * NH + k], h1[k], a);
    if (a > 0.f) m2 |= 1ull << j;
    st[2 * NH + j] = fmaxf(a, 0.f);
    y = fmaf(ws[OW3 + j], fmaxf(a, 0.f), y);
  }
  const float e = y - T[q];
  sloss[s] = e * e;
  const float dy = 2.f * e / (float)count;
  st[4 * NH] = dy;
  float dz1[NH];
#pragma unroll
  for (int k = 0; k < NH; k++) dz1[k] = 0.f;
#pragma unroll 1
  for (int j = 0; j < NH; j++) {
    const float dz2 = ((m2 >> j) & 1ull) ? dy * ws[OW3 + j] : 0.f;
    st[3 * NH + j] = dz2;
#pragma unroll
    for (int k = 0; k < NH; k++) dz1[k] = fmaf(ws[OW2 + j * NH + k], dz2, dz1[k]);
  }
#pragma unroll
  for (int k = 0; k < NH; k++) st[NH + k] = ((m1 >> k) & 1ull) ? dz1[k] : 0.f;
}

// weight gradients, one thread per parameter, summed over the batch in a
// fixed order (deterministic)
__global__ void mlp_wgrad_kernel(const float *__restrict__ fmean, const float *__restrict__ fstd,
                                 const float *__restrict__ X, const uint32_t *__restrict__ idx,
                                 size_t start, int count, const float *__restrict__ stash,
                                 float *__restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NP) return;
  float g = 0.f;
  if (p < OB1) {
    const int j = p / NIN, i = p % NIN;
    const float m = fmean[i], sd = fstd[i];
    for (int s = 0; s < count; s++) {
      const float x = (X[(size_t)idx[start + s] * NIN + i] - m) / sd;
      g = fmaf(stash[(size_t)s * kStash + NH + j], x, g);
    }
  } else if (p < OW2) {
    const int j = p - OB1;
    for (int s = 0; s < count; s++) g += stash[(size_t)s * kStash + NH + j];
  } else if (p < OB2) {
    const int j = (p - OW2) / NH, k = (p - OW2) % NH;
    for (int s = 0; s < count; s++)
      g = fmaf(stash[(size_t)s * kStash + 3 * NH + j], stash[(size_t)s * kStash + k], g);
  } else if (p < OW3) {
    const int j = p - OB2;
    for (int s = 0; s < count; s++) g += stash[(size_t)s * kStash + 3 * NH + j];
  } else if (p < OB3) {
    const int k = p - OW3;
    for (int s = 0; s < count; s++)
      g = fmaf(stash[(size_t)s * kStash + 4 * NH], stash[(size_t)s * kStash + 2 * NH + k], g);
  } else {
    for (int s = 0; s < count; s++) g += stash[(size_t)s * kStash + 4 * NH];
  }
  grad[p] = g;
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------
// selection and correction chunks
// ---------------------------------------------------------------------------
__global__ void select_kernel(const uint32_t *__restrict__ cells, const uint32_t *__restrict__ cnt,
                              const uint32_t *__restrict__ cs, const float *__restrict__ score,
                              const float *__restrict__ pred, int mode, float thr,
                              uint32_t *__restrict__ nchunk, uint8_t *__restrict__ sel,
                              uint32_t *__restrict__ nsel) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cnt[0]) return;
  bool s = false;
  if (mode == CT2G_SELECT_ALL) s = true;
  else if (mode == CT2G_SELECT_FIXED) s = score[c] > thr;
  else if (mode == CT2G_SELECT_MLP) s = pred[c] > thr;
  const uint32_t key = cells[c];
  const uint32_t n = cs[key + 1] - cs[key];
  nchunk[c] = s ? (n + 31) / 32 : 0u;
  sel[c] = s ? 1 : 0;
  if (s) atomicAdd(nsel, 1u);
}

__global__ void chunk_list_kernel(const uint32_t *__restrict__ cells,
                                  const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ cs,
                                  const uint32_t *__restrict__ nchunk,
                                  const uint32_t *__restrict__ first, uint2 *__restrict__ chunks) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cnt[0] || !nchunk[c]) return;
  const uint32_t key = cells[c];
  const uint32_t n = cs[key + 1] - cs[key];
  for (uint32_t j = 0; j < nchunk[c]; j++)
    chunks[first[c] + j] = make_uint2(c, ((32u * j) << 8) | min(32u, n - 32u * j));
}

// ---- block-walk widening (bwidth_ext <= 4) ---------------------------------
// selected cells -> 0/1 flags over the range's upper bound (scan: rank)
__global__ void sel_flag_kernel(const uint32_t *__restrict__ cnt, const uint8_t *__restrict__ sel,
                                size_t nr, uint32_t *__restrict__ flag) {
  const size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nr) flag[c] = (c < cnt[0] && sel[c]) ? 1u : 0u;
}

__global__ void sel_list_kernel(const uint32_t *__restrict__ cnt, const uint8_t *__restrict__ sel,
                                const uint32_t *__restrict__ rank, uint32_t *__restrict__ sel_cells) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < cnt[0] && sel[c]) sel_cells[rank[c]] = c;
}

// particles of the selected cells (one thread per selected cell)
__global__ void sink_flag_kernel(const uint32_t *__restrict__ cnt,
                                 const uint32_t *__restrict__ sel_cells,
                                 const uint32_t *__restrict__ cells, const uint32_t *__restrict__ cs,
                                 uint32_t begin, uint32_t *__restrict__ pflag) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cnt[1]) return;
  const uint32_t key = cells[sel_cells[j]];
  for (uint32_t i = cs[key]; i < cs[key + 1]; i++) pflag[i - begin] = 1u;
}

__global__ void sink_list_kernel(const uint32_t *__restrict__ cnt,
                                 const uint32_t *__restrict__ sel_cells,
                                 const uint32_t *__restrict__ cells, const uint32_t *__restrict__ cs,
                                 uint32_t begin, const uint32_t *__restrict__ pscan,
                                 uint32_t *__restrict__ ssink, uint32_t *__restrict__ scell) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cnt[1]) return;
  const uint32_t key = cells[sel_cells[j]];
  for (uint32_t i = cs[key]; i < cs[key + 1]; i++) {
    const uint32_t q = pscan[i - begin];
    ssink[q] = i;
    scell[q] = j;
  }
}

// chunk starts over the sink list: the first selected sink of every 4x4x4
// cell block and every 32nd one after it
__global__ void sink_chunk_flag_kernel(const uint32_t *__restrict__ keys,
                                       const uint32_t *__restrict__ cs,
                                       const uint32_t *__restrict__ pflag,
                                       const uint32_t *__restrict__ pscan, uint32_t begin,
                                       size_t nr, uint32_t *__restrict__ cflag) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr || !pflag[i]) return;
  const uint32_t q = pscan[i];
  const uint32_t f = cs[keys[i] & ~63u] - begin;  // first particle of the block (<= i)
  cflag[q] = ((q - pscan[f]) % 32u) == 0u ? 1u : 0u;
}

__global__ void sink_chunk_fill_kernel(const uint32_t *__restrict__ nsink_ptr,
                                       const uint32_t *__restrict__ cflag,
                                       const uint32_t *__restrict__ cscan,
                                       const uint32_t *__restrict__ ssink,
                                       const uint32_t *__restrict__ keys,
                                       const uint32_t *__restrict__ cs,
                                       const uint32_t *__restrict__ pscan, uint32_t begin,
                                       size_t nr, uint2 *__restrict__ chunks) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nsink = *nsink_ptr;
  if (q >= nsink || !cflag[q]) return;
  const uint32_t i = ssink[q] - begin;
  const uint32_t e = cs[(keys[i] | 63u) + 1] - begin;  // past the block
  const uint32_t qe = e < nr ? pscan[e] : nsink;
  chunks[cscan[q]] = make_uint2(q, min(32u, qe - q));
}

// the selected cells' sinks for the widened direct sum: cells of at least
// dense_cell particles as dense-style chunks (every 32nd particle of the cell
// starts one: dflag), the rest listed one by one (sflag)
__global__ void shell_split_kernel(const uint32_t *__restrict__ cnt,
                                   const uint32_t *__restrict__ sel_cells,
                                   const uint32_t *__restrict__ cells,
                                   const uint32_t *__restrict__ cs, uint32_t begin,
                                   uint32_t dense_cell, uint32_t *__restrict__ dflag,
                                   uint32_t *__restrict__ sflag) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cnt[1]) return;
  const uint32_t key = cells[sel_cells[j]];
  const uint32_t c0 = cs[key], c1 = cs[key + 1];
  if (c1 - c0 >= dense_cell) {
    for (uint32_t i = c0; i < c1; i += 32) dflag[i - begin] = 1u;
  } else {
    for (uint32_t i = c0; i < c1; i++) sflag[i - begin] = 1u;
  }
}

// (first particle, count) of each dense-style chunk
__global__ void shell_dense_fill_kernel(const uint32_t *__restrict__ dflag,
                                        const uint32_t *__restrict__ dscan,
                                        const uint32_t *__restrict__ keys,
                                        const uint32_t *__restrict__ cs, uint32_t begin, size_t nr,
                                        uint2 *__restrict__ list) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr || !dflag[i]) return;
  const uint32_t g = begin + (uint32_t)i;
  list[dscan[i]] = make_uint2(g, min(32u, cs[keys[i] + 1] - g));
}

// the listed (sparse) sinks, in particle order
__global__ void shell_sparse_list_kernel(const uint32_t *__restrict__ sflag,
                                         const uint32_t *__restrict__ sscan, uint32_t begin,
                                         size_t nr, uint32_t *__restrict__ list) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nr && sflag[i]) list[sscan[i]] = begin + (uint32_t)i;
}

// the mesh's Taylor term of the shell, once per selected cell: warp per
// cell, lanes over the shell offsets
template <int P>
__global__ void __launch_bounds__(256) shell_m2l_kernel(
    const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ sel_cells,
    const uint32_t *__restrict__ cells, const float *__restrict__ mc,
    const uint32_t *__restrict__ idx, CellGeo geo, const int *__restrict__ shell,
    const float *__restrict__ shellG, int nshell, float *__restrict__ lsub) {
  constexpr int NC = ct2g_ncomp(P);
  constexpr Mg2lPairs<P> T{};
  const int lane = threadIdx.x & 31;
  const uint32_t nsel = cnt[1];
  for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nsel;
       j += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t key = cells[sel_cells[j]];
    uint32_t box;
    int ix, iy, iz;
    geo.decode(key, box, ix, iy, iz);
    float L[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) L[k] = 0.f;
    for (int s = lane; s < nshell; s += 32) {
      const int4 o = reinterpret_cast<const int4 *>(shell)[s];
      const uint32_t c2 = idx[geo.key(box, ix + o.x, iy + o.y, iz + o.z)];
      if (c2 == ~0u) continue;
      float Mv[NC];
#pragma unroll
      for (int k = 0; k < NC; k++) Mv[k] = mc[(size_t)c2 * NC + k];
      const float *G = shellG + (size_t)s * NC;
#pragma unroll
      for (int q = 0; q < Mg2lPairs<P>::NP; q++) L[T.a[q]] = fmaf(__ldg(G + T.ab[q]), Mv[T.b[q]], L[T.a[q]]);
    }
#pragma unroll
    for (int k = 0; k < NC; k++) L[k] = warp_sum(L[k]);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < NC; k++) lsub[(size_t)j * NC + k] = L[k];
  }
}

// removes the shell's mesh term from every selected sink
template <int P, bool POT>
__global__ void shell_l2p_kernel(const uint32_t *__restrict__ cnt, const uint32_t *__restrict__ ssink,
                                 const uint32_t *__restrict__ scell, const uint32_t *__restrict__ keys,
                                 uint32_t begin, int mbits, const float4 *__restrict__ src,
                                 const float *__restrict__ lsub, const float *__restrict__ box_gm,
                                 float *__restrict__ ofx, float *__restrict__ ofy,
                                 float *__restrict__ ofz, float *__restrict__ opot) {
  constexpr int NC = ct2g_ncomp(P);
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cnt[4]) return;
  const uint32_t i = ssink[q];
  const float *Lc = lsub + (size_t)scell[q] * NC;
  const float4 t = src[i];
  const float GM = box_gm[keys[i - begin] >> (3 * mbits)];
  float fx, fy, fz, ph;
  ct2g_l2p<P>([&](int k) { return __ldg(Lc + k); }, t.x, t.y, t.z, fx, fy, fz, ph);
  ofx[i] -= GM * fx;
  ofy[i] -= GM * fy;
  ofz[i] -= GM * fz;
  if (POT) opot[i] -= GM * ph;
}

// Shell correction, one warp per chunk of <= 32 sinks of a selected cell,
// persistent over the device-held chunk count (cnt[2], work counter cnt[3]).
// Lanes walk the shell offsets 32 at a time: each lane adds its source
// cell's Taylor term to a lane-partial expansion, then the warp sums the
// cells' particles directly (sources staged in shared memory, broadcast).
template <int P, int KERNEL, bool POT>
__global__ void __launch_bounds__(256) shell_kernel(
    const uint2 *__restrict__ chunks, uint32_t *__restrict__ cnt,
    const uint32_t *__restrict__ cells, const uint32_t *__restrict__ cs,
    const float4 *__restrict__ src, const float *__restrict__ grid, int64_t CB, CellGeo geo,
    const int *__restrict__ shell, const float *__restrict__ shellG, int nshell, float soft,
    const float *__restrict__ box_gm, float *__restrict__ ofx, float *__restrict__ ofy,
    float *__restrict__ ofz, float *__restrict__ opot) {
  constexpr int NC = ct2g_ncomp(P);
  constexpr Mg2lPairs<P> T{};
  __shared__ float4 sbuf[8][32];
  const int lane = threadIdx.x & 31;
  float4 *sb = sbuf[threadIdx.x >> 5];
  const uint32_t nch = cnt[2];
  const float hc = 1.0f / (float)(1 << geo.mbits);
  const float h2 = soft * soft, hinv = 1.f / soft, hinv3 = hinv * hinv * hinv;
  for (;;) {
    uint32_t ch = 0;
    if (lane == 0) ch = atomicAdd(cnt + 3, 1u);
    ch = __shfl_sync(0xffffffffu, ch, 0);
    if (ch >= nch) break;
    const uint2 cd = chunks[ch];
    const uint32_t key = cells[cd.x];
    uint32_t box;
    int ix, iy, iz;
    geo.decode(key, box, ix, iy, iz);
    const uint32_t count = cd.y & 255u, first = cd.y >> 8;
    const bool act = (uint32_t)lane < count;
    const uint32_t i = cs[key] + first + (act ? (uint32_t)lane : 0u);
    const float4 si = src[i];
    const float GM = box_gm[box];
    float L[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) L[k] = 0.f;
    float nx = 0.f, ny = 0.f, nz = 0.f, np = 0.f;
    for (int g0 = 0; g0 < nshell; g0 += 32) {
      const int s = g0 + lane;
      int4 o = make_int4(0, 0, 0, 0);
      uint32_t jb = 0, je = 0;
      if (s < nshell) {
        o = reinterpret_cast<const int4 *>(shell)[s];
        const uint32_t k2 = geo.key(box, ix + o.x, iy + o.y, iz + o.z);
        jb = cs[k2];
        je = cs[k2 + 1];
      }
      if (je > jb) {
        // the mesh's primary-image term of this source cell
        const int64_t r2c = geo.rowmajor(box, ix + o.x, iy + o.y, iz + o.z);
        float Mv[NC];
#pragma unroll
        for (int k = 0; k < NC; k++) Mv[k] = grid[(int64_t)k * CB + r2c];
        const float *G = shellG + (size_t)s * NC;
#pragma unroll
        for (int q = 0; q < Mg2lPairs<P>::NP; q++) L[T.a[q]] = fmaf(__ldg(G + T.ab[q]), Mv[T.b[q]], L[T.a[q]]);
      }
      unsigned hb = __ballot_sync(0xffffffffu, je > jb);
      while (hb) {
        const int t = __ffs(hb) - 1;
        hb &= hb - 1;
        const uint32_t j0 = __shfl_sync(0xffffffffu, jb, t), j1 = __shfl_sync(0xffffffffu, je, t);
        const int ox = __shfl_sync(0xffffffffu, o.x, t), oy = __shfl_sync(0xffffffffu, o.y, t),
                  oz = __shfl_sync(0xffffffffu, o.z, t);
        const float xs = si.x - (float)ox * hc, ys = si.y - (float)oy * hc,
                    zs = si.z - (float)oz * hc;
        float4 nxt = __ldg(src + min(j0 + lane, j1 - 1));
        for (uint32_t jj = j0; jj < j1; jj += 32) {
          const int cn = (int)min(32u, j1 - jj);
          __syncwarp();
          sb[lane] = nxt;
          __syncwarp();
          if (jj + 32 < j1) nxt = __ldg(src + min(jj + 32 + lane, j1 - 1));
#pragma unroll 4
          for (int u = 0; u < cn; u++) {
            const float4 q = sb[u];
            ct2g_pair_term<KERNEL, POT>(xs - q.x, ys - q.y, zs - q.z, h2, hinv, hinv3, nx, ny,
                                        nz, np, true);
          }
        }
      }
    }
#pragma unroll
    for (int k = 0; k < NC; k++) L[k] = warp_sum(L[k]);
    if (act) {
      float fx, fy, fz, ph;
      ct2g_l2p<P>([&](int k) { return L[k]; }, si.x, si.y, si.z, fx, fy, fz, ph);
      ofx[i] += GM * (nx - fx);
      ofy[i] += GM * (ny - fy);
      ofz[i] += GM * (nz - fz);
      if (POT) opot[i] += GM * (np - ph);
    }
  }
}

// per-cell target: log10 of the rms over the cell's sinks of
// |F_wide - F_plain| / |F_wide|
__global__ void target_kernel(const uint32_t *__restrict__ cells, const uint32_t *__restrict__ cnt,
                              const uint32_t *__restrict__ cs, const float *__restrict__ fx,
                              const float *__restrict__ fy, const float *__restrict__ fz,
                              const float *__restrict__ ex, const float *__restrict__ ey,
                              const float *__restrict__ ez, float *__restrict__ T) {
  const int lane = threadIdx.x & 31;
  const uint32_t ncell = cnt[0];
  for (uint32_t ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < ncell;
       ci += (gridDim.x * blockDim.x) >> 5) {
    const uint32_t key = cells[ci];
    const uint32_t c0 = cs[key], c1 = cs[key + 1];
    float acc = 0.f;
    for (uint32_t i = c0 + lane; i < c1; i += 32) {
      const float dx = ex[i] - fx[i], dy = ey[i] - fy[i], dz = ez[i] - fz[i];
      const float w2 = ex[i] * ex[i] + ey[i] * ey[i] + ez[i] * ez[i];
      acc += (dx * dx + dy * dy + dz * dz) / fmaxf(w2, 1e-30f);
    }
    acc = warp_sum(acc);
    if (lane == 0) T[ci] = log10f(fmaxf(sqrtf(acc / (float)(c1 - c0)), 1e-10f));
  }
}

// per-feature mean and standard deviation of the training set (one block
// per feature, fixed summation order)
__global__ void norm_stats_kernel(const float *__restrict__ X, size_t n, float *__restrict__ mean,
                                  float *__restrict__ sdev) {
  __shared__ double s1[256], s2[256];
  const int f = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (size_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double v = X[i * NIN + f];
    a += v;
    b += v * v;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double m = s1[0] / (double)n;
    const double v = s2[0] / (double)n - m * m;
    mean[f] = (float)m;
    sdev[f] = (float)fmax(sqrt(fmax(v, 0.0)), 1e-6);
  }
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, __nv_bfloat16 *__restrict__ wbf, float lr,
                            float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NP) return;
  const float b1 = 0.9f, b2 = 0.999f;
  m[i] = b1 * m[i] + (1.f - b1) * g[i];
  v[i] = b2 * v[i] + (1.f - b2) * g[i] * g[i];
  p[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + 1e-8f);
  wbf[i] = __float2bfloat16_rn(p[i]);
}

__global__ void to_bf16_kernel(const float *__restrict__ p, __nv_bfloat16 *__restrict__ w, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = __float2bfloat16_rn(p[i]);
}

__global__ void loss_sum_kernel(const float *__restrict__ l, int n, float *__restrict__ out) {
  __shared__ float s[256];
  float a = 0.f;
  for (int i = threadIdx.x; i < n; i += 256) a += l[i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0] / (float)n;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
int free_learn_cells(ct2g_learn *L) {
  void *ptrs[] = {L->cells, L->flags, L->scan, L->X, L->score, L->pred, L->sel, L->chunks,
                  L->ex, L->ey, L->ez, L->sel_cells, L->pflag, L->pscan, L->ssink, L->scell,
                  L->cflag, L->cscan, L->lsub, L->dchunks, L->ssink2};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  L->sel_cells = L->pflag = L->pscan = L->ssink = L->scell = L->cflag = L->cscan = nullptr;
  L->dchunks = nullptr;
  L->ssink2 = nullptr;
  L->lsub = nullptr;
  if (L->mc) cudaFree(L->mc);
  L->mc = nullptr;
  L->cells = L->flags = L->scan = nullptr;
  L->X = L->score = L->pred = L->ex = L->ey = L->ez = nullptr;
  L->sel = nullptr;
  L->chunks = nullptr;
  L->cap = 0;
  return CT2G_OK;
}

int learn_cells_alloc(ct2g_ctx *ctx) {
  ct2g_learn *L = ctx->learn;
  const size_t cap = std::max<size_t>(ctx->cap, 1);
  if (L->cap >= cap) return CT2G_OK;
  free_learn_cells(L);
#define A(ptr, bytes) CT2G_CUDA(ctx, cudaMalloc(&(ptr), (bytes)))
  A(L->cells, cap * 4);
  A(L->flags, cap * 4);
  A(L->scan, cap * 4);
  A(L->X, cap * NIN * 4);
  A(L->score, cap * 4);
  A(L->pred, cap * 4);
  A(L->sel, cap);
  A(L->chunks, cap * sizeof(uint2));
  A(L->dchunks, cap * sizeof(uint2));
  A(L->ssink2, cap * 4);
  A(L->ex, cap * 4);
  A(L->ey, cap * 4);
  A(L->ez, cap * 4);
  A(L->sel_cells, cap * 4);
  A(L->pflag, cap * 4);
  A(L->pscan, cap * 4);
  A(L->ssink, cap * 4);
  A(L->scell, cap * 4);
  A(L->cflag, cap * 4);
  A(L->cscan, cap * 4);
  A(L->lsub, cap * sizeof(float) * ctx->nc);
  A(L->mc, cap * sizeof(float) * ctx->nc);
  if (L->idx_cap < (size_t)ctx->CB) {
    if (L->idx) cudaFree(L->idx);
    L->idx = nullptr;
    L->idx_cap = 0;
    A(L->idx, sizeof(uint32_t) * (size_t)ctx->CB);
    L->idx_cap = (size_t)ctx->CB;
  }
#undef A
  L->cap = cap;
  ctx->epoch++;
  return CT2G_OK;
}

CellGeo geo_of(const ct2g_ctx *ctx) {
  return CellGeo{ctx->mbits, (uint32_t)(ctx->C - 1)};
}

// occupied cells of the range -> L->cells, count in L->d_cnt[0]
int occupied_cells(ct2g_ctx *ctx) {
  ct2g_learn *L = ctx->learn;
  const size_t nr = ctx->n - ctx->rung_begin;
  cudaStream_t st = ctx->stream;
  CT2G_CUDA(ctx, cudaMemsetAsync(L->d_cnt, 0, sizeof(uint32_t) * 4, st));
  if (nr == 0) return CT2G_OK;
  run_flag_kernel<<<ct2g_div_up(nr, 256), 256, 0, st>>>(ctx->keys, nr, L->flags);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, L->flags, L->scan, nr, L->d_cnt, 0));
  run_list_kernel<<<ct2g_div_up(nr, 256), 256, 0, st>>>(ctx->keys, nr, L->flags, L->scan, L->cells);
  CT2G_LAUNCHED(ctx);
  // key -> record index and the compact moment records
  CT2G_CUDA(ctx, cudaMemsetAsync(L->idx, 0xFF, sizeof(uint32_t) * (size_t)ctx->CB, st));
  cell_index_kernel<<<ct2g_div_up(nr, 256), 256, 0, st>>>(L->cells, L->d_cnt, L->idx);
  CT2G_LAUNCHED(ctx);
  compact_moments_kernel<<<ct2g_div_up(nr, 256), 256, 0, st>>>(L->cells, L->d_cnt, ctx->grid,
                                                               ctx->CB, geo_of(ctx), ctx->nc,
                                                               L->mc);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

unsigned warp_grid(ct2g_ctx *ctx, size_t nitems) {
  // warps per item, at most 16 blocks of 256 threads per SM
  const size_t blocks = std::min<size_t>((nitems + 7) / 8, (size_t)ctx->num_sms * 16);
  return (unsigned)std::max<size_t>(blocks, 1);
}

template <int P>
int launch_features(ct2g_ctx *ctx, const float *fx, const float *fy, const float *fz) {
  ct2g_learn *L = ctx->learn;
  const size_t nr = ctx->n - ctx->rung_begin;
  features_kernel<P><<<warp_grid(ctx, nr), 256, 0, ctx->stream>>>(
      L->cells, L->d_cnt, ctx->cell_start, L->mc, L->idx, geo_of(ctx), L->d_shell, L->nshell,
      fx, fy, fz, ctx->box_off, ctx->box_gm, L->X, L->score);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

int features(ct2g_ctx *ctx, const float *fx, const float *fy, const float *fz) {
  switch (ctx->p) {
    case 1: return launch_features<1>(ctx, fx, fy, fz);
    case 2: return launch_features<2>(ctx, fx, fy, fz);
    case 3: return launch_features<3>(ctx, fx, fy, fz);
    case 4: return launch_features<4>(ctx, fx, fy, fz);
    case 5: return launch_features<5>(ctx, fx, fy, fz);
    case 6: return launch_features<6>(ctx, fx, fy, fz);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "unsupported order");
}

int infer(ct2g_ctx *ctx) {
  ct2g_learn *L = ctx->learn;
  const size_t nr = ctx->n - ctx->rung_begin;
  const size_t smem = sizeof(float) * NP;
  CT2G_TRY(ct2g_smem_attrs(ctx, mlp_infer_kernel, smem));
  const unsigned blocks = (unsigned)std::max<size_t>(
      1, std::min<size_t>((nr + 255) / 256, (size_t)ctx->num_sms * 4));
  mlp_infer_kernel<<<blocks, 256, smem, ctx->stream>>>(L->wbf, L->fmean, L->fstd, L->X, L->d_cnt,
                                                       L->pred);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// selection (count in d_cnt[1]); with `lists`, the per-cell chunk list of
// the cell-walk form too (count in d_cnt[2]); work counter d_cnt[3] reset
int build_chunks(ct2g_ctx *ctx, int mode, float thr, bool lists) {
  ct2g_learn *L = ctx->learn;
  const size_t nr = ctx->n - ctx->rung_begin;
  cudaStream_t st = ctx->stream;
  CT2G_CUDA(ctx, cudaMemsetAsync(L->d_cnt + 1, 0, sizeof(uint32_t) * 3, st));
  if (nr == 0) return CT2G_OK;
  CT2G_CUDA(ctx, cudaMemsetAsync(L->flags, 0, sizeof(uint32_t) * nr, st));
  select_kernel<<<ct2g_div_up(nr, 256), 256, 0, st>>>(L->cells, L->d_cnt, ctx->cell_start,
                                                      L->score, L->pred, mode, thr, L->flags,
                                                      L->sel, L->d_cnt + 1);
  CT2G_LAUNCHED(ctx);
  if (!lists) return CT2G_OK;
  CT2G_TRY(ct2g_scan_exclusive(ctx, L->flags, L->scan, nr, L->d_cnt + 2, 0));
  chunk_list_kernel<<<ct2g_div_up(nr, 256), 256, 0, st>>>(L->cells, L->d_cnt, ctx->cell_start,
                                                          L->flags, L->scan, L->chunks);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

template <int P, int K, bool POT>
int launch_shell1(ct2g_ctx *ctx, float *fx, float *fy, float *fz, float *pot) {
  ct2g_learn *L = ctx->learn;
  auto k = shell_kernel<P, K, POT>;
  int per_sm = 0;
  CT2G_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, 0));
  const size_t nr = ctx->n - ctx->rung_begin;
  const size_t blocks = std::max<size_t>(
      1, std::min<size_t>((size_t)std::max(1, per_sm) * ctx->num_sms, (nr + 255) / 256));
  k<<<(unsigned)blocks, 256, 0, ctx->stream>>>(
      L->chunks, L->d_cnt, L->cells, ctx->cell_start, ctx->src, ctx->grid, ctx->CB, geo_of(ctx),
      L->d_shell, L->d_shellG, L->nshell, ctx->opt.hsoft, ctx->box_gm, fx, fy, fz, pot);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

template <int P>
int launch_shell_p(ct2g_ctx *ctx, bool pot, float *fx, float *fy, float *fz, float *po) {
  if (ctx->opt.kernel == CT2G_SOFT_SPHERE)
    return pot ? launch_shell1<P, CT2G_SOFT_SPHERE, true>(ctx, fx, fy, fz, po)
               : launch_shell1<P, CT2G_SOFT_SPHERE, false>(ctx, fx, fy, fz, po);
  return pot ? launch_shell1<P, CT2G_SOFT_PLUMMER, true>(ctx, fx, fy, fz, po)
             : launch_shell1<P, CT2G_SOFT_PLUMMER, false>(ctx, fx, fy, fz, po);
}

int shell_correct(ct2g_ctx *ctx, bool pot, float *fx, float *fy, float *fz, float *po) {
  switch (ctx->p) {
    case 1: return launch_shell_p<1>(ctx, pot, fx, fy, fz, po);
    case 2: return launch_shell_p<2>(ctx, pot, fx, fy, fz, po);
    case 3: return launch_shell_p<3>(ctx, pot, fx, fy, fz, po);
    case 4: return launch_shell_p<4>(ctx, pot, fx, fy, fz, po);
    case 5: return launch_shell_p<5>(ctx, pot, fx, fy, fz, po);
    case 6: return launch_shell_p<6>(ctx, pot, fx, fy, fz, po);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "unsupported order");
}

template <int P>
int widen_block_p(ct2g_ctx *ctx, bool pot, float *fx, float *fy, float *fz, float *po) {
  ct2g_learn *L = ctx->learn;
  const size_t nr = ctx->n - ctx->rung_begin;
  const uint32_t begin = (uint32_t)ctx->rung_begin;
  cudaStream_t st = ctx->stream;
  const unsigned T = 256, G = ct2g_div_up(nr, T);
  sel_flag_kernel<<<G, T, 0, st>>>(L->d_cnt, L->sel, nr, L->flags);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, L->flags, L->scan, nr, L->d_cnt + 1, 0));
  sel_list_kernel<<<G, T, 0, st>>>(L->d_cnt, L->sel, L->scan, L->sel_cells);
  CT2G_LAUNCHED(ctx);
  CT2G_CUDA(ctx, cudaMemsetAsync(L->pflag, 0, sizeof(uint32_t) * nr, st));
  sink_flag_kernel<<<G, T, 0, st>>>(L->d_cnt, L->sel_cells, L->cells, ctx->cell_start, begin,
                                    L->pflag);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, L->pflag, L->pscan, nr, L->d_cnt + 4, 0));
  sink_list_kernel<<<G, T, 0, st>>>(L->d_cnt, L->sel_cells, L->cells, ctx->cell_start, begin,
                                    L->pscan, L->ssink, L->scell);
  CT2G_LAUNCHED(ctx);
  // the widened direct sum: selected dense cells through the near kernel's
  // dense path (chunks of one cell, count d_cnt[5], work counter d_cnt[6]),
  // the sinks of the other selected cells (count d_cnt[7]) in sparse-style
  // chunks per 4x4x4 block (count d_cnt[2], work counter d_cnt[3]); flags,
  // scan, pflag and pscan are free again here
  CT2G_CUDA(ctx, cudaMemsetAsync(L->flags, 0, sizeof(uint32_t) * nr, st));
  CT2G_CUDA(ctx, cudaMemsetAsync(L->pflag, 0, sizeof(uint32_t) * nr, st));
  shell_split_kernel<<<G, T, 0, st>>>(L->d_cnt, L->sel_cells, L->cells, ctx->cell_start, begin,
                                      ctx->dense_cell, L->flags, L->pflag);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, L->flags, L->scan, nr, L->d_cnt + 5, 0));
  shell_dense_fill_kernel<<<G, T, 0, st>>>(L->flags, L->scan, ctx->keys, ctx->cell_start, begin,
                                           nr, L->dchunks);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, L->pflag, L->pscan, nr, L->d_cnt + 7, 0));
  shell_sparse_list_kernel<<<G, T, 0, st>>>(L->pflag, L->pscan, begin, nr, L->ssink2);
  CT2G_LAUNCHED(ctx);
  CT2G_CUDA(ctx, cudaMemsetAsync(L->cflag, 0, sizeof(uint32_t) * nr, st));
  sink_chunk_flag_kernel<<<G, T, 0, st>>>(ctx->keys, ctx->cell_start, L->pflag, L->pscan, begin,
                                          nr, L->cflag);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, L->cflag, L->cscan, nr, L->d_cnt + 2, 0));
  sink_chunk_fill_kernel<<<G, T, 0, st>>>(L->d_cnt + 7, L->cflag, L->cscan, L->ssink2, ctx->keys,
                                          ctx->cell_start, L->pscan, begin, nr, L->chunks);
  CT2G_LAUNCHED(ctx);
  CT2G_CUDA(ctx, cudaMemsetAsync(L->d_cnt + 3, 0, sizeof(uint32_t), st));
  CT2G_CUDA(ctx, cudaMemsetAsync(L->d_cnt + 6, 0, sizeof(uint32_t), st));
  shell_m2l_kernel<P><<<warp_grid(ctx, nr), 256, 0, st>>>(
      L->d_cnt, L->sel_cells, L->cells, L->mc, L->idx, geo_of(ctx), L->d_shell, L->d_shellG,
      L->nshell, L->lsub);
  CT2G_LAUNCHED(ctx);
  const float bw = ctx->opt.bwidth, bx = L->bw_ext;
  CT2G_TRY(ct2g_near_dense_window(ctx, L->dchunks, L->d_cnt + 5, L->d_cnt + 6, L->d_stm, pot, fx,
                                  fy, fz, po));
  CT2G_TRY(ct2g_near_window(ctx, L->chunks, L->d_cnt + 2, L->d_cnt + 3, L->ssink2, L->d_stm,
                            bw * bw, bx * bx, pot, fx, fy, fz, po));
  if (pot)
    shell_l2p_kernel<P, true><<<G, T, 0, st>>>(L->d_cnt, L->ssink, L->scell, ctx->keys, begin,
                                                ctx->mbits, ctx->src, L->lsub, ctx->box_gm, fx, fy,
                                                fz, po);
  else
    shell_l2p_kernel<P, false><<<G, T, 0, st>>>(L->d_cnt, L->ssink, L->scell, ctx->keys, begin,
                                                 ctx->mbits, ctx->src, L->lsub, ctx->box_gm, fx, fy,
                                                 fz, po);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

// widen the direct sum of the selected cells (selection already made)
int widen(ct2g_ctx *ctx, int mode, float thr, bool pot, float *fx, float *fy, float *fz,
          float *po) {
  ct2g_learn *L = ctx->learn;
  CT2G_TRY(build_chunks(ctx, mode, thr, !L->d_stm));
  if (!L->d_stm) return shell_correct(ctx, pot, fx, fy, fz, po);
  switch (ctx->p) {
    case 2: return widen_block_p<2>(ctx, pot, fx, fy, fz, po);
    case 3: return widen_block_p<3>(ctx, pot, fx, fy, fz, po);
    case 4: return widen_block_p<4>(ctx, pot, fx, fy, fz, po);
    case 5: return widen_block_p<5>(ctx, pot, fx, fy, fz, po);
    case 6: return widen_block_p<6>(ctx, pot, fx, fy, fz, po);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "unsupported order");
}

ct2g_learn *need_learn(ct2g_ctx *ctx) {
  if (!ctx->learn) ct2g_fail(ctx, CT2G_ESTATE, "learned correction not enabled (ct2g_learned_enable)");
  return ctx->learn;
}

int mlp_upload_bf16(ct2g_ctx *ctx) {
  ct2g_learn *L = ctx->learn;
  to_bf16_kernel<<<ct2g_div_up(NP, 256), 256, 0, ctx->stream>>>(L->params, L->wbf, NP);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

int stash_alloc(ct2g_ctx *ctx, size_t batch) {
  ct2g_learn *L = ctx->learn;
  if (L->stash_cap >= batch) return CT2G_OK;
  if (L->stash) cudaFree(L->stash);
  if (L->sloss) cudaFree(L->sloss);
  L->stash = nullptr;
  L->sloss = nullptr;
  L->stash_cap = 0;
  CT2G_CUDA(ctx, cudaMalloc(&L->stash, sizeof(float) * kStash * batch));
  CT2G_CUDA(ctx, cudaMalloc(&L->sloss, sizeof(float) * (batch + 1)));
  L->stash_cap = batch;
  return CT2G_OK;
}

// one optimisation batch (or, with lr == 0, only the gradient)
int mlp_batch(ct2g_ctx *ctx, const float *X, const float *T, const uint32_t *idx, size_t start,
              int count, float lr, float *loss_dev) {
  ct2g_learn *L = ctx->learn;
  cudaStream_t st = ctx->stream;
  const size_t smem = sizeof(float) * NP;
  CT2G_TRY(ct2g_smem_attrs(ctx, mlp_fwdbwd_kernel, smem));
  mlp_fwdbwd_kernel<<<ct2g_div_up(count, 128), 128, smem, st>>>(
      L->wbf, L->fmean, L->fstd, X, T, idx, start, count, L->stash, L->sloss);
  CT2G_LAUNCHED(ctx);
  mlp_wgrad_kernel<<<ct2g_div_up(NP, 128), 128, 0, st>>>(L->fmean, L->fstd, X, idx, start, count,
                                                          L->stash, L->grad);
  CT2G_LAUNCHED(ctx);
  if (loss_dev) {
    loss_sum_kernel<<<1, 256, 0, st>>>(L->sloss, count, loss_dev);
    CT2G_LAUNCHED(ctx);
  }
  if (lr > 0.f) {
    L->adam_t++;
    const float c1 = 1.f - std::pow(0.9f, (float)L->adam_t);
    const float c2 = 1.f - std::pow(0.999f, (float)L->adam_t);
    adam_kernel<<<ct2g_div_up(NP, 256), 256, 0, st>>>(L->params, L->grad, L->am, L->av, L->wbf,
                                                      lr, c1, c2);
    CT2G_LAUNCHED(ctx);
  }
  return CT2G_OK;
}

}  // namespace

bool ct2g_learned_active(const ct2g_ctx *ctx) {
  return ctx->learn && ctx->learn->mode != CT2G_SELECT_NONE;
}

int ct2g_learned_resize(ct2g_ctx *ctx) {
  if (!ctx->learn) return CT2G_OK;
  return learn_cells_alloc(ctx);
}

void ct2g_learned_free(ct2g_ctx *ctx) {
  ct2g_learn *L = ctx->learn;
  if (!L) return;
  free_learn_cells(L);
  void *ptrs[] = {L->d_shell, L->d_shellG, L->d_stm, L->idx, L->d_cnt, L->params, L->grad, L->am, L->av, L->wbf,
                  L->fmean, L->fstd, L->tX, L->tT, L->stash, L->sloss, L->tidx};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete L;
  ctx->learn = nullptr;
}

// After the plain forces: select cells and widen their direct sum.
int ct2g_learned_apply(ct2g_ctx *ctx, bool pot) {
  ct2g_learn *L = ctx->learn;
  if (!L || L->mode == CT2G_SELECT_NONE || ctx->n == ctx->rung_begin) return CT2G_OK;
  if (L->mode == CT2G_SELECT_MLP && !L->have_mlp)
    return ct2g_fail(ctx, CT2G_ESTATE, "MLP selection without trained or loaded weights");
  CT2G_TRY(occupied_cells(ctx));
  if (L->mode == CT2G_SELECT_FIXED || L->mode == CT2G_SELECT_MLP)
    CT2G_TRY(features(ctx, ctx->fx, ctx->fy, ctx->fz));
  if (L->mode == CT2G_SELECT_MLP) CT2G_TRY(infer(ctx));
  return widen(ctx, L->mode, L->threshold, pot, ctx->fx, ctx->fy, ctx->fz, ctx->pot);
}

extern "C" {

int ct2g_learned_enable(ct2g_ctx *ctx, float bwidth_ext) {
  CT2G_TRY(ct2g_check(ctx));
  const float bw = ctx->opt.bwidth;
  if (ctx->p < 2) return ct2g_fail(ctx, CT2G_EINVAL, "the features need order >= 2");
  if (!(bwidth_ext > bw) || bwidth_ext > 8.f || 2.f * bwidth_ext + 1.f > (float)ctx->M)
    return ct2g_fail(ctx, CT2G_EINVAL, "bwidth_ext must be in (bwidth, 8] and fit the mesh");
  if (!ctx->learn) {
    ctx->learn = new ct2g_learn();
    ct2g_learn *L = ctx->learn;
    CT2G_CUDA(ctx, cudaMalloc(&L->d_cnt, sizeof(uint32_t) * 8));
    CT2G_CUDA(ctx, cudaMemset(L->d_cnt, 0, sizeof(uint32_t) * 8));
    CT2G_CUDA(ctx, cudaMalloc(&L->params, sizeof(float) * NP));
    CT2G_CUDA(ctx, cudaMalloc(&L->grad, sizeof(float) * NP));
    CT2G_CUDA(ctx, cudaMalloc(&L->am, sizeof(float) * NP));
    CT2G_CUDA(ctx, cudaMalloc(&L->av, sizeof(float) * NP));
    CT2G_CUDA(ctx, cudaMalloc(&L->wbf, sizeof(__nv_bfloat16) * NP));
    CT2G_CUDA(ctx, cudaMalloc(&L->fmean, sizeof(float) * NIN));
    CT2G_CUDA(ctx, cudaMalloc(&L->fstd, sizeof(float) * NIN));
  }
  ct2g_learn *L = ctx->learn;
  if (L->d_shell) cudaFree(L->d_shell);
  if (L->d_shellG) cudaFree(L->d_shellG);
  L->d_shell = nullptr;
  L->d_shellG = nullptr;
  // shell offsets, nearest first, and three distance bins of equal size
  std::vector<std::array<int, 3>> offs;
  const int B = (int)std::floor(bwidth_ext);
  const double b2 = (double)bw * bw, x2 = (double)bwidth_ext * bwidth_ext;
  for (int i = -B; i <= B; i++)
    for (int j = -B; j <= B; j++)
      for (int k = -B; k <= B; k++) {
        const double d2 = (double)(i * i + j * j + k * k);
        if (d2 > b2 && d2 <= x2) offs.push_back({i, j, k});
      }
  std::stable_sort(offs.begin(), offs.end(), [](const std::array<int, 3> &a, const std::array<int, 3> &b) {
    return a[0] * a[0] + a[1] * a[1] + a[2] * a[2] < b[0] * b[0] + b[1] * b[1] + b[2] * b[2];
  });
  L->nshell = (int)offs.size();
  std::vector<int> o4(4 * offs.size()), o3(3 * offs.size());
  for (size_t s = 0; s < offs.size(); s++) {
    const int bin = (int)std::min<size_t>(2, 3 * s / std::max<size_t>(offs.size(), 1));
    for (int a = 0; a < 3; a++) {
      o4[4 * s + a] = offs[s][a];
      o3[3 * s + a] = offs[s][a];
    }
    o4[4 * s + 3] = bin;
  }
  CT2G_CUDA(ctx, cudaMalloc(&L->d_shell, sizeof(int) * std::max<size_t>(o4.size(), 4)));
  CT2G_CUDA(ctx, cudaMalloc(&L->d_shellG, sizeof(float) * std::max<size_t>(offs.size() * ctx->nc, 1)));
  if (!offs.empty())
    CT2G_CUDA(ctx, cudaMemcpy(L->d_shell, o4.data(), sizeof(int) * o4.size(), cudaMemcpyHostToDevice));
  CT2G_TRY(ct2g_shell_greens(ctx, o3, L->d_shellG));
  // shell cells of each neighbouring 4x4x4 block per in-block position (the
  // block walk reaches 4 cells in every direction)
  if (L->d_stm) cudaFree(L->d_stm);
  L->d_stm = nullptr;
  if (bwidth_ext <= 4.f) {
    std::vector<unsigned long long> m(64 * 27, 0ull);
    auto pos = [](int b, int &x, int &y, int &z) {
      x = ((b >> 2) & 1) | ((b >> 4) & 2);
      y = ((b >> 1) & 1) | ((b >> 3) & 2);
      z = (b & 1) | ((b >> 2) & 2);
    };
    for (int p = 0; p < 64; p++) {
      int px, py, pz;
      pos(p, px, py, pz);
      for (int o = 0; o < 27; o++)
        for (int b = 0; b < 64; b++) {
          int bx, by, bz;
          pos(b, bx, by, bz);
          const int ox = 4 * (o / 9 - 1) + bx - px, oy = 4 * ((o / 3) % 3 - 1) + by - py,
                    oz = 4 * (o % 3 - 1) + bz - pz;
          const double d2 = (double)(ox * ox + oy * oy + oz * oz);
          if (d2 > b2 && d2 <= x2) m[p * 27 + o] |= 1ull << b;
        }
    }
    CT2G_CUDA(ctx, cudaMalloc(&L->d_stm, sizeof(unsigned long long) * m.size()));
    CT2G_CUDA(ctx, cudaMemcpy(L->d_stm, m.data(), sizeof(unsigned long long) * m.size(),
                              cudaMemcpyHostToDevice));
  }
  L->bw_ext = bwidth_ext;
  CT2G_TRY(learn_cells_alloc(ctx));
  ctx->epoch++;
  return CT2G_OK;
}

int ct2g_learned_select(ct2g_ctx *ctx, int mode, float threshold) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  if (mode < CT2G_SELECT_NONE || mode > CT2G_SELECT_ALL) return ct2g_fail(ctx, CT2G_EINVAL, "bad selection mode");
  if (mode == CT2G_SELECT_MLP && !L->have_mlp)
    return ct2g_fail(ctx, CT2G_ESTATE, "no MLP weights (train or load them first)");
  L->mode = mode;
  L->threshold = threshold;
  ctx->epoch++;  // mode and threshold are launch arguments of a recorded step
  ctx->forces_valid = false;
  return CT2G_OK;
}

int ct2g_learned_collect(ct2g_ctx *ctx, size_t *ncells) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  if (!ctx->grid_valid) return ct2g_fail(ctx, CT2G_ESTATE, "particle_to_grid has not run since the particles moved");
  CT2G_TRY(learn_cells_alloc(ctx));
  const size_t nr = ctx->n - ctx->rung_begin;
  cudaStream_t st = ctx->stream;
  // plain forces; the moment grid is formed first (the features and the
  // shell's Taylor term read it), so the far field does not fuse P2M away
  if (!ctx->moments_valid) {
    CT2G_TRY(ct2g_p2m(ctx));
    ctx->moments_valid = true;
    ctx->expansions_valid = false;
  }
  const int mode = L->mode;
  L->mode = CT2G_SELECT_NONE;
  int rc = ct2g_all_forces(ctx, false);
  L->mode = mode;
  CT2G_TRY(rc);
  ctx->forces_valid = true;
  ctx->pot_valid = false;
  // features from the plain forces; widened forces with every cell corrected
  CT2G_TRY(occupied_cells(ctx));
  CT2G_TRY(features(ctx, ctx->fx, ctx->fy, ctx->fz));
  CT2G_CUDA(ctx, cudaMemcpyAsync(L->ex, ctx->fx, ctx->n * 4, cudaMemcpyDeviceToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(L->ey, ctx->fy, ctx->n * 4, cudaMemcpyDeviceToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(L->ez, ctx->fz, ctx->n * 4, cudaMemcpyDeviceToDevice, st));
  CT2G_TRY(widen(ctx, CT2G_SELECT_ALL, 0.f, false, L->ex, L->ey, L->ez, nullptr));
  // append (features, target) to the training set
  uint32_t nc = 0;
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, L->d_cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  nc = ctx->h_pinned[0];
  if (L->tn + nc > L->tcap) {
    const size_t ncap = std::max<size_t>(2 * L->tcap, L->tn + nc);
    float *nX = nullptr, *nT = nullptr;
    uint32_t *nI = nullptr;
    CT2G_CUDA(ctx, cudaMalloc(&nX, sizeof(float) * NIN * ncap));
    CT2G_CUDA(ctx, cudaMalloc(&nT, sizeof(float) * ncap));
    CT2G_CUDA(ctx, cudaMalloc(&nI, sizeof(uint32_t) * ncap));
    if (L->tn) {
      CT2G_CUDA(ctx, cudaMemcpyAsync(nX, L->tX, sizeof(float) * NIN * L->tn, cudaMemcpyDeviceToDevice, st));
      CT2G_CUDA(ctx, cudaMemcpyAsync(nT, L->tT, sizeof(float) * L->tn, cudaMemcpyDeviceToDevice, st));
    }
    CT2G_CUDA(ctx, cudaStreamSynchronize(st));
    if (L->tX) cudaFree(L->tX);
    if (L->tT) cudaFree(L->tT);
    if (L->tidx) cudaFree(L->tidx);
    L->tX = nX;
    L->tT = nT;
    L->tidx = nI;
    L->tcap = ncap;
  }
  if (nc) {
    CT2G_CUDA(ctx, cudaMemcpyAsync(L->tX + L->tn * NIN, L->X, sizeof(float) * NIN * nc,
                                   cudaMemcpyDeviceToDevice, st));
    target_kernel<<<warp_grid(ctx, nc), 256, 0, st>>>(L->cells, L->d_cnt, ctx->cell_start, ctx->fx,
                                                       ctx->fy, ctx->fz, L->ex, L->ey, L->ez,
                                                       L->tT + L->tn);
    CT2G_LAUNCHED(ctx);
  }
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  L->tn += nc;
  (void)nr;
  if (ncells) *ncells = nc;
  return CT2G_OK;
}

int ct2g_learned_dataset(ct2g_ctx *ctx, float *X, float *T, size_t cap, size_t *n) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  if (n) *n = L->tn;
  if (!X && !T) return CT2G_OK;
  const size_t m = std::min(cap, L->tn);
  if (X && m) CT2G_CUDA(ctx, cudaMemcpy(X, L->tX, sizeof(float) * NIN * m, cudaMemcpyDeviceToHost));
  if (T && m) CT2G_CUDA(ctx, cudaMemcpy(T, L->tT, sizeof(float) * m, cudaMemcpyDeviceToHost));
  return CT2G_OK;
}

int ct2g_learned_clear(ct2g_ctx *ctx) {
  if (!ctx) return CT2G_EINVAL;
  if (ctx->learn) ctx->learn->tn = 0;
  return CT2G_OK;
}

int ct2g_mlp_init(ct2g_ctx *ctx, uint64_t seed) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  std::vector<float> p(NP, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](int off, int fan_in, int count) {
    const float a = std::sqrt(6.f / (float)fan_in);  // He-uniform for ReLU layers
    std::uniform_real_distribution<float> u(-a, a);
    for (int i = 0; i < count; i++) p[off + i] = u(rng);
  };
  fill(OW1, NIN, NH * NIN);
  fill(OW2, NH, NH * NH);
  fill(OW3, NH, NH);
  p[OB3] = -5.f;  // typical log10 residual
  std::vector<float> m(NIN, 0.f), s(NIN, 1.f);
  CT2G_CUDA(ctx, cudaMemcpy(L->params, p.data(), sizeof(float) * NP, cudaMemcpyHostToDevice));
  CT2G_CUDA(ctx, cudaMemset(L->am, 0, sizeof(float) * NP));
  CT2G_CUDA(ctx, cudaMemset(L->av, 0, sizeof(float) * NP));
  CT2G_CUDA(ctx, cudaMemcpy(L->fmean, m.data(), sizeof(float) * NIN, cudaMemcpyHostToDevice));
  CT2G_CUDA(ctx, cudaMemcpy(L->fstd, s.data(), sizeof(float) * NIN, cudaMemcpyHostToDevice));
  L->adam_t = 0;
  CT2G_TRY(mlp_upload_bf16(ctx));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  L->have_mlp = true;
  return CT2G_OK;
}

int ct2g_mlp_set(ct2g_ctx *ctx, const float *params, const float *fmean, const float *fstd) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  if (!params || !fmean || !fstd) return ct2g_fail(ctx, CT2G_EINVAL, "null MLP arrays");
  for (int i = 0; i < NIN; i++)
    if (!(fstd[i] > 0.f)) return ct2g_fail(ctx, CT2G_EINVAL, "feature scales must be > 0");
  CT2G_CUDA(ctx, cudaMemcpy(L->params, params, sizeof(float) * NP, cudaMemcpyHostToDevice));
  CT2G_CUDA(ctx, cudaMemcpy(L->fmean, fmean, sizeof(float) * NIN, cudaMemcpyHostToDevice));
  CT2G_CUDA(ctx, cudaMemcpy(L->fstd, fstd, sizeof(float) * NIN, cudaMemcpyHostToDevice));
  CT2G_CUDA(ctx, cudaMemset(L->am, 0, sizeof(float) * NP));
  CT2G_CUDA(ctx, cudaMemset(L->av, 0, sizeof(float) * NP));
  L->adam_t = 0;
  CT2G_TRY(mlp_upload_bf16(ctx));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  L->have_mlp = true;
  return CT2G_OK;
}

int ct2g_mlp_get(ct2g_ctx *ctx, float *params, float *fmean, float *fstd) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  if (!L->have_mlp) return ct2g_fail(ctx, CT2G_ESTATE, "no MLP weights");
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (params) CT2G_CUDA(ctx, cudaMemcpy(params, L->params, sizeof(float) * NP, cudaMemcpyDeviceToHost));
  if (fmean) CT2G_CUDA(ctx, cudaMemcpy(fmean, L->fmean, sizeof(float) * NIN, cudaMemcpyDeviceToHost));
  if (fstd) CT2G_CUDA(ctx, cudaMemcpy(fstd, L->fstd, sizeof(float) * NIN, cudaMemcpyDeviceToHost));
  return CT2G_OK;
}

int ct2g_mlp_train(ct2g_ctx *ctx, int epochs, int batch, float lr, uint64_t seed, int normalize,
                   float *loss) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  if (!L->have_mlp) CT2G_TRY(ct2g_mlp_init(ctx, seed));
  if (L->tn == 0) return ct2g_fail(ctx, CT2G_ESTATE, "empty training set (ct2g_learned_collect)");
  if (epochs < 0 || batch < 1 || batch > (1 << 20) || !(lr >= 0.f))
    return ct2g_fail(ctx, CT2G_EINVAL, "bad training arguments");
  cudaStream_t st = ctx->stream;
  if (normalize) {
    norm_stats_kernel<<<NIN, 256, 0, st>>>(L->tX, L->tn, L->fmean, L->fstd);
    CT2G_LAUNCHED(ctx);
  }
  CT2G_TRY(stash_alloc(ctx, (size_t)batch));
  std::vector<uint32_t> idx(L->tn);
  for (size_t i = 0; i < L->tn; i++) idx[i] = (uint32_t)i;
  std::mt19937_64 rng(seed);
  float *dloss = L->sloss + batch;  // spare slot past the per-sample losses
  float last = 0.f;
  for (int e = 0; e < epochs; e++) {
    std::shuffle(idx.begin(), idx.end(), rng);
    CT2G_CUDA(ctx, cudaMemcpyAsync(L->tidx, idx.data(), sizeof(uint32_t) * L->tn,
                                   cudaMemcpyHostToDevice, st));
    for (size_t s = 0; s < L->tn; s += (size_t)batch) {
      const int cnt = (int)std::min<size_t>(batch, L->tn - s);
      CT2G_TRY(mlp_batch(ctx, L->tX, L->tT, L->tidx, s, cnt, lr, nullptr));
    }
    CT2G_CUDA(ctx, cudaStreamSynchronize(st));  // idx is reused next epoch
  }
  // loss over the whole set with the final weights
  double acc = 0.0;
  for (size_t i = 0; i < L->tn; i++) idx[i] = (uint32_t)i;
  CT2G_CUDA(ctx, cudaMemcpyAsync(L->tidx, idx.data(), sizeof(uint32_t) * L->tn, cudaMemcpyHostToDevice, st));
  for (size_t s = 0; s < L->tn; s += (size_t)batch) {
    const int cnt = (int)std::min<size_t>(batch, L->tn - s);
    CT2G_TRY(mlp_batch(ctx, L->tX, L->tT, L->tidx, s, cnt, 0.f, dloss));
    float h = 0.f;
    CT2G_CUDA(ctx, cudaMemcpyAsync(&h, dloss, sizeof(float), cudaMemcpyDeviceToHost, st));
    CT2G_CUDA(ctx, cudaStreamSynchronize(st));
    acc += (double)h * cnt;
  }
  last = (float)(acc / (double)L->tn);
  if (loss) *loss = last;
  return CT2G_OK;
}

int ct2g_mlp_gradients(ct2g_ctx *ctx, const float *X, const float *T, size_t n, float *grad,
                       float *loss) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  if (!L->have_mlp) return ct2g_fail(ctx, CT2G_ESTATE, "no MLP weights");
  if (!X || !T || !grad || n == 0 || n > (1u << 20)) return ct2g_fail(ctx, CT2G_EINVAL, "bad gradient arguments");
  CT2G_TRY(stash_alloc(ctx, n));
  float *dX = nullptr, *dT = nullptr;
  uint32_t *dI = nullptr;
  std::vector<uint32_t> idx(n);
  for (size_t i = 0; i < n; i++) idx[i] = (uint32_t)i;
  int rc = CT2G_OK;
  cudaError_t e = cudaMalloc(&dX, sizeof(float) * NIN * n);
  if (e == cudaSuccess) e = cudaMalloc(&dT, sizeof(float) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dI, sizeof(uint32_t) * n);
  if (e == cudaSuccess) e = cudaMemcpy(dX, X, sizeof(float) * NIN * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dT, T, sizeof(float) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dI, idx.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) rc = ct2g_cuda_fail(ctx, e, "gradient inputs");
  if (rc == CT2G_OK) rc = mlp_batch(ctx, dX, dT, dI, 0, (int)n, 0.f, L->sloss + n);
  if (rc == CT2G_OK) {
    e = cudaMemcpyAsync(grad, L->grad, sizeof(float) * NP, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && loss)
      e = cudaMemcpyAsync(loss, L->sloss + n, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = ct2g_cuda_fail(ctx, e, "gradient outputs");
  }
  cudaStreamSynchronize(ctx->stream);
  if (dX) cudaFree(dX);
  if (dT) cudaFree(dT);
  if (dI) cudaFree(dI);
  return rc;
}

int ct2g_learned_cells(ct2g_ctx *ctx, uint32_t *keys, float *X, float *score, float *pred,
                       uint8_t *selected, size_t cap, size_t *ncells, size_t *nselected) {
  CT2G_TRY(ct2g_check(ctx));
  ct2g_learn *L = need_learn(ctx);
  if (!L) return CT2G_ESTATE;
  uint32_t c[2] = {0, 0};
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  CT2G_CUDA(ctx, cudaMemcpy(c, L->d_cnt, sizeof(c), cudaMemcpyDeviceToHost));
  if (ncells) *ncells = c[0];
  if (nselected) *nselected = c[1];
  const size_t m = std::min<size_t>(cap, c[0]);
  if (m == 0) return CT2G_OK;
  if (keys) CT2G_CUDA(ctx, cudaMemcpy(keys, L->cells, 4 * m, cudaMemcpyDeviceToHost));
  if (X) CT2G_CUDA(ctx, cudaMemcpy(X, L->X, 4 * NIN * m, cudaMemcpyDeviceToHost));
  if (score) CT2G_CUDA(ctx, cudaMemcpy(score, L->score, 4 * m, cudaMemcpyDeviceToHost));
  if (pred) CT2G_CUDA(ctx, cudaMemcpy(pred, L->pred, 4 * m, cudaMemcpyDeviceToHost));
  if (selected) CT2G_CUDA(ctx, cudaMemcpy(selected, L->sel, m, cudaMemcpyDeviceToHost));
  return CT2G_OK;
}

}  // extern "C"
