// Internal declarations shared by the ct2g CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ct2g.h"

#define CT2G_TWO_M32 2.3283064365386963e-10

// ---------------------------------------------------------------------------
// Multi-indices n = (nx, ny, nz), |n| <= P: ordered by degree, then nx
// descending, then ny descending.  idx = T(d) + (d-nx)(d-nx+1)/2 + nz with
// T(d) = d(d+1)(d+2)/6.  (The same ordering as the CPU oracle.)
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ct2g_ncomp(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }
__host__ __device__ constexpr int ct2g_mi_index(int nx, int ny, int nz) {
  return (nx + ny + nz) * (nx + ny + nz + 1) * (nx + ny + nz + 2) / 6 +
         (ny + nz) * (ny + nz + 1) / 2 + nz;
}

// ---------------------------------------------------------------------------
// Morton keys: cell (i,j,k) -> bits interleaved from the most significant, x
// first.  The reference's recursive bisection (src/particle.cpp:89-114,
// depth d splitting dimension d%3) lays its leaves out in exactly this order.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t ct2g_spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ __forceinline__ uint32_t ct2g_compact3(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030c30c3u;
  v = (v | (v >> 4)) & 0x0300f00fu;
  v = (v | (v >> 8)) & 0x030000ffu;
  v = (v | (v >> 16)) & 0x3ffu;
  return v;
}
__host__ __device__ __forceinline__ uint32_t ct2g_morton(uint32_t i, uint32_t j, uint32_t k) {
  return (ct2g_spread3(i) << 2) | (ct2g_spread3(j) << 1) | ct2g_spread3(k);
}

template <int P>
struct MiTable {
  static constexpr int NC = ct2g_ncomp(P);
  int nx[NC];
  int ny[NC];
  int nz[NC];
  int deg[NC];
  constexpr MiTable() : nx(), ny(), nz(), deg() {
    int k = 0;
    for (int d = 0; d <= P; d++)
      for (int a = d; a >= 0; a--)
        for (int b = d - a; b >= 0; b--) {
          nx[k] = a;
          ny[k] = b;
          nz[k] = d - a - b;
          deg[k] = d;
          k++;
        }
  }
};

// L2P: evaluate the local expansion L (accessor L(k) -> coefficient k) at
// offset t from the cell centre: F_i = sum_a L_{a+e_i} t^a/a! (without GM),
// potential -sum_a L_a t^a/a!
template <int P, typename LA>
__device__ __forceinline__ void ct2g_l2p(const LA &Lacc, float tx, float ty, float tz, float &fx,
                                         float &fy, float &fz, float &pot) {
  constexpr MiTable<P> T{};
  constexpr int NC = MiTable<P>::NC;
  float L[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) L[k] = Lacc(k);
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

// Softened pair acceleration (src/kick.cpp:44-60) of a sink at offset d from
// a source, accumulated into (ax, ay, az) and the potential ap; `on` false
// adds exact zeros (masked lanes keep their summation order).
template <int KERNEL, bool POT>
__device__ __forceinline__ void ct2g_pair_term(float dx, float dy, float dz, float h2, float hinv,
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

// The (a, b) pairs with |a|+|b| <= P, grouped by a: since multi-indices are
// ordered by degree, the b of one a are exactly the first ncomp(P-|a|).
template <int P>
struct Mg2lPairs {
  static constexpr int NC = ct2g_ncomp(P);
  static constexpr int count() {
    int n = 0;
    for (int d = 0; d <= P; d++) n += (ct2g_ncomp(d) - (d ? ct2g_ncomp(d - 1) : 0)) * ct2g_ncomp(P - d);
    return n;
  }
  static constexpr int NP = count();
  int a[NP], b[NP], ab[NP], odd[NP], first[NP], last[NP];
  constexpr Mg2lPairs() : a(), b(), ab(), odd(), first(), last() {
    MiTable<P> T{};
    int i = 0;
    for (int ia = 0; ia < NC; ia++) {
      const int nb = ct2g_ncomp(P - T.deg[ia]);
      for (int ib = 0; ib < nb; ib++) {
        a[i] = ia;
        b[i] = ib;
        ab[i] = ct2g_mi_index(T.nx[ia] + T.nx[ib], T.ny[ia] + T.ny[ib], T.nz[ia] + T.nz[ib]);
        odd[i] = (T.deg[ia] + T.deg[ib]) & 1;
        first[i] = ib == 0;
        last[i] = ib == nb - 1;
        i++;
      }
    }
  }
};
template <int P>
struct Mg2lTab {
  static constexpr Mg2lPairs<P> t{};
};

// One (a, b) term of L_a = sum_b G_{a+b} M_b (src/particle.cpp:244-250).
// G_n is real for even |n| and i*g for odd |n| (parity of D^n phi); g[n * GS]
// is that real factor.  Every index is a compile-time constant, so m[], a
// register g[] and acc stay in registers; L_a goes to out[a].
template <int P, int GS, int I>
__device__ __forceinline__ void ct2g_mg2l_term(const float2 *m, const float *g, float2 &acc,
                                               float2 *out) {
  constexpr int A = Mg2lTab<P>::t.a[I], B = Mg2lTab<P>::t.b[I], AB = Mg2lTab<P>::t.ab[I];
  constexpr bool FIRST = Mg2lTab<P>::t.first[I] != 0, LAST = Mg2lTab<P>::t.last[I] != 0,
                 ODD = Mg2lTab<P>::t.odd[I] != 0;
  if constexpr (FIRST) acc = make_float2(0.f, 0.f);
  const float gv = g[AB * GS];
  const float2 mb = m[B];
  if constexpr (!ODD) {
    acc.x = fmaf(gv, mb.x, acc.x);
    acc.y = fmaf(gv, mb.y, acc.y);
  } else {  // i*g*(mx + i my) = (-g my, g mx)
    acc.x = fmaf(-gv, mb.y, acc.x);
    acc.y = fmaf(gv, mb.x, acc.y);
  }
  if constexpr (LAST) out[A] = acc;
}

template <int P, int GS, int... I>
__device__ __forceinline__ void ct2g_mg2l_all(const float2 *m, const float *g, float2 *out,
                                              std::integer_sequence<int, I...>) {
  float2 acc = make_float2(0.f, 0.f);
  (ct2g_mg2l_term<P, GS, I>(m, g, acc, out), ...);
}

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------
struct FftPlanBufs;

struct ct2g_ctx {
  ct2g_options opt;
  int mbits = 0;
  int M = 0;       // mesh cells per dim
  int64_t C = 0;   // mesh^3
  int64_t CK = 0;  // mesh*mesh*ldk: spectrum entries per component
  int ldk = 0;     // spectrum row pitch along the halved axis: mesh/2+2 (even)
  int p = 0;
  int nc = 0;      // ncomp(p)
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  // the near field's own stream when it overlaps the mesh solve, and the
  // events that fork it from and join it back to `stream`
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // host-state steps (ct2g_kick_drift_host): the velocity and rung upload
  // runs on copy_stream after ev_pos (positions landed) and signals ev_vel,
  // which the step waits for just before it gathers the velocities
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_pos = nullptr, ev_vel = nullptr;
  bool defer_vel = false;    // binning leaves the velocity/rung gather for later
  bool vel_pending = false;  // ... and that gather has not run yet
  cudaEvent_t ev[8] = {};
  float stage_ms[8] = {};
  std::string err;
  uint64_t launches = 0;
  uint64_t interactions = 0;

  // particle store (current order) and the sort target buffers
  size_t n = 0, cap = 0;
  uint32_t *x = nullptr, *y = nullptr, *z = nullptr, *id = nullptr;
  float *vx = nullptr, *vy = nullptr, *vz = nullptr;
  int8_t *rung = nullptr;
  uint32_t *x2 = nullptr, *y2 = nullptr, *z2 = nullptr, *id2 = nullptr;
  float *vx2 = nullptr, *vy2 = nullptr, *vz2 = nullptr;
  int8_t *rung2 = nullptr;
  // binning scratch
  uint32_t *keys = nullptr, *keys2 = nullptr, *vals = nullptr, *vals2 = nullptr;
  uint32_t *hist = nullptr;   // radix digit histograms
  uint32_t *scan_tmp = nullptr;
  size_t scan_tmp_words = 0;
  uint32_t *cell_start = nullptr;  // [C+1] indexed by Morton key, absolute indices
  unsigned long long *occ = nullptr;  // [C/64] occupancy bits of 4x4x4 cell blocks
  unsigned long long *stmask = nullptr;  // [64][27] stencil bits per (in-block cell, block offset)
  float4 *src = nullptr;           // per sorted particle: offset from own cell centre
  uint2 *chunks = nullptr;         // near-field warp chunks (start, count): dense ones
                                   // (particle index) then sparse ones (sparse_list index)
  uint32_t *sparse_list = nullptr; // particles of sparse cells, in order
  uint32_t *flags = nullptr;
  // work-list sizes stay on the device, so a step needs no host readback:
  // [0] dense chunks, [1] sparse sinks, [2] sparse chunks, [3] and [4] the
  // dense and sparse near-field work counters, [5] scan total scratch,
  // [6] sticky device error (a status code a kernel left)
  uint32_t *d_counts = nullptr;
  uint32_t dense_cell = 16;  // cells with at least this many particles get their own chunks
  int near_blocks_per_sm = 0;  // persistent near-field grid: blocks per SM (0: occupancy)
  int fft_tile = 0;            // y/x FFT pass tile width (0: default)
  int split_mg2l = 0;          // 1: X passes and MG2L as three launches, not one
  int sparse_path = 2;         // sparse sinks: 0 one per lane, 1 per-block warp chunks, 2 the
                               // same chunks with their sources streamed in windows (Plummer;
                               // the sphere kernel takes 1)
  int overlap = 0;             // 1: near field on stream2, concurrent with the mesh solve
  int mg2l_greens_direct = 0;  // 1: the fused x pass reads the Green's values from HBM
  int near_chunks_per_warp = 0;  // overlap: chunks a near-field warp takes before its block exits
  int plane_pipe = 0;          // > 0: z and y passes as one plane pipeline, this lag in planes
  int cols_tma = 1;            // 1: FP32 column FFT passes move their tiles by TMA
  int p2m_compact = 0;         // 1: P2M into compact per-cell records before the z pass
  int x_tma = 2;               // fused x pass inputs: 1 tensor + bulk copies, 2 cp.async
                               // column + bulk Green's copy, 0 per-thread loads
  // tensor map of the spectrum's x-pass columns (a CUtensorMap, built once)
  alignas(64) unsigned char xmap[128] = {};
  int xmap_bw = 0;             // box width (floats) the map was built for (0: none)
  int pipe_discard = 1;        // the pipeline's inverse z lines drop the L2 lines they read
  struct ct2g_batch *self_batch = nullptr;  // graph of ct2g_kick_drift
  struct ct2g_learn *learn = nullptr;       // learned near-field correction
  bool fft_tc = false;                      // y/x FFT passes on the tensor cores
  unsigned char *tc_tables = nullptr;       // their DFT matrices and twiddles

  // independent periodic boxes sharing the mesh: box b holds particles
  // [box_off[b], box_off[b+1]); its cells are keys (b << 3*mbits) | morton
  int nbox = 1;
  int boxbits = 0;
  int64_t CB = 0;                    // nbox * C
  std::vector<uint64_t> h_box_off;   // [nbox+1]
  std::vector<float> h_box_gm;       // [nbox]: G x particle mass
  bool boxes_set = true;
  uint32_t *box_off = nullptr;       // device [nbox+1]
  float *box_gm = nullptr;           // device [nbox]
  uint64_t epoch = 0;                // bumped when buffers or parameters change
  bool capturing = false;            // recording a CUDA graph: no events, no host reads
  // forces
  float *fx = nullptr, *fy = nullptr, *fz = nullptr, *pot = nullptr;
  // near-field accelerations while they run beside the mesh solve (overlap)
  float *nfx = nullptr, *nfy = nullptr, *nfz = nullptr, *npot = nullptr;
  // plane pipeline counters: per direction an item counter, a spare word and
  // one count per plane (nbox * mesh planes)
  uint32_t *pipe_sync = nullptr;
  // compact P2M: per occupied cell NC floats (capacity: one cell per
  // particle), the occupied cells' rank per 4x4x4 block, and the list of
  // cells summed by a warp (count first)
  float *cmom = nullptr;
  uint32_t *blk_rank = nullptr;
  uint32_t *p2m_big = nullptr;
  int *d_maxrung = nullptr;
  unsigned long long *d_inter = nullptr;
  uint32_t *h_pinned = nullptr;  // small pinned host scratch
  // mesh
  float *grid = nullptr;    // [nc][nbox][C] real: moments, then expansions
  // spectrum of the mesh solve, all components of a k-point side by side:
  // [box][qi][qj][qk][nc], qk < ldk (the slots qk > N/2 are zero padding)
  float2 *spec = nullptr;
  float *greens = nullptr;  // [nc][CK] real-or-imag, shared by the boxes
  // the same table in column order for the fused X pass + MG2L:
  // [qj][qk <= N/2][nc][qi]
  float *greens_x = nullptr;
  float2 *tw32 = nullptr;   // twiddles exp(-2 pi i k/M), k < M/2
  double2 *tw64 = nullptr;
  int tw_n = 0;
  // stencil
  int nstencil = 0;
  int *d_stencil = nullptr;  // [nstencil][3]

  // state
  size_t rung_begin = 0;
  std::vector<size_t> rung_stack;
  bool grid_valid = false;     // cell_start / src / chunks valid for current range
  bool moments_valid = false;
  bool expansions_valid = false;
  bool greens_valid = false;
  bool forces_valid = false;
  bool pot_valid = false;        // potential computed with the current forces
  bool has_particles = false;
};

// ---------------------------------------------------------------------------
// Error plumbing
// ---------------------------------------------------------------------------
int ct2g_fail(ct2g_ctx *ctx, int code, const std::string &msg);
int ct2g_cuda_fail(ct2g_ctx *ctx, cudaError_t e, const char *what);

#define CT2G_CUDA(ctx, call)                                       \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return ct2g_cuda_fail((ctx), e_, #call); \
  } while (0)

#define CT2G_LAUNCHED(ctx)                                                 \
  do {                                                                     \
    (ctx)->launches++;                                                     \
    cudaError_t e_ = cudaGetLastError();                                   \
    if (e_ != cudaSuccess) return ct2g_cuda_fail((ctx), e_, "kernel launch"); \
  } while (0)

#define CT2G_TRY(expr)        \
  do {                        \
    int rc_ = (expr);         \
    if (rc_ != CT2G_OK) return rc_; \
  } while (0)

// ---------------------------------------------------------------------------
// Stage entry points (implemented across the .cu files)
// ---------------------------------------------------------------------------
int ct2g_alloc_particles(ct2g_ctx *ctx, size_t n);
int ct2g_alloc_mesh(ct2g_ctx *ctx);
// exclusive scan (+ offset) of n uint32 values; in may equal out
// (total_dev: optional device word that receives the sum)
int ct2g_scan_exclusive(ct2g_ctx *ctx, const uint32_t *in, uint32_t *out, size_t n,
                        uint32_t *total_dev, uint32_t offset);
// words of scan scratch for n inputs
size_t ct2g_scan_scratch_words(size_t n);
// stage-time event k, skipped while a graph is recorded
void ct2g_mark(ct2g_ctx *ctx, int k);
int ct2g_bin_range(ct2g_ctx *ctx);
// the velocity/rung half of a gather that binning deferred (ctx->defer_vel)
int ct2g_gather_velocities(ct2g_ctx *ctx);
int ct2g_check(ct2g_ctx *ctx);  // valid context; selects its device
// the compact P2M records for the particle capacity (no-op when present)
int ct2g_alloc_p2m_compact(ct2g_ctx *ctx);
// resident blocks per SM of `kernel` (threads, dynamic shared memory) from its
// own registers and shared memory at the maximum carveout
int ct2g_blocks_per_sm(ct2g_ctx *ctx, const void *kernel, int threads, size_t dyn_smem);
// waits for the stream, then reports a status a kernel left in d_counts[6]
int ct2g_device_error(ct2g_ctx *ctx);
// tensor-core FFT passes (ct2g_fft_tc.cu)
bool ct2g_fft_tc_supported(int N);
int ct2g_fft_tc_prepare(ct2g_ctx *ctx);
int ct2g_fft_cols_tc(ct2g_ctx *ctx, float2 *spec, int N, size_t nouter, size_t ostride,
                     size_t rstride, size_t ncols, bool inv);
// learned correction (ct2g_learned.cu): applied after the plain forces
int ct2g_learned_apply(ct2g_ctx *ctx, bool pot);
int ct2g_learned_resize(ct2g_ctx *ctx);  // per-cell arrays follow the particle capacity
void ct2g_learned_free(ct2g_ctx *ctx);
// near-field direct sum of listed sinks over the cell window lo2 < |o|^2 <=
// hi2 (ct2g_near.cu); sparse-style chunks, persistent over *nch / *work
int ct2g_near_window(ct2g_ctx *ctx, const uint2 *chunks, const uint32_t *nch, uint32_t *work,
                     const uint32_t *slist, const unsigned long long *stm, float lo2, float hi2,
                     bool pot, float *fx, float *fy, float *fz, float *po);
// the same over the stencil masks stm for dense-style chunks (<= 32
// consecutive sinks of one cell, (first particle, count)), persistent over
// *nch / *work
int ct2g_near_dense_window(ct2g_ctx *ctx, const uint2 *chunks, const uint32_t *nch,
                           uint32_t *work, const unsigned long long *stm, bool pot, float *fx,
                           float *fy, float *fz, float *po);
// D^n phi_eps(-o h) for the offsets o (x,y,z triples) -> d_out[nshell][nc]
int ct2g_shell_greens(ct2g_ctx *ctx, const std::vector<int> &offs3, float *d_out);
// far field of the current range into the force buffers (P2M if needed, mesh
// solve with the fused inverse z pass + L2P)
int ct2g_far_field(ct2g_ctx *ctx, bool pot);
int ct2g_build_greens(ct2g_ctx *ctx);
int ct2g_p2m(ct2g_ctx *ctx);
// mesh solve; fused_l2p: the inverse z pass evaluates the far field of every
// particle of the current range straight into the force buffers (the
// expansion grid is not written)
// p2m: where the forward z pass takes the moments from --
// CT2G_P2M_GRID the moment grid (already computed);
// CT2G_P2M_FUSED computed inside the pass, not stored (ctx->grid then holds
//   no moments);
// CT2G_P2M_FUSED_STORE computed inside the pass and also written to the grid
// CT2G_P2M_COMPACT computed by a cell-parallel pass into compact per-cell
// records (ctx->cmom) that the z pass reads (tuning p2m_compact)
enum { CT2G_P2M_GRID = 0, CT2G_P2M_FUSED = 1, CT2G_P2M_FUSED_STORE = 2, CT2G_P2M_COMPACT = 3 };
int ct2g_mesh_solve(ct2g_ctx *ctx, bool fused_l2p, bool pot, int p2m = CT2G_P2M_GRID);
// Mesh-solve transforms on ctx->spec (ct2g_fft.cu).  Forward: the z pass
// (taking the moments as src says, CT2G_P2M_*), the Y pass, and the X pass
// unless the X passes are fused with MG2L.  ct2g_spec_mg2l: the fused X pass
// + MG2L + inverse X pass, or MG2L alone.  Inverse: the inverse X pass (when
// not fused), the Y pass and the z pass (L2P inside it when l2p, else into
// the expansion grid).
int ct2g_spec_forward(ct2g_ctx *ctx, int src);
int ct2g_spec_mg2l(ct2g_ctx *ctx);
int ct2g_spec_inverse(ct2g_ctx *ctx, bool l2p, bool pot);
// the X passes and MG2L run as one kernel for this context
bool ct2g_mg2l_fused(const ct2g_ctx *ctx);
// MG2L alone on ctx->spec (ct2g_mesh.cu)
int ct2g_mg2l_split(ct2g_ctx *ctx);
// floats of ctx->greens_x
size_t ct2g_greens_x_floats(const ct2g_ctx *ctx);
// the learned correction will run on the next force computation
bool ct2g_learned_active(const ct2g_ctx *ctx);
// near-field forces of the current range added to the far field already in
// the force buffers; pot: also the potential (diagnostics)
int ct2g_forces(ct2g_ctx *ctx, bool pot);
// far field and near field of the current range (the mesh solve, then or
// beside it the near field, per ctx->overlap)
int ct2g_all_forces(ct2g_ctx *ctx, bool pot);
int ct2g_update(ct2g_ctx *ctx, const ct2g_kick_params *p, int *max_rung, bool fuse_drift,
                float drift_dt, float drift_scale);
int ct2g_drift_all(ct2g_ctx *ctx, float dt, float scale);
int ct2g_twiddles(ct2g_ctx *ctx, int N);
// batched 3D FFTs on device buffers, on ctx->stream; spectrum rows (along the
// halved axis) hold ld >= N/2+1 complex values
int ct2g_fft_r2c_f32(ct2g_ctx *ctx, const float *in, float2 *out, int N, int batch, int ld);
int ct2g_fft_c2r_f32(ct2g_ctx *ctx, float2 *in, float *out, int N, int batch, int ld);
int ct2g_fft_c2c_f32(ct2g_ctx *ctx, float2 *a, int N, int batch, bool inv);
int ct2g_fft_r2c_f64(ct2g_ctx *ctx, const double *in, double2 *out, int N, int batch, int ld);
int ct2g_fft_c2r_f64(ct2g_ctx *ctx, double2 *in, double *out, int N, int batch, int ld);

static inline unsigned ct2g_div_up(size_t a, size_t b) { return (unsigned)((a + b - 1) / b); }

// a kernel's dynamic shared memory, with all of the unified L1 offered as
// shared memory so that the occupancy the launch sizes assume is reachable
template <typename K>
int ct2g_smem_attrs(ct2g_ctx *ctx, K kernel, size_t smem) {
  CT2G_CUDA(ctx, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CT2G_CUDA(ctx, cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                      (int)cudaSharedmemCarveoutMaxShared));
  return CT2G_OK;
}
