/*
 * ct2g.h -- C ABI of the B200-native ct2 gravity step.
 *
 * Plain C types only (pointers, sizes, scalars); no torch or C++ types.  One
 * context owns one GPU's particle store (SoA, resident in HBM), the mesh
 * buffers, the cached Green's tensor and one CUDA stream.  A context is not
 * thread-safe; separate contexts are independent.  Every entry point returns
 * a status (CT2G_OK == 0) and ct2g_last_error() describes the last failure.
 *
 * Each declaration names the reference interface it replaces (dmarce1/ct2,
 * file:line within that project).  The reference keeps its particles in
 * process-global arrays (src/particle.cpp:17-25, cosmictiger/particle.hpp:22-56)
 * mutated in place by particle_to_grid / kick / drift; here they live in the
 * context and cross the boundary through ct2g_upload_* / ct2g_download_*.
 * Like the reference, particle_to_grid leaves the store in cell order; the ids
 * returned by ct2g_download_particles map it back to upload order.
 */
#ifndef CT2G_H_
#define CT2G_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CT2G_OK 0
#define CT2G_EINVAL 1   /* bad argument or option                              */
#define CT2G_ENOMEM 2   /* device allocation failed                            */
#define CT2G_ECUDA 3    /* CUDA runtime error                                  */
#define CT2G_ESTATE 4   /* call out of order (e.g. kick before particle_to_grid)*/
#define CT2G_ETIMEOUT 5 /* a bounded device-side wait gave up                  */
#define CT2G_ENODEV 6   /* no usable sm_100 device                             */

/* softening kernels */
#define CT2G_SOFT_PLUMMER 0 /* 1/sqrt(r^2+h^2) for every pair                      */
#define CT2G_SOFT_SPHERE 1  /* the reference's compact uniform-sphere kernel,      */
                            /* src/kick.cpp:52-60: Newtonian beyond r = h          */

#define CT2G_MAX_ORDER 6

/* Options: the fields of the reference's struct options read by the gravity
 * step (cosmictiger/options.hpp:14-32; defaults src/options.cpp:50-62,88),
 * plus the mesh / order / kernel choices the reference leaves to Ncell and to
 * sfmm.  Ncell = cbrt(count/ppcell)+4 (src/particle.cpp:355) becomes an
 * explicit power-of-two `mesh`; PORDER (cosmictiger/cosmictiger.hpp:16)
 * becomes the runtime `order`. */
typedef struct {
  float bwidth;         /* direct-sum stencil: cell offsets |o|^2 <= bwidth^2      */
  float hsoft;          /* softening length, box units                             */
  float eta;            /* rung accuracy parameter                                 */
  float GM;             /* G * particle mass; 0 -> 1/nparts at upload              */
  int mesh;             /* cells per dimension: power of two, 8..512               */
  int order;            /* multipole expansion order p, 1..CT2G_MAX_ORDER          */
  int kernel;           /* CT2G_SOFT_*                                             */
  int device;           /* CUDA device ordinal                                     */
  size_t max_particles; /* capacity reserved at create (0: sized by first upload)  */
} ct2g_options;

/* kick parameters, field for field cosmictiger/kick.hpp:10-20 */
typedef struct {
  int ascending;
  int descending;
  int top;
  int first;
  int rung;
  float t0;
  float eta;
  float max_dt;
  float scale;
} ct2g_kick_params;

typedef struct ct2g_ctx ct2g_ctx;

/* Reference defaults (src/options.cpp:50-62): bwidth 3, hsoft 1/50, eta 0.15;
 * plus mesh 64, order 4, Plummer kernel, device 0. */
void ct2g_default_options(ct2g_options *opt);

/* Context lifetime; replaces the reference's process-global particle and
 * option state (src/particle.cpp:17-25, src/options.cpp:14,36-42). */
int ct2g_create(const ct2g_options *opt, ct2g_ctx **out);
int ct2g_destroy(ct2g_ctx *ctx);
const char *ct2g_last_error(const ct2g_ctx *ctx);
const char *ct2g_status_string(int status);
/* get_options() (cosmictiger/options.hpp:34) */
int ct2g_get_options(const ct2g_ctx *ctx, ct2g_options *out);
/* change hsoft / eta / GM without rebuilding (GM <= 0 keeps the current value) */
int ct2g_set_params(ct2g_ctx *ctx, float hsoft, float eta, float GM);

/* Particle store: replaces particle_allocate + particles_init + the SoA
 * accessors (src/particle.cpp:273-288,364-374; cosmictiger/particle.hpp:22-56).
 * Host pointers; rung may be NULL (all 0).  Assigns ids 0..n-1. */
int ct2g_upload_particles(ct2g_ctx *ctx, const uint32_t *x, const uint32_t *y,
                          const uint32_t *z, const float *vx, const float *vy,
                          const float *vz, const int8_t *rung, size_t n);
/* Host pointers; any may be NULL.  Current (cell-sorted) order. */
int ct2g_download_particles(ct2g_ctx *ctx, uint32_t *x, uint32_t *y, uint32_t *z,
                            float *vx, float *vy, float *vz, int8_t *rung,
                            uint32_t *ids);
/* particle_count() (src/particle.cpp:27) */
size_t ct2g_particle_count(const ct2g_ctx *ctx);

/* particle_to_grid() (src/particle.cpp:349-362; cosmictiger/particle.hpp:62):
 * stable sort of the current range [rung_begin, n) by cell.  Each particle
 * lands in the leaf the reference's bisection (particle.cpp:69-114) reaches,
 * and the cells follow one another in the bisection's (Morton, x-major bit
 * interleave) order; inside a cell the previous order is kept. */
int ct2g_particle_to_grid(ct2g_ctx *ctx);
/* particle_get_cell(i,j,k) (cosmictiger/particle.hpp:70) for every cell at
 * once: host int64 [mesh^3] each, indexed (i*mesh+j)*mesh+k, absolute
 * particle index ranges [begin, end). */
int ct2g_download_cells(ct2g_ctx *ctx, int64_t *cell_begin, int64_t *cell_end);

/* particle_compute_multipoles (src/particle.cpp:180-209): per-cell Cartesian
 * moments about the cell centre, accumulated in FP64, stored FP32. */
int ct2g_compute_multipoles(ct2g_ctx *ctx);
/* host float[ncomp(order)][mesh^3] */
int ct2g_download_multipoles(ct2g_ctx *ctx, float *out);

/* particle_compute_expansions (src/particle.cpp:211-271): forward r2c FFT of
 * every moment grid, Green's multiply (MG2L, particle.cpp:244-250) with the
 * cached k-space Green's tensor (particle_greens, particle.cpp:116-178),
 * inverse c2r FFT into per-cell local expansions. */
int ct2g_compute_expansions(ct2g_ctx *ctx);
/* host float[ncomp(order)][mesh^3]: particle_get_expansion
 * (cosmictiger/particle.hpp:71) for every cell */
int ct2g_download_expansions(ct2g_ctx *ctx, float *out);
/* host float[ncomp(order)][mesh][mesh][mesh/2+1]: the k-space Green's tensor,
 * normalised by 1/mesh^3; real part for even |n|, imaginary part for odd |n| */
int ct2g_download_greens(ct2g_ctx *ctx, float *out);

/* Forces of the current range (L2P far field + direct-sum near field,
 * src/kick.cpp:19-74), without touching velocities. */
int ct2g_compute_forces(ct2g_ctx *ctx);
/* host float[n] each, current order; pot may be NULL.  Accelerations include
 * GM.  Entries outside the current range are zero.  The potential is computed
 * by ct2g_compute_forces only (ct2g_kick skips it; it then reads as zero). */
int ct2g_download_forces(ct2g_ctx *ctx, float *fx, float *fy, float *fz, float *pot);
/* host float[n] each: replaces the force buffer (for update-only tests) */
int ct2g_upload_forces(ct2g_ctx *ctx, const float *fx, const float *fy, const float *fz);
/* velocity + rung update of kick_cell (src/kick.cpp:75-99) from the force
 * buffer, over the current range; *max_rung receives the largest new rung */
int ct2g_kick_update(ct2g_ctx *ctx, const ct2g_kick_params *p, int *max_rung);

/* int kick(const kick_params&) (cosmictiger/kick.hpp:24, src/kick.cpp:105-125):
 * forces + update over the current range; returns the max rung in *max_rung.
 * Requires ct2g_particle_to_grid (and the mesh stages, which it runs if the
 * expansions are stale). */
int ct2g_kick(ct2g_ctx *ctx, const ct2g_kick_params *p, int *max_rung);

/* void drift(float dt, float scale) (cosmictiger/drift.hpp:12,
 * src/drift.cpp:4-18): x += fixed32(v * dt/scale) for every particle */
int ct2g_drift(ct2g_ctx *ctx, float dt, float scale);

/* int kick_step(int& minrung, int max_rung, double scale, double adot,
 * double tau, double t0, int minrung0, bool nocrop) (cosmictiger/kick.hpp:23,
 * src/main.cpp:8-92): the rung-hierarchical KDK step, GPU-resident.
 * *minrung is updated like the reference's reference argument; the return
 * value of the reference goes to *out_max_rung (may be NULL).  That value is
 * the max_rung argument itself: in the reference the max_rung that each level
 * declares from kick() (main.cpp:68) shadows the parameter and has gone out of
 * scope at the return (main.cpp:90).  The highest rung after the step, which
 * the next call's max_rung should be, is ct2g_rung_counts' *nrungs - 1.  The
 * rung stack carries over between calls as in the reference: a call whose
 * max_rung is above minrung pops one level per rung above it, pushed by the
 * previous call's descending levels (CT2G_ESTATE if the stack runs out). */
int ct2g_kick_step(ct2g_ctx *ctx, int *minrung, int max_rung, double scale, double adot,
                   double tau, double t0, int minrung0, int nocrop, int *out_max_rung);

/* One kick + drift of every particle: particle_to_grid, kick (far field, near
 * field, velocity and rung update) and drift -- the body of the reference's
 * single-level step (src/main.cpp:49,68,81 at one rung level:
 * particle_to_grid(), kick(kparams), drift(dt, scale)).  flags & CT2G_STEP_GRAPH: the sequence is recorded once
 * into a CUDA graph and replayed while the parameters, the particle count and
 * the buffers stay the same (any change records it again); the step then needs
 * no host round trip.  *max_rung (may be NULL: no wait) gets kick()'s return
 * value; with NULL the call returns as soon as the work is queued. */
#define CT2G_STEP_GRAPH 1
int ct2g_kick_drift(ct2g_ctx *ctx, const ct2g_kick_params *p, float dt, float scale, int flags,
                    int *max_rung);

/* One kick + drift from host state to host state: the same step as
 * ct2g_upload_particles (same n as the last upload), ct2g_kick_drift and
 * ct2g_download_particles in a row, with the same results bit for bit, but
 * with the velocity and rung upload overlapping binning and the force solve
 * (they are gathered into cell order just before the update).  No
 * counterpart in the reference, whose particles live in host memory.
 * Inputs: host arrays of n particles (rung may be NULL: all 0); ids are set
 * to 0..n-1 in input order, as an upload does, and the box counts of a box
 * context stay as set.  Outputs: host arrays in the new (cell-sorted) order,
 * any may be NULL; ids_out maps them back to input order.  Pinned host
 * memory gives the copies their full rate.  *max_rung (may be NULL) gets
 * kick()'s return value.  Returns once the outputs are written. */
int ct2g_kick_drift_host(ct2g_ctx *ctx, const ct2g_kick_params *p, float dt, float scale,
                         int flags, const uint32_t *x, const uint32_t *y, const uint32_t *z,
                         const float *vx, const float *vy, const float *vz, const int8_t *rung,
                         size_t n, uint32_t *x_out, uint32_t *y_out, uint32_t *z_out,
                         float *vx_out, float *vy_out, float *vz_out, int8_t *rung_out,
                         uint32_t *ids_out, int *max_rung);

/* Many independent periodic boxes.  No counterpart in the reference (one box
 * per process there).  A box context holds nbox unit boxes that share the
 * mesh, order, stencil and softening of *opt (so they share one Green's
 * table); each box has its own particles and its own GM.  Upload the boxes'
 * particles concatenated box after box with ct2g_upload_particles, then call
 * ct2g_set_boxes with the per-box counts (summing to the upload) and GM
 * (G x particle mass) before particle_to_grid.  Particles stay inside their
 * box's range of the store.  Requires 3*log2(mesh) + ceil(log2(nbox)) <= 32.
 * Grid downloads hold [component][box][cell]; ct2g_download_cells gives
 * nbox*mesh^3 ranges, box-major.  Rung levels (ct2g_sort_by_rung,
 * ct2g_kick_step) need nbox == 1. */
int ct2g_create_boxes(const ct2g_options *opt, int nbox, ct2g_ctx **ctx);
int ct2g_set_boxes(ct2g_ctx *ctx, const uint64_t *counts, const float *GM);
int ct2g_box_count(const ct2g_ctx *ctx);

/* A batch: several contexts on one device (e.g. box contexts of different
 * meshes) stepped together by ONE graph launch on the first context's stream;
 * each context's stages run on its own stream inside the graph, so the
 * contexts overlap on the GPU.  No counterpart in the reference. */
typedef struct ct2g_batch ct2g_batch;
int ct2g_batch_create(ct2g_ctx *const *ctxs, int nctx, ct2g_batch **out);
/* kick + drift of every context, as ct2g_kick_drift with CT2G_STEP_GRAPH;
 * *max_rung (may be NULL: no wait) = the largest over the contexts */
int ct2g_batch_kick_drift(ct2g_batch *b, const ct2g_kick_params *p, float dt, float scale,
                          int *max_rung);
/* device time (ms) of the last batch launch; waits for it */
int ct2g_batch_last_ms(ct2g_batch *b, float *ms);
int ct2g_batch_destroy(ct2g_batch *b);

/* Tunable launch shapes of a context (no counterpart in the reference):
 * dense_cell -- cells with at least this many particles get their own sink
 * chunks, the sinks of sparser cells take the sparse path; near_blocks_per_sm
 * -- blocks per SM of the persistent near-field grid (0: occupancy limit);
 * fft_tile -- columns per tile of the y/x FFT passes (0: default); split_mg2l
 * -- 1 runs the X FFT passes and the Green's-function multiply as three
 * kernels, 0 (the default) as one wherever a spectrum column of all
 * components fits in shared memory; sparse_path -- 2 (the default): the
 * sparse sinks of a 4x4x4 cell block share a warp; the candidate cells of
 * the union of their stencils go in windows of 32, every lane tabulates
 * which of them lie in its own stencil, and the window's sources are
 * streamed in full batches of 32 staged in shared memory, each evaluated by
 * every lane times its table entry (the Plummer kernel; the sphere kernel
 * takes 1); 1: the same chunks, the union walked cell by cell, each cell's
 * sources staged as their own batch; 0: one sparse sink per warp lane, each
 * lane walking its own stencil and reading its own sources (no masked work,
 * but every lane gathers its own sources through the L1 cache); overlap -- 1: the near field runs on a second stream
 * beside the mesh solve (from the end of binning to the L2P pass) into its
 * own buffers, added to the far field afterwards in the same order as the
 * serial form (0), so both give the same forces bit for bit; the per-stage
 * times then show only the part of the near field the mesh solve did not
 * hide; mg2l_greens_direct -- 1: the fused x pass + Green's multiply reads
 * the Green's values straight from HBM inside the contraction instead of
 * staging each column in shared memory first (one more block per SM; the
 * same results); near_chunks_per_warp -- with overlap, > 0: a near-field warp
 * takes at most this many sink chunks before its block exits, so that the
 * mesh solve's blocks (on the context stream, which has the higher priority)
 * get SMs in between; 0: the near-field grid is persistent; plane_pipe --
 * D > 0 (up to 16): the forward z pass (with P2M) and y pass run as one
 * persistent kernel that hands out the z lines and y tiles of the x planes
 * in turn, the y tiles of a plane D planes after its z lines, each waiting
 * (bounded) for its plane's z lines, so that the y pass reads the plane from
 * L2; the inverse y pass and z pass (with L2P) likewise, the z lines dropping
 * the L2 lines they have read (PTX discard.global.L2) instead of letting them
 * be written back; the same results as 0 (separate passes); meshes 64-256
 * with the FP32 passes (others run the separate passes); cols_tma -- 1 (the
 * default): every FP32 column FFT pass with 16-byte aligned rows (the mesh's
 * y passes, the r2c / c2r / complex 3D FFT entry points) moves each tile
 * (all N rows x 32 complex columns; 16 with fft_tile 16 or at N = 512) by
 * tiled bulk tensor copies (TMA) in and out, three tiles in flight per
 * block (N 64-512); 0: every thread copies its share of each tile
 * (cp.async, two tiles in flight); the same results; x_tma -- 1: the fused x
 * pass + Green's multiply brings each spectrum column in by one tiled bulk
 * tensor copy and its Green's column by one bulk copy (meshes 64-256, FP32
 * passes; with mg2l_greens_direct the Green's values are read by the
 * contraction instead, and three blocks fit per SM); 2 (the default): the
 * column by per-thread cp.async copies, all in flight at once, into rows NC complex
 * apart (the tensor copy's 16-byte-multiple rows put the contraction's
 * shared-memory reads into a few banks); 0: per-thread loads inside the
 * first transform step; the same results; p2m_compact -- 1: the cells'
 * multipole moments are summed by a cell-parallel pass (the thread of a
 * cell's first particle, a warp per cell of more than 6 particles) into
 * compact records
 * of the occupied cells (capacity: NC floats per particle), which the
 * forward z pass then reads; 0 (the default): the z pass sums them itself,
 * a line's cells at a time; the same results. */
typedef struct {
  int dense_cell;
  int near_blocks_per_sm;
  int fft_tile;
  int split_mg2l;
  int sparse_path;
  int overlap;
  int mg2l_greens_direct;
  int near_chunks_per_warp;
  int plane_pipe;
  int cols_tma;
  int x_tma;
  int p2m_compact;
} ct2g_tuning;
int ct2g_get_tuning(const ct2g_ctx *ctx, ct2g_tuning *t);
int ct2g_set_tuning(ct2g_ctx *ctx, const ct2g_tuning *t);
/* Autotuner: times ct2g_kick_drift (graph replays) on the context's current
 * particles for candidate tunings, keeps the fastest and restores the
 * particles afterwards.  cache_path (may be NULL): a text file of
 * "key dense_cell near_blocks_per_sm fft_tile sparse_path overlap
 * mg2l_greens_direct near_chunks_per_warp plane_pipe cols_tma x_tma p2m_compact ms"
 * lines; a hit for this
 * context's key (mesh, order, bwidth, boxes, particle-count octave) is used
 * without timing, a miss is appended.  *out (may be NULL) gets the choice. */
int ct2g_autotune(ct2g_ctx *ctx, const ct2g_kick_params *p, float dt, float scale,
                  const char *cache_path, ct2g_tuning *out);

/* Learned near-field correction.  No counterpart in the reference.
 *
 * For selected sink cells the direct sum is widened from the stencil
 * |o|^2 <= bwidth^2 to |o|^2 <= bwidth_ext^2: the shell's particles are summed
 * exactly and the mesh's Taylor term for those cells is subtracted, so a
 * selected cell gets the forces of the method run with bwidth_ext.  Cells are
 * selected by CT2G_SELECT_FIXED (score = the shell's monopole pull relative to
 * the sink's force, above `threshold`), CT2G_SELECT_MLP (an MLP of 24 per-cell
 * moment and density features -> 64 -> 64 -> 1, BF16 weights, FP32
 * accumulation, predicts log10 of the cell's rms relative force residual;
 * selected above `threshold`) or CT2G_SELECT_ALL.  Once a mode is set, every
 * force computation (ct2g_compute_forces, ct2g_kick, ct2g_kick_drift) applies
 * it.  Training: ct2g_learned_collect computes, for the current state, the
 * plain forces, the widened forces with every cell corrected, and appends
 * one (features, log10 residual) sample per occupied cell to the device
 * training set; ct2g_mlp_train runs Adam on it with the library's own
 * forward and backward kernels.  Parameters: W1[64][24], b1[64], W2[64][64],
 * b2[64], W3[64], b3 (CT2G_MLP_NPARAM floats); features are normalised by
 * (x - fmean) / fstd. */
#define CT2G_SELECT_NONE 0
#define CT2G_SELECT_FIXED 1
#define CT2G_SELECT_MLP 2
#define CT2G_SELECT_ALL 3
#define CT2G_MLP_NIN 24
#define CT2G_MLP_NHID 64
#define CT2G_MLP_NPARAM 5825
/* shell tables for bwidth < bwidth_ext <= 8 (2*bwidth_ext+1 <= mesh); order >= 2 */
int ct2g_learned_enable(ct2g_ctx *ctx, float bwidth_ext);
int ct2g_learned_select(ct2g_ctx *ctx, int mode, float threshold);
/* after particle_to_grid; *ncells = samples added */
int ct2g_learned_collect(ct2g_ctx *ctx, size_t *ncells);
/* training set: *n samples; copies min(cap, n) rows of X [n][24] and T [n] */
int ct2g_learned_dataset(ct2g_ctx *ctx, float *X, float *T, size_t cap, size_t *n);
int ct2g_learned_clear(ct2g_ctx *ctx);
/* cells of the last selection pass: keys, features, fixed-criterion scores,
 * MLP predictions, selected flags (each may be NULL; min(cap, ncells) rows) */
int ct2g_learned_cells(ct2g_ctx *ctx, uint32_t *keys, float *X, float *score, float *pred,
                       uint8_t *selected, size_t cap, size_t *ncells, size_t *nselected);
int ct2g_mlp_init(ct2g_ctx *ctx, uint64_t seed);
int ct2g_mlp_set(ct2g_ctx *ctx, const float *params, const float *fmean, const float *fstd);
int ct2g_mlp_get(ct2g_ctx *ctx, float *params, float *fmean, float *fstd);
/* epochs of Adam over the training set in shuffled batches; normalize != 0
 * first sets fmean/fstd from the set; *loss = final mean squared error */
int ct2g_mlp_train(ct2g_ctx *ctx, int epochs, int batch, float lr, uint64_t seed, int normalize,
                   float *loss);
/* gradient of the mean squared error over n host samples (raw features X
 * [n][24], targets T[n]) at the current weights, as the training step
 * computes it: grad[CT2G_MLP_NPARAM], *loss */
int ct2g_mlp_gradients(ct2g_ctx *ctx, const float *X, const float *T, size_t n, float *grad,
                       float *loss);

/* Rung bookkeeping (src/particle.cpp:31-57,320-347). */
int ct2g_sort_by_rung(ct2g_ctx *ctx, int minrung);        /* particle_sort_by_rung   */
int ct2g_push_rungs(ct2g_ctx *ctx);                       /* particle_push_rungs     */
int ct2g_pop_rungs(ct2g_ctx *ctx);                        /* particle_pop_rungs      */
int ct2g_set_minrung(ct2g_ctx *ctx, int minrung);         /* particle_set_minrung    */
int ct2g_current_range(ct2g_ctx *ctx, size_t *begin, size_t *end); /* particle_current_range */
/* particle_rung_counts: counts[0..nmax) (host); *nrungs = highest rung + 1 */
int ct2g_rung_counts(ct2g_ctx *ctx, size_t *counts, int nmax, int *nrungs);

/* 3D FFTs, replacing fft_r2c_3d / fft_c2r_3d (cosmictiger/fft.hpp:28-29;
 * src/fft/fft_r2c_3d.cpp, src/fft/fft_c2r_3d.cpp) in FP64 with the
 * reference's split-plane halfcomplex layout (src/particle.cpp:220,236-237):
 * xin[N^3] real, index (i*N+j)*N+k; xout[2*dimag], dimag = N*N*(N/2+1), real
 * parts at [0,dimag) and imaginary parts at [dimag,2*dimag), index
 * (i*N+j)*(N/2+1)+k.  Forward: X(q) = sum_r x(r) exp(-2 pi i q.r/N).
 * c2r is the unnormalised inverse (c2r(r2c(x)) = N^3 x).  Host pointers;
 * batch transforms of consecutive arrays.  N: power of two, 4..512. */
int ct2g_fft_r2c_3d(ct2g_ctx *ctx, const double *xin, double *xout, int N, int batch);
int ct2g_fft_c2r_3d(ct2g_ctx *ctx, const double *xin, double *xout, int N, int batch);
/* The reference's 1D FFT surface (cosmictiger/fft.hpp:18-27), computed on the
 * GPU in FP64; host arrays, transformed in place.  Several independent
 * sequences ("lanes") interleave element by element like the reference's
 * 4-lane SIMD type: real element n of lane l at X[n*lanes + l]; complex
 * element n at X[(2n)*lanes + l] (real part) and X[(2n+1)*lanes + l]
 * (imaginary part).  Inputs arrive in bit-reversed order (scrambled, as
 * src/fft/fft_test.cpp:81-159 prepares them); dir = +1 is the forward DFT
 * sum_n x(n) exp(-2 pi i n k/N), dir = -1 the same with exp(+2 pi i n k/N)
 * (the reference's dir = -1 path is not a usable transform; this is the one
 * its inverse twiddle table, src/fft/twiddles.cpp:44-56, describes).
 * N: power of two, 2..8192.
 *   ct2g_fft1d_real:    fft_real(fft_float*, N, dir) with lanes = 1 and
 *                       fft_real(fft_simd*, N, dir) with lanes = 4
 *                       (fft.hpp:25-26, src/fft/fft_real_scalar.cpp,
 *                       fft_real_vector.cpp); output in halfcomplex order:
 *                       X[0], Re X(1)..Re X(N/2), Im X(N/2-1)..Im X(1).
 *   ct2g_fft1d_complex: fft_complex(complex<fft_simd>*, N, dir) with lanes =
 *                       4 (fft.hpp:27, src/fft/fft_complex_vector.cpp);
 *                       output in natural order. */
int ct2g_fft1d_real(ct2g_ctx *ctx, double *X, int N, int lanes, int dir);
int ct2g_fft1d_complex(ct2g_ctx *ctx, double *X, int N, int lanes, int dir);
/* scramble(X, N1, N2, N3) (fft.hpp:21, src/fft/scramble.cpp:26-43): in each
 * of N1 blocks of N2 rows of N3 values, row j trades places with row
 * bitrev(j).  N2: power of two. */
int ct2g_scramble(ct2g_ctx *ctx, double *X, int N1, int N2, int N3);
/* transpose_yz(X, N) (fft.hpp:18, src/fft/transpose.cpp:7-31,118-120): X[ix][iy][iz]
 * becomes X[ix][iz][iy].  (The reference swaps every pair twice, which leaves
 * X unchanged; this is the transpose its 3D drivers rely on.)  N <= 512. */
int ct2g_transpose_yz(ct2g_ctx *ctx, double *X, int N);
/* transpose_r2c(xin, xout, N) (fft.hpp:19, src/fft/transpose.cpp:33-72):
 * xin[N][N][N] holds halfcomplex rows along y; xout receives the split planes,
 * re[(ix*N+iz)*(N/2+1)+iy] = xin[ix][iy][iz] and im[same] = xin[ix][N-iy][iz]
 * (0 at iy = 0, N/2) at offset N*N*(N/2+1).  N even, <= 512. */
int ct2g_transpose_r2c(ct2g_ctx *ctx, const double *xin, double *xout, int N);
/* transpose_c2r(xin, xout, N) (fft.hpp:20, src/fft/transpose.cpp:74-116):
 * the inverse of ct2g_transpose_r2c.  (The reference reads its input with a
 * row stride of N where transpose_r2c writes N/2+1, and starts its z loop at
 * the block's y coordinate; this is the inverse both are meant to be.) */
int ct2g_transpose_c2r(ct2g_ctx *ctx, const double *xin, double *xout, int N);
/* cos_twiddles / sin_twiddles / inv_sin_twiddles (fft.hpp:22-24,
 * src/fft/twiddles.cpp): out[n] = cos(-2 pi n/N) (which 0), sin(-2 pi n/N)
 * (which 1), sin(2 pi n/N) (which 2), n < N. */
int ct2g_twiddles(ct2g_ctx *ctx, int which, int N, double *out);
/* The device-pointer entry points below queue their kernels on the context's
 * stream (ct2g_stream), a non-blocking stream created at the highest stream
 * priority: it is not ordered with the legacy default stream nor with the
 * caller's streams.  A caller that fills or reads the buffers on a stream of
 * its own makes the context's stream wait for that stream first (an event)
 * and its own stream wait for the context's afterwards. */
/* FP32 device-pointer variant on the context stream, interleaved complex
 * output (float2[batch][N][N][N/2+1]); dir = +1 forward r2c, -1 inverse c2r */
int ct2g_fft3d_f32_dev(ct2g_ctx *ctx, int dir, void *d_real, void *d_complex, int N,
                       int batch);
/* Complex-to-complex 3D FFT of `batch` device grids float2[batch][N][N][N]
 * (k contiguous), in place, FP32, on the context's stream: dir = +1 forward
 * (exp(-2 pi i q.r/N)), -1 the unnormalised inverse.  With CT2G_FFT_TC_BF16X3
 * set (and N equal to the context's mesh) the y and x passes run on the
 * tensor cores.  No counterpart in the reference.  N: power of two, 4..512;
 * the grid 16-byte aligned. */
int ct2g_fft3d_c2c_f32_dev(ct2g_ctx *ctx, int dir, void *d_data, int N, int batch);
/* Cloud-in-cell deposit of the context's particles (unit mass) onto four
 * complex device grids float2[4][N][N][N] (zeroed first): the real parts hold
 * the CIC mass and the three first moments about each mesh point (offsets in
 * mesh units), the imaginary parts zero.  A particle at x lies between mesh
 * points floor(xN - 1/2) and the next, with linear weights per axis.  No
 * counterpart in the reference. */
int ct2g_cic_deposit(ct2g_ctx *ctx, int N, void *d_grid);

/* FP64 Ewald direct sum over ALL particles of the context as sources, at the
 * given sink positions (host, fixed32): the force truth.  f: host double[3*ns]
 * (interleaved xyz), pot: host double[ns] or NULL.  Same kernel/softening/GM
 * as the context. */
int ct2g_ewald_direct(ct2g_ctx *ctx, const uint32_t *sx, const uint32_t *sy,
                      const uint32_t *sz, size_t ns, double alpha, double rcut, int kmax,
                      double *f, double *pot);

/* Allocation-free FP64 Ewald direct sum.  No counterpart in the reference.
 * For callers that cannot allocate device memory themselves (a framework that
 * owns all device memory, a loop where cudaMalloc is not allowed): every
 * pointer is a DEVICE pointer owned by the caller -- sources qx,qy,qz[nq],
 * sinks sx,sy,sz[ns] (fixed32), outputs f[3*ns] (interleaved xyz) and pot[ns]
 * (both required) -- and the only scratch, the structure factor, lives in a
 * static device array of the library (about 0.94 MB per GPU, held until the
 * process exits).  kmax must be <= 24, the size that array holds; larger
 * values return CT2G_EINVAL, as do more than 65535*4096 sources.  The first
 * call on a device looks the array up (cudaGetSymbolAddress), so make it
 * before any stream capture.  Calls share the array: calls that overlap on
 * the GPU race.  Work is queued on `stream` (a cudaStream_t, or NULL for the
 * default stream); nothing is allocated.  The calling thread's current device
 * is the same on return as on entry; an error already pending from the
 * caller's own work is left in place and the call returns CT2G_ECUDA without
 * running. */
int ct2g_ewald_direct_noalloc(int device, const uint32_t *qx, const uint32_t *qy,
                              const uint32_t *qz, size_t nq, const uint32_t *sx,
                              const uint32_t *sy, const uint32_t *sz, size_t ns, int kernel,
                              double soft, double GM, double alpha, double rcut, int kmax,
                              double *f, double *pot, void *stream);

/* Self-test of the tcgen05 building blocks (tensor memory, UMMA descriptors,
 * MMA completion) the tensor-core passes use.  No counterpart in the
 * reference.  One CTA computes D[128][N] = A[128][K] * B[N][K]^T with the
 * operands rounded to BF16 and FP32 accumulation; host arrays, row-major;
 * N in {32, 64}, K in {16, 32, 64, 96}.  CT2G_ETIMEOUT if the MMA did not
 * complete within the kernel's bounded wait. */
int ct2g_tc_selftest(int device, const float *A, const float *B, int N, int K, float *D);

/* Failure-path self-test.  No counterpart in the reference.  Queues on the
 * context's stream a kernel whose threads wait, `polls` times each (1..2^22,
 * a few ns apart), on an mbarrier that nothing arrives at; the wait gives up
 * and the kernel records CT2G_ETIMEOUT in the context's device error word,
 * the path the tensor-core passes take when an MMA completion does not
 * arrive.  The next ct2g_synchronize reports CT2G_ETIMEOUT and clears it; the
 * context stays usable. */
int ct2g_wait_selftest(ct2g_ctx *ctx, uint32_t polls);

/* FFT arithmetic of the mesh solve (precision form).  No counterpart in the
 * reference.  CT2G_FFT_FP32 (default): every pass on the CUDA cores in FP32.
 * CT2G_FFT_TC_BF16X3: the y and x passes as radix-R2 x radix-16 DFT matrix
 * products on the tensor cores (tcgen05), operands split into BF16 hi + lo
 * parts (three products per term, FP32 accumulation); meshes 256 and 512.
 * Applies to every later mesh solve of the context and to ct2g_fft3d_f32_dev. */
#define CT2G_FFT_FP32 0
#define CT2G_FFT_TC_BF16X3 1
int ct2g_set_fft_mode(ct2g_ctx *ctx, int mode);

/* Stream and timing helpers.  ct2g_synchronize also reports a status a
 * kernel left behind (CT2G_ETIMEOUT: a bounded device-side wait gave up). */
void *ct2g_stream(ct2g_ctx *ctx);   /* the context's cudaStream_t */
int ct2g_synchronize(ct2g_ctx *ctx);
/* Per-stage device times (ms) of the last ct2g_kick / ct2g_kick_step call:
 * [0] bin, [1] P2M, [2] forward FFT, [3] MG2L, [4] inverse FFT, [5] forces,
 * [6] kick update + drift.  n >= 7. */
int ct2g_stage_times(ct2g_ctx *ctx, float *ms, int n);
/* Number of kernel launches issued by this context since creation. */
uint64_t ct2g_launch_count(const ct2g_ctx *ctx);
/* Near-field pair interactions of the last force computation (exact count). */
uint64_t ct2g_interaction_count(const ct2g_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* CT2G_H_ */
