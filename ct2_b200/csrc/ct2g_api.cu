// C ABI: context lifetime, particle store, stage entry points, the
// rung-hierarchical kick_step driver (src/main.cpp:8-92) and rung bookkeeping
// (src/particle.cpp:31-57,320-347).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ct2g_internal.cuh"

int ct2g_upload_stencil(ct2g_ctx *ctx, const std::vector<int> &st4);
int ct2g_fft_init(ct2g_ctx *ctx);

int ct2g_fail(ct2g_ctx *ctx, int code, const std::string &msg) {
  if (ctx) ctx->err = msg;
  return code;
}

int ct2g_cuda_fail(ct2g_ctx *ctx, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
  if (ctx) ctx->err = m;
  return e == cudaErrorMemoryAllocation ? CT2G_ENOMEM : CT2G_ECUDA;
}

namespace {

// stable partition of [b, e) by rung < minrung (front) / >= minrung (back)
__global__ void rung_flag_kernel(const int8_t *__restrict__ rung, size_t b, size_t nr,
                                 int minrung, uint32_t *__restrict__ flags) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nr) flags[i] = rung[b + i] < minrung ? 1u : 0u;
}

__global__ void rung_scatter_kernel(const uint32_t *__restrict__ flags,
                                    const uint32_t *__restrict__ fscan, size_t b, size_t nr,
                                    uint32_t nlow, uint32_t *__restrict__ perm) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  uint32_t dst = flags[i] ? fscan[i] : nlow + ((uint32_t)i - fscan[i]);
  perm[dst] = (uint32_t)i;
}

template <typename T>
__global__ void permute_kernel(const uint32_t *__restrict__ perm, size_t b, size_t nr,
                               const T *__restrict__ in, T *__restrict__ out) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nr) out[b + i] = in[b + perm[i]];
}

__global__ void rung_count_kernel(const int8_t *__restrict__ rung, size_t n,
                                  unsigned long long *__restrict__ counts) {
  __shared__ unsigned int c[128];
  if (threadIdx.x < 128) c[threadIdx.x] = 0;
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    int r = rung[i];
    atomicAdd(&c[r & 127], 1u);
  }
  __syncthreads();
  if (threadIdx.x < 128 && c[threadIdx.x]) atomicAdd(&counts[threadIdx.x], (unsigned long long)c[threadIdx.x]);
}

__global__ void set_minrung_kernel(int8_t *__restrict__ rung, size_t n, int minrung) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && rung[i] < minrung) rung[i] = (int8_t)minrung;
}

__global__ void iota_kernel(uint32_t *__restrict__ id, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) id[i] = (uint32_t)i;
}

bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

void free_particles(ct2g_ctx *ctx) {
  void *ptrs[] = {ctx->x, ctx->y, ctx->z, ctx->id, ctx->vx, ctx->vy, ctx->vz, ctx->rung,
                  ctx->x2, ctx->y2, ctx->z2, ctx->id2, ctx->vx2, ctx->vy2, ctx->vz2, ctx->rung2,
                  ctx->keys, ctx->keys2, ctx->vals, ctx->vals2, ctx->hist, ctx->src,
                  ctx->chunks, ctx->sparse_list, ctx->flags, ctx->fx,
                  ctx->fy, ctx->fz,
                  ctx->pot, ctx->nfx, ctx->nfy, ctx->nfz, ctx->npot, ctx->cmom, ctx->p2m_big};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  ctx->x = ctx->y = ctx->z = ctx->id = nullptr;
  ctx->vx = ctx->vy = ctx->vz = nullptr;
  ctx->rung = nullptr;
  ctx->x2 = ctx->y2 = ctx->z2 = ctx->id2 = nullptr;
  ctx->vx2 = ctx->vy2 = ctx->vz2 = nullptr;
  ctx->rung2 = nullptr;
  ctx->keys = ctx->keys2 = ctx->vals = ctx->vals2 = ctx->hist = nullptr;
  ctx->src = nullptr;
  ctx->chunks = nullptr;
  ctx->sparse_list = ctx->flags = nullptr;
  ctx->fx = ctx->fy = ctx->fz = ctx->pot = nullptr;
  ctx->nfx = ctx->nfy = ctx->nfz = ctx->npot = nullptr;
  ctx->cmom = nullptr;
  ctx->p2m_big = nullptr;
  ctx->cap = 0;
}

int check(ct2g_ctx *ctx) {
  if (!ctx) return CT2G_EINVAL;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ct2g_cuda_fail(ctx, e, "cudaSetDevice");
  return CT2G_OK;
}

int ensure_grid(ct2g_ctx *ctx) {
  if (!ctx->has_particles) return ct2g_fail(ctx, CT2G_ESTATE, "no particles uploaded");
  if (!ctx->grid_valid) return ct2g_fail(ctx, CT2G_ESTATE, "particle_to_grid has not run since the particles moved");
  return CT2G_OK;
}

}  // namespace

void ct2g_mark(ct2g_ctx *ctx, int k) {
  if (!ctx->capturing) cudaEventRecord(ctx->ev[k], ctx->stream);
}

int ct2g_check(ct2g_ctx *ctx) { return check(ctx); }

// compact P2M records for the particle capacity: NC floats per occupied
// cell (at most one cell per particle) and the big-cell list (count first;
// a big cell holds more than 6 particles, so at most cap / 7 of them)
int ct2g_alloc_p2m_compact(ct2g_ctx *ctx) {
  if (ctx->cmom || ctx->cap == 0) return CT2G_OK;
  if (ctx->capturing) return ct2g_fail(ctx, CT2G_ESTATE, "compact P2M records not allocated before recording");
  CT2G_CUDA(ctx, cudaMalloc(&ctx->cmom, sizeof(float) * ctx->nc * ctx->cap));
  cudaError_t e = cudaMalloc(&ctx->p2m_big, sizeof(uint32_t) * (ctx->cap / 7 + 2));
  if (e != cudaSuccess) {
    cudaFree(ctx->cmom);
    ctx->cmom = nullptr;
    return ct2g_cuda_fail(ctx, e, "compact P2M big-cell list");
  }
  ctx->epoch++;
  return CT2G_OK;
}

// resident blocks per SM of a kernel from its registers, its shared memory
// (static + dynamic + the 1 KB the system reserves per block) against the
// SM's maximum carveout, and its threads
int ct2g_blocks_per_sm(ct2g_ctx *ctx, const void *kernel, int threads, size_t dyn_smem) {
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  int smem_sm = 0, regs_sm = 0, threads_sm = 0;
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, ctx->device);
  cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, ctx->device);
  cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, ctx->device);
  // registers are allocated per warp in units of 256
  const int regs_warp = ((std::max(1, fa.numRegs) * 32 + 255) / 256) * 256;
  const int warps = (threads + 31) / 32;
  const int by_regs = regs_sm / std::max(1, regs_warp * warps);
  const int by_smem = smem_sm / (int)std::max<size_t>(1, dyn_smem + fa.sharedSizeBytes + 1024);
  const int by_threads = threads_sm / std::max(1, threads);
  return std::max(1, std::min(std::min(by_regs, by_smem), by_threads));
}

int ct2g_device_error(ct2g_ctx *ctx) {
  uint32_t e = 0;
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  CT2G_CUDA(ctx, cudaMemcpy(&e, ctx->d_counts + 6, sizeof(e), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(ctx->d_counts + 6, 0, sizeof(uint32_t));
    return ct2g_fail(ctx, (int)e, "a device-side wait gave up (tensor-core pass)");
  }
  return CT2G_OK;
}

// far field of the current range into the force buffers: moments (if the
// grid does not hold them), then the mesh solve whose inverse z pass
// evaluates L2P for every particle (the moments stay in the grid)
int ct2g_far_field(ct2g_ctx *ctx, bool pot) {
  CT2G_TRY(ensure_grid(ctx));
  ct2g_mark(ctx, 1);
  if (ctx->moments_valid) return ct2g_mesh_solve(ctx, true, pot, CT2G_P2M_GRID);
  // the moments are formed inside the forward z pass; the learned correction
  // reads the moment grid, so then the pass stores them too
  ctx->expansions_valid = false;
  if (ct2g_learned_active(ctx)) {
    CT2G_TRY(ct2g_mesh_solve(ctx, true, pot, CT2G_P2M_FUSED_STORE));
    ctx->moments_valid = true;
    return CT2G_OK;
  }
  return ct2g_mesh_solve(ctx, true, pot, CT2G_P2M_FUSED);
}

// upload the box table (offsets and GM) of the context
static int upload_boxes(ct2g_ctx *ctx) {
  std::vector<uint32_t> off(ctx->nbox + 1);
  for (int b = 0; b <= ctx->nbox; b++) off[b] = (uint32_t)ctx->h_box_off[b];
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->box_off, off.data(), sizeof(uint32_t) * off.size(),
                                 cudaMemcpyHostToDevice, ctx->stream));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->box_gm, ctx->h_box_gm.data(),
                                 sizeof(float) * ctx->h_box_gm.size(), cudaMemcpyHostToDevice,
                                 ctx->stream));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // kernels read the table from device memory: a recorded graph stays valid
  return CT2G_OK;
}

int ct2g_alloc_particles(ct2g_ctx *ctx, size_t n) {
  if (n <= ctx->cap) return CT2G_OK;
  free_particles(ctx);
  ctx->epoch++;
  const size_t cap = n;
  const size_t ntiles = (cap + 4095) / 4096;
#define A(ptr, bytes) CT2G_CUDA(ctx, cudaMalloc(&(ptr), (bytes)))
  A(ctx->x, cap * 4);
  A(ctx->y, cap * 4);
  A(ctx->z, cap * 4);
  A(ctx->id, cap * 4);
  A(ctx->vx, cap * 4);
  A(ctx->vy, cap * 4);
  A(ctx->vz, cap * 4);
  A(ctx->rung, cap);
  A(ctx->x2, cap * 4);
  A(ctx->y2, cap * 4);
  A(ctx->z2, cap * 4);
  A(ctx->id2, cap * 4);
  A(ctx->vx2, cap * 4);
  A(ctx->vy2, cap * 4);
  A(ctx->vz2, cap * 4);
  A(ctx->rung2, cap);
  A(ctx->keys, cap * 4);
  A(ctx->keys2, cap * 4);
  A(ctx->vals, cap * 4);
  A(ctx->vals2, cap * 4);
  A(ctx->hist, ntiles * 256 * 4);
  A(ctx->src, cap * sizeof(float4));
  A(ctx->chunks, cap * sizeof(uint2));
  A(ctx->sparse_list, cap * 4);
  A(ctx->flags, cap * 4);
  A(ctx->fx, cap * 4);
  A(ctx->fy, cap * 4);
  A(ctx->fz, cap * 4);
  A(ctx->pot, cap * 4);
  A(ctx->nfx, cap * 4);
  A(ctx->nfy, cap * 4);
  A(ctx->nfz, cap * 4);
  A(ctx->npot, cap * 4);
#undef A
  ctx->cap = cap;
  if (ctx->p2m_compact) CT2G_TRY(ct2g_alloc_p2m_compact(ctx));
  // scan scratch for the largest scan of a step (radix histograms, cell
  // ranges, per-particle flags), so that no step allocates
  const size_t words = ct2g_scan_scratch_words(
      std::max<size_t>(std::max<size_t>(ntiles * 256, (size_t)ctx->CB + 1), cap));
  if (ctx->scan_tmp_words < words) {
    if (ctx->scan_tmp) cudaFree(ctx->scan_tmp);
    ctx->scan_tmp = nullptr;
    ctx->scan_tmp_words = 0;
    CT2G_CUDA(ctx, cudaMalloc(&ctx->scan_tmp, sizeof(uint32_t) * words));
    ctx->scan_tmp_words = words;
  }
  return ct2g_learned_resize(ctx);
}

int ct2g_alloc_mesh(ct2g_ctx *ctx) {
  const size_t nb = (size_t)ctx->nbox;
  CT2G_CUDA(ctx, cudaMalloc(&ctx->cell_start, sizeof(uint32_t) * (ctx->CB + 1)));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->occ, sizeof(unsigned long long) * (ctx->CB / 64)));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->stmask, sizeof(unsigned long long) * 64 * 27));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->grid, sizeof(float) * ctx->nc * nb * ctx->C));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->spec, sizeof(float2) * ctx->nc * nb * ctx->CK));
  ctx->xmap_bw = 0;  // the x-pass tensor map describes the spectrum's address
  CT2G_CUDA(ctx, cudaMalloc(&ctx->d_counts, sizeof(uint32_t) * 8));
  CT2G_CUDA(ctx, cudaMemset(ctx->d_counts, 0, sizeof(uint32_t) * 8));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->pipe_sync, sizeof(uint32_t) * 2 * (2 + nb * ctx->M)));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->blk_rank, sizeof(uint32_t) * (ctx->CB / 64)));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->box_off, sizeof(uint32_t) * (nb + 1)));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->box_gm, sizeof(float) * nb));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->greens, sizeof(float) * ctx->nc * ctx->CK));
  CT2G_CUDA(ctx, cudaMalloc(&ctx->greens_x, sizeof(float) * ct2g_greens_x_floats(ctx)));
  return CT2G_OK;
}

extern "C" {

void ct2g_default_options(ct2g_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->bwidth = 3.0f;
  o->hsoft = 1.0f / 50.0f;
  o->eta = 0.15f;
  o->GM = 0.0f;
  o->mesh = 64;
  o->order = 4;
  o->kernel = CT2G_SOFT_PLUMMER;
  o->device = 0;
  o->max_particles = 0;
}

const char *ct2g_status_string(int s) {
  switch (s) {
    case CT2G_OK: return "ok";
    case CT2G_EINVAL: return "invalid argument";
    case CT2G_ENOMEM: return "out of device memory";
    case CT2G_ECUDA: return "CUDA error";
    case CT2G_ESTATE: return "call out of order";
    case CT2G_ETIMEOUT: return "device wait timed out";
    case CT2G_ENODEV: return "no usable sm_100 device";
  }
  return "unknown status";
}

const char *ct2g_last_error(const ct2g_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int ct2g_create(const ct2g_options *opt, ct2g_ctx **out) { return ct2g_create_boxes(opt, 1, out); }

int ct2g_create_boxes(const ct2g_options *opt, int nbox, ct2g_ctx **out) {
  if (!opt || !out) return CT2G_EINVAL;
  *out = nullptr;
  if (nbox < 1) return CT2G_EINVAL;
  if (!is_pow2(opt->mesh) || opt->mesh < 8 || opt->mesh > 512) return CT2G_EINVAL;
  if (opt->order < 1 || opt->order > CT2G_MAX_ORDER) return CT2G_EINVAL;
  if (!(opt->bwidth >= 0.f) || 2.0f * opt->bwidth + 1.0f > (float)opt->mesh || opt->bwidth > 4.0f)
    return CT2G_EINVAL;
  if (!(opt->hsoft > 0.f)) return CT2G_EINVAL;
  if (opt->kernel != CT2G_SOFT_PLUMMER && opt->kernel != CT2G_SOFT_SPHERE) return CT2G_EINVAL;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= opt->device || opt->device < 0) {
    cudaGetLastError();
    return CT2G_ENODEV;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, opt->device) != cudaSuccess || prop.major < 10) return CT2G_ENODEV;
  ct2g_ctx *ctx = new ct2g_ctx();
  ctx->opt = *opt;
  ctx->device = opt->device;
  ctx->num_sms = prop.multiProcessorCount;
  ctx->M = opt->mesh;
  while ((1 << ctx->mbits) < ctx->M) ctx->mbits++;
  ctx->C = (int64_t)ctx->M * ctx->M * ctx->M;
  ctx->ldk = ctx->M / 2 + 2;  // even, so spectrum rows start on 16-byte boundaries
  ctx->CK = (int64_t)ctx->M * ctx->M * ctx->ldk;
  ctx->p = opt->order;
  ctx->nc = ct2g_ncomp(ctx->p);
  ctx->nbox = nbox;
  while ((1 << ctx->boxbits) < nbox) ctx->boxbits++;
  ctx->CB = ctx->C * nbox;
  if (3 * ctx->mbits + ctx->boxbits > 32) {
    delete ctx;
    return CT2G_EINVAL;  // cell keys are 32 bits: box index above the Morton key
  }
  ctx->h_box_off.assign(nbox + 1, 0);
  ctx->h_box_gm.assign(nbox, opt->GM);
  ctx->boxes_set = nbox == 1;
  int rc = CT2G_OK;
  do {
    if (cudaSetDevice(ctx->device) != cudaSuccess) { rc = CT2G_ENODEV; break; }
    // the context stream at the highest priority, the near field's own stream
    // at the lowest: when both have blocks waiting, the mesh solve's go first
    int prio_least = 0, prio_greatest = 0;
    cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    if (cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_greatest) != cudaSuccess) { rc = CT2G_ECUDA; break; }
    if (cudaStreamCreateWithPriority(&ctx->stream2, cudaStreamNonBlocking, prio_least) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_pos, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->ev_vel, cudaEventDisableTiming) != cudaSuccess) {
      rc = CT2G_ECUDA;
      break;
    }
    // ev_vel always holds a record: a step that waits on it without a
    // host-state upload finds it complete
    if (cudaEventRecord(ctx->ev_vel, ctx->copy_stream) != cudaSuccess) { rc = CT2G_ECUDA; break; }
    for (auto &e : ctx->ev)
      if (cudaEventCreate(&e) != cudaSuccess) { rc = CT2G_ECUDA; break; }
    if (rc) break;
    if (cudaMallocHost(&ctx->h_pinned, 64) != cudaSuccess) { rc = CT2G_ECUDA; break; }
    if (cudaMalloc(&ctx->d_maxrung, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&ctx->d_inter, sizeof(unsigned long long)) != cudaSuccess) { rc = CT2G_ENOMEM; break; }
    if ((rc = ct2g_alloc_mesh(ctx)) != CT2G_OK) break;
    if ((rc = ct2g_fft_init(ctx)) != CT2G_OK) break;
    // near-field stencil: integer offsets |o|^2 <= bwidth^2 (the fixed form
    // of particle_cell_neighbors, src/particle.cpp:302-318)
    std::vector<int> st;
    const int B = (int)std::floor(opt->bwidth);
    const double bw2 = (double)opt->bwidth * (double)opt->bwidth;
    for (int i = -B; i <= B; i++)
      for (int j = -B; j <= B; j++)
        for (int k = -B; k <= B; k++)
          if ((double)(i * i + j * j + k * k) <= bw2) {
            st.push_back(i);
            st.push_back(j);
            st.push_back(k);
            st.push_back(0);
          }
    ctx->nstencil = (int)(st.size() / 4);
    if ((rc = ct2g_upload_stencil(ctx, st)) != CT2G_OK) break;
    // stencil bits per (in-block Morton position p, block offset (dX,dY,dZ)):
    // cells b of the neighbouring 4x4x4 block with |4 d + pos(b) - pos(p)|^2 <= bwidth^2
    {
      std::vector<unsigned long long> m(64 * 27, 0ull);
      auto pos = [](int b, int &x, int &y, int &z) {
        x = ((b >> 2) & 1) | ((b >> 4) & 2);
        y = ((b >> 1) & 1) | ((b >> 3) & 2);
        z = (b & 1) | ((b >> 2) & 2);
      };
      for (int p = 0; p < 64; p++) {
        int px, py, pz;
        pos(p, px, py, pz);
        for (int o = 0; o < 27; o++) {
          const int dX = o / 9 - 1, dY = (o / 3) % 3 - 1, dZ = o % 3 - 1;
          for (int b = 0; b < 64; b++) {
            int bx, by, bz;
            pos(b, bx, by, bz);
            const int ox = 4 * dX + bx - px, oy = 4 * dY + by - py, oz = 4 * dZ + bz - pz;
            if ((double)(ox * ox + oy * oy + oz * oz) <= bw2) m[p * 27 + o] |= 1ull << b;
          }
        }
      }
      if (cudaMemcpy(ctx->stmask, m.data(), sizeof(unsigned long long) * m.size(),
                     cudaMemcpyHostToDevice) != cudaSuccess) { rc = CT2G_ECUDA; break; }
    }
    if (opt->max_particles && (rc = ct2g_alloc_particles(ctx, opt->max_particles)) != CT2G_OK) break;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { rc = CT2G_ECUDA; break; }
  } while (0);
  if (rc != CT2G_OK) {
    cudaGetLastError();
    ct2g_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return CT2G_OK;
}

int ct2g_destroy(ct2g_ctx *ctx) {
  if (!ctx) return CT2G_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_particles(ctx);
  if (ctx->self_batch) ct2g_batch_destroy(ctx->self_batch);
  ct2g_learned_free(ctx);
  void *ptrs[] = {ctx->cell_start, ctx->occ, ctx->stmask, ctx->grid, ctx->spec, ctx->greens,
                  ctx->greens_x,                  ctx->tw32, ctx->tw64, ctx->d_counts, ctx->box_off, ctx->box_gm, ctx->tc_tables,
                  ctx->d_maxrung, ctx->d_inter, ctx->scan_tmp, ctx->pipe_sync, ctx->blk_rank};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
  for (auto &e : ctx->ev)
    if (e) cudaEventDestroy(e);
  if (ctx->stream2) cudaStreamSynchronize(ctx->stream2);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  if (ctx->ev_pos) cudaEventDestroy(ctx->ev_pos);
  if (ctx->ev_vel) cudaEventDestroy(ctx->ev_vel);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  if (ctx->stream2) cudaStreamDestroy(ctx->stream2);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return CT2G_OK;
}

int ct2g_get_options(const ct2g_ctx *ctx, ct2g_options *out) {
  if (!ctx || !out) return CT2G_EINVAL;
  *out = ctx->opt;
  return CT2G_OK;
}

int ct2g_set_boxes(ct2g_ctx *ctx, const uint64_t *counts, const float *GM) {
  CT2G_TRY(check(ctx));
  if (!counts || !GM) return ct2g_fail(ctx, CT2G_EINVAL, "null box table");
  if (!ctx->has_particles) return ct2g_fail(ctx, CT2G_ESTATE, "upload the particles first");
  uint64_t sum = 0;
  for (int b = 0; b < ctx->nbox; b++) {
    if (!(GM[b] > 0.f)) return ct2g_fail(ctx, CT2G_EINVAL, "box GM must be > 0");
    ctx->h_box_off[b] = sum;
    sum += counts[b];
  }
  if (sum != ctx->n) return ct2g_fail(ctx, CT2G_EINVAL, "box counts do not add up to the upload");
  ctx->h_box_off[ctx->nbox] = sum;
  ctx->h_box_gm.assign(GM, GM + ctx->nbox);
  CT2G_TRY(upload_boxes(ctx));
  ctx->boxes_set = true;
  ctx->grid_valid = ctx->moments_valid = ctx->expansions_valid = ctx->forces_valid = false;
  return CT2G_OK;
}

int ct2g_box_count(const ct2g_ctx *ctx) { return ctx ? ctx->nbox : 0; }

int ct2g_set_params(ct2g_ctx *ctx, float hsoft, float eta, float GM) {
  if (!ctx) return CT2G_EINVAL;
  if (!(hsoft > 0.f) || !(eta > 0.f)) return ct2g_fail(ctx, CT2G_EINVAL, "hsoft and eta must be > 0");
  if (hsoft != ctx->opt.hsoft) {
    ctx->greens_valid = false;  // the far-field kernel depends on the softening
    ctx->expansions_valid = false;
  }
  ctx->opt.hsoft = hsoft;
  ctx->opt.eta = eta;
  ctx->forces_valid = false;
  ctx->epoch++;
  if (GM > 0.f) {
    ctx->opt.GM = GM;
    if (ctx->nbox == 1) {
      ctx->h_box_gm[0] = GM;
      CT2G_TRY(check(ctx));
      CT2G_TRY(upload_boxes(ctx));
    }
  }
  return CT2G_OK;
}

int ct2g_upload_particles(ct2g_ctx *ctx, const uint32_t *x, const uint32_t *y, const uint32_t *z,
                          const float *vx, const float *vy, const float *vz, const int8_t *rung,
                          size_t n) {
  CT2G_TRY(check(ctx));
  if (!x || !y || !z || !vx || !vy || !vz) return ct2g_fail(ctx, CT2G_EINVAL, "null particle array");
  if (n >= 0x7fffffffu) return ct2g_fail(ctx, CT2G_EINVAL, "too many particles");
  CT2G_TRY(ct2g_alloc_particles(ctx, std::max<size_t>(n, 1)));
  cudaStream_t st = ctx->stream;
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->x, x, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->y, y, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->z, z, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vx, vx, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vy, vy, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vz, vz, n * 4, cudaMemcpyHostToDevice, st));
  if (rung)
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->rung, rung, n, cudaMemcpyHostToDevice, st));
  else
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->rung, 0, n, st));
  if (n) {
    iota_kernel<<<ct2g_div_up(n, 256), 256, 0, st>>>(ctx->id, n);
    CT2G_LAUNCHED(ctx);
  }
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  ctx->n = n;
  if (!(ctx->opt.GM > 0.f)) ctx->opt.GM = n ? 1.0f / (float)n : 0.f;
  if (ctx->nbox == 1) {
    ctx->h_box_off[0] = 0;
    ctx->h_box_off[1] = n;
    ctx->h_box_gm[0] = ctx->opt.GM;
    CT2G_TRY(upload_boxes(ctx));
  } else {
    ctx->boxes_set = false;  // ct2g_set_boxes must describe this upload
  }
  ctx->rung_begin = 0;
  ctx->rung_stack.clear();
  ctx->has_particles = true;
  ctx->grid_valid = ctx->moments_valid = ctx->expansions_valid = ctx->forces_valid = false;
  return CT2G_OK;
}

int ct2g_download_particles(ct2g_ctx *ctx, uint32_t *x, uint32_t *y, uint32_t *z, float *vx,
                            float *vy, float *vz, int8_t *rung, uint32_t *ids) {
  CT2G_TRY(check(ctx));
  const size_t n = ctx->n;
  cudaStream_t st = ctx->stream;
  if (x) CT2G_CUDA(ctx, cudaMemcpyAsync(x, ctx->x, n * 4, cudaMemcpyDeviceToHost, st));
  if (y) CT2G_CUDA(ctx, cudaMemcpyAsync(y, ctx->y, n * 4, cudaMemcpyDeviceToHost, st));
  if (z) CT2G_CUDA(ctx, cudaMemcpyAsync(z, ctx->z, n * 4, cudaMemcpyDeviceToHost, st));
  if (vx) CT2G_CUDA(ctx, cudaMemcpyAsync(vx, ctx->vx, n * 4, cudaMemcpyDeviceToHost, st));
  if (vy) CT2G_CUDA(ctx, cudaMemcpyAsync(vy, ctx->vy, n * 4, cudaMemcpyDeviceToHost, st));
  if (vz) CT2G_CUDA(ctx, cudaMemcpyAsync(vz, ctx->vz, n * 4, cudaMemcpyDeviceToHost, st));
  if (rung) CT2G_CUDA(ctx, cudaMemcpyAsync(rung, ctx->rung, n, cudaMemcpyDeviceToHost, st));
  if (ids) CT2G_CUDA(ctx, cudaMemcpyAsync(ids, ctx->id, n * 4, cudaMemcpyDeviceToHost, st));
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  return CT2G_OK;
}

// One kick + drift from host state to host state.  Positions and ids go
// first on the context stream (binning needs them at once); the velocities
// and rungs follow on copy_stream while binning and the force solve run,
// and the step waits for them (ev_vel) only where it gathers them into cell
// order, just before the update.  Then the state comes back.
int ct2g_kick_drift_host(ct2g_ctx *ctx, const ct2g_kick_params *p, float dt, float scale,
                         int flags, const uint32_t *x, const uint32_t *y, const uint32_t *z,
                         const float *vx, const float *vy, const float *vz, const int8_t *rung,
                         size_t n, uint32_t *xo, uint32_t *yo, uint32_t *zo, float *vxo,
                         float *vyo, float *vzo, int8_t *rungo, uint32_t *ido, int *max_rung) {
  CT2G_TRY(check(ctx));
  if (!p) return ct2g_fail(ctx, CT2G_EINVAL, "null kick params");
  if (!x || !y || !z || !vx || !vy || !vz) return ct2g_fail(ctx, CT2G_EINVAL, "null particle array");
  if (!ctx->has_particles || n != ctx->n)
    return ct2g_fail(ctx, CT2G_ESTATE, "host-state step: n must equal the uploaded particle count");
  cudaStream_t st = ctx->stream, cs = ctx->copy_stream;
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->x, x, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->y, y, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->z, z, n * 4, cudaMemcpyHostToDevice, st));
  if (n) {
    iota_kernel<<<ct2g_div_up(n, 256), 256, 0, st>>>(ctx->id, n);
    CT2G_LAUNCHED(ctx);
  }
  // the velocity upload starts once everything queued before it on the
  // context stream (earlier steps included) and the position upload are done
  CT2G_CUDA(ctx, cudaEventRecord(ctx->ev_pos, st));
  CT2G_CUDA(ctx, cudaStreamWaitEvent(cs, ctx->ev_pos, 0));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vx, vx, n * 4, cudaMemcpyHostToDevice, cs));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vy, vy, n * 4, cudaMemcpyHostToDevice, cs));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vz, vz, n * 4, cudaMemcpyHostToDevice, cs));
  if (rung)
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->rung, rung, n, cudaMemcpyHostToDevice, cs));
  else
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->rung, 0, n, cs));
  CT2G_CUDA(ctx, cudaEventRecord(ctx->ev_vel, cs));
  // what an upload resets
  ctx->rung_begin = 0;
  ctx->rung_stack.clear();
  ctx->grid_valid = ctx->moments_valid = ctx->expansions_valid = ctx->forces_valid = false;
  const int rc = ct2g_kick_drift(ctx, p, dt, scale, flags, nullptr);
  if (rc != CT2G_OK) {
    cudaStreamSynchronize(cs);  // the host arrays stay in use until the copies end
    return rc;
  }
  if (xo) CT2G_CUDA(ctx, cudaMemcpyAsync(xo, ctx->x, n * 4, cudaMemcpyDeviceToHost, st));
  if (yo) CT2G_CUDA(ctx, cudaMemcpyAsync(yo, ctx->y, n * 4, cudaMemcpyDeviceToHost, st));
  if (zo) CT2G_CUDA(ctx, cudaMemcpyAsync(zo, ctx->z, n * 4, cudaMemcpyDeviceToHost, st));
  if (vxo) CT2G_CUDA(ctx, cudaMemcpyAsync(vxo, ctx->vx, n * 4, cudaMemcpyDeviceToHost, st));
  if (vyo) CT2G_CUDA(ctx, cudaMemcpyAsync(vyo, ctx->vy, n * 4, cudaMemcpyDeviceToHost, st));
  if (vzo) CT2G_CUDA(ctx, cudaMemcpyAsync(vzo, ctx->vz, n * 4, cudaMemcpyDeviceToHost, st));
  if (rungo) CT2G_CUDA(ctx, cudaMemcpyAsync(rungo, ctx->rung, n, cudaMemcpyDeviceToHost, st));
  if (ido) CT2G_CUDA(ctx, cudaMemcpyAsync(ido, ctx->id, n * 4, cudaMemcpyDeviceToHost, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, ctx->d_maxrung, sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  if (max_rung) *max_rung = (int)ctx->h_pinned[0];
  return CT2G_OK;
}

size_t ct2g_particle_count(const ct2g_ctx *ctx) { return ctx ? ctx->n : 0; }

int ct2g_particle_to_grid(ct2g_ctx *ctx) {
  CT2G_TRY(check(ctx));
  if (!ctx->has_particles) return ct2g_fail(ctx, CT2G_ESTATE, "no particles uploaded");
  ct2g_mark(ctx, 0);
  return ct2g_bin_range(ctx);
}

int ct2g_download_cells(ct2g_ctx *ctx, int64_t *cell_begin, int64_t *cell_end) {
  CT2G_TRY(check(ctx));
  if (!cell_begin || !cell_end) return ct2g_fail(ctx, CT2G_EINVAL, "null output");
  CT2G_TRY(ensure_grid(ctx));
  std::vector<uint32_t> h(ctx->CB + 1);
  CT2G_CUDA(ctx, cudaMemcpyAsync(h.data(), ctx->cell_start, sizeof(uint32_t) * h.size(),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const uint32_t M = (uint32_t)ctx->M;
  for (int b = 0; b < ctx->nbox; b++)
    for (uint32_t i = 0; i < M; i++)
      for (uint32_t j = 0; j < M; j++)
        for (uint32_t k = 0; k < M; k++) {
          const uint32_t key = ((uint32_t)b << (3 * ctx->mbits)) | ct2g_morton(i, j, k);
          const size_t c = (size_t)b * ctx->C + ((size_t)i * M + j) * M + k;
          cell_begin[c] = h[key];
          cell_end[c] = h[key + 1];
        }
  return CT2G_OK;
}

int ct2g_compute_multipoles(ct2g_ctx *ctx) {
  CT2G_TRY(check(ctx));
  CT2G_TRY(ensure_grid(ctx));
  CT2G_TRY(ct2g_p2m(ctx));
  ctx->moments_valid = true;
  ctx->expansions_valid = false;
  return CT2G_OK;
}

int ct2g_download_multipoles(ct2g_ctx *ctx, float *out) {
  CT2G_TRY(check(ctx));
  if (!out) return ct2g_fail(ctx, CT2G_EINVAL, "null output");
  if (!ctx->moments_valid) return ct2g_fail(ctx, CT2G_ESTATE, "moments not computed (or already transformed)");
  CT2G_CUDA(ctx, cudaMemcpyAsync(out, ctx->grid, sizeof(float) * ctx->nc * ctx->CB,
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CT2G_OK;
}

int ct2g_compute_expansions(ct2g_ctx *ctx) {
  CT2G_TRY(check(ctx));
  CT2G_TRY(ensure_grid(ctx));
  if (!ctx->moments_valid) CT2G_TRY(ct2g_compute_multipoles(ctx));
  CT2G_TRY(ct2g_mesh_solve(ctx, false, false));
  ctx->moments_valid = false;  // the grid now holds the expansions
  ctx->expansions_valid = true;
  return CT2G_OK;
}

int ct2g_download_expansions(ct2g_ctx *ctx, float *out) {
  CT2G_TRY(check(ctx));
  if (!out) return ct2g_fail(ctx, CT2G_EINVAL, "null output");
  if (!ctx->expansions_valid) return ct2g_fail(ctx, CT2G_ESTATE, "expansions not computed");
  CT2G_CUDA(ctx, cudaMemcpyAsync(out, ctx->grid, sizeof(float) * ctx->nc * ctx->CB,
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CT2G_OK;
}

int ct2g_download_greens(ct2g_ctx *ctx, float *out) {
  CT2G_TRY(check(ctx));
  if (!out) return ct2g_fail(ctx, CT2G_EINVAL, "null output");
  CT2G_TRY(ct2g_build_greens(ctx));
  std::vector<float> h((size_t)ctx->nc * ctx->CK);
  CT2G_CUDA(ctx, cudaMemcpyAsync(h.data(), ctx->greens, sizeof(float) * h.size(),
                                 cudaMemcpyDeviceToHost, ctx->stream));
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const size_t NH = ctx->M / 2 + 1, rows = (size_t)ctx->nc * ctx->M * ctx->M;
  for (size_t r = 0; r < rows; r++)
    std::memcpy(out + r * NH, h.data() + r * ctx->ldk, sizeof(float) * NH);
  return CT2G_OK;
}

int ct2g_compute_forces(ct2g_ctx *ctx) {
  CT2G_TRY(check(ctx));
  CT2G_TRY(ct2g_all_forces(ctx, true));
  ctx->forces_valid = true;
  ctx->pot_valid = true;
  return CT2G_OK;
}

int ct2g_download_forces(ct2g_ctx *ctx, float *fx, float *fy, float *fz, float *pot) {
  CT2G_TRY(check(ctx));
  const size_t n = ctx->n;
  cudaStream_t st = ctx->stream;
  if (fx) CT2G_CUDA(ctx, cudaMemcpyAsync(fx, ctx->fx, n * 4, cudaMemcpyDeviceToHost, st));
  if (fy) CT2G_CUDA(ctx, cudaMemcpyAsync(fy, ctx->fy, n * 4, cudaMemcpyDeviceToHost, st));
  if (fz) CT2G_CUDA(ctx, cudaMemcpyAsync(fz, ctx->fz, n * 4, cudaMemcpyDeviceToHost, st));
  if (pot) CT2G_CUDA(ctx, cudaMemcpyAsync(pot, ctx->pot, n * 4, cudaMemcpyDeviceToHost, st));
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  return CT2G_OK;
}

int ct2g_upload_forces(ct2g_ctx *ctx, const float *fx, const float *fy, const float *fz) {
  CT2G_TRY(check(ctx));
  if (!fx || !fy || !fz) return ct2g_fail(ctx, CT2G_EINVAL, "null force array");
  const size_t n = ctx->n;
  cudaStream_t st = ctx->stream;
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->fx, fx, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->fy, fy, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->fz, fz, n * 4, cudaMemcpyHostToDevice, st));
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  ctx->forces_valid = true;
  return CT2G_OK;
}

int ct2g_kick_update(ct2g_ctx *ctx, const ct2g_kick_params *p, int *max_rung) {
  CT2G_TRY(check(ctx));
  if (!p) return ct2g_fail(ctx, CT2G_EINVAL, "null kick params");
  if (p->rung < 0 || p->rung > 30) return ct2g_fail(ctx, CT2G_EINVAL, "rung out of range");
  if (!ctx->forces_valid) return ct2g_fail(ctx, CT2G_ESTATE, "no forces to apply");
  return ct2g_update(ctx, p, max_rung, false, 0.f, 1.f);
}

int ct2g_kick(ct2g_ctx *ctx, const ct2g_kick_params *p, int *max_rung) {
  CT2G_TRY(check(ctx));
  if (!p) return ct2g_fail(ctx, CT2G_EINVAL, "null kick params");
  if (p->rung < 0 || p->rung > 30) return ct2g_fail(ctx, CT2G_EINVAL, "rung out of range");
  CT2G_TRY(ct2g_all_forces(ctx, false));
  ctx->pot_valid = false;
  ct2g_mark(ctx, 6);
  ctx->forces_valid = true;
  CT2G_TRY(ct2g_update(ctx, p, max_rung, false, 0.f, 1.f));
  ct2g_mark(ctx, 7);
  return CT2G_OK;
}

int ct2g_drift(ct2g_ctx *ctx, float dt, float scale) {
  CT2G_TRY(check(ctx));
  if (!(scale != 0.f)) return ct2g_fail(ctx, CT2G_EINVAL, "scale must be nonzero");
  return ct2g_drift_all(ctx, dt, scale);
}

int ct2g_sort_by_rung(ct2g_ctx *ctx, int minrung) {
  CT2G_TRY(check(ctx));
  if (ctx->nbox > 1) return ct2g_fail(ctx, CT2G_EINVAL, "rung levels need a single-box context");
  if (minrung == 0) {
    ctx->rung_begin = 0;
    return CT2G_OK;
  }
  const size_t b = ctx->rung_begin, nr = ctx->n - b;
  if (nr == 0) return CT2G_OK;
  CT2G_TRY(ct2g_alloc_particles(ctx, ctx->n));
  cudaStream_t st = ctx->stream;
  const unsigned T = 256, G = ct2g_div_up(nr, T);
  rung_flag_kernel<<<G, T, 0, st>>>(ctx->rung, b, nr, minrung, ctx->flags);
  CT2G_LAUNCHED(ctx);
  CT2G_TRY(ct2g_scan_exclusive(ctx, ctx->flags, ctx->vals2, nr, ctx->d_counts + 5, 0));
  CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, ctx->d_counts + 5, sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, st));
  CT2G_CUDA(ctx, cudaStreamSynchronize(st));
  const uint32_t nlow = ctx->h_pinned[0];
  rung_scatter_kernel<<<G, T, 0, st>>>(ctx->flags, ctx->vals2, b, nr, nlow, ctx->vals);
  CT2G_LAUNCHED(ctx);
  permute_kernel<uint32_t><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->x, ctx->x2);
  permute_kernel<uint32_t><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->y, ctx->y2);
  permute_kernel<uint32_t><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->z, ctx->z2);
  permute_kernel<uint32_t><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->id, ctx->id2);
  permute_kernel<float><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->vx, ctx->vx2);
  permute_kernel<float><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->vy, ctx->vy2);
  permute_kernel<float><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->vz, ctx->vz2);
  permute_kernel<int8_t><<<G, T, 0, st>>>(ctx->vals, b, nr, ctx->rung, ctx->rung2);
  ctx->launches += 7;
  CT2G_LAUNCHED(ctx);
  if (b > 0) {
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->x2, ctx->x, b * 4, cudaMemcpyDeviceToDevice, st));
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->y2, ctx->y, b * 4, cudaMemcpyDeviceToDevice, st));
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->z2, ctx->z, b * 4, cudaMemcpyDeviceToDevice, st));
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->id2, ctx->id, b * 4, cudaMemcpyDeviceToDevice, st));
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vx2, ctx->vx, b * 4, cudaMemcpyDeviceToDevice, st));
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vy2, ctx->vy, b * 4, cudaMemcpyDeviceToDevice, st));
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->vz2, ctx->vz, b * 4, cudaMemcpyDeviceToDevice, st));
    CT2G_CUDA(ctx, cudaMemcpyAsync(ctx->rung2, ctx->rung, b, cudaMemcpyDeviceToDevice, st));
  }
  std::swap(ctx->x, ctx->x2);
  std::swap(ctx->y, ctx->y2);
  std::swap(ctx->z, ctx->z2);
  std::swap(ctx->id, ctx->id2);
  std::swap(ctx->vx, ctx->vx2);
  std::swap(ctx->vy, ctx->vy2);
  std::swap(ctx->vz, ctx->vz2);
  std::swap(ctx->rung, ctx->rung2);
  ctx->epoch++;  // the store moved to the other buffers
  ctx->rung_begin = b + nlow;
  ctx->grid_valid = ctx->moments_valid = ctx->expansions_valid = ctx->forces_valid = false;
  return CT2G_OK;
}

int ct2g_push_rungs(ct2g_ctx *ctx) {
  if (!ctx) return CT2G_EINVAL;
  ctx->rung_stack.push_back(ctx->rung_begin);
  return CT2G_OK;
}

int ct2g_pop_rungs(ct2g_ctx *ctx) {
  if (!ctx) return CT2G_EINVAL;
  if (ctx->rung_stack.empty()) return ct2g_fail(ctx, CT2G_ESTATE, "rung stack empty");
  ctx->rung_begin = ctx->rung_stack.back();
  ctx->rung_stack.pop_back();
  ctx->grid_valid = ctx->moments_valid = ctx->expansions_valid = ctx->forces_valid = false;
  return CT2G_OK;
}

int ct2g_set_minrung(ct2g_ctx *ctx, int minrung) {
  CT2G_TRY(check(ctx));
  if (ctx->n == 0) return CT2G_OK;
  set_minrung_kernel<<<ct2g_div_up(ctx->n, 256), 256, 0, ctx->stream>>>(ctx->rung, ctx->n, minrung);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

int ct2g_current_range(ct2g_ctx *ctx, size_t *begin, size_t *end) {
  if (!ctx) return CT2G_EINVAL;
  if (begin) *begin = ctx->rung_begin;
  if (end) *end = ctx->n;
  return CT2G_OK;
}

int ct2g_rung_counts(ct2g_ctx *ctx, size_t *counts, int nmax, int *nrungs) {
  CT2G_TRY(check(ctx));
  unsigned long long *d = nullptr;
  CT2G_CUDA(ctx, cudaMalloc(&d, sizeof(unsigned long long) * 128));
  cudaMemsetAsync(d, 0, sizeof(unsigned long long) * 128, ctx->stream);
  if (ctx->n) {
    rung_count_kernel<<<std::min<unsigned>(ct2g_div_up(ctx->n, 256), 1024), 256, 0, ctx->stream>>>(ctx->rung, ctx->n, d);
    ctx->launches++;
  }
  unsigned long long h[128];
  cudaError_t e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess) return ct2g_cuda_fail(ctx, e, "rung counts");
  int top = 0;
  for (int r = 0; r < 128; r++)
    if (h[r]) top = r + 1;
  if (nrungs) *nrungs = top;
  for (int r = 0; r < nmax && counts; r++) counts[r] = r < 128 ? (size_t)h[r] : 0;
  return CT2G_OK;
}

// kick_step, src/main.cpp:8-92, with the GPU stages; the level bookkeeping,
// clip_top rule and push/pop order are the reference's.
int ct2g_kick_step(ct2g_ctx *ctx, int *minrung_io, int max_rung, double scale, double adot,
                   double tau, double t0, int minrung0, int nocrop, int *out_max_rung) {
  CT2G_TRY(check(ctx));
  if (!minrung_io) return ct2g_fail(ctx, CT2G_EINVAL, "null minrung");
  int &minrung = *minrung_io;
  // every level above minrung pops a range pushed by an earlier call's
  // descending levels; refuse before any work if the stack is short (the
  // reference would read an empty std::stack, particle.cpp:31-34)
  if (max_rung > minrung && ctx->rung_stack.size() < (size_t)(max_rung - minrung))
    return ct2g_fail(ctx, CT2G_ESTATE,
                     "kick_step: the rung stack holds fewer levels than max_rung - minrung");
  std::vector<int> levels(std::max(max_rung - minrung, 0) + 1);
  int k = 0;
  for (int i = max_rung; i > minrung; i--) levels[k++] = i;
  levels[k++] = minrung;
  bool ascending = true, clip_top = false, top = false;
  int mr = 0;
  for (size_t li = 0; li < levels.size(); li++) {
    if (levels[li] == minrung) {
      ascending = false;
      top = true;
    } else {
      top = false;
    }
    if (!ascending && !top) CT2G_TRY(ct2g_push_rungs(ctx));
    if (!ascending) CT2G_TRY(ct2g_sort_by_rung(ctx, levels[li]));
    if (top && minrung == minrung0) {
      size_t counts[128];
      int nr = 0;
      CT2G_TRY(ct2g_rung_counts(ctx, counts, 128, &nr));
      if (nr > minrung0 + 1) {
        size_t fast = 0, slow = counts[minrung0];
        for (int i = minrung0 + 1; i < nr; i++) fast += counts[i];
        if (3 * fast > slow) clip_top = !nocrop;
      }
    }
    CT2G_TRY(ct2g_particle_to_grid(ctx));
    ct2g_kick_params kp;
    kp.top = (clip_top && levels[li] == minrung0 + 1) ? 1 : (top ? 1 : 0);
    kp.ascending = (ascending || top) ? 1 : 0;
    kp.descending = (clip_top && top) ? 0 : ((!ascending || top) ? 1 : 0);
    kp.eta = ctx->opt.eta;
    kp.scale = (float)scale;
    kp.first = tau == 0.0 ? 1 : 0;
    kp.rung = levels[li];
    kp.t0 = (float)t0;
    kp.max_dt = (float)(0.01f / adot);
    CT2G_TRY(ct2g_kick(ctx, &kp, &mr));
    if (clip_top && top) CT2G_TRY(ct2g_set_minrung(ctx, minrung0 + 1));
    if (clip_top && top) {
      levels.push_back(minrung0 + 1);
    } else if (!ascending || top) {
      if (mr > levels[li]) levels.push_back(levels[li] + 1);
    }
    if ((!ascending || top) && !(clip_top && top)) {
      const double dt = t0 / (double)(1 << levels[li]);
      CT2G_TRY(ct2g_drift(ctx, (float)dt, (float)scale));
    }
    if (ascending && !top) CT2G_TRY(ct2g_pop_rungs(ctx));
  }
  if (clip_top) minrung++;
  // the reference returns its max_rung argument: the max_rung declared in
  // its loop body (main.cpp:68) shadows the parameter and is out of scope at
  // the return (main.cpp:90)
  if (out_max_rung) *out_max_rung = max_rung;
  return CT2G_OK;
}

int ct2g_fft_r2c_3d(ct2g_ctx *ctx, const double *xin, double *xout, int N, int batch) {
  CT2G_TRY(check(ctx));
  if (!xin || !xout || batch < 1 || !is_pow2(N) || N < 4 || N > 512)
    return ct2g_fail(ctx, CT2G_EINVAL, "fft_r2c_3d: bad arguments");
  const size_t n3 = (size_t)N * N * N, nk = (size_t)N * N * (N / 2 + 1);
  double *din = nullptr;
  double2 *dout = nullptr;
  CT2G_CUDA(ctx, cudaMalloc(&din, sizeof(double) * n3 * batch));
  cudaError_t e = cudaMalloc(&dout, sizeof(double2) * nk * batch);
  if (e != cudaSuccess) {
    cudaFree(din);
    return ct2g_cuda_fail(ctx, e, "fft_r2c_3d alloc");
  }
  int rc = CT2G_OK;
  std::vector<double2> h(nk * batch);
  e = cudaMemcpyAsync(din, xin, sizeof(double) * n3 * batch, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    rc = ct2g_fft_r2c_f64(ctx, din, dout, N, batch, N / 2 + 1);
    if (rc == CT2G_OK) {
      e = cudaMemcpyAsync(h.data(), dout, sizeof(double2) * nk * batch, cudaMemcpyDeviceToHost, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
  }
  cudaFree(din);
  cudaFree(dout);
  if (rc != CT2G_OK) return rc;
  if (e != cudaSuccess) return ct2g_cuda_fail(ctx, e, "fft_r2c_3d");
  // split planes: re at [0,dimag), im at [dimag, 2 dimag)
  for (int b = 0; b < batch; b++) {
    double *o = xout + (size_t)b * 2 * nk;
    for (size_t q = 0; q < nk; q++) {
      o[q] = h[b * nk + q].x;
      o[nk + q] = h[b * nk + q].y;
    }
  }
  return CT2G_OK;
}

int ct2g_fft_c2r_3d(ct2g_ctx *ctx, const double *xin, double *xout, int N, int batch) {
  CT2G_TRY(check(ctx));
  if (!xin || !xout || batch < 1 || !is_pow2(N) || N < 4 || N > 512)
    return ct2g_fail(ctx, CT2G_EINVAL, "fft_c2r_3d: bad arguments");
  const size_t n3 = (size_t)N * N * N, nk = (size_t)N * N * (N / 2 + 1);
  std::vector<double2> h(nk * batch);
  for (int b = 0; b < batch; b++) {
    const double *i = xin + (size_t)b * 2 * nk;
    for (size_t q = 0; q < nk; q++) h[b * nk + q] = make_double2(i[q], i[nk + q]);
  }
  double *dout = nullptr;
  double2 *din = nullptr;
  CT2G_CUDA(ctx, cudaMalloc(&din, sizeof(double2) * nk * batch));
  cudaError_t e = cudaMalloc(&dout, sizeof(double) * n3 * batch);
  if (e != cudaSuccess) {
    cudaFree(din);
    return ct2g_cuda_fail(ctx, e, "fft_c2r_3d alloc");
  }
  int rc = CT2G_OK;
  e = cudaMemcpyAsync(din, h.data(), sizeof(double2) * nk * batch, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    rc = ct2g_fft_c2r_f64(ctx, din, dout, N, batch, N / 2 + 1);
    if (rc == CT2G_OK) {
      e = cudaMemcpyAsync(xout, dout, sizeof(double) * n3 * batch, cudaMemcpyDeviceToHost, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    }
  }
  cudaFree(din);
  cudaFree(dout);
  if (rc != CT2G_OK) return rc;
  if (e != cudaSuccess) return ct2g_cuda_fail(ctx, e, "fft_c2r_3d");
  return CT2G_OK;
}

int ct2g_fft3d_f32_dev(ct2g_ctx *ctx, int dir, void *d_real, void *d_complex, int N, int batch) {
  CT2G_TRY(check(ctx));
  if (!d_real || !d_complex || batch < 1 || !is_pow2(N) || N < 4 || N > 512)
    return ct2g_fail(ctx, CT2G_EINVAL, "fft3d_f32_dev: bad arguments");
  if (dir > 0)
    return ct2g_fft_r2c_f32(ctx, (const float *)d_real, (float2 *)d_complex, N, batch, N / 2 + 1);
  return ct2g_fft_c2r_f32(ctx, (float2 *)d_complex, (float *)d_real, N, batch, N / 2 + 1);
}

void *ct2g_stream(ct2g_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int ct2g_synchronize(ct2g_ctx *ctx) {
  CT2G_TRY(check(ctx));
  return ct2g_device_error(ctx);
}

int ct2g_set_fft_mode(ct2g_ctx *ctx, int mode) {
  CT2G_TRY(check(ctx));
  if (mode == CT2G_FFT_FP32) {
    ctx->fft_tc = false;
  } else if (mode == CT2G_FFT_TC_BF16X3) {
    if (!ct2g_fft_tc_supported(ctx->M)) return ct2g_fail(ctx, CT2G_EINVAL, "the tensor-core FFT supports meshes 256 and 512");
    CT2G_TRY(ct2g_fft_tc_prepare(ctx));
    ctx->fft_tc = true;
  } else {
    return ct2g_fail(ctx, CT2G_EINVAL, "unknown FFT mode");
  }
  ctx->epoch++;
  ctx->expansions_valid = ctx->forces_valid = false;
  return CT2G_OK;
}

int ct2g_stage_times(ct2g_ctx *ctx, float *ms, int n) {
  CT2G_TRY(check(ctx));
  if (!ms || n < 7) return ct2g_fail(ctx, CT2G_EINVAL, "need 7 slots");
  CT2G_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < 7; k++) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, ctx->ev[k], ctx->ev[k + 1]) != cudaSuccess) {
      cudaGetLastError();
      t = -1.f;
    }
    ms[k] = t;
  }
  return CT2G_OK;
}

uint64_t ct2g_launch_count(const ct2g_ctx *ctx) { return ctx ? ctx->launches : 0; }

uint64_t ct2g_interaction_count(const ct2g_ctx *ctx) {
  if (!ctx || !ctx->d_inter) return 0;
  unsigned long long v = 0;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaMemcpy(&v, ctx->d_inter, sizeof(v), cudaMemcpyDeviceToHost);
  return v;
}

}  // extern "C"
