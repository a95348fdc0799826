// FP64 Ewald direct sum on the GPU: the force truth the method is measured
// against at sizes the CPU cannot reach (every source against a sample of
// sinks).  Same split as the CPU oracle's ct2o_ewald_direct:
//   a_i = GM sum_j [grad kernel(d) - grad(1/r)(d) + grad(erfc(alpha r)/r)(d) [r<rc]]
//       + GM sum_k w(k) (-2 pi k) Im(e^{2 pi i k.x_i} conj S(k)),
// d the minimum-image displacement, w(k) = exp(-pi^2 k^2/alpha^2)/(pi k^2).
#include "ct2g_internal.cuh"

namespace {

constexpr int kSinkThreads = 128;
constexpr int kSrcChunk = 4096;
// source chunks ride on grid.y (at most 65535), which bounds the source count
constexpr size_t kMaxSources = (size_t)65535 * kSrcChunk;

__global__ void ewald_real_kernel(const uint32_t *__restrict__ sx, const uint32_t *__restrict__ sy,
                                  const uint32_t *__restrict__ sz, size_t ns,
                                  const uint32_t *__restrict__ qx, const uint32_t *__restrict__ qy,
                                  const uint32_t *__restrict__ qz, size_t nq, int kernel,
                                  double h, double alpha, double rc2, double *__restrict__ f,
                                  double *__restrict__ pot) {
  __shared__ uint32_t tx[kSrcChunk / 4], ty[kSrcChunk / 4], tz[kSrcChunk / 4];
  const size_t i = (size_t)blockIdx.x * kSinkThreads + threadIdx.x;
  const size_t j0 = (size_t)blockIdx.y * kSrcChunk;
  const size_t j1 = min(nq, j0 + kSrcChunk);
  const bool act = i < ns;
  const uint32_t xi = act ? sx[i] : 0, yi = act ? sy[i] : 0, zi = act ? sz[i] : 0;
  const double spi = 1.7724538509055160273;
  const double h2 = h * h;
  double fx = 0, fy = 0, fz = 0, ph = 0;
  for (size_t t0 = j0; t0 < j1; t0 += kSrcChunk / 4) {
    const int nt = (int)min((size_t)(kSrcChunk / 4), j1 - t0);
    __syncthreads();
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
      tx[t] = qx[t0 + t];
      ty[t] = qy[t0 + t];
      tz[t] = qz[t0 + t];
    }
    __syncthreads();
    if (!act) continue;
    for (int t = 0; t < nt; t++) {
      const double dx = (double)(int32_t)(xi - tx[t]) * CT2G_TWO_M32;
      const double dy = (double)(int32_t)(yi - ty[t]) * CT2G_TWO_M32;
      const double dz = (double)(int32_t)(zi - tz[t]) * CT2G_TWO_M32;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 == 0.0) {
        ph += (kernel == CT2G_SOFT_SPHERE ? 1.5 / h : 1.0 / h) - 2.0 * alpha / spi;
        continue;
      }
      const double r = sqrt(r2), ri = 1.0 / r, ri3 = ri * ri * ri;
      double g, pk;
      if (kernel == CT2G_SOFT_SPHERE) {
        if (r2 < h2) {
          g = 1.0 / (h * h2);
          pk = 1.5 / h - 0.5 * r2 / (h * h2);
        } else {
          g = ri3;
          pk = ri;
        }
      } else {
        const double s = 1.0 / sqrt(r2 + h2);
        g = s * s * s;
        pk = s;
      }
      double gc = g - ri3, pc = pk - ri;
      if (r2 < rc2) {
        const double ec = erfc(alpha * r);
        gc += (ec + 2.0 * alpha * r / spi * exp(-alpha * alpha * r2)) * ri3;
        pc += ec * ri;
      }
      fx -= dx * gc;
      fy -= dy * gc;
      fz -= dz * gc;
      ph += pc;
    }
  }
  if (act) {
    atomicAdd(f + 3 * i + 0, fx);
    atomicAdd(f + 3 * i + 1, fy);
    atomicAdd(f + 3 * i + 2, fz);
    atomicAdd(pot + i, ph);
  }
}

// S(k) = sum_j exp(2 pi i k.x_j): one thread per k, a chunk of sources each
__global__ void ewald_sk_kernel(const int *__restrict__ kv, int nk, const uint32_t *__restrict__ qx,
                                const uint32_t *__restrict__ qy, const uint32_t *__restrict__ qz,
                                size_t nq, double *__restrict__ S) {
  __shared__ double px[1024], py[1024], pz[1024];
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t j0 = (size_t)blockIdx.y * kSrcChunk;
  const size_t j1 = min(nq, j0 + kSrcChunk);
  const bool act = q < nk;
  const double kx = act ? kv[3 * q] : 0, ky = act ? kv[3 * q + 1] : 0, kz = act ? kv[3 * q + 2] : 0;
  double sr = 0, si = 0;
  for (size_t t0 = j0; t0 < j1; t0 += 1024) {
    const int nt = (int)min((size_t)1024, j1 - t0);
    __syncthreads();
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
      px[t] = qx[t0 + t] * CT2G_TWO_M32;
      py[t] = qy[t0 + t] * CT2G_TWO_M32;
      pz[t] = qz[t0 + t] * CT2G_TWO_M32;
    }
    __syncthreads();
    if (!act) continue;
    for (int t = 0; t < nt; t++) {
      double s, c;
      sincospi(2.0 * (kx * px[t] + ky * py[t] + kz * pz[t]), &s, &c);
      sr += c;
      si += s;
    }
  }
  if (act) {
    atomicAdd(S + 2 * q, sr);
    atomicAdd(S + 2 * q + 1, si);
  }
}

__global__ void ewald_kspace_kernel(const uint32_t *__restrict__ sx, const uint32_t *__restrict__ sy,
                                    const uint32_t *__restrict__ sz, size_t ns,
                                    const int *__restrict__ kv, int nk, const double *__restrict__ S,
                                    double alpha, double nq, double *__restrict__ f,
                                    double *__restrict__ pot) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const double x = sx[i] * CT2G_TWO_M32, y = sy[i] * CT2G_TWO_M32, z = sz[i] * CT2G_TWO_M32;
  const double pi = 3.14159265358979323846;
  double fx = 0, fy = 0, fz = 0, ph = 0;
  for (int q = 0; q < nk; q++) {
    const double kx = kv[3 * q], ky = kv[3 * q + 1], kz = kv[3 * q + 2];
    double s, c;
    sincospi(2.0 * (kx * x + ky * y + kz * z), &s, &c);
    const double k2 = kx * kx + ky * ky + kz * kz;
    const double w = exp(-pi * pi * k2 / (alpha * alpha)) / (pi * k2);
    const double re = c * S[2 * q] + s * S[2 * q + 1];
    const double im = s * S[2 * q] - c * S[2 * q + 1];
    const double a = 2.0 * w * (-2.0 * pi) * im;
    fx += a * kx;
    fy += a * ky;
    fz += a * kz;
    ph += 2.0 * w * re;
  }
  f[3 * i + 0] += fx;
  f[3 * i + 1] += fy;
  f[3 * i + 2] += fz;
  // potential: real part accumulated ph_real (sum of kernel-style terms);
  // final pot = -GM (ph_real + ph_k - pi/alpha^2 nq), scaled on the host
  pot[i] += ph - pi / (alpha * alpha) * nq;
}

}  // namespace

extern "C" int ct2g_ewald_direct(ct2g_ctx *ctx, const uint32_t *sx, const uint32_t *sy,
                                 const uint32_t *sz, size_t ns, double alpha, double rcut,
                                 int kmax, double *f, double *pot) {
  if (!ctx) return CT2G_EINVAL;
  CT2G_CUDA(ctx, cudaSetDevice(ctx->device));
  if (!sx || !sy || !sz || !f || ns == 0) return ct2g_fail(ctx, CT2G_EINVAL, "ewald: bad arguments");
  if (!ctx->has_particles) return ct2g_fail(ctx, CT2G_ESTATE, "no particles uploaded");
  if (!(alpha > 0) || !(rcut > 0) || rcut > 0.5 || kmax < 1 || kmax > 64)
    return ct2g_fail(ctx, CT2G_EINVAL, "ewald: bad split parameters");
  if (ctx->n > kMaxSources) return ct2g_fail(ctx, CT2G_EINVAL, "ewald: more than 65535*4096 sources");
  std::vector<int> kv;
  for (int kx = 0; kx <= kmax; kx++)
    for (int ky = -kmax; ky <= kmax; ky++)
      for (int kz = -kmax; kz <= kmax; kz++) {
        if (kx == 0 && (ky < 0 || (ky == 0 && kz <= 0))) continue;
        if (kx * kx + ky * ky + kz * kz > kmax * kmax) continue;
        kv.push_back(kx);
        kv.push_back(ky);
        kv.push_back(kz);
      }
  const int nk = (int)(kv.size() / 3);
  uint32_t *d_s = nullptr;
  double *d_f = nullptr, *d_p = nullptr, *d_S = nullptr;
  int *d_k = nullptr;
  int rc = CT2G_OK;
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  do {
    if ((e = cudaMalloc(&d_s, sizeof(uint32_t) * 3 * ns)) != cudaSuccess ||
        (e = cudaMalloc(&d_f, sizeof(double) * 3 * ns)) != cudaSuccess ||
        (e = cudaMalloc(&d_p, sizeof(double) * ns)) != cudaSuccess ||
        (e = cudaMalloc(&d_S, sizeof(double) * 2 * nk)) != cudaSuccess ||
        (e = cudaMalloc(&d_k, sizeof(int) * 3 * nk)) != cudaSuccess) {
      rc = ct2g_cuda_fail(ctx, e, "ewald alloc");
      break;
    }
    cudaMemcpyAsync(d_s, sx, 4 * ns, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_s + ns, sy, 4 * ns, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_s + 2 * ns, sz, 4 * ns, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_k, kv.data(), sizeof(int) * 3 * nk, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_f, 0, sizeof(double) * 3 * ns, st);
    cudaMemsetAsync(d_p, 0, sizeof(double) * ns, st);
    cudaMemsetAsync(d_S, 0, sizeof(double) * 2 * nk, st);
    const size_t nq = ctx->n;
    dim3 g1(ct2g_div_up(ns, kSinkThreads), ct2g_div_up(nq, kSrcChunk));
    ewald_real_kernel<<<g1, kSinkThreads, 0, st>>>(d_s, d_s + ns, d_s + 2 * ns, ns, ctx->x, ctx->y,
                                                   ctx->z, nq, ctx->opt.kernel, ctx->opt.hsoft,
                                                   alpha, rcut * rcut, d_f, d_p);
    dim3 g2(ct2g_div_up(nk, 128), ct2g_div_up(nq, kSrcChunk));
    ewald_sk_kernel<<<g2, 128, 0, st>>>(d_k, nk, ctx->x, ctx->y, ctx->z, nq, d_S);
    ewald_kspace_kernel<<<ct2g_div_up(ns, 128), 128, 0, st>>>(d_s, d_s + ns, d_s + 2 * ns, ns, d_k,
                                                             nk, d_S, alpha, (double)nq, d_f, d_p);
    ctx->launches += 3;
    if ((e = cudaGetLastError()) != cudaSuccess) {
      rc = ct2g_cuda_fail(ctx, e, "ewald kernels");
      break;
    }
    std::vector<double> hp(ns);
    if ((e = cudaMemcpyAsync(f, d_f, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hp.data(), d_p, sizeof(double) * ns, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
      rc = ct2g_cuda_fail(ctx, e, "ewald readback");
      break;
    }
    const double GM = ctx->opt.GM;
    for (size_t i = 0; i < 3 * ns; i++) f[i] *= GM;
    if (pot)
      for (size_t i = 0; i < ns; i++) pot[i] = -GM * hp[i];
  } while (0);
  cudaStreamSynchronize(st);
  if (d_s) cudaFree(d_s);
  if (d_f) cudaFree(d_f);
  if (d_p) cudaFree(d_p);
  if (d_S) cudaFree(d_S);
  if (d_k) cudaFree(d_k);
  return rc;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the FP64 Ewald direct sum.
//
// For callers that cannot call cudaMalloc -- code that runs inside a
// framework which owns all device memory, or a loop where allocation is not
// allowed -- ct2g_ewald_direct_noalloc takes device pointers for its inputs
// and outputs and keeps its only scratch, the structure factor S(k), in the
// file-scope device array below.  Every GPU that loads the library holds the
// array (kNoallocBox complex doubles, about 0.94 MB) until the process exits.
// In host code g_noalloc_sk is only a host-side stand-in, never a device
// address: the address comes from cudaGetSymbolAddress, taken once per device
// on the first call there (so that first call should come before any stream
// capture).  All calls share the array, and calls that overlap on the GPU
// race on it; each call clears it before use.
// ---------------------------------------------------------------------------
#include <mutex>

#define CT2G_NOALLOC_KMAX 24
namespace {
constexpr int kNoallocSide = 2 * CT2G_NOALLOC_KMAX + 1;
constexpr int kNoallocBox = (CT2G_NOALLOC_KMAX + 1) * kNoallocSide * kNoallocSide;
}  // namespace

static __device__ __align__(256) double2 g_noalloc_sk[kNoallocBox];

namespace {

std::mutex g_noalloc_mu;
double2 *g_noalloc_ptr[128] = {};

// k-vector of box index q for a given kmax: kx in [0,K], ky,kz in [-K,K];
// valid when in the half space (kx>0, or kx==0 && (ky>0 || ky==0 && kz>0))
// and |k| <= K
__device__ __forceinline__ bool noalloc_k(int q, int K, int &kx, int &ky, int &kz) {
  const int side = 2 * K + 1;
  kx = q / (side * side);
  ky = (q / side) % side - K;
  kz = q % side - K;
  if (kx == 0 && (ky < 0 || (ky == 0 && kz <= 0))) return false;
  return kx * kx + ky * ky + kz * kz <= K * K;
}

__global__ void noalloc_sk_kernel(int K, const uint32_t *__restrict__ qx,
                                  const uint32_t *__restrict__ qy, const uint32_t *__restrict__ qz,
                                  size_t nq, double2 *__restrict__ S) {
  __shared__ double px[1024], py[1024], pz[1024];
  const int nbox = (K + 1) * (2 * K + 1) * (2 * K + 1);
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const size_t j0 = (size_t)blockIdx.y * kSrcChunk;
  const size_t j1 = min(nq, j0 + kSrcChunk);
  int kx = 0, ky = 0, kz = 0;
  const bool act = q < nbox && noalloc_k(q, K, kx, ky, kz);
  double sr = 0, si = 0;
  for (size_t t0 = j0; t0 < j1; t0 += 1024) {
    const int nt = (int)min((size_t)1024, j1 - t0);
    __syncthreads();
    for (int t = threadIdx.x; t < nt; t += blockDim.x) {
      px[t] = qx[t0 + t] * CT2G_TWO_M32;
      py[t] = qy[t0 + t] * CT2G_TWO_M32;
      pz[t] = qz[t0 + t] * CT2G_TWO_M32;
    }
    __syncthreads();
    if (!act) continue;
    for (int t = 0; t < nt; t++) {
      double s, c;
      sincospi(2.0 * (kx * px[t] + ky * py[t] + kz * pz[t]), &s, &c);
      sr += c;
      si += s;
    }
  }
  if (act) {
    atomicAdd(&S[q].x, sr);
    atomicAdd(&S[q].y, si);
  }
}

__global__ void noalloc_kspace_kernel(const uint32_t *__restrict__ sx,
                                      const uint32_t *__restrict__ sy,
                                      const uint32_t *__restrict__ sz, size_t ns, int K,
                                      const double2 *__restrict__ S, double alpha, double nq,
                                      double GM, double *__restrict__ f, double *__restrict__ pot) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ns) return;
  const double x = sx[i] * CT2G_TWO_M32, y = sy[i] * CT2G_TWO_M32, z = sz[i] * CT2G_TWO_M32;
  const double pi = 3.14159265358979323846;
  const int nbox = (K + 1) * (2 * K + 1) * (2 * K + 1);
  double fx = 0, fy = 0, fz = 0, ph = 0;
  for (int q = 0; q < nbox; q++) {
    int kx, ky, kz;
    if (!noalloc_k(q, K, kx, ky, kz)) continue;
    double s, c;
    sincospi(2.0 * (kx * x + ky * y + kz * z), &s, &c);
    const double k2 = (double)(kx * kx + ky * ky + kz * kz);
    const double w = exp(-pi * pi * k2 / (alpha * alpha)) / (pi * k2);
    const double2 Sq = S[q];
    const double re = c * Sq.x + s * Sq.y;
    const double im = s * Sq.x - c * Sq.y;
    const double a = 2.0 * w * (-2.0 * pi) * im;
    fx += a * kx;
    fy += a * ky;
    fz += a * kz;
    ph += 2.0 * w * re;
  }
  // the real-space kernel has accumulated into f and pot; finish and scale
  f[3 * i + 0] = GM * (f[3 * i + 0] + fx);
  f[3 * i + 1] = GM * (f[3 * i + 1] + fy);
  f[3 * i + 2] = GM * (f[3 * i + 2] + fz);
  pot[i] = -GM * (pot[i] + ph - pi / (alpha * alpha) * nq);
}

}  // namespace

extern "C" int ct2g_ewald_direct_noalloc(int device, const uint32_t *qx, const uint32_t *qy,
                                         const uint32_t *qz, size_t nq, const uint32_t *sx,
                                         const uint32_t *sy, const uint32_t *sz, size_t ns,
                                         int kernel, double soft, double GM, double alpha,
                                         double rcut, int kmax, double *f, double *pot,
                                         void *stream) {
  if (!qx || !qy || !qz || !sx || !sy || !sz || !f || !pot || nq == 0 || ns == 0)
    return CT2G_EINVAL;
  if (kmax < 1 || kmax > CT2G_NOALLOC_KMAX) return CT2G_EINVAL;  // scratch holds kmax <= 24
  if (nq > kMaxSources) return CT2G_EINVAL;
  if (!(alpha > 0) || !(rcut > 0) || rcut > 0.5 || !(soft > 0)) return CT2G_EINVAL;
  if (kernel != CT2G_SOFT_PLUMMER && kernel != CT2G_SOFT_SPHERE) return CT2G_EINVAL;
  if (device < 0 || device >= 128) return CT2G_EINVAL;
  // an error the caller's own work left pending is theirs: report it without
  // clearing it, and run nothing
  if (cudaPeekAtLastError() != cudaSuccess) return CT2G_ECUDA;
  // the caller's current device is put back on every return
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) {
    cudaGetLastError();
    return CT2G_ENODEV;
  }
  struct Restore {
    int dev;
    ~Restore() {
      if (dev >= 0) cudaSetDevice(dev);
    }
  } restore{prev};
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return CT2G_ENODEV;
  }
  double2 *S = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[device]) {
      double2 *ptr = nullptr;
      if (cudaGetSymbolAddress((void **)&ptr, g_noalloc_sk) != cudaSuccess || !ptr) {
        cudaGetLastError();
        return CT2G_ECUDA;
      }
      g_noalloc_ptr[device] = ptr;
    }
    S = g_noalloc_ptr[device];
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int nbox = (kmax + 1) * (2 * kmax + 1) * (2 * kmax + 1);
  // the outputs accumulate, and S keeps the previous call's sums: clear all
  // (no error was pending on entry, so any error here is this call's own)
  if (cudaMemsetAsync(S, 0, sizeof(double2) * nbox, st) != cudaSuccess ||
      cudaMemsetAsync(f, 0, sizeof(double) * 3 * ns, st) != cudaSuccess ||
      cudaMemsetAsync(pot, 0, sizeof(double) * ns, st) != cudaSuccess) {
    cudaGetLastError();
    return CT2G_ECUDA;
  }
  dim3 g1(ct2g_div_up(ns, kSinkThreads), ct2g_div_up(nq, kSrcChunk));
  ewald_real_kernel<<<g1, kSinkThreads, 0, st>>>(sx, sy, sz, ns, qx, qy, qz, nq, kernel, soft,
                                                 alpha, rcut * rcut, f, pot);
  dim3 g2(ct2g_div_up(nbox, 128), ct2g_div_up(nq, kSrcChunk));
  noalloc_sk_kernel<<<g2, 128, 0, st>>>(kmax, qx, qy, qz, nq, S);
  noalloc_kspace_kernel<<<ct2g_div_up(ns, 128), 128, 0, st>>>(sx, sy, sz, ns, kmax, S, alpha,
                                                             (double)nq, GM, f, pot);
  if (cudaGetLastError() != cudaSuccess) return CT2G_ECUDA;
  return CT2G_OK;
}
