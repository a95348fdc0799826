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
