// Mesh stages of the gravity step:
//   P2M    per-cell moments about the cell centre, FP64 accumulate
//          (particle_compute_multipoles, src/particle.cpp:180-209)
//   Green  k-space Green's tensor with the near zone zeroed and Ewald images
//          (particle_greens, src/particle.cpp:116-178), built once per context
//   MG2L   per-k contraction L_a = sum_b G_{a+b} M_b (src/particle.cpp:244-250)
//   solve  forward FFT -> MG2L -> inverse FFT (particle_compute_expansions,
//          src/particle.cpp:211-271)
//
// The reference takes the multipole algebra from the un-vendored sfmm
// library.  Here it is the Cartesian Taylor form: with s = x_j - centre(src),
// t = x - centre(sink), R = centre(sink) - centre(src),
//   M_b = sum_j (-s_j)^b / b!,   L_a = sum_b D^{a+b} phi(R) M_b,
//   phi(x) = -GM sum_a L_a t^a/a!,   F_i = GM sum_a L_{a+e_i} t^a/a!,
// truncated at |a|+|b| <= p, the cell-centre sums done as one periodic
// convolution per (a, b) on the mesh.
#include <utility>

#include "ct2g_internal.cuh"

namespace {

// ---------------------------------------------------------------------------
// P2M: one thread per cell (particles are cell-sorted, so no atomics).
// Thread t is row-major cell t % C of box t / C; moments are per unit mass
// (the box's GM is applied to the forces).
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) p2m_kernel(const uint32_t *__restrict__ x,
                                                  const uint32_t *__restrict__ y,
                                                  const uint32_t *__restrict__ z,
                                                  const uint32_t *__restrict__ cs, int mbits,
                                                  int64_t CB, float *__restrict__ grid) {
  constexpr MiTable<P> T{};
  constexpr int NC = MiTable<P>::NC;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // box * C + row-major cell
  if (c >= CB) return;
  const uint32_t M1 = (1u << mbits) - 1u;
  const uint32_t cx = (uint32_t)(c >> (2 * mbits)) & M1, cy = (uint32_t)(c >> mbits) & M1,
                 cz = (uint32_t)c & M1;
  const uint32_t box = (uint32_t)(c >> (3 * mbits));
  const uint32_t key = (box << (3 * mbits)) | ct2g_morton(cx, cy, cz);
  const uint32_t b = cs[key], e = cs[key + 1];
  double acc[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) acc[k] = 0.0;
  const int sh = 32 - mbits;
  const uint32_t halfc = 1u << (sh - 1);
  const uint32_t ux = (cx << sh) + halfc, uy = (cy << sh) + halfc, uz = (cz << sh) + halfc;
  for (uint32_t i = b; i < e; i++) {
    // -s, exactly from the fixed-point difference
    const double sx = -(double)(int32_t)(x[i] - ux) * CT2G_TWO_M32;
    const double sy = -(double)(int32_t)(y[i] - uy) * CT2G_TWO_M32;
    const double sz = -(double)(int32_t)(z[i] - uz) * CT2G_TWO_M32;
    double px[P + 1], py[P + 1], pz[P + 1];
    px[0] = py[0] = pz[0] = 1.0;
#pragma unroll
    for (int q = 1; q <= P; q++) {
      px[q] = px[q - 1] * sx * (1.0 / q);
      py[q] = py[q - 1] * sy * (1.0 / q);
      pz[q] = pz[q - 1] * sz * (1.0 / q);
    }
#pragma unroll
    for (int k = 0; k < NC; k++) acc[k] += px[T.nx[k]] * py[T.ny[k]] * pz[T.nz[k]];
  }
#pragma unroll
  for (int k = 0; k < NC; k++) grid[(int64_t)k * CB + c] = (float)acc[k];
}

// ---------------------------------------------------------------------------
// MG2L alone (the precision form, and orders or meshes whose fused X pass
// does not fit in shared memory): one thread per k-point, in place.  A block's
// 128 k-points are one contiguous run of the spectrum ([k-point][nc]), staged
// through shared memory so that both the load and the store are coalesced;
// each thread's Green's values go to a private smem column.  blockIdx.y is
// the box; the boxes share G.  The zero-padding slots qk > N/2 are skipped.
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) mg2l_kernel(float2 *__restrict__ spec,
                                                   const float *__restrict__ G, int64_t CK,
                                                   int ldk, int nh) {
  constexpr int NC = ct2g_ncomp(P);
  extern __shared__ __align__(16) unsigned char smraw[];
  float2 *sm = reinterpret_cast<float2 *>(smraw);       // [128][NC]
  float *gs = reinterpret_cast<float *>(sm + 128 * NC);  // [NC][128]
  const int64_t q0 = (int64_t)blockIdx.x * 128;
  const int np = (int)min((int64_t)128, CK - q0);
  float2 *run = spec + ((int64_t)blockIdx.y * CK + q0) * NC;
  for (int e = threadIdx.x; e < np * NC; e += 128) sm[e] = run[e];
  const int64_t q = q0 + threadIdx.x;
  if (threadIdx.x < np) {
#pragma unroll
    for (int k = 0; k < NC; k++) gs[k * 128 + threadIdx.x] = __ldg(G + (int64_t)k * CK + q);
  }
  __syncthreads();
  if (threadIdx.x < np && (int)(q % ldk) < nh) {
    float2 m[NC];
#pragma unroll
    for (int k = 0; k < NC; k++) m[k] = sm[threadIdx.x * NC + k];
    ct2g_mg2l_all<P, 128>(m, gs + threadIdx.x, sm + threadIdx.x * NC,
                          std::make_integer_sequence<int, Mg2lPairs<P>::NP>{});
  }
  __syncthreads();
  for (int e = threadIdx.x; e < np * NC; e += 128) run[e] = sm[e];
}

// ctx->greens [nc][CK] -> ctx->greens_x: column (qj, qk), qk <= N/2, holds
// the column's values as [nc][qi]
__global__ void greens_cols_kernel(const float *__restrict__ G, int64_t CK, int N, int ldk,
                                   int nc, float *__restrict__ gx) {
  const int nh = N / 2 + 1;
  const int64_t gcol = (int64_t)nc * N;
  const int64_t total = (int64_t)N * nh * gcol;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t colid = e / gcol;
    const int r = (int)(e - colid * gcol);
    const int qj = (int)(colid / nh), qk = (int)(colid % nh);
    const int k = r / N, qi = r % N;
    gx[e] = G[(int64_t)k * CK + ((int64_t)qi * N + qj) * ldk + qk];
  }
}

// ---------------------------------------------------------------------------
// Green's tensor, FP64, runtime tables (built once per context)
// ---------------------------------------------------------------------------
constexpr int kMaxTerms = 16;
struct DTerm {
  int mx, my, mz, j;
  double coef;
};

// f^[j] = (r^-1 d/dr)^j f for the softened kernels and erf(alpha r)/r
__device__ void radial_plummer(double r2, double eps, int jmax, double *f) {
  double s2 = r2 + eps * eps;
  double inv = 1.0 / s2, base = 1.0 / sqrt(s2);
  double df = 1.0;  // (2j-1)!!
  for (int j = 0; j <= jmax; j++) {
    if (j > 0) df *= (2 * j - 1);
    f[j] = ((j & 1) ? -df : df) * base;
    base *= inv;
  }
}

__device__ void radial_sphere(double r2, double h, int jmax, double *f) {
  if (r2 >= h * h) {
    radial_plummer(r2, 0.0, jmax, f);
    return;
  }
  const double h3 = h * h * h;
  for (int j = 0; j <= jmax; j++) f[j] = 0.0;
  f[0] = 1.5 / h - 0.5 * r2 / h3;
  if (jmax >= 1) f[1] = -1.0 / h3;
}

__device__ void radial_erf(double r2, double alpha, int jmax, double *f) {
  const double a2 = alpha * alpha;
  const double spi = 1.7724538509055160273;
  if (a2 * r2 < 4.0) {
    // power series in u = r^2
    const double pre = 2.0 * alpha / spi;
    double p2 = 1.0;
    for (int j = 0; j <= jmax; j++) {
      double sum = 0.0, term = 1.0;
      for (int k = j; k < j + 80; k++) {
        double t = term / (2 * k + 1);
        sum += (k & 1) ? -t : t;
        term *= a2 * r2 / (k - j + 1);
        if (term < 1e-30 * fabs(sum) && k > j + 4) break;
      }
      f[j] = pre * p2 * sum;
      p2 *= 2.0 * a2;
    }
  } else {
    // 1/r - erfc(alpha r)/r with Smith's recursion for the erfc part
    const double r = sqrt(r2);
    const double ex = exp(-a2 * r2);
    double B = erfc(alpha * r) / r;
    double Aj = 1.0 / r;
    double twoa2j = 1.0;
    for (int j = 0; j <= jmax; j++) {
      if (j > 0) {
        twoa2j *= 2.0 * a2;
        B = ((2 * j - 1) * B + twoa2j / (alpha * spi) * ex) / r2;
        Aj *= (2 * j - 1) / r2;
      }
      f[j] = ((j & 1) ? -1.0 : 1.0) * (Aj - B);
    }
  }
}

__device__ __forceinline__ double ipow(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; i++) r *= x;
  return r;
}

// real-space part for components [k0, k0+K) at every lattice offset
__global__ void greens_real_kernel(int mbits, int p, int kernel, double soft, double bw2,
                                   double alpha, const DTerm *__restrict__ terms,
                                   const int *__restrict__ nterms, int k0, int K,
                                   double *__restrict__ out) {
  const int M = 1 << mbits;
  const int64_t C = (int64_t)M * M * M;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  int o[3] = {(int)(c >> (2 * mbits)), (int)((c >> mbits) & (M - 1)), (int)(c & (M - 1))};
  for (int d = 0; d < 3; d++)
    if (o[d] >= M / 2) o[d] -= M;
  const double h = 1.0 / M;
  const double R[3] = {o[0] * h, o[1] * h, o[2] * h};
  const double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
  const bool near = (double)(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]) <= bw2;
  double fe[CT2G_MAX_ORDER + 1], fk[CT2G_MAX_ORDER + 1], f[CT2G_MAX_ORDER + 1];
  radial_erf(r2, alpha, p, fe);
  if (!near) {
    if (kernel == CT2G_SOFT_SPHERE)
      radial_sphere(r2, soft, p, fk);
    else
      radial_plummer(r2, soft, p, fk);
  }
  for (int j = 0; j <= p; j++) f[j] = (near ? 0.0 : fk[j]) - fe[j];
  for (int kk = 0; kk < K; kk++) {
    const int k = k0 + kk;
    double g = 0.0;
    for (int t = 0; t < nterms[k]; t++) {
      const DTerm d = terms[k * kMaxTerms + t];
      g += d.coef * ipow(R[0], d.mx) * ipow(R[1], d.my) * ipow(R[2], d.mz) * f[d.j];
    }
    if (k == 0) g -= 3.14159265358979323846 / (alpha * alpha);
    out[(int64_t)kk * C + c] = g;
  }
}

// D^n phi_eps(R) of the softened kernel alone (no near-zone exclusion, no
// Ewald split) at R = -o h for a list of lattice offsets o: the primary-image
// term the mesh holds for a source cell at offset o from the sink cell
__global__ void shell_greens_kernel(int nshell, const int *__restrict__ offs, int mbits, int p,
                                    int nc, int kernel, double soft,
                                    const DTerm *__restrict__ terms,
                                    const int *__restrict__ nterms, float *__restrict__ out) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nshell) return;
  const double h = 1.0 / (double)(1 << mbits);
  const double R[3] = {-offs[3 * s] * h, -offs[3 * s + 1] * h, -offs[3 * s + 2] * h};
  const double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
  double f[CT2G_MAX_ORDER + 1];
  if (kernel == CT2G_SOFT_SPHERE)
    radial_sphere(r2, soft, p, f);
  else
    radial_plummer(r2, soft, p, f);
  for (int k = 0; k < nc; k++) {
    double g = 0.0;
    for (int t = 0; t < nterms[k]; t++) {
      const DTerm d = terms[k * kMaxTerms + t];
      g += d.coef * ipow(R[0], d.mx) * ipow(R[1], d.my) * ipow(R[2], d.mz) * f[d.j];
    }
    out[(size_t)s * nc + k] = (float)g;
  }
}

// combine the FFT of the real-space part with the folded Ewald k-space sum
// (spectrum rows hold ldk entries; those past M/2 are padding, set to zero)
__global__ void greens_finish_kernel(int mbits, int p, double alpha, int kmax,
                                     const int *__restrict__ mi, int k0, int K, int ldk,
                                     const double2 *__restrict__ spec64, float *__restrict__ G) {
  const int M = 1 << mbits;
  const int NH = M / 2 + 1;
  const int64_t CK = (int64_t)M * M * ldk;
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= CK) return;
  const int qx = (int)(q / ((int64_t)M * ldk)), qy = (int)((q / ldk) % M), qz = (int)(q % ldk);
  if (qz >= NH) {
    for (int kk = 0; kk < K; kk++) G[(int64_t)(k0 + kk) * CK + q] = 0.f;
    return;
  }
  const double norm = 1.0 / ((double)M * M * M);
  double acc[64];
  for (int kk = 0; kk < K; kk++) {
    const int k = k0 + kk;
    const int deg = mi[3 * k] + mi[3 * k + 1] + mi[3 * k + 2];
    const double2 v = spec64[(int64_t)kk * CK + q];
    acc[kk] = ((deg & 1) ? v.y : v.x) * norm;
  }
  // aliases kv == q (mod M) with |kv| <= kmax, kv != 0
  const double pi = 3.14159265358979323846;
  const double K2 = (double)kmax * kmax;
  auto first = [&](int qd) {  // smallest alias of qd (in [0,M)) that is >= -kmax
    int t = qd;
    while (t - M >= -kmax) t -= M;
    return t;
  };
  for (int kx = first(qx); kx <= kmax; kx += M)
    for (int ky = first(qy); ky <= kmax; ky += M)
      for (int kz = first(qz); kz <= kmax; kz += M) {
        const double k2 = (double)kx * kx + (double)ky * ky + (double)kz * kz;
        if (k2 == 0.0 || k2 > K2) continue;
        const double w = exp(-pi * pi * k2 / (alpha * alpha)) / (pi * k2);
        const double kv[3] = {2 * pi * kx, 2 * pi * ky, 2 * pi * kz};
        for (int kk = 0; kk < K; kk++) {
          const int k = k0 + kk;
          const int *n = mi + 3 * k;
          const int deg = n[0] + n[1] + n[2];
          const double s = ((deg / 2) & 1) ? -1.0 : 1.0;
          acc[kk] += s * w * ipow(kv[0], n[0]) * ipow(kv[1], n[1]) * ipow(kv[2], n[2]);
        }
      }
  for (int kk = 0; kk < K; kk++) G[(int64_t)(k0 + kk) * CK + q] = (float)acc[kk];
}

double factd(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; i++) r *= i;
  return r;
}

template <int P>
int launch_p2m(ct2g_ctx *ctx) {
  const unsigned T = 128;
  p2m_kernel<P><<<ct2g_div_up(ctx->CB, T), T, 0, ctx->stream>>>(
      ctx->x, ctx->y, ctx->z, ctx->cell_start, ctx->mbits, ctx->CB, ctx->grid);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

template <int P>
int launch_mg2l(ct2g_ctx *ctx) {
  constexpr int NC = ct2g_ncomp(P);
  const size_t smem = (sizeof(float2) + sizeof(float)) * 128 * NC;
  auto k = mg2l_kernel<P>;
  CT2G_TRY(ct2g_smem_attrs(ctx, k, smem));
  const dim3 grid(ct2g_div_up(ctx->CK, 128), (unsigned)ctx->nbox);
  k<<<grid, 128, smem, ctx->stream>>>(ctx->spec, ctx->greens, ctx->CK, ctx->ldk, ctx->M / 2 + 1);
  CT2G_LAUNCHED(ctx);
  return CT2G_OK;
}

}  // namespace

// Green's-table Ewald split (box units), as in the CPU oracle
static const double kGreensAlpha = 12.0;
static const int kGreensKmax = 36;

// D^n f = sum_m n!/(m!(n-2m)! 2^|m|) R^(n-2m) f^[|n|-|m|]: one DTerm per m,
// per multi-index of degree <= p; mi holds the multi-indices
static void build_dterms(int p, std::vector<DTerm> &terms, std::vector<int> &nterms,
                         std::vector<int> &mi) {
  const int nc = ct2g_ncomp(p);
  terms.assign((size_t)nc * kMaxTerms, DTerm{});
  nterms.assign(nc, 0);
  mi.assign(3 * nc, 0);
  {
    int k = 0;
    for (int d = 0; d <= p; d++)
      for (int a = d; a >= 0; a--)
        for (int b = d - a; b >= 0; b--) {
          int n[3] = {a, b, d - a - b};
          mi[3 * k] = n[0];
          mi[3 * k + 1] = n[1];
          mi[3 * k + 2] = n[2];
          int t = 0;
          for (int mx = 0; 2 * mx <= n[0]; mx++)
            for (int my = 0; 2 * my <= n[1]; my++)
              for (int mz = 0; 2 * mz <= n[2]; mz++) {
                int m[3] = {mx, my, mz};
                double c = 1.0;
                for (int q = 0; q < 3; q++)
                  c *= factd(n[q]) / (factd(m[q]) * factd(n[q] - 2 * m[q]));
                c /= (double)(1 << (mx + my + mz));
                DTerm &dt = terms[(size_t)k * kMaxTerms + t];
                dt.mx = n[0] - 2 * mx;
                dt.my = n[1] - 2 * my;
                dt.mz = n[2] - 2 * mz;
                dt.j = d - mx - my - mz;
                dt.coef = c;
                t++;
              }
          nterms[k] = t;
          k++;
        }
  }
}

int ct2g_shell_greens(ct2g_ctx *ctx, const std::vector<int> &offs3, float *d_out) {
  const int nshell = (int)(offs3.size() / 3);
  if (nshell == 0) return CT2G_OK;
  std::vector<DTerm> terms;
  std::vector<int> nterms, mi;
  build_dterms(ctx->p, terms, nterms, mi);
  DTerm *d_terms = nullptr;
  int *d_nterms = nullptr, *d_offs = nullptr;
  cudaError_t e = cudaMalloc(&d_terms, sizeof(DTerm) * terms.size());
  if (e == cudaSuccess) e = cudaMalloc(&d_nterms, sizeof(int) * nterms.size());
  if (e == cudaSuccess) e = cudaMalloc(&d_offs, sizeof(int) * offs3.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(d_terms, terms.data(), sizeof(DTerm) * terms.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_nterms, nterms.data(), sizeof(int) * nterms.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(d_offs, offs3.data(), sizeof(int) * offs3.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    shell_greens_kernel<<<ct2g_div_up(nshell, 64), 64, 0, ctx->stream>>>(
        nshell, d_offs, ctx->mbits, ctx->p, ctx->nc, ctx->opt.kernel, ctx->opt.hsoft, d_terms,
        d_nterms, d_out);
    ctx->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (d_terms) cudaFree(d_terms);
  if (d_nterms) cudaFree(d_nterms);
  if (d_offs) cudaFree(d_offs);
  if (e != cudaSuccess) return ct2g_cuda_fail(ctx, e, "shell Green's table");
  return CT2G_OK;
}

int ct2g_build_greens(ct2g_ctx *ctx) {
  if (ctx->greens_valid) return CT2G_OK;
  if (ctx->capturing) return ct2g_fail(ctx, CT2G_ESTATE, "Green's table not built before recording");
  const int p = ctx->p, nc = ctx->nc, M = ctx->M;
  std::vector<DTerm> terms;
  std::vector<int> nterms, mi;
  build_dterms(p, terms, nterms, mi);
  DTerm *d_terms = nullptr;
  int *d_nterms = nullptr, *d_mi = nullptr;
  double *rs = nullptr;
  double2 *sp = nullptr;
  int rc = CT2G_OK;
  const int K = std::min(nc, M >= 512 ? 2 : (M >= 256 ? 8 : 16));
  auto cleanup = [&]() {
    cudaStreamSynchronize(ctx->stream);
    if (d_terms) cudaFree(d_terms);
    if (d_nterms) cudaFree(d_nterms);
    if (d_mi) cudaFree(d_mi);
    if (rs) cudaFree(rs);
    if (sp) cudaFree(sp);
  };
  do {
    cudaError_t e;
    if ((e = cudaMalloc(&d_terms, sizeof(DTerm) * terms.size())) != cudaSuccess ||
        (e = cudaMalloc(&d_nterms, sizeof(int) * nc)) != cudaSuccess ||
        (e = cudaMalloc(&d_mi, sizeof(int) * 3 * nc)) != cudaSuccess ||
        (e = cudaMalloc(&rs, sizeof(double) * (size_t)K * ctx->C)) != cudaSuccess ||
        (e = cudaMalloc(&sp, sizeof(double2) * (size_t)K * ctx->CK)) != cudaSuccess) {
      rc = ct2g_cuda_fail(ctx, e, "greens scratch allocation");
      break;
    }
    cudaMemcpyAsync(d_terms, terms.data(), sizeof(DTerm) * terms.size(), cudaMemcpyHostToDevice,
                    ctx->stream);
    cudaMemcpyAsync(d_nterms, nterms.data(), sizeof(int) * nc, cudaMemcpyHostToDevice,
                    ctx->stream);
    cudaMemcpyAsync(d_mi, mi.data(), sizeof(int) * 3 * nc, cudaMemcpyHostToDevice, ctx->stream);
    const double soft = ctx->opt.hsoft;
    const double bw2 = (double)ctx->opt.bwidth * (double)ctx->opt.bwidth;
    for (int k0 = 0; k0 < nc && rc == CT2G_OK; k0 += K) {
      const int kk = std::min(K, nc - k0);
      greens_real_kernel<<<ct2g_div_up(ctx->C, 128), 128, 0, ctx->stream>>>(
          ctx->mbits, p, ctx->opt.kernel, soft, bw2, kGreensAlpha, d_terms, d_nterms, k0, kk,
          rs);
      ctx->launches++;
      if ((e = cudaGetLastError()) != cudaSuccess) {
        rc = ct2g_cuda_fail(ctx, e, "greens_real_kernel");
        break;
      }
      rc = ct2g_fft_r2c_f64(ctx, rs, sp, M, kk, ctx->ldk);
      if (rc != CT2G_OK) break;
      greens_finish_kernel<<<ct2g_div_up(ctx->CK, 128), 128, 0, ctx->stream>>>(
          ctx->mbits, p, kGreensAlpha, kGreensKmax, d_mi, k0, kk, ctx->ldk, sp, ctx->greens);
      ctx->launches++;
      if ((e = cudaGetLastError()) != cudaSuccess) {
        rc = ct2g_cuda_fail(ctx, e, "greens_finish_kernel");
        break;
      }
    }
  } while (0);
  cleanup();
  if (rc == CT2G_OK && ctx->greens_x) {
    greens_cols_kernel<<<4 * ctx->num_sms, 256, 0, ctx->stream>>>(ctx->greens, ctx->CK, M,
                                                                 ctx->ldk, nc, ctx->greens_x);
    ctx->launches++;
  }
  if (rc == CT2G_OK) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ct2g_cuda_fail(ctx, e, "greens build");
    ctx->greens_valid = true;
  }
  return rc;
}

size_t ct2g_greens_x_floats(const ct2g_ctx *ctx) {
  return (size_t)ctx->M * (ctx->M / 2 + 1) * ctx->nc * ctx->M;
}

int ct2g_mg2l_split(ct2g_ctx *ctx) {
  switch (ctx->p) {
    case 1: return launch_mg2l<1>(ctx);
    case 2: return launch_mg2l<2>(ctx);
    case 3: return launch_mg2l<3>(ctx);
    case 4: return launch_mg2l<4>(ctx);
    case 5: return launch_mg2l<5>(ctx);
    case 6: return launch_mg2l<6>(ctx);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "unsupported order");
}

int ct2g_p2m(ct2g_ctx *ctx) {
  switch (ctx->p) {
    case 1: return launch_p2m<1>(ctx);
    case 2: return launch_p2m<2>(ctx);
    case 3: return launch_p2m<3>(ctx);
    case 4: return launch_p2m<4>(ctx);
    case 5: return launch_p2m<5>(ctx);
    case 6: return launch_p2m<6>(ctx);
  }
  return ct2g_fail(ctx, CT2G_EINVAL, "unsupported order");
}

// forward FFT of the moments, MG2L, inverse FFT into the expansions (the
// expansion grid, or straight into the forces)
int ct2g_mesh_solve(ct2g_ctx *ctx, bool fused_l2p, bool pot, int p2m) {
  CT2G_TRY(ct2g_build_greens(ctx));
  ct2g_mark(ctx, 2);
  CT2G_TRY(ct2g_spec_forward(ctx, p2m));
  ct2g_mark(ctx, 3);
  CT2G_TRY(ct2g_spec_mg2l(ctx));
  ct2g_mark(ctx, 4);
  if (fused_l2p) {
    // every particle of the range gets its far field; others read zero
    const size_t n = ctx->n;
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->fx, 0, n * 4, ctx->stream));
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->fy, 0, n * 4, ctx->stream));
    CT2G_CUDA(ctx, cudaMemsetAsync(ctx->fz, 0, n * 4, ctx->stream));
    if (pot) CT2G_CUDA(ctx, cudaMemsetAsync(ctx->pot, 0, n * 4, ctx->stream));
  }
  CT2G_TRY(ct2g_spec_inverse(ctx, fused_l2p, pot));
  ct2g_mark(ctx, 5);
  return CT2G_OK;
}
