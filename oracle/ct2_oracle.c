/*
 * ct2_oracle.c -- CPU restatement of the ct2 gravity step, used ONLY as test
 * infrastructure (the checker for the CUDA path, and the timed CPU baseline).
 * Nothing in the product library links or calls this file.
 *
 * What it restates (reference = dmarce1/ct2, file:line within that project):
 *   - cell binning: recursive bisection of particle_to_grid / particle_sort_by_pos
 *     (src/particle.cpp:69-114, 349-362) with the z-index defect fixed
 *     (cells[I0][I1][I2] instead of cells[I0][I1][I1], particle.cpp:92) and a
 *     power-of-two mesh; plus the stable counting-sort order the GPU produces.
 *   - P2M per-cell moments about the cell centre (particle.cpp:180-209), in FP64.
 *   - the real-space Green's tensor with the near zone zeroed and Ewald images
 *     added (particle.cpp:116-178), made consistent with the direct-sum stencil.
 *   - L2P + direct-sum near field + velocity/rung update (src/kick.cpp:3-103),
 *     with the source-loop, force-reduction and lane-index defects fixed.
 *   - drift (src/drift.cpp:4-18).
 *   - an FP64 Ewald direct sum: the force truth the method is judged against.
 *
 * The reference's multipole arithmetic (P2M, MG2L, L2P, greens, greens_ewald)
 * lives in the un-vendored "sfmm" library (no version pin exists), so this file
 * restates the published Cartesian-Taylor FMM algorithm instead: parity of the
 * multipole basis is UNPINNED against sfmm; the physics is pinned by the Ewald
 * direct sum (itself pinned by the simple-cubic Madelung constant) and by the
 * known-answer tests under tests/.
 *
 * Build: see oracle/Makefile (gcc -O3 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define TWO_M32 2.3283064365386963e-10 /* 2^-32 */

/* ------------------------------------------------------------------------ */
/* multi-indices n=(nx,ny,nz), |n|<=p, ordered by degree, then nx descending,  */
/* then ny descending.  idx = T(d) + (d-nx)(d-nx+1)/2 + nz, T(d)=d(d+1)(d+2)/6 */
/* ------------------------------------------------------------------------ */
int ct2o_ncomp(int p) { return (p + 1) * (p + 2) * (p + 3) / 6; }

int ct2o_mi_index(int nx, int ny, int nz) {
  int d = nx + ny + nz;
  return d * (d + 1) * (d + 2) / 6 + (d - nx) * (d - nx + 1) / 2 + nz;
}

void ct2o_mi_table(int p, int *nxyz) {
  int k = 0;
  for (int d = 0; d <= p; d++)
    for (int nx = d; nx >= 0; nx--)
      for (int ny = d - nx; ny >= 0; ny--) {
        nxyz[3 * k + 0] = nx;
        nxyz[3 * k + 1] = ny;
        nxyz[3 * k + 2] = d - nx - ny;
        k++;
      }
}

static double dfact(int n) { /* n!! for n>=-1 */
  double r = 1.0;
  for (int i = n; i > 1; i -= 2) r *= i;
  return r;
}
static double fact(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; i++) r *= i;
  return r;
}

/* ------------------------------------------------------------------------ */
/* Binning                                                                   */
/* ------------------------------------------------------------------------ */

/* Morton key of cell (i,j,k): bits interleaved from the most significant,
 * x first, then y, then z.  This is the order in which the reference's
 * recursive bisection (particle.cpp:89-114) lays the leaves out in the
 * particle array: depth d splits dimension d%3 at the midpoint
 * fixed32((I+N/2)/Ncell) = (I+N/2) << (32-mbits) (particle.cpp:103), lower
 * half first. */
static uint32_t spread3(uint32_t v) {
  uint32_t r = 0;
  for (int b = 0; b < 10; b++) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}
static uint32_t compact3(uint32_t v) {
  uint32_t r = 0;
  for (int b = 0; b < 10; b++) r |= ((v >> (3 * b)) & 1u) << b;
  return r;
}
uint32_t ct2o_morton(uint32_t i, uint32_t j, uint32_t k) {
  return (spread3(i) << 2) | (spread3(j) << 1) | spread3(k);
}
void ct2o_morton_decode(uint32_t key, uint32_t *i, uint32_t *j, uint32_t *k) {
  *i = compact3(key >> 2);
  *j = compact3(key >> 1);
  *k = compact3(key);
}

/* cell key of a fixed-point position on a 2^mbits mesh: the Morton key of
 * its top mbits bits per axis */
void ct2o_cell_keys(const uint32_t *x, const uint32_t *y, const uint32_t *z,
                    int64_t n, int mbits, uint32_t *key) {
  const int sh = 32 - mbits;
  for (int64_t i = 0; i < n; i++) key[i] = ct2o_morton(x[i] >> sh, y[i] >> sh, z[i] >> sh);
}

/* stable counting sort by Morton key: perm[k] = original index of the k-th
 * particle in cell order; cell_start[key] (ncells+1 entries) indexed by the
 * Morton key. */
void ct2o_bin_stable(const uint32_t *key, int64_t n, int64_t ncells,
                     int64_t *perm, int64_t *cell_start) {
  memset(cell_start, 0, sizeof(int64_t) * (ncells + 1));
  for (int64_t i = 0; i < n; i++) cell_start[key[i] + 1]++;
  for (int64_t c = 0; c < ncells; c++) cell_start[c + 1] += cell_start[c];
  int64_t *fill = (int64_t *)malloc(sizeof(int64_t) * ncells);
  memcpy(fill, cell_start, sizeof(int64_t) * ncells);
  for (int64_t i = 0; i < n; i++) perm[fill[key[i]]++] = i;
  free(fill);
}

/* Restatement of particle_sort_by_pos (particle.cpp:69-87): the reference's
 * Hoare-style partition of [lo,hi) on coordinate dim against xmid; returns the
 * split.  Operates on an index array (ids) instead of swapping 7 SoA arrays. */
static int64_t bisect_partition(int64_t *ids, const uint32_t *pos, int64_t lo,
                                int64_t hi, uint32_t xmid) {
  while (lo < hi) {
    if (pos[ids[lo]] >= xmid) {
      while (lo != hi) {
        hi--;
        if (pos[ids[hi]] < xmid) {
          int64_t t = ids[hi];
          ids[hi] = ids[lo];
          ids[lo] = t;
          break;
        }
      }
    }
    lo++;
  }
  return hi;
}

/* Restatement of the recursive particle_to_grid (particle.cpp:89-114) for a
 * power-of-two mesh M = 2^mbits, z-index defect fixed.  ids: the particle
 * order (in/out); cell_begin/cell_end: leaf ranges indexed (i*M+j)*M+k. */
static void bisect_rec(int64_t *ids, const uint32_t *const pos[3], int64_t lo,
                       int64_t hi, int I[3], int N[3], int depth, int mbits,
                       int64_t *cb, int64_t *ce) {
  const int M = 1 << mbits;
  if (N[0] * N[1] * N[2] == 1) {
    int64_t c = ((int64_t)I[0] * M + I[1]) * M + I[2];
    cb[c] = lo;
    ce[c] = hi;
    return;
  }
  const int xdim = depth % 3;
  int No2[3] = {N[0], N[1], N[2]};
  No2[xdim] >>= 1;
  int Il[3] = {I[0], I[1], I[2]}, Ir[3] = {I[0], I[1], I[2]};
  Ir[xdim] += No2[xdim];
  uint32_t xmid = (uint32_t)((uint64_t)(I[xdim] + No2[xdim]) << (32 - mbits));
  int64_t mid = bisect_partition(ids, pos[xdim], lo, hi, xmid);
  bisect_rec(ids, pos, mid, hi, Ir, No2, depth + 1, mbits, cb, ce);
  bisect_rec(ids, pos, lo, mid, Il, No2, depth + 1, mbits, cb, ce);
}

void ct2o_bin_bisect(const uint32_t *x, const uint32_t *y, const uint32_t *z,
                     int64_t n, int mbits, int64_t *ids, int64_t *cell_begin,
                     int64_t *cell_end) {
  const uint32_t *pos[3] = {x, y, z};
  for (int64_t i = 0; i < n; i++) ids[i] = i;
  int I[3] = {0, 0, 0}, N[3] = {1 << mbits, 1 << mbits, 1 << mbits};
  bisect_rec(ids, pos, 0, n, I, N, 0, mbits, cell_begin, cell_end);
}

/* ------------------------------------------------------------------------ */
/* P2M: M_b(c) = sum_j (-s_j)^b / b!, s_j = x_j - centre(c)  (unit masses)   */
/* particle.cpp:180-209; computed in FP64.  Mgrid layout [ncomp][M^3].       */
/* ------------------------------------------------------------------------ */
static double center_offset(uint32_t u, int64_t cidx, int mbits) {
  /* centre of cell cidx along one axis in fixed point: (c + 1/2) * 2^(32-m) */
  uint32_t cu = (uint32_t)(((uint64_t)cidx << (32 - mbits)) + (1ull << (31 - mbits)));
  return (double)(int32_t)(u - cu) * TWO_M32;
}

void ct2o_p2m(const uint32_t *x, const uint32_t *y, const uint32_t *z,
              const int64_t *cell_start, int mbits, int p, double *Mgrid) {
  const int M = 1 << mbits;
  const int64_t C = (int64_t)M * M * M;
  const int nc = ct2o_ncomp(p);
  int *mi = (int *)malloc(sizeof(int) * 3 * nc);
  ct2o_mi_table(p, mi);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t c = 0; c < C; c++) {
    double acc[220];
    for (int k = 0; k < nc; k++) acc[k] = 0.0;
    const int64_t ci = c / ((int64_t)M * M), cj = (c / M) % M, ck = c % M;
    const uint32_t key = ct2o_morton((uint32_t)ci, (uint32_t)cj, (uint32_t)ck);
    for (int64_t i = cell_start[key]; i < cell_start[key + 1]; i++) {
      double s[3];
      s[0] = -center_offset(x[i], ci, mbits);
      s[1] = -center_offset(y[i], cj, mbits);
      s[2] = -center_offset(z[i], ck, mbits);
      double pw[3][12];
      for (int d = 0; d < 3; d++) {
        pw[d][0] = 1.0;
        for (int q = 1; q <= p; q++) pw[d][q] = pw[d][q - 1] * s[d] / q;
      }
      for (int k = 0; k < nc; k++)
        acc[k] += pw[0][mi[3 * k]] * pw[1][mi[3 * k + 1]] * pw[2][mi[3 * k + 2]];
    }
    for (int k = 0; k < nc; k++) Mgrid[(int64_t)k * C + c] = acc[k];
  }
  free(mi);
}

/* ------------------------------------------------------------------------ */
/* Radial-kernel derivative tables.                                          */
/*   For radial f, D^n f(R) = sum_{m<=n/2} n!/(m!(n-2m)! 2^|m|) R^(n-2m)     */
/*                            * f^[|n|-|m|](r),  f^[j] = (r^-1 d/dr)^j f.     */
/* ------------------------------------------------------------------------ */

/* f^[j] for the softened kernel (r^2+eps^2)^-1/2 (eps=0: Newtonian 1/r) */
static void radial_plummer(double r2, double eps, int jmax, double *f) {
  double s2 = r2 + eps * eps;
  double inv = 1.0 / s2, base = 1.0 / sqrt(s2);
  for (int j = 0; j <= jmax; j++) {
    f[j] = ((j & 1) ? -1.0 : 1.0) * dfact(2 * j - 1) * base;
    base *= inv;
  }
}

/* f^[j] for erf(alpha r)/r.  Series in u=r^2 for alpha r < 2, otherwise
 * 1/r - erfc(alpha r)/r with Smith's recursion for the erfc part. */
static void radial_erf(double r2, double alpha, int jmax, double *f) {
  const double a2 = alpha * alpha;
  const double spi = 1.7724538509055160273;
  if (a2 * r2 < 4.0) {
    const double pre = 2.0 * alpha / spi;
    for (int j = 0; j <= jmax; j++) {
      /* f^[j] = pre * 2^j * sum_{k>=j} (-1)^k alpha^{2k} u^{k-j} / ((k-j)! (2k+1)) */
      double sum = 0.0, term = 1.0; /* term = (a2 u)^(k-j)/(k-j)! */
      for (int k = j; k < j + 80; k++) {
        double t = term / (2 * k + 1);
        sum += (k & 1) ? -t : t;
        term *= a2 * r2 / (k - j + 1);
        if (term < 1e-30 * fabs(sum) && k > j + 4) break;
      }
      f[j] = pre * pow(2.0 * a2, j) * sum;
    }
  } else {
    const double r = sqrt(r2);
    const double ex = exp(-a2 * r2);
    double B = erfc(alpha * r) / r; /* B_0 */
    double Aj = 1.0 / r;            /* (2j-1)!!/r^(2j+1) */
    double twoa2j = 1.0;
    for (int j = 0; j <= jmax; j++) {
      if (j > 0) {
        twoa2j *= 2.0 * a2;
        B = ((2 * j - 1) * B + twoa2j / (alpha * spi) * ex) / r2;
        Aj *= (2 * j - 1) / r2;
      }
      /* (r^-1 d/dr)^j [1/r - erfc/r] = (-1)^j (A_j - B_j) */
      f[j] = ((j & 1) ? -1.0 : 1.0) * (Aj - B);
    }
  }
}

/* f^[j] for the reference's compact "uniform sphere" kernel (kick.cpp:52-60):
 * phi = 1.5/h - 0.5 r^2/h^3 for r<h, 1/r outside. */
static void radial_sphere(double r2, double h, int jmax, double *f) {
  if (r2 >= h * h) {
    radial_plummer(r2, 0.0, jmax, f);
    return;
  }
  const double h3 = h * h * h;
  for (int j = 0; j <= jmax; j++) f[j] = 0.0;
  f[0] = 1.5 / h - 0.5 * r2 / h3;
  if (jmax >= 1) f[1] = -1.0 / h3;
}

/* expansion of D^n into (m, coefficient) terms, generic over the kernel */
typedef struct {
  int nterm;
  int mono[64][3];
  int j[64];
  double coef[64];
} dterms_t;

static void build_dterms(int p, dterms_t *T) {
  const int nc = ct2o_ncomp(p);
  int *mi = (int *)malloc(sizeof(int) * 3 * nc);
  ct2o_mi_table(p, mi);
  for (int k = 0; k < nc; k++) {
    const int *n = mi + 3 * k;
    int t = 0;
    for (int mx = 0; 2 * mx <= n[0]; mx++)
      for (int my = 0; 2 * my <= n[1]; my++)
        for (int mz = 0; 2 * mz <= n[2]; mz++) {
          double c = 1.0;
          int m[3] = {mx, my, mz};
          for (int d = 0; d < 3; d++) c *= fact(n[d]) / (fact(m[d]) * fact(n[d] - 2 * m[d]));
          c /= (double)(1 << (mx + my + mz));
          T[k].mono[t][0] = n[0] - 2 * mx;
          T[k].mono[t][1] = n[1] - 2 * my;
          T[k].mono[t][2] = n[2] - 2 * mz;
          T[k].j[t] = n[0] + n[1] + n[2] - mx - my - mz;
          T[k].coef[t] = c;
          t++;
        }
    T[k].nterm = t;
  }
  free(mi);
}

static double ipow(double x, int e) {
  double r = 1.0;
  for (int i = 0; i < e; i++) r *= x;
  return r;
}

/* kernel ids */
#define CT2O_KERNEL_PLUMMER 0
#define CT2O_KERNEL_SPHERE 1

/* Real-space part of the Green's tensor on the M^3 lattice of cell offsets,
 * G_n(R) = [R not in near zone] D^n phi_soft(R) - D^n erf(alpha|R|)/|R|
 *          (+ the constant -pi/alpha^2 on G_0),
 * the Ewald k-space part being added in Fourier space (ct2o_greens_kfold).
 * Near zone = integer min-image offsets o with |o|^2 <= bwidth^2: the SAME set
 * the direct sum visits, so no pair is counted twice or missed (the reference
 * excluded j^2+k^2+l^2<=10 without wrap, particle.cpp:136, against a
 * bwidth^2 stencil, particle.cpp:311).  Layout [ncomp][M^3], offset index
 * (i*M+j)*M+k with i the min-image-wrapped x offset. */
void ct2o_greens_real(int mbits, int p, int kernel, double soft, double bwidth,
                      double alpha, double *G) {
  const int M = 1 << mbits;
  const int64_t C = (int64_t)M * M * M;
  const int nc = ct2o_ncomp(p);
  dterms_t *T = (dterms_t *)malloc(sizeof(dterms_t) * nc);
  build_dterms(p, T);
  const double h = 1.0 / M;
  const double bw2 = bwidth * bwidth;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < C; c++) {
    int o[3] = {(int)(c / ((int64_t)M * M)), (int)((c / M) % M), (int)(c % M)};
    for (int d = 0; d < 3; d++)
      if (o[d] >= M / 2) o[d] -= M;
    const double R[3] = {o[0] * h, o[1] * h, o[2] * h};
    const double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2];
    const int near = (double)(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]) <= bw2;
    double fe[16], fk[16], f[16];
    radial_erf(r2, alpha, p, fe);
    if (!near) {
      if (kernel == CT2O_KERNEL_SPHERE)
        radial_sphere(r2, soft, p, fk);
      else
        radial_plummer(r2, soft, p, fk);
    }
    for (int j = 0; j <= p; j++) f[j] = (near ? 0.0 : fk[j]) - fe[j];
    for (int k = 0; k < nc; k++) {
      double g = 0.0;
      for (int t = 0; t < T[k].nterm; t++)
        g += T[k].coef[t] * ipow(R[0], T[k].mono[t][0]) * ipow(R[1], T[k].mono[t][1]) *
             ipow(R[2], T[k].mono[t][2]) * f[T[k].j[t]];
      if (k == 0) g -= M_PI / (alpha * alpha);
      G[(int64_t)k * C + c] = g;
    }
  }
  free(T);
}

/* Ewald k-space part of the Green's tensor, folded onto the r2c grid of the
 * M^3 mesh:  out_n(q) = sum_{k != 0, k == q mod M, |k|<=Kmax}
 *                         (2 pi i)^|n| k^n exp(-pi^2 k^2/alpha^2) / (pi k^2).
 * This is the mesh DFT of the k-space Ewald sum sampled at the lattice,
 * divided by M^3.  Even |n|: value is real; odd |n|: purely imaginary; the
 * real (even) or imaginary (odd) part is stored.  Layout [ncomp][M][M][M/2+1]. */
void ct2o_greens_kfold(int mbits, int p, double alpha, int Kmax, double *out) {
  const int M = 1 << mbits;
  const int Mh = M / 2 + 1;
  const int64_t Ck = (int64_t)M * M * Mh;
  const int nc = ct2o_ncomp(p);
  int *mi = (int *)malloc(sizeof(int) * 3 * nc);
  ct2o_mi_table(p, mi);
  memset(out, 0, sizeof(double) * nc * Ck);
  const double K2max = (double)Kmax * Kmax;
  /* parallel over kx residue classes to avoid write races */
#pragma omp parallel for schedule(dynamic, 1)
  for (int qx = 0; qx < M; qx++) {
    for (int kx = -Kmax; kx <= Kmax; kx++) {
      if ((((kx % M) + M) % M) != qx) continue;
      for (int ky = -Kmax; ky <= Kmax; ky++)
        for (int kz = -Kmax; kz <= Kmax; kz++) {
          double k2 = (double)kx * kx + (double)ky * ky + (double)kz * kz;
          if (k2 == 0.0 || k2 > K2max) continue;
          int qz = ((kz % M) + M) % M;
          if (qz >= Mh) continue; /* only the stored half */
          int qy = ((ky % M) + M) % M;
          double w = exp(-M_PI * M_PI * k2 / (alpha * alpha)) / (M_PI * k2);
          const int64_t base = ((int64_t)qx * M + qy) * Mh + qz;
          const double kv[3] = {2 * M_PI * kx, 2 * M_PI * ky, 2 * M_PI * kz};
          for (int c = 0; c < nc; c++) {
            const int *n = mi + 3 * c;
            int d = n[0] + n[1] + n[2];
            /* i^d: real for even d (sign (-1)^(d/2)), imaginary for odd d */
            double s = ((d / 2) & 1) ? -1.0 : 1.0;
            out[(int64_t)c * Ck + base] +=
                s * w * ipow(kv[0], n[0]) * ipow(kv[1], n[1]) * ipow(kv[2], n[2]);
          }
        }
    }
  }
  free(mi);
}

/* ------------------------------------------------------------------------ */
/* L2P + near field (kick.cpp:3-68), FP64 restatement.                       */
/*   far:  F_i = GM * sum_a L_{a+e_i}(c) t^a/a!,   pot = -GM sum_a L_a t^a/a! */
/*   near: F = -GM sum_{j in stencil} d_ij * kernel'(r),  d_ij = x_i - x_j    */
/* Particles are the cell-sorted arrays; Lgrid layout [ncomp][M^3] (real).    */
/* ------------------------------------------------------------------------ */
void ct2o_forces(const uint32_t *x, const uint32_t *y, const uint32_t *z,
                 const int64_t *cell_start, int mbits, int p, const double *Lgrid,
                 int kernel, double soft, double bwidth, double GM,
                 double *ffar, double *fnear, double *pot) {
  const int M = 1 << mbits;
  const int64_t C = (int64_t)M * M * M;
  const int nc = ct2o_ncomp(p);
  int *mi = (int *)malloc(sizeof(int) * 3 * nc);
  ct2o_mi_table(p, mi);
  /* stencil offsets */
  int B = (int)floor(bwidth);
  int nst = 0;
  int(*st)[3] = malloc(sizeof(int[3]) * (2 * B + 1) * (2 * B + 1) * (2 * B + 1));
  for (int i = -B; i <= B; i++)
    for (int j = -B; j <= B; j++)
      for (int k = -B; k <= B; k++)
        if ((double)(i * i + j * j + k * k) <= bwidth * bwidth) {
          st[nst][0] = i;
          st[nst][1] = j;
          st[nst][2] = k;
          nst++;
        }
  const double h = soft, h2 = soft * soft, hinv3 = 1.0 / (soft * soft * soft);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t key = 0; key < C; key++) {
    if (cell_start[key] == cell_start[key + 1]) continue;
    uint32_t ui, uj, uk;
    ct2o_morton_decode((uint32_t)key, &ui, &uj, &uk);
    const int ci = (int)ui, cj = (int)uj, ck = (int)uk;
    const int64_t c = ((int64_t)ci * M + cj) * M + ck; /* row-major cell */
    double L[220];
    if (Lgrid)
      for (int k = 0; k < nc; k++) L[k] = Lgrid[(int64_t)k * C + c];
    for (int64_t i = cell_start[key]; i < cell_start[key + 1]; i++) {
      double fo[3] = {0, 0, 0}, po = 0.0;
      if (Lgrid) {
        double t[3] = {center_offset(x[i], ci, mbits), center_offset(y[i], cj, mbits),
                       center_offset(z[i], ck, mbits)};
        double pw[3][12];
        for (int d = 0; d < 3; d++) {
          pw[d][0] = 1.0;
          for (int q = 1; q <= p; q++) pw[d][q] = pw[d][q - 1] * t[d] / q;
        }
        for (int k = 0; k < nc; k++) {
          const int *n = mi + 3 * k;
          const double mono = pw[0][n[0]] * pw[1][n[1]] * pw[2][n[2]];
          po -= L[k] * mono;
          int d = n[0] + n[1] + n[2];
          if (d < p) {
            fo[0] += L[ct2o_mi_index(n[0] + 1, n[1], n[2])] * mono;
            fo[1] += L[ct2o_mi_index(n[0], n[1] + 1, n[2])] * mono;
            fo[2] += L[ct2o_mi_index(n[0], n[1], n[2] + 1)] * mono;
          }
        }
        if (ffar) {
          ffar[3 * i + 0] = GM * fo[0];
          ffar[3 * i + 1] = GM * fo[1];
          ffar[3 * i + 2] = GM * fo[2];
        }
      }
      double fn[3] = {0, 0, 0}, pn = 0.0;
      for (int s = 0; s < nst; s++) {
        int nb[3] = {(ci + st[s][0] + M) % M, (cj + st[s][1] + M) % M, (ck + st[s][2] + M) % M};
        int64_t cn = ct2o_morton((uint32_t)nb[0], (uint32_t)nb[1], (uint32_t)nb[2]);
        for (int64_t j = cell_start[cn]; j < cell_start[cn + 1]; j++) {
          double d[3] = {(double)(int32_t)(x[i] - x[j]) * TWO_M32,
                         (double)(int32_t)(y[i] - y[j]) * TWO_M32,
                         (double)(int32_t)(z[i] - z[j]) * TWO_M32};
          double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
          double g, ph;
          if (kernel == CT2O_KERNEL_SPHERE) {
            if (r2 < h2) {
              g = hinv3;
              ph = 1.5 / h - 0.5 * r2 * hinv3;
            } else {
              double ri = 1.0 / sqrt(r2);
              g = ri * ri * ri;
              ph = ri;
            }
          } else {
            double ri = 1.0 / sqrt(r2 + h2);
            g = ri * ri * ri;
            ph = ri;
          }
          fn[0] -= d[0] * g;
          fn[1] -= d[1] * g;
          fn[2] -= d[2] * g;
          pn -= ph;
        }
      }
      if (fnear) {
        fnear[3 * i + 0] = GM * fn[0];
        fnear[3 * i + 1] = GM * fn[1];
        fnear[3 * i + 2] = GM * fn[2];
      }
      if (pot) pot[i] = GM * (po + pn);
    }
  }
  free(st);
  free(mi);
}

/* ------------------------------------------------------------------------ */
/* Velocity + rung update of kick_cell (kick.cpp:75-99), with the lane-index  */
/* defect fixed (f.force[d][i] -> this particle's force).  The velocity is    */
/* advanced in FP64 and stored as FP32.  ceil(log2(t0/dt)) is taken exactly   */
/* from the float's exponent bits.  Returns the max rung.                     */
/* ------------------------------------------------------------------------ */
static int ceil_log2_exact(float v) {
  /* exact ceil(log2(v)) for finite v > 0 */
  int e;
  float m = frexpf(v, &e); /* v = m * 2^e, m in [0.5,1) */
  return (m == 0.5f) ? e - 1 : e;
}

int ct2o_kick_update(float *vx, float *vy, float *vz, int8_t *rung,
                     const float *fx, const float *fy, const float *fz, int64_t n,
                     int ascending, int descending, int top, int first, int prung,
                     float t0, float eta, float max_dt, float scale, float hsoft) {
  int max_rung = 0;
  const float sgn = top ? 1.f : -1.f;
  for (int64_t i = 0; i < n; i++) {
    double v[3] = {vx[i], vy[i], vz[i]};
    const double f[3] = {fx[i], fy[i], fz[i]};
    if (ascending && !first) {
      const float dt = 0.5f * t0 / (float)(1 << prung);
      for (int d = 0; d < 3; d++) v[d] += (double)sgn * f[d] * (double)dt;
    }
    if (descending) {
      float g2 = fx[i] * fx[i];
      g2 = g2 + fy[i] * fy[i];
      g2 = g2 + fz[i] * fz[i];
      float dt = fminf(eta * sqrtf(scale * hsoft / sqrtf(g2)), t0);
      dt = fminf(max_dt, dt);
      int r = rung[i];
      int up = (ceil_log2_exact(t0 / dt) > prung) ? 1 : 0;
      int nr = prung + up;
      if (r - 1 > nr) nr = r - 1;
      rung[i] = (int8_t)nr;
      if (nr > max_rung) max_rung = nr;
      const float dth = 0.5f * t0 / (float)(1 << prung);
      for (int d = 0; d < 3; d++) v[d] += (double)sgn * f[d] * (double)dth;
    }
    vx[i] = (float)v[0];
    vy[i] = (float)v[1];
    vz[i] = (float)v[2];
  }
  return max_rung;
}

/* drift (drift.cpp:4-18): x += fixed32(v * dt/scale); the float displacement
 * is scaled by 2^32 and truncated toward zero, wrapping mod 2^32. */
void ct2o_drift(uint32_t *x, uint32_t *y, uint32_t *z, const float *vx,
                const float *vy, const float *vz, int64_t n, float dt, float scale) {
  const float lambda = dt / scale;
  for (int64_t i = 0; i < n; i++) {
    float d[3] = {vx[i] * lambda, vy[i] * lambda, vz[i] * lambda};
    uint32_t *p[3] = {x + i, y + i, z + i};
    for (int k = 0; k < 3; k++) {
      float s = d[k] * 4294967296.0f;
      int64_t q = (int64_t)s; /* truncation toward zero */
      *p[k] += (uint32_t)q;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* FP64 Ewald direct sum: the force truth.                                   */
/*   a_i = GM sum_j [ grad kernel(d) - grad 1/r(d) + grad erfc(a r)/r [r<rc] ]*/
/*       + GM sum_k w(k) (-2 pi k) Im(e^{2 pi i k.x_i} conj S(k)),            */
/*   w(k) = exp(-pi^2 k^2/alpha^2)/(pi k^2),  S(k) = sum_j e^{2 pi i k.x_j}.  */
/* d is the min-image displacement, so softening acts on the nearest image.  */
/* Sinks are given as fixed-point positions; sources likewise.               */
/* ------------------------------------------------------------------------ */
void ct2o_ewald_direct(const uint32_t *sx, const uint32_t *sy, const uint32_t *sz,
                       int64_t ns, const uint32_t *qx, const uint32_t *qy,
                       const uint32_t *qz, int64_t nq, int kernel, double soft,
                       double GM, double alpha, double rcut, int Kmax, double *fx,
                       double *fy, double *fz, double *pot) {
  const double h = soft, h2 = soft * soft;
  const double rc2 = rcut * rcut;
  const double spi = 1.7724538509055160273;
  /* real space */
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < ns; i++) {
    double f[3] = {0, 0, 0}, ph = 0.0;
    for (int64_t j = 0; j < nq; j++) {
      double d[3] = {(double)(int32_t)(sx[i] - qx[j]) * TWO_M32,
                     (double)(int32_t)(sy[i] - qy[j]) * TWO_M32,
                     (double)(int32_t)(sz[i] - qz[j]) * TWO_M32};
      double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 == 0.0) {
        /* self (or coincident) pair: zero force; potential self terms */
        ph += (kernel == CT2O_KERNEL_SPHERE ? 1.5 / h : 1.0 / h) - 2.0 * alpha / spi;
        continue;
      }
      double r = sqrt(r2), ri = 1.0 / r;
      double g, pk; /* kernel force factor and potential */
      if (kernel == CT2O_KERNEL_SPHERE) {
        if (r2 < h2) {
          g = 1.0 / (h * h2);
          pk = 1.5 / h - 0.5 * r2 / (h * h2);
        } else {
          g = ri * ri * ri;
          pk = ri;
        }
      } else {
        double s = 1.0 / sqrt(r2 + h2);
        g = s * s * s;
        pk = s;
      }
      /* kernel minus Newton */
      double gc = g - ri * ri * ri, pc = pk - ri;
      if (r2 < rc2) {
        double ec = erfc(alpha * r);
        gc += (ec + 2.0 * alpha * r / spi * exp(-alpha * alpha * r2)) * ri * ri * ri;
        pc += ec * ri;
      }
      f[0] -= d[0] * gc;
      f[1] -= d[1] * gc;
      f[2] -= d[2] * gc;
      ph += pc;
    }
    fx[i] = GM * f[0];
    fy[i] = GM * f[1];
    fz[i] = GM * f[2];
    if (pot) pot[i] = -GM * ph;
  }
  /* k space: half space of k (kx>0, or kx==0&&ky>0, or kx==ky==0&&kz>0) */
  const int K = Kmax, W = 2 * K + 1;
  int64_t nk = 0;
  for (int kx = 0; kx <= K; kx++)
    for (int ky = -K; ky <= K; ky++)
      for (int kz = -K; kz <= K; kz++) {
        if (kx == 0 && (ky < 0 || (ky == 0 && kz <= 0))) continue;
        if (kx * kx + ky * ky + kz * kz > K * K) continue;
        nk++;
      }
  int *kv = (int *)malloc(sizeof(int) * 3 * nk);
  double *Sre = (double *)calloc(nk, sizeof(double));
  double *Sim = (double *)calloc(nk, sizeof(double));
  nk = 0;
  for (int kx = 0; kx <= K; kx++)
    for (int ky = -K; ky <= K; ky++)
      for (int kz = -K; kz <= K; kz++) {
        if (kx == 0 && (ky < 0 || (ky == 0 && kz <= 0))) continue;
        if (kx * kx + ky * ky + kz * kz > K * K) continue;
        kv[3 * nk] = kx;
        kv[3 * nk + 1] = ky;
        kv[3 * nk + 2] = kz;
        nk++;
      }
  /* structure factor, parallel over source blocks with per-thread partials */
#pragma omp parallel
  {
    double *pr = (double *)calloc(nk, sizeof(double));
    double *pi = (double *)calloc(nk, sizeof(double));
    double *er = (double *)malloc(sizeof(double) * 3 * W);
    double *ei = (double *)malloc(sizeof(double) * 3 * W);
#pragma omp for schedule(static)
    for (int64_t j = 0; j < nq; j++) {
      const double xq[3] = {qx[j] * TWO_M32, qy[j] * TWO_M32, qz[j] * TWO_M32};
      for (int d = 0; d < 3; d++)
        for (int k = -K; k <= K; k++) {
          er[d * W + k + K] = cos(2 * M_PI * k * xq[d]);
          ei[d * W + k + K] = sin(2 * M_PI * k * xq[d]);
        }
      for (int64_t q = 0; q < nk; q++) {
        const int a = kv[3 * q] + K, b = W + kv[3 * q + 1] + K, c = 2 * W + kv[3 * q + 2] + K;
        double r1 = er[a] * er[b] - ei[a] * ei[b], i1 = er[a] * ei[b] + ei[a] * er[b];
        pr[q] += r1 * er[c] - i1 * ei[c];
        pi[q] += r1 * ei[c] + i1 * er[c];
      }
    }
#pragma omp critical
    for (int64_t q = 0; q < nk; q++) {
      Sre[q] += pr[q];
      Sim[q] += pi[q];
    }
    free(pr);
    free(pi);
    free(er);
    free(ei);
  }
#pragma omp parallel
  {
    double *er = (double *)malloc(sizeof(double) * 3 * W);
    double *ei = (double *)malloc(sizeof(double) * 3 * W);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < ns; i++) {
      const double xs[3] = {sx[i] * TWO_M32, sy[i] * TWO_M32, sz[i] * TWO_M32};
      for (int d = 0; d < 3; d++)
        for (int k = -K; k <= K; k++) {
          er[d * W + k + K] = cos(2 * M_PI * k * xs[d]);
          ei[d * W + k + K] = sin(2 * M_PI * k * xs[d]);
        }
      double f[3] = {0, 0, 0}, ph = 0.0;
      for (int64_t q = 0; q < nk; q++) {
        const int a = kv[3 * q] + K, b = W + kv[3 * q + 1] + K, c = 2 * W + kv[3 * q + 2] + K;
        double r1 = er[a] * er[b] - ei[a] * ei[b], i1 = er[a] * ei[b] + ei[a] * er[b];
        double cr = r1 * er[c] - i1 * ei[c], ci = r1 * ei[c] + i1 * er[c];
        double k2 = (double)kv[3 * q] * kv[3 * q] + (double)kv[3 * q + 1] * kv[3 * q + 1] +
                    (double)kv[3 * q + 2] * kv[3 * q + 2];
        double w = exp(-M_PI * M_PI * k2 / (alpha * alpha)) / (M_PI * k2);
        /* e^{ikx_i} conj(S) */
        double re = cr * Sre[q] + ci * Sim[q];
        double im = ci * Sre[q] - cr * Sim[q];
        /* half-space: each k stands for +k and -k -> factor 2 */
        for (int d = 0; d < 3; d++) f[d] += 2.0 * w * (-2.0 * M_PI * kv[3 * q + d]) * im;
        ph += 2.0 * w * re;
      }
      fx[i] += GM * f[0];
      fy[i] += GM * f[1];
      fz[i] += GM * f[2];
      if (pot) pot[i] -= GM * (ph - M_PI / (alpha * alpha) * (double)nq);
    }
    free(er);
    free(ei);
  }
  free(kv);
  free(Sre);
  free(Sim);
}
