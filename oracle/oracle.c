/*
 * CPU oracle for the FP64 GEMM / SYRK / rotation path — TEST INFRASTRUCTURE
 * (see oracle.h). Parity of these loops with the reference is pinned by
 * tests/test_oracle.py against the reference's own kernels built from its
 * sources (oracle/_ref) and against the committed golden vectors.
 */
#include "oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>

static int clamp_threads(int n) { return n < 1 ? 1 : n; }

/* ------------------------------------------------------------ naive loops */
void oracle_gemm_naive(int64_t M, int64_t N, int64_t K, const double* A, const double* B,
                       double* D, double alpha, double gamma, int nthreads) {
  /* gemm_opt.cpp:467-475: i outer, j, then k; sum += A[i + k*M] * B[k*N + j]. */
#pragma omp parallel for schedule(static) num_threads(clamp_threads(nthreads))
  for (int64_t i = 0; i < M; ++i) {
    for (int64_t j = 0; j < N; ++j) {
      double sum = 0.0;
      for (int64_t k = 0; k < K; ++k) sum += A[i + k * M] * B[k * N + j];
      D[i * N + j] = alpha * sum + gamma;
    }
  }
}

void oracle_syrk_naive(int64_t K, int64_t M, const double* A, double* C, double alpha,
                       double beta, int nthreads) {
  /* syrk_crsp.cpp:360-372: m1 outer, m2 >= m1, k inner. */
#pragma omp parallel for schedule(dynamic, 1) num_threads(clamp_threads(nthreads))
  for (int64_t m1 = 0; m1 < M; ++m1) {
    for (int64_t m2 = m1; m2 < M; ++m2) {
      double sum = 0.0;
      const double* a1 = A + (m1 / 16) * K * 16 + m1 % 16;
      const double* a2 = A + (m2 / 16) * K * 16 + m2 % 16;
      for (int64_t k = 0; k < K; ++k) sum += a1[k * 16] * a2[k * 16];
      C[m1 + m2 * M] = alpha * sum + beta * C[m1 + m2 * M];
    }
  }
}

void oracle_rot_naive(int64_t Nd, int64_t nb, const double* A, const double* Q, double* D,
                      int nthreads) {
  /* trp_3d_test.cpp:57-65: g outer, bp, then b; grid_packed_get / band_packed_set
   * index maps of trp_3d_test.cpp:31-49. */
#pragma omp parallel for schedule(static) num_threads(clamp_threads(nthreads))
  for (int64_t g = 0; g < Nd; ++g) {
    for (int64_t bp = 0; bp < nb; ++bp) {
      double sum = 0.0;
      const double* arow = A + (g / 16) * nb * 16 + g % 16;
      for (int64_t b = 0; b < nb; ++b) sum += arow[b * 16] * Q[b * nb + bp];
      D[(bp / 16) * Nd * 16 + g * 16 + bp % 16] = sum;
    }
  }
}

/* ------------------------------------------------------- double-double */
/* TwoSum (Knuth): s + e = a + b exactly. */
static inline void two_sum(double a, double b, double* s, double* e) {
  double x = a + b;
  double z = x - a;
  *e = (a - (x - z)) + (b - z);
  *s = x;
}

/* TwoProduct via fma: p + e = a * b exactly. */
static inline void two_prod(double a, double b, double* p, double* e) {
  double x = a * b;
  *e = fma(a, b, -x);
  *p = x;
}

/* Dot2 over K terms, then alpha * (s + c) + gamma in double-double. */
static double dot2_elem(int64_t K, const double* x, int64_t sx, const double* y, int64_t sy,
                        double alpha, double gamma) {
  double s = 0.0, c = 0.0;
  for (int64_t k = 0; k < K; ++k) {
    double p, ep, es;
    two_prod(x[k * sx], y[k * sy], &p, &ep);
    two_sum(s, p, &s, &es);
    c += es + ep;
  }
  /* Normalise (s, c), multiply by alpha, add gamma. */
  double hi, lo;
  two_sum(s, c, &hi, &lo);
  double ph, pl;
  two_prod(alpha, hi, &ph, &pl);
  pl += alpha * lo;
  double sh, sl;
  two_sum(ph, gamma, &sh, &sl);
  sl += pl;
  return sh + sl;
}

void oracle_dot2_gemm(int64_t M, int64_t N, int64_t K, const double* X, int64_t sxi,
                      int64_t sxk, const double* Y, int64_t syk, int64_t syj, double* out,
                      int64_t soi, int64_t soj, double alpha, double gamma, int nthreads) {
#pragma omp parallel for collapse(2) schedule(static) num_threads(clamp_threads(nthreads))
  for (int64_t i = 0; i < M; ++i)
    for (int64_t j = 0; j < N; ++j)
      out[i * soi + j * soj] = dot2_elem(K, X + i * sxi, sxk, Y + j * syj, syk, alpha, gamma);
}

void oracle_dot2_sampled(int64_t npos, const int64_t* ii, const int64_t* jj, int64_t K,
                         const double* X, int64_t sxi, int64_t sxk, const double* Y,
                         int64_t syk, int64_t syj, double* out, double alpha, double gamma,
                         int nthreads) {
#pragma omp parallel for schedule(dynamic, 4) num_threads(clamp_threads(nthreads))
  for (int64_t t = 0; t < npos; ++t)
    out[t] = dot2_elem(K, X + ii[t] * sxi, sxk, Y + jj[t] * syj, syk, alpha, gamma);
}

/* ---------------------------------------------------------- layouts */
void oracle_pack(int64_t R, int64_t K, const double* X, int64_t sr, int64_t sk, int T,
                 double* Xp) {
  int64_t tiles = (R + T - 1) / T;
  for (int64_t t = 0; t < tiles; ++t)
    for (int64_t k = 0; k < K; ++k)
      for (int64_t i = 0; i < T; ++i) {
        int64_t r = t * T + i;
        Xp[(t * K + k) * T + i] = r < R ? X[r * sr + k * sk] : 0.0;
      }
}

void oracle_init_A_packed_rand(int64_t K, int64_t M, double* A, int seed) {
  /* syrk_crsp.cpp:381-394: one rand() per live entry, in [tm][k][ml] order. */
  srand(seed);
  int64_t tiles = (M + 15) / 16;
  for (int64_t tm = 0; tm < tiles; ++tm)
    for (int64_t k = 0; k < K; ++k)
      for (int ml = 0; ml < 16; ++ml) {
        int64_t m = tm * 16 + ml;
        A[(tm * K + k) * 16 + ml] = m < M ? (double)(rand() % 100) / 100.0 : 0.0;
      }
}

/* ------------------------------------------------------------- stencil */
void oracle_stencil_ext(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                        const double* ext, const double* A, const double* cx, const double* cy,
                        const double* cz, double c0, double* out, int out_tile, int nthreads) {
  const int64_t K = ni * nj * nk;
  const int64_t ni_ex = ni + 2 * FDn, nj_ex = nj + 2 * FDn, nk_ex = nk + 2 * FDn;
  const int64_t K_ex = ni_ex * nj_ex * nk_ex;
  const int64_t sj = ni_ex, sk = ni_ex * nj_ex;
#pragma omp parallel for schedule(static) num_threads(clamp_threads(nthreads))
  for (int64_t g = 0; g < K; ++g) {
    const int64_t i = g % ni, j = (g / ni) % nj, k = g / (ni * nj);
    const int64_t gx = (i + FDn) + (j + FDn) * sj + (k + FDn) * sk;
    const double a = A[g] + c0;
    for (int64_t b = 0; b < nb; ++b) {
      const double* s = ext + (b / 16) * K_ex * 16 + b % 16;
      double res = s[gx * 16] * a;
      for (int r = 1; r <= FDn; ++r) {
        res = fma(s[(gx + r) * 16] + s[(gx - r) * 16], cx[r], res);
        res = fma(s[(gx + r * sj) * 16] + s[(gx - r * sj) * 16], cy[r], res);
        res = fma(s[(gx + r * sk) * 16] + s[(gx - r * sk) * 16], cz[r], res);
      }
      out[((b / out_tile) * K + g) * out_tile + b % out_tile] = res;
    }
  }
}

static inline int64_t wrap(int64_t x, int64_t n) { return ((x % n) + n) % n; }

void oracle_halo_periodic(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                          const double* local, double* ext) {
  const int64_t K = ni * nj * nk;
  const int64_t ni_ex = ni + 2 * FDn, nj_ex = nj + 2 * FDn, nk_ex = nk + 2 * FDn;
  const int64_t K_ex = ni_ex * nj_ex * nk_ex, tiles = (nb + 15) / 16;
  for (int64_t t = 0; t < tiles; ++t)
    for (int64_t gx = 0; gx < K_ex; ++gx) {
      const int64_t ix = gx % ni_ex, jx = (gx / ni_ex) % nj_ex, kx = gx / (ni_ex * nj_ex);
      const int64_t g = wrap(ix - FDn, ni) + wrap(jx - FDn, nj) * ni + wrap(kx - FDn, nk) * ni * nj;
      for (int l = 0; l < 16; ++l) ext[(t * K_ex + gx) * 16 + l] = local[(t * K + g) * 16 + l];
    }
}

/* ----------------------------------------------------------- projector */
/* Rounding as the reference compiles (g++ contracts a*b + c in C++ by
 * default; determined against the in-place build): the forward dot products
 * unfused, the block update fma(dv, sum, C), the backward products fused. */
void oracle_nloc_project(int64_t P, const uint32_t* nrow, const uint32_t* ncol,
                         const int32_t* atom, const uint32_t* offsets, const uint32_t* index,
                         const int64_t* row_off, const double* chi, const int64_t* chi_off,
                         const double* gamma, const int64_t* gam_off, int64_t nb, int64_t K,
                         double dv, const double* psi16, double* out, int out_tile) {
  if (P <= 0 || offsets[P] == 0) return;
  double* C = (double*)calloc((size_t)offsets[P] * nb, sizeof(double));
  for (int64_t p = 0; p < P; ++p) { /* gather + C += dv chi^T filtered */
    const int64_t nr = nrow[p], nc = ncol[p];
    if (nr == 0 || nc == 0) continue;
    const uint32_t* idx = index + row_off[p];
    const double* X = chi + chi_off[p];
    double* Cb = C + (int64_t)offsets[p] * nb;
    for (int64_t n = 0; n < nb; ++n)
      for (int64_t m = 0; m < nc; ++m) {
        double sum = 0.0;
        for (int64_t k = 0; k < nr; ++k)
          sum = sum + X[k + m * nr] * psi16[((n / 16) * K + idx[k]) * 16 + n % 16];
        Cb[m + n * nc] = fma(dv, sum, 1.0 * Cb[m + n * nc]);
      }
  }
  int32_t a = atom[0] - 1; /* gamma on each change of atom index */
  for (int64_t p = 0; p < P; ++p) {
    if (a == atom[p]) continue;
    a = atom[p];
    double* Cb = C + (int64_t)offsets[p] * nb;
    const double* gm = gamma + gam_off[p];
    for (int64_t b = 0; b < nb; ++b)
      for (int64_t j = 0; j < ncol[p]; ++j) Cb[j + b * ncol[p]] *= gm[j];
  }
  for (int64_t p = 0; p < P; ++p) { /* temp = chi C, scatter-add */
    const int64_t nr = nrow[p], nc = ncol[p];
    if (nr == 0 || nc == 0) continue;
    const uint32_t* idx = index + row_off[p];
    const double* X = chi + chi_off[p];
    const double* Cb = C + (int64_t)offsets[p] * nb;
    double* t = (double*)malloc((size_t)nr * nb * sizeof(double));
    for (int64_t n = 0; n < nb; ++n) {
      for (int64_t m = 0; m < nr; ++m) t[m + n * nr] = 0.0;
      for (int64_t k = 0; k < nc; ++k) {
        const double bv = 1.0 * Cb[k + n * nc];
        for (int64_t m = 0; m < nr; ++m) t[m + n * nr] = fma(X[m + k * nr], bv, t[m + n * nr]);
      }
    }
    for (int64_t b = 0; b < nb; ++b)
      for (int64_t r = 0; r < nr; ++r)
        out[((b / out_tile) * K + idx[r]) * out_tile + b % out_tile] += t[r + b * nr];
    free(t);
  }
  free(C);
}
