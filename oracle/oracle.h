/*
 * CPU oracle for the FP64 GEMM / SYRK / rotation path — TEST INFRASTRUCTURE.
 *
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg use
 * this library, and only as a checker or as the timed CPU baseline; the
 * product (libskgemm.so) never links or calls it.
 *
 * Two families:
 *  - "naive": restatements of the reference's own portable reference loops,
 *    same loop order and accumulation order, for the CPU baseline and for
 *    parity with the reference's known-answer tests;
 *  - "dot2": every dot product accumulated in double-double (Ogita, Rump and
 *    Oishi, "Accurate sum and dot product", SIAM J. Sci. Comput. 26(6), 2005,
 *    algorithm Dot2: TwoProduct via fma + TwoSum), then rounded once. This is
 *    the accurate oracle the 1e-13 relative-Frobenius gate is measured
 *    against; its own error is about u + K*u^2 relative.
 */
#ifndef SKGEMM_ORACLE_H
#define SKGEMM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* gemm_opt.cpp:467-475 (= gemm_crsp.cpp:475-483): A column-major M x K,
 * B row-major K x N, D row-major, D[i*N+j] = alpha*sum_k A[i+k*M]*B[k*N+j] + gamma.
 * nthreads > 1 parallelises the outer i loop (a restatement, not the
 * reference's serial loop); the per-element accumulation order is unchanged. */
void oracle_gemm_naive(int64_t M, int64_t N, int64_t K, const double* A, const double* B,
                       double* D, double alpha, double gamma, int nthreads);

/* syrk_crsp.cpp:355-373: A packed16 [ceil(M/16)][K][16], C column-major,
 * upper triangle C[m1 + m2*M] = alpha*sum + beta*C[m1 + m2*M], m1 <= m2. */
void oracle_syrk_naive(int64_t K, int64_t M, const double* A_packed, double* C, double alpha,
                       double beta, int nthreads);

/* trp_3d_test.cpp:55-66: A grid-packed [Nd/16][nb][16], Q row-major nb x nb,
 * D band-packed [nb/16][Nd][16], D(g,b') = sum_b A(g,b) Q[b*nb+b']. */
void oracle_rot_naive(int64_t Nd, int64_t nb, const double* A_grid, const double* Q,
                      double* D_band, int nthreads);

/* Accurate general product on strided dense operands:
 *   R(i,j) = alpha * sum_k X[i*sxi + k*sxk] * Y[k*syk + j*syj] + gamma
 * written to out[i*soi + j*soj], for i < M, j < N. Every sum is a Dot2
 * double-double accumulation; alpha*sum + gamma is formed in double-double
 * and rounded once. */
void oracle_dot2_gemm(int64_t M, int64_t N, int64_t K, const double* X, int64_t sxi,
                      int64_t sxk, const double* Y, int64_t syk, int64_t syj, double* out,
                      int64_t soi, int64_t soj, double alpha, double gamma, int nthreads);

/* Same arithmetic for a list of (i, j) output positions only (large problems
 * checked on a sample of entries). out[t] receives element (ii[t], jj[t]). */
void oracle_dot2_sampled(int64_t npos, const int64_t* ii, const int64_t* jj, int64_t K,
                         const double* X, int64_t sxi, int64_t sxk, const double* Y,
                         int64_t syk, int64_t syj, double* out, double alpha, double gamma,
                         int nthreads);

/* Layout maps of the reference, applied on the CPU. */
/* gemm_opt.cpp:342-371 packing, extended to ceil(R/T) panels with zero padding:
 * Xp[(r/T)*K*T + k*T + r%T] = X[r*sr + k*sk]. */
void oracle_pack(int64_t R, int64_t K, const double* X, int64_t sr, int64_t sk, int T,
                 double* Xp);

/* syrk_crsp.cpp:379-395 init_A_packed: srand(seed); entries rand()%100/100
 * in [tm][k][ml] order, zero for padding rows (host C library rand()). */
void oracle_init_A_packed_rand(int64_t K, int64_t M, double* A_packed, int seed);

/* H Psi stencil on extended (halo-padded) band-packed Psi, restating
 * calc_laplacian_extended_packed_16to32 / _16to16
 * (include/stencil_extended_packed.hpp:47-181, :276-): grid point
 * g = i + j*ni + k*ni*nj, g_ex its extended index (offset FDn per axis),
 * per band b < nb:
 *   res = ext[g_ex] * (A[g] + c0);
 *   for r = 1..FDn: res = fma(ext[g_ex+r] + ext[g_ex-r], cx[r], res),
 *                   then the same along y (stride ni_ex) and z (ni_ex*nj_ex),
 * the SVE kernels' operation order (x, y, z for each r; svmla is fused).
 * ext: [ceil(nb/16)][K_ex][16]; out: [ceil(nb/T)][K][T], T = out_tile (16
 * or 32); lanes b >= nb of out are left untouched. */
void oracle_stencil_ext(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                        const double* ext, const double* A, const double* cx, const double* cy,
                        const double* cz, double c0, double* out, int out_tile, int nthreads);

/* Single-rank periodic halo: copy_interior_to_extended_packed
 * (include/halo_packed.hpp:93-124) plus the periodic wrap of the no-MPI path
 * (:350-393): ext[(t*K_ex + g_ex)*16 + l] = local[(t*K + g)*16 + l] with
 * g = ((i_ex - FDn) mod ni) + ((j_ex - FDn) mod nj)*ni + ((k_ex - FDn) mod nk)*ni*nj. */
void oracle_halo_periodic(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                          const double* local, double* ext);

/* Nonlocal projector, restating Hamiltonian::nloc_project_vectors_packed /
 * _16to16 (include/nloc_packed_opt2.hpp:226-445, the sequential form) in its
 * loop and rounding order, without fused multiply-adds: per projector p (rows
 * index[row_off[p] ..], coefficients chi col-major nrow x ncol at chi_off[p],
 * block at offsets[p]): C_p[j + b*ncol] = C_p + dv * sum_r chi[r + j*nrow] *
 * psi(index[r], b) (gemm_aTb, :143-176); then, on every change of atom index
 * in projector order, C_p *= gamma_p per column; then temp = chi * C_p (gemm_ab,
 * :181-224) scatter-added into out[(b/T)*K + index[r]][b%T] (:85-135).
 * Rounding of the reference as compiled (C++ contracts a*b + c): forward
 * sums unfused, the block update fma(dv, sum, C), backward sums fused. */
void oracle_nloc_project(int64_t P, const uint32_t* nrow, const uint32_t* ncol,
                         const int32_t* atom, const uint32_t* offsets, const uint32_t* index,
                         const int64_t* row_off, const double* chi, const int64_t* chi_off,
                         const double* gamma, const int64_t* gam_off, int64_t nb, int64_t K,
                         double dv, const double* psi16, double* out, int out_tile);

#ifdef __cplusplus
}
#endif

#endif
