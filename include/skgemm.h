/*
 * skgemm — C ABI of the B200 (sm_100a) FP64 Stream-K GEMM / SYRK / rotation
 * library for the dense subspace steps of a real-space DFT eigensolver
 * (S = Psi^T Psi, Hs = Psi^T (H Psi), Psi' = Psi Q).
 *
 * The entry points mirror the static C++ entry points of the reference
 * (shriramch/stream-k-gemm), which are host-side, blocking, FP64 and operate
 * on caller-owned buffers in the reference's packed layouts:
 *
 *   packed16 (band-tile, "A" of GEMM/SYRK):  X[(m/16)*K*16 + k*16 + m%16] = X(k, m)
 *   packed32 (band-tile, "B" of GEMM):       X[(n/32)*K*32 + k*32 + n%32] = X(k, n)
 *   grid-packed (rotation input):            A[(g/16)*nb*16 + b*16 + g%16]
 *   band-packed (rotation output):           D[(b/16)*Nd*16 + g*16 + b%16]
 *
 * Differences from the reference, all deliberate:
 *   - Remainders are computed. A packed16 buffer holds ceil(M/16) tiles and a
 *     packed32 buffer ceil(N/32) tiles (padding rows may hold any finite or
 *     non-finite value: they only feed output rows/columns that are not
 *     stored). The reference drops M%16 rows and N%32 columns of the GEMM
 *     (gemm_opt.cpp:318, :249) and its SYRK stores past C when M%16 != 0
 *     (syrk_crsp.cpp:152-165); here every stored element is in bounds.
 *   - SYRK applies alpha and beta exactly once: C = alpha*A^T*A + beta*C on the
 *     upper triangle. The reference scales only the last K chunk by alpha when
 *     K > 256 (sme_syrk.hpp:123-133); both agree for alpha = 1.
 *   - Sizes are int64_t (the reference uses int).
 *   - Every call returns a status (the reference has none).
 *
 * Host-pointer entry points are blocking: they stage inputs into device memory
 * (pinned or pageable host memory both work), run, copy the result back and
 * synchronise. The *_dev entry points take device pointers and a CUDA stream
 * (cudaStream_t passed as void*, NULL = legacy default stream) and are
 * asynchronous; device-side failures of an asynchronous call (a bounded wait
 * that ran out) are reported by skgemm_stream_status().
 */
#ifndef SKGEMM_H
#define SKGEMM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define SKGEMM_OK 0
#define SKGEMM_ERR_INVALID_ARG (-1)    /* bad shape, NULL pointer, bad option */
#define SKGEMM_ERR_OOM (-2)            /* device memory or HBM budget exhausted */
#define SKGEMM_ERR_CUDA (-3)           /* CUDA runtime / driver error */
#define SKGEMM_ERR_DEVICE_TIMEOUT (-4) /* a bounded device-side wait expired */
#define SKGEMM_ERR_NO_DEVICE (-5)      /* no sm_100 device visible */
#define SKGEMM_ERR_UNSUPPORTED (-6)    /* valid request this build cannot serve */

/* ------------------------------------------------------------- precision */
/* SKGEMM_PREC_NATIVE: FP64 DMMA tensor cores, Stream-K. The plain method and
 * the drop-in for the reference call.
 * SKGEMM_PREC_OZAKI_I8: Ozaki scheme II (Chinese-remainder reconstruction) —
 * operands scaled to integers, reduced modulo `slices` pairwise-coprime
 * moduli <= 256, INT8 x INT8 -> INT32 products on tcgen05 tensor cores,
 * FP64 reconstruction. */
#define SKGEMM_PREC_NATIVE 0
#define SKGEMM_PREC_OZAKI_I8 1
/* Per problem, whichever of native and Ozaki INT8 is faster: in batched
 * plans by the cost model, confirmed by timing when the plan tunes; in the
 * single-problem _opt entries and skgemm_dsubspace_packed_dev by the cost
 * model (slices_used_out = 0 reports that native ran). */
#define SKGEMM_PREC_AUTO 2
/* SKGEMM_PREC_OZAKI_BF16: the same Ozaki scheme II with the residues stored
 * as BF16 and kind::f16 products (FP32 accumulation over at most 1024
 * products, exact, summed in INT32): results identical to _OZAKI_I8 bit for
 * bit, at half its tensor throughput. Rotation: nb <= 1024. */
#define SKGEMM_PREC_OZAKI_BF16 3

typedef struct skgemm_options {
  int precision;        /* SKGEMM_PREC_* */
  int slices;           /* Ozaki: number of moduli; 0 = choose automatically */
  double err_bound_out; /* out: a-priori bound of the relative Frobenius error
                           contributed by the split (0 for native) */
  int slices_used_out;  /* out: moduli actually used */
} skgemm_options_t;

/* -------------------------------------------------- library / diagnostics */
const char* skgemm_version(void);
/* Message of the most recent failing call on this host thread. */
const char* skgemm_last_error(void);
/* Synchronise `stream` and report (then clear) device-side failures of the
 * asynchronous calls issued on it since the last check. */
int skgemm_stream_status(void* stream);
/* Measured FP64 tensor-core (DMMA m16n8k8) throughput of the current device,
 * TFLOP/s, from a register-resident peak loop; the analogue of the
 * reference's FMOPA peak probe (sme_peak_microbench.cpp:16-61). */
int skgemm_probe_fp64_peak(double* tflops_out);
/* Diagnostic of the failure path: enqueues on `stream` one CTA whose bounded
 * device wait (an mbarrier nothing arrives on) runs out after budget_ms
 * (0 < budget_ms <= 1000), the same mechanism every kernel wait uses (their
 * budgets are 4-8 s): the kernel records the timeout in the stream's device
 * error word and returns, the GPU context stays usable, and the next
 * skgemm_stream_status(stream) returns SKGEMM_ERR_DEVICE_TIMEOUT (and clears
 * the word). No counterpart in the reference. */
int skgemm_diag_expire_wait(double budget_ms, void* stream);
/* The same for the Stream-K fixup's flag wait (the wait of the CTA that
 * finishes a tile for the partial tiles of the CTAs after it; budget 4 s in
 * the kernels): one thread runs that wait, with budget_ms (0 < budget_ms <=
 * 1000), on a flag nothing sets; the timeout is recorded, the kernel returns
 * and the next skgemm_stream_status(stream) returns
 * SKGEMM_ERR_DEVICE_TIMEOUT. No counterpart in the reference. */
int skgemm_diag_expire_fixup_wait(double budget_ms, void* stream);
/* Per-kernel timing, off by default. skgemm_kernel_timing(1) clears the
 * record and starts recording: every launch of the FP64 Stream-K and Ozaki
 * kernels is then bracketed by two CUDA events on its own stream (a few
 * microseconds each, so time the workload itself with timing off).
 * skgemm_kernel_timing(0) stops recording. skgemm_kernel_timing_report
 * synchronises the recorded events, writes one line per kernel name,
 * "<name> <launches> <total_ms>\n", into buf (NUL-terminated), clears the
 * record and returns the number of lines (negative: a status). No
 * counterpart in the reference. */
int skgemm_kernel_timing(int enable);
int skgemm_kernel_timing_report(char* buf, int64_t len);
/* 1 when the process runs in debug fill mode (environment
 * SKGEMM_DEBUG_FILL=1 at the first call): every scratch buffer of the library
 * is filled with 0xFF bytes when allocated and again at the start of each
 * call that uses it, so that a read of scratch not written first shows in
 * the results (which are otherwise unchanged). Costs a fill per call. No
 * counterpart in the reference. */
int skgemm_debug_fill(void);
/* Measured INT8 tensor-core (tcgen05.mma kind::i8, 128x256x32) throughput of
 * the current device, TOP/s; the roofline denominator of the Ozaki path. */
int skgemm_probe_i8_peak(double* tops_out);

/* Exact INT8 GEMM on tcgen05 tensor cores: C[i*ldc + j] = sum_k A[i*lda + k] *
 * B[j*ldb + k] in int32 (both operands K-major int8; device pointers). The
 * engine of the Ozaki path, exposed for callers with integer data. Requires
 * |result| < 2^31 (guaranteed for K <= 131072). No counterpart in the
 * reference (which is FP64 only). */
int skgemm_igemm_s8_dev(int64_t M, int64_t N, int64_t K, const int8_t* A, int64_t lda,
                        const int8_t* B, int64_t ldb, int32_t* C, int64_t ldc, void* stream);

/* --------------------------------------------------------------- GEMM */
/* D = alpha * A * B + gamma (gamma added to every element).
 * A column-major M x K (A[i + k*M]), B row-major K x N (B[k*N + j]),
 * D row-major M x N (D[i*N + j]). Host pointers.
 * Replaces gemm<double>::compute_test (gemm_opt.cpp:376-392) and the Stream-K
 * check's gemm<double>::compute_test (gemm_crsp.cpp:369-385). */
int skgemm_dgemm(int64_t M, int64_t N, int64_t K, const double* A_colmajor,
                 const double* B_rowmajor, double* D_rowmajor, double alpha,
                 double gamma);

/* Same contract on packed operands: A packed16 (ceil(M/16) tiles), B packed32
 * (ceil(N/32) tiles), D row-major. Host pointers.
 * Replaces gemm<double>::compute_packed (gemm_opt.cpp:314-337) and
 * gemm<double>::compute_streamk_packed (gemm_crsp.cpp:316-337). */
int skgemm_dgemm_packed(int64_t M, int64_t N, int64_t K, const double* A_packed16,
                        const double* B_packed32, double* D_rowmajor, double alpha,
                        double gamma);

/* Device-pointer, stream-ordered forms of the two calls above.
 * ldd = row stride of D (>= N). */
int skgemm_dgemm_dev(int64_t M, int64_t N, int64_t K, const double* A_colmajor,
                     int64_t lda, const double* B_rowmajor, int64_t ldb, double* D,
                     int64_t ldd, double alpha, double gamma, void* stream);
int skgemm_dgemm_packed_dev(int64_t M, int64_t N, int64_t K, const double* A_packed16,
                            const double* B_packed32, double* D, int64_t ldd,
                            double alpha, double gamma, void* stream);
/* Allocation-free form of skgemm_dgemm_packed_dev, for callers that cannot
 * allocate device memory at call time: applications that reserve the device's
 * memory in their own pool up front, code whose device footprint must stay
 * fixed after start-up, or loops that cannot take the synchronisation of
 * cudaMalloc / cudaFree. No counterpart in the reference (whose drivers
 * allocate every buffer themselves).
 * Same contract as skgemm_dgemm_packed_dev (native FP64, 128 x 128 tiles);
 * the result agrees with it within FP64 rounding (relative Frobenius error
 * <= 1e-13), not bit for bit, since the regular entry may pick 64 x 64 tiles
 * and so a different Stream-K split. Its Stream-K scratch is a static device
 * array of 148 partial-tile slots (19.4 MB), held on each GPU where the
 * library's no-alloc code has been loaded until the process exits; a launch
 * that needs more slots (a device with more than 148 SMs) is rejected with
 * SKGEMM_ERR_INVALID_ARG. With CUDA's lazy module loading (the default) the
 * first call on a device loads that array and the kernel's code, taking
 * their device memory then: make that first call (an empty one, M = 0 or
 * N = 0, is enough) before reserving the rest of the device's memory. The
 * first call also looks up the array's device address (cudaGetSymbolAddress)
 * with that device current. Every call on a device shares its array, so calls
 * on one device are serialised by a per-device lock, and each call returns
 * only after its kernel has finished (it synchronises `stream`): it cannot be
 * issued while `stream` is being captured. A device-side wait that ran out is
 * reported as SKGEMM_ERR_DEVICE_TIMEOUT. */
int skgemm_dgemm_packed_dev_noalloc(int64_t M, int64_t N, int64_t K,
                                    const double* A_packed16, const double* B_packed32,
                                    double* D, int64_t ldd, double alpha, double gamma,
                                    void* stream);
/* Packed GEMM with a precision selector (native or Ozaki). */
int skgemm_dgemm_packed_dev_opt(int64_t M, int64_t N, int64_t K,
                                const double* A_packed16, const double* B_packed32,
                                double* D, int64_t ldd, double alpha, double gamma,
                                skgemm_options_t* opts, void* stream);

/* --------------------------------------------------------------- SYRK */
/* C = alpha * A^T * A + beta * C on the upper triangle (m1 <= m2) of the
 * column-major M x M matrix C (C[m1 + m2*M]); A packed16 K x M. The strict
 * lower triangle of C is not touched. beta == 0 does not read C.
 * Replaces sme_syrk<double>::compute (include/sme_syrk.hpp:137-149) and the
 * 8-ZA check sme_syrk<double>::compute (syrk_crsp.cpp:306-348). Host pointers. */
int skgemm_dsyrk_packed(int64_t K, int64_t M, const double* A_packed16,
                        double* C_colmajor, double alpha, double beta);
/* Device-pointer form; ldc = column stride of C (>= M). */
int skgemm_dsyrk_packed_dev(int64_t K, int64_t M, const double* A_packed16, double* C,
                            int64_t ldc, double alpha, double beta, void* stream);
int skgemm_dsyrk_packed_dev_opt(int64_t K, int64_t M, const double* A_packed16,
                                double* C, int64_t ldc, double alpha, double beta,
                                skgemm_options_t* opts, void* stream);

/* ------------------------------------------------------- subspace pair */
/* S = Psi^T Psi (upper triangle of the column-major nb x nb S, column stride
 * lds) and Hs = Psi^T (H Psi) (row-major nb x nb, row stride ldh) from one
 * band-packed Psi (packed16, K = Ng grid points x M = nb states) and a
 * 32-band-packed H Psi: the two products of one CheFSI subspace step, which
 * the reference computes with two calls on the same Psi
 * (sme_syrk<double>::compute, include/sme_syrk.hpp:137, then
 * gemm<double>::compute_packed, gemm_opt.cpp:314). Results equal those two
 * calls (alpha = 1, beta = gamma = 0). With the Ozaki precision Psi is
 * split once and its residues serve both products. */
int skgemm_dsubspace_packed_dev(int64_t K, int64_t M, const double* Psi_packed16,
                                const double* HPsi_packed32, double* S, int64_t lds,
                                double* Hs, int64_t ldh, skgemm_options_t* opts,
                                void* stream);

/* ----------------------------------------------------- subspace rotation */
/* D = A * Q: Psi' = Psi Q. A grid-packed Nd x nb, Q row-major nb x nb,
 * D band-packed Nd x nb. No scaling (the CheFSI rotation never needs it).
 * Host pointers. Nd % 16 == 0 and nb % 16 == 0 are required by the packed
 * layouts themselves (the reference further requires nb % 32 == 0,
 * sme_trp_3d.hpp:108-109).
 * Replaces sme_gemm_trp_3d<double>::compute (include/sme_trp_3d.hpp:194-215). */
int skgemm_drot(int64_t Nd, int64_t nb, const double* A_gridpacked,
                const double* Q_rowmajor, double* D_bandpacked);
/* Host-pointer forms of the three reference calls with a precision selector
 * (skgemm_options_t, NULL = native): the reference's blocking, host-memory
 * interface on the Ozaki path. Native runs the same pipelined copies as the
 * calls without `_opt`. Ozaki GEMM and SYRK upload their operands whole (the
 * split scales each row by its norm over all of K) and run one device call;
 * the Ozaki rotation keeps the row-chunked pipeline (each grid row is scaled
 * by its own norm, so chunks give the same bits). Results equal the `_dev_opt`
 * entries' bit for bit; AUTO is resolved once per call. Same references as
 * skgemm_dgemm_packed, skgemm_dsyrk_packed and skgemm_drot. */
int skgemm_dgemm_packed_opt(int64_t M, int64_t N, int64_t K, const double* A_packed16,
                            const double* B_packed32, double* D_rowmajor, double alpha,
                            double gamma, skgemm_options_t* opts);
int skgemm_dsyrk_packed_opt(int64_t K, int64_t M, const double* A_packed16,
                            double* C_colmajor, double alpha, double beta,
                            skgemm_options_t* opts);
int skgemm_drot_opt(int64_t Nd, int64_t nb, const double* A_gridpacked,
                    const double* Q_rowmajor, double* D_bandpacked, skgemm_options_t* opts);
int skgemm_drot_dev(int64_t Nd, int64_t nb, const double* A_gridpacked,
                    const double* Q_rowmajor, double* D_bandpacked, void* stream);
int skgemm_drot_dev_opt(int64_t Nd, int64_t nb, const double* A_gridpacked,
                        const double* Q_rowmajor, double* D_bandpacked,
                        skgemm_options_t* opts, void* stream);

/* The rotation on band-packed Psi, A_band[(b/16)*Nd*16 + g*16 + b%16] (the
 * layout SYRK and GEMM read), so a CheFSI step keeps one copy of Psi: the
 * band -> grid transposition that skgemm_drot_dev's input needs
 * (sme_pack<double>::band_to_grid_tile, include/sme_pack.hpp:232-249) is
 * folded into the operand loads. Output and options as skgemm_drot_dev /
 * skgemm_drot_dev_opt, and equal to them on the grid-packed copy, bit for
 * bit. Nd and nb multiples of 16. */
int skgemm_drot_band_dev(int64_t Nd, int64_t nb, const double* A_bandpacked,
                         const double* Q_rowmajor, double* D_bandpacked, void* stream);
int skgemm_drot_band_dev_opt(int64_t Nd, int64_t nb, const double* A_bandpacked,
                             const double* Q_rowmajor, double* D_bandpacked,
                             skgemm_options_t* opts, void* stream);

/* ------------------------------------------------------ layout converters */
/* Device-side packing, the B200 counterpart of gemm<double>::pack_A / pack_B
 * (gemm_opt.cpp:342-371): strided dense X(r, k) = X[r*sr + k*sk] ->
 * packed-T panels X[(r/T)*K*T + k*T + r%T], T in {16, 32}, zero padding for
 * r >= R. */
int skgemm_pack_dev(int64_t R, int64_t K, const double* X, int64_t sr, int64_t sk,
                    int T, double* X_packed, void* stream);
/* The inverse: packed-T panels -> strided dense X(r, k) = X[r*sr + k*sk] for
 * r < R (sme_pack<double>::unpack_c16 / unpack_r16 generalised,
 * include/sme_pack.hpp:109-156). */
int skgemm_unpack_dev(int64_t R, int64_t K, const double* X_packed, int T, double* X,
                      int64_t sr, int64_t sk, void* stream);
/* The reference's C converters linalg_pack_c16_f64 / linalg_pack_r16_f64 /
 * linalg_unpack_c16_f64 / linalg_unpack_r16_f64 (include/sme_pack.hpp:
 * 319-329) on device pointers: column-major [Nd, nb] (src[g + b*Nd]; the
 * row-major [nb, Nd] of the r16 names is the same bytes) <-> grid-packed
 * [Nd/16][nb][16]. Nd must be a multiple of 16 (the reference drops the
 * remainder rows; these return SKGEMM_ERR_INVALID_ARG). */
int skgemm_pack_c16_dev(int64_t Nd, int64_t nb, const double* src, double* dst, void* stream);
int skgemm_pack_r16_dev(int64_t Nd, int64_t nb, const double* src, double* dst, void* stream);
int skgemm_unpack_c16_dev(int64_t Nd, int64_t nb, const double* src, double* dst, void* stream);
int skgemm_unpack_r16_dev(int64_t Nd, int64_t nb, const double* src, double* dst, void* stream);
/* The same four converters under the reference's own names and signatures
 * (include/sme_pack.hpp:316-352: `void f(const int Nd, const int nb, const
 * double* src, double* dst)`), for callers linked against those names. Host
 * pointers; blocking (staged through device memory, converted on the GPU).
 * As in the reference, only the first 16 * floor(Nd/16) grid points are
 * converted (its g_tiles = Nd / 16) and the dense side keeps the column
 * stride Nd; unpacking leaves the remaining rows of dst unchanged. They
 * return nothing, like the reference: a refused call (negative sizes, a null
 * pointer, no usable device) leaves dst unchanged and its reason is read
 * with skgemm_last_error(), which is empty after a call that succeeded. */
void linalg_pack_c16_f64(const int Nd, const int nb, const double* src, double* dst);
void linalg_pack_r16_f64(const int Nd, const int nb, const double* src, double* dst);
void linalg_unpack_c16_f64(const int Nd, const int nb, const double* src, double* dst);
void linalg_unpack_r16_f64(const int Nd, const int nb, const double* src, double* dst);
/* Band-packed <-> grid-packed conversion of an Nd x nb block of states
 * (sme_pack<double>::band_to_grid_tile / grid_to_band_tile,
 * include/sme_pack.hpp:232-313). */
int skgemm_band_to_grid_dev(int64_t Nd, int64_t nb, const double* src_band,
                            double* dst_grid, void* stream);
int skgemm_grid_to_band_dev(int64_t Nd, int64_t nb, const double* src_grid,
                            double* dst_band, void* stream);

/* ----------------------------------------------- H Psi producer (stencil) */
/* The 6th-order finite-difference stencil of the kinetic part of H on
 * extended (halo-padded) band-packed Psi: calc_laplacian_extended_packed_16to32
 * (out_tile 32: the 32-band-packed B operand of skgemm_dgemm_packed, so that
 * Hs = Psi^T (H Psi) follows on the device) and _16to16 (out_tile 16),
 * include/stencil_extended_packed.hpp:47-181, :276-. Grid point
 * g = i + j*ni + k*ni*nj, extended index g_ex = (i+FDn) + (j+FDn)*ni_ex +
 * (k+FDn)*ni_ex*nj_ex with ni_ex = ni + 2*FDn (likewise nj_ex, nk_ex):
 *   out[g, b] = ext[g_ex, b]*(A_diag[g] + coef_0)
 *             + sum_{r=1..FDn} coef_x[r]*(ext[g_ex+r, b] + ext[g_ex-r, b])
 *             + the same along y (stride ni_ex) and z (stride ni_ex*nj_ex),
 * in the reference's SVE operation order (the results equal it bit for bit).
 * psi_ext16: [ceil(nb/16)][ni_ex*nj_ex*nk_ex][16]; A_diag: [ni*nj*nk];
 * coef_x/y/z: host arrays of FDn + 1 doubles (entry 0 unused); out:
 * [ceil(nb/T)][ni*nj*nk][T], T = out_tile, lanes b >= nb left untouched.
 * FDn must be 6 (the reference's kernels); other radii return
 * SKGEMM_ERR_UNSUPPORTED. psi_ext16, A_diag and out must be 16-byte aligned
 * (the arrays are read by TMA), and ni*nj*nk < 2^31. Asynchronous on `stream`;
 * a device-side wait that ran out is reported by skgemm_stream_status. */
int skgemm_stencil_ext_dev(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                           const double* psi_ext16, const double* A_diag,
                           const double* coef_x, const double* coef_y, const double* coef_z,
                           double coef_0, double* out, int out_tile, void* stream);
/* Single-rank periodic extension of band-packed Psi [ceil(nb/16)][ni*nj*nk][16]
 * into that extended array: the interior copy (copy_interior_to_extended_packed,
 * include/halo_packed.hpp:93-124) and the no-MPI periodic wrap (:350-393).
 * FDn <= ni, nj, nk. */
int skgemm_halo_periodic_dev(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                             const double* psi_local16, double* psi_ext16, void* stream);

/* ------------------------------------------ nonlocal projector (V_nloc) */
/* The nonlocal part of H (Hamiltonian::nloc_project_vectors_packed and
 * _16to16, include/nloc_packed_opt2.hpp:226-445) on the device. A handle
 * holds the projector set, the reference's Effective_potential_nloc:
 * projector p has nrow[p] grid rows (its entries of `index`, concatenated in
 * projector order, each < K), coefficients chi (column-major nrow x ncol,
 * concatenated), gamma (ncol values, concatenated), atom index atom[p] and a
 * coefficient block at column offsets[p] (offsets[P] = total columns;
 * projectors sharing a block — the periodic images of one atom — accumulate
 * into it and must have the same ncol). Host arrays, copied at creation. */
typedef struct skgemm_nloc* skgemm_nloc_t;
int skgemm_nloc_create(int64_t P, const uint32_t* nrow, const uint32_t* ncol,
                       const int32_t* atom, const uint32_t* offsets, const uint32_t* index,
                       const double* chi, const double* gamma, int64_t K, skgemm_nloc_t* out);
/* out += V_nloc psi: psi 16-band-packed [ceil(nb/16)][K][16]; out
 * 32-band-packed (out_tile 32: H Psi, the GEMM's B operand) or 16-band-packed
 * (out_tile 16). Device pointers; dv the grid volume element. Per projector:
 * gather, C += dv chi^T psi; gamma scaling on every change of atom index in
 * projector order; scatter-add of chi C. The single-rank all-reduce is the
 * identity. Results equal the reference's bit for bit. A handle's calls must
 * not run concurrently on two streams (they share its scratch). */
int skgemm_nloc_apply_dev(skgemm_nloc_t h, int64_t nb, double dv, const double* psi16,
                          double* out, int out_tile, void* stream);
void skgemm_nloc_destroy(skgemm_nloc_t h);

/* ------------------------------------------------------ batched (grouped) */
/* Many independent GEMM / SYRK / rotation problems of uneven sizes (k-points,
 * spin blocks) in ONE persistent Stream-K launch: the MAC-loop iterations of
 * all problems are concatenated and split evenly over the CTAs, so small and
 * large problems share the GPU without tail waves. No counterpart in the
 * reference, whose drivers call one problem at a time (the CheFSI loop calls
 * sme_syrk<double>::compute and gemm<double>::compute_packed per k-point).
 * Each item uses the contract of the single-problem _dev call it names. */
#define SKGEMM_OP_GEMM_PACKED 0 /* skgemm_dgemm_packed_dev: M, N, K, A packed16,
                                   B packed32, D row-major (ldd), alpha, beta=gamma */
#define SKGEMM_OP_SYRK_PACKED 1 /* skgemm_dsyrk_packed_dev: M (= N), K, A packed16,
                                   C column-major upper (ldd), alpha, beta */
#define SKGEMM_OP_ROT 2         /* skgemm_drot_dev: M = Nd, N = nb (K ignored),
                                   A grid-packed, B = Q row-major, D band-packed */

typedef struct skgemm_batch_item {
  int op; /* SKGEMM_OP_* */
  int64_t M, N, K;
  const double* A;
  const double* B; /* unused for SYRK */
  double* D;
  int64_t ldd; /* unused for ROT */
  double alpha;
  double beta; /* GEMM: gamma (scalar added); SYRK: beta; ROT: unused */
} skgemm_batch_item_t;

/* Plan options. Zero-initialised options = autotune everything, capture a
 * graph. Out fields report the chosen configuration. */
typedef struct skgemm_plan_options {
  int tile;      /* output tile: 128 (128x128), 64 (64x64) or 0 = autotune */
  int grid;      /* persistent CTAs (Stream-K split factor); 0 = all SMs x occupancy */
  int order;     /* problem order: 1 = as given, 2 = most work first, 0 = autotune */
  int no_tune;   /* 1: do not time candidates, pick by the cost model alone */
  int no_graph;  /* 1: plain stream launches instead of a CUDA graph */
  int precision; /* SKGEMM_PREC_NATIVE (default), _OZAKI_I8, _OZAKI_BF16 or _AUTO */
  int slices;    /* Ozaki moduli, 0 = automatic (accuracy target 1e-13) */
  int ozaki_problems_out; /* problems the plan runs on the Ozaki path */
  int tile_out, grid_out, order_out;
  int candidates_timed_out;
  double tuned_ms_out; /* device time of the chosen configuration (ms), 0 if untimed */
  double model_efficiency_out; /* useful MACs / issued MACs of the chosen tiles */
  int graph_kernels_out; /* kernel nodes in the captured graph (0 without a graph) */
} skgemm_plan_options_t;

typedef struct skgemm_plan* skgemm_plan_t;

/* Builds a plan for `n` items on the current device: validates every item,
 * chooses each problem's precision (SKGEMM_PREC_AUTO: native FP64 in the
 * grouped launch, or the Ozaki split with the moduli count the accuracy
 * target needs), builds the problem table and TMA descriptors in device
 * memory, chooses the tile shape, problem order and grid (autotuning times the candidate
 * configurations on the items' own buffers, so outputs hold unspecified
 * values afterwards, except SYRK outputs with beta != 0, which are restored),
 * and captures [flag reset, grouped launch] in a CUDA graph. Pointers in
 * `items` are bound into the plan. `stream` orders the tuning runs. Results of
 * tuning are cached per batch signature for the process. */
int skgemm_plan_create(const skgemm_batch_item_t* items, int n, skgemm_plan_options_t* opts,
                       void* stream, skgemm_plan_t* plan_out);
/* Enqueues the batch on `stream` (a graph launch, or plain launches). */
int skgemm_plan_run(skgemm_plan_t plan, void* stream);
/* Synchronises `stream` and reports (then clears) device-side failures of the
 * plan's launches. */
int skgemm_plan_status(skgemm_plan_t plan, void* stream);
/* The path each of the plan's `n` items runs on: prec_out[i] =
 * SKGEMM_PREC_NATIVE, _OZAKI_I8 or _OZAKI_BF16 (n must equal the item count). */
int skgemm_plan_precisions(skgemm_plan_t plan, int* prec_out, int n);
/* Releases the plan (synchronises the device first: its launches may still be
 * in flight). */
void skgemm_plan_destroy(skgemm_plan_t plan);

/* One-shot grouped launch of `n` items without tuning or graph (cost-model
 * configuration); asynchronous on `stream`, check with skgemm_stream_status. */
int skgemm_batch_dev(const skgemm_batch_item_t* items, int n, void* stream);

/* Host-only view of a grouped schedule (no device needed): for tile 128 or
 * 64, problem order `order` (1 or 2) and `grid` CTAs, writes the problem
 * order (perm_out[n]), the first MAC-loop iteration of each problem in the
 * concatenated space (iter_begin_out[n+1], in perm order), and the useful /
 * issued MAC ratio. Items with a zero dimension get zero iterations. */
int skgemm_batch_schedule(const skgemm_batch_item_t* items, int n, int tile, int order,
                          int* perm_out, int64_t* iter_begin_out, double* efficiency_out);
/* The autotuner's choices persisted across processes: plans tuned in this
 * process (per batch signature: device name, plan options, each item's op
 * and shape) are written by skgemm_tune_cache_save as a JSON file (one entry
 * per line: key, tile, order, grid, per-item Ozaki flags); a later process
 * on the same device type loads them with skgemm_tune_cache_load and its
 * skgemm_plan_create skips the timing runs of those batches (an entry is
 * used only where it matches the plan's items and candidates). Both return
 * the number of entries written / read, or a negative status (unreadable or
 * malformed file: nothing is loaded). skgemm_tune_cache_clear forgets them.
 * The reference has compile-time tiles only (gemm_opt.cpp:37-47); no
 * counterpart. */
int skgemm_tune_cache_save(const char* path);
int skgemm_tune_cache_load(const char* path);
int skgemm_tune_cache_clear(void);

/* ------------------------------------------------------------- serving */
/* A serving engine for subspace requests: each request is the sequence
 * S = Psi^T Psi (SYRK), Hs = Psi^T (H Psi) (GEMM), Psi' = Psi Q (rotation) on
 * its own Psi, H Psi and Q, which stay resident on the device across the
 * three steps. Requests are admitted in arrival order when a contiguous block
 * of the HBM budget is free for all their buffers; admitted requests overlap
 * on the device (native FP64: continuous batching of the ready steps of all
 * admitted requests into grouped persistent launches; Ozaki: concurrent
 * request streams). Inputs are synthetic and seeded: Psi and H Psi entries
 * N(0,1)/sqrt(Ng), Q entries uniform[-1,1], each a pure function of
 * (seed, index), so a request's result does not depend on what else runs.
 * No counterpart in the reference. */
typedef struct skgemm_serve_request {
  int64_t Ng;       /* grid points, multiple of 16 */
  int64_t nb;       /* states, multiple of 16 (<= 2048 for Ozaki) */
  double arrival_s; /* arrival time, seconds after the start of the run */
  uint64_t seed;
  /* Optional host copies (NULL = not kept): results S (nb*nb column-major,
   * upper triangle valid), Hs (nb*nb row-major), Psi' (band-packed Ng x nb),
   * and the inputs Psi (band-packed), H Psi (packed32), Q (row-major). */
  double* S_out;
  double* Hs_out;
  double* Psi_out;
  double* Psi_in_out;
  double* HPsi_in_out;
  double* Q_in_out;
  double admit_s; /* out: admission time */
  double done_s;  /* out: completion time (device clock, CUDA events) */
} skgemm_serve_request_t;

#define SKGEMM_SERVE_FIFO 0
#define SKGEMM_SERVE_SMALLEST 1
/* Highest response ratio next: the waiting request with the largest wait per
 * unit of its own work (ties: least work). A large request ages in proportion
 * to its size, so it cannot starve behind a stream of small ones. */
#define SKGEMM_SERVE_RATIO 2

typedef struct skgemm_serve_options {
  int precision;           /* SKGEMM_PREC_NATIVE or SKGEMM_PREC_OZAKI_I8 */
  int slices;              /* Ozaki moduli, 0 = automatic */
  double hbm_budget_bytes; /* request data + engine scratch; 0 = 150e9 */
  int max_inflight;        /* native: admitted requests at once (0 = 64) */
  int ozaki_streams;       /* Ozaki: concurrent request streams (0 = 2) */
  double max_batch_tflop;  /* native: work cap of one grouped launch (0 = 2 TFLOP) */
  int realtime;            /* 1: release requests at arrival_s (wall clock); 0: all at 0 */
  int policy;              /* admission order among waiting requests:
                              SKGEMM_SERVE_FIFO (0, arrival order),
                              SKGEMM_SERVE_SMALLEST (least work first, aged) or
                              SKGEMM_SERVE_RATIO (largest wait / work first) */
  double aging_s;          /* SMALLEST: a request's work counts / (1 + wait / aging_s),
                              so a long wait always ends (0 = 1 s, which on a B200 at
                              ~93% load gave a lower p50 and p99 than arrival order) */
  /* skgemm_serve_simulate only: throughput model (0 = defaults) */
  double sim_native_tflops, sim_ozaki_tflops, sim_gen_gbs;
  /* out */
  double makespan_s;          /* last completion */
  double flop;                /* S: nb^2 Ng, Hs: 2 nb^2 Ng, rotation: 2 Ng nb^2 */
  int batches;                /* grouped launches (native) */
  double mean_batch_problems; /* problems per grouped launch */
  double peak_admitted_bytes; /* peak request data held */
  double scratch_bytes;       /* engine scratch counted against the budget */
} skgemm_serve_options_t;

/* Runs `n` requests to completion on the current device (blocking). */
int skgemm_serve_run(skgemm_serve_request_t* reqs, int n, skgemm_serve_options_t* opts);
/* Same scheduler on a virtual clock with a throughput model instead of the
 * GPU (no device needed): admission, batching and latency accounting. */
int skgemm_serve_simulate(skgemm_serve_request_t* reqs, int n, skgemm_serve_options_t* opts);

/* Releases the per-stream scratch the library keeps for `stream` (Stream-K
 * partial slots, Ozaki residue buffers); synchronises the stream first. */
int skgemm_stream_release(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SKGEMM_H */
