// Reference gemm_opt.cpp (M-tile data-parallel FP64 GEMM, D = alpha*A*B + gamma)
// compiled unchanged on the host with the SME emulation shim.
// Exports: gemm<double>::compute_test (gemm_opt.cpp:376), compute_packed
// (gemm_opt.cpp:314), pack_A/pack_B (gemm_opt.cpp:342,359) and the file's own
// four known-answer tests (test_gemm, gemm_opt.cpp:432, cases at :517-520).
#include "ref_prelude.hpp"
#define main skgemm_ref_gemm_opt_main
#include "gemm_opt.cpp"
#undef main

SKREF_EXPORT void ref_gemm_opt_compute_test(int M, int N, int K, const double* A,
                                            const double* B, double* D,
                                            double alpha, double gamma) {
  gemm<double>::compute_test(M, N, K, A, B, D, alpha, gamma);
}
SKREF_EXPORT void ref_gemm_opt_compute_packed(int M, int N, int K, const double* Ap,
                                              const double* Bp, double* D,
                                              double alpha, double gamma) {
  gemm<double>::compute_packed(M, N, K, Ap, Bp, D, alpha, gamma);
}
SKREF_EXPORT void ref_gemm_opt_pack_A(int M, int K, const double* A, double* Ap) {
  gemm<double>::pack_A(M, K, A, Ap);
}
SKREF_EXPORT void ref_gemm_opt_pack_B(int N, int K, const double* B, double* Bp) {
  gemm<double>::pack_B(N, K, B, Bp);
}
SKREF_EXPORT int ref_gemm_opt_selftest() {
  int passed = 0;
  passed += test_gemm<double>(32, 64, 128, 1.0, 0.0);
  passed += test_gemm<double>(32, 64, 4096, 1.0, 0.0);
  passed += test_gemm<double>(32, 64, 4096, 2.0, 0.5);
  passed += test_gemm<double>(64, 128, 2048, 1.0, 0.0);
  return passed;
}
