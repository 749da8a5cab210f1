// Reference gemm_crsp.cpp (K-split "Stream-K" FP64 GEMM with a P-way partial
// reduction) compiled unchanged on the host with the SME emulation shim.
// Exports compute_test (gemm_crsp.cpp:369), compute_streamk_packed (:316) and
// the file's four known-answer tests (test_gemm :437, cases :555-565).
#include "ref_prelude.hpp"
#define main skgemm_ref_gemm_crsp_main
#include "gemm_crsp.cpp"
#undef main

SKREF_EXPORT void ref_gemm_crsp_compute_test(int M, int N, int K, const double* A,
                                             const double* B, double* D,
                                             double alpha, double gamma) {
  gemm<double>::compute_test(M, N, K, A, B, D, alpha, gamma);
}
SKREF_EXPORT void ref_gemm_crsp_compute_streamk_packed(int M, int N, int K,
                                                       const double* Ap,
                                                       const double* Bp, double* D,
                                                       double alpha, double gamma) {
  gemm<double>::compute_streamk_packed(M, N, K, Ap, Bp, D, alpha, gamma);
}
SKREF_EXPORT int ref_gemm_crsp_selftest() {
  int passed = 0;
  passed += test_gemm<double>(32, 64, 128, 1.0, 0.0);
  passed += test_gemm<double>(32, 64, 4096, 1.0, 0.0);
  passed += test_gemm<double>(32, 64, 4096, 2.0, 0.5);
  passed += test_gemm<double>(64, 128, 2048, 1.0, 0.0);
  return passed;
}
