// Reference syrk_crsp.cpp (8-ZA FP64 SYRK with 3-D blocking, plus its naive
// syrk_reference and seeded init_A_packed) compiled unchanged with the SME
// emulation shim. Exports compute (syrk_crsp.cpp:306), syrk_reference (:355),
// init_A_packed (:379, srand/rand of the host C library) and the file's own
// test driver (main, :425-528, run with no arguments = the five test cases).
#include "ref_prelude.hpp"
#define main skgemm_ref_syrk_crsp_main
#include "syrk_crsp.cpp"
#undef main

SKREF_EXPORT void ref_syrk_crsp_compute(int K, int M, const double* Ap, double* C,
                                        double alpha, double beta) {
  sme_syrk<double>::compute(K, M, Ap, C, alpha, beta);
}
SKREF_EXPORT void ref_syrk_crsp_reference(int K, int M, const double* Ap, double* C,
                                          double alpha, double beta) {
  syrk_reference<double>(K, M, Ap, C, alpha, beta);
}
SKREF_EXPORT void ref_syrk_crsp_init_A_packed(int K, int M, double* Ap, int seed) {
  init_A_packed<double>(K, M, Ap, seed);
}
SKREF_EXPORT int ref_syrk_crsp_selftest() {
  char name[] = "syrk_crsp";
  char* argv[] = {name, nullptr};
  return skgemm_ref_syrk_crsp_main(1, argv) == 0 ? 1 : 0;
}
