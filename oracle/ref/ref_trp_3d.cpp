// Reference rotation Psi' = Psi*Q: include/sme_trp_3d.hpp (grid-packed in,
// band-packed out) and its checker trp_3d_test.cpp (naive compute_reference and
// test_correctness), compiled unchanged with the SME emulation shim.
// Exports sme_gemm_trp_3d<double>::compute (sme_trp_3d.hpp:194),
// compute_reference (trp_3d_test.cpp:56) and the file's six correctness cases
// (trp_3d_test.cpp:237-239).
#include "ref_prelude.hpp"
#define main skgemm_ref_trp_3d_main
#include "trp_3d_test.cpp"
#undef main

SKREF_EXPORT void ref_trp_3d_compute(int Nd, int nb, const double* A_grid,
                                     const double* Q, double* D_band) {
  sme_gemm_trp_3d<double>::compute(Nd, nb, A_grid, Q, D_band);
}
SKREF_EXPORT void ref_trp_3d_reference(int Nd, int nb, const double* A_grid,
                                       const double* Q, double* D_band) {
  compute_reference<double>(Nd, nb, A_grid, Q, D_band);
}
SKREF_EXPORT int ref_trp_3d_selftest() {
  const int cases[6][2] = {{64, 32}, {256, 64}, {512, 128}, {1024, 256}, {2048, 128}, {4096, 128}};
  int passed = 0;
  for (auto& c : cases) passed += test_correctness<double>(c[0], c[1]);
  return passed;
}
