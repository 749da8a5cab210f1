// Reference include/sme_syrk.hpp (4-ZA FP64 SYRK, C = alpha*A^T*A + beta*C,
// upper triangle, C column-major) compiled unchanged with the SME emulation shim.
// Exports sme_syrk<double>::compute (sme_syrk.hpp:137).
#include "ref_prelude.hpp"
#include "sme_syrk.hpp"

SKREF_EXPORT void ref_sme_syrk_compute(int K, int M, const double* Ap, double* C,
                                       double alpha, double beta) {
  sme_syrk<double>::compute(K, M, Ap, C, alpha, beta);
}
