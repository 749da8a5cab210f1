// Reference nonlocal projector: include/nloc_packed_opt2.hpp
// (Hamiltonian::nloc_project_vectors_packed 16->32 and _16to16), compiled
// unchanged through its test file nloc_packed_opt2_test.cpp, which supplies
// the MPI and projector-structure mocks (single rank).
#include "ref_prelude.hpp"
#define main skgemm_ref_nloc_main
#include "nloc_packed_opt2_test.cpp"
#undef main

// P projectors, flattened: projector p has nrow[p] grid rows index[row_off[p]
// .. +nrow[p]], coefficients chi (col-major nrow x ncol) at chi_off[p], gamma
// (ncol) at gam_off[p], atom atom[p], and its coefficient block at
// offsets[p] (offsets[P] = total columns).
SKREF_EXPORT void ref_nloc_project(int P, const unsigned* nrow, const unsigned* ncol,
                                   const int* atom, const unsigned* offsets,
                                   const unsigned* index, const long long* row_off,
                                   const double* chi, const long long* chi_off,
                                   const double* gamma, const long long* gam_off, int nb, int K,
                                   double dv, const double* psi16, double* out, int out_tile) {
  Effective_potential_nloc<double> V;
  for (int p = 0; p < P; ++p) {
    Nloc_projector<double> pr;
    pr.nrow = nrow[p];
    pr.ncol = ncol[p];
    pr.atom_index = atom[p];
    pr.chi.nrow = nrow[p];
    pr.chi.ncol = ncol[p];
    pr.chi.data = const_cast<double*>(chi + chi_off[p]);
    pr.gamma.size = ncol[p];
    pr.gamma.data = const_cast<double*>(gamma + gam_off[p]);
    pr.index.assign(index + row_off[p], index + row_off[p] + nrow[p]);
    V.nloc_projectors.push_back(std::move(pr));
  }
  V.offsets.assign(offsets, offsets + P + 1);
  if (out_tile == 32)
    Hamiltonian::nloc_project_vectors_packed<double>(out, psi16, V, nb, K, dv, MPI_COMM_WORLD);
  else
    Hamiltonian::nloc_project_vectors_packed_16to16<double>(out, psi16, V, nb, K, dv,
                                                            MPI_COMM_WORLD);
}
