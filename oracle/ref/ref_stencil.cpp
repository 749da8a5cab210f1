// Reference H*Psi producer: include/stencil_extended_packed.hpp (the FDn = 6
// SVE kernels 16->32 and 16->16 and the scalar version for any FDn), compiled
// unchanged with the SVE emulation shim.
#include "ref_prelude.hpp"
#include "include/stencil_extended_packed.hpp"

using Stencil_method::Packed::calc_laplacian_extended_packed_16to16;
using Stencil_method::Packed::calc_laplacian_extended_packed_16to32;
using Stencil_method::Packed::calc_laplacian_extended_packed_16to32_scalar;

SKREF_EXPORT void ref_stencil_16to32(const double* ext, double* out, const double* A, int ni,
                                     int nj, int nk, int nb, int FDn, const double* cx,
                                     const double* cy, const double* cz, double c0) {
  calc_laplacian_extended_packed_16to32(ext, out, A, ni, nj, nk, nb, FDn, cx, cy, cz, c0);
}
SKREF_EXPORT void ref_stencil_16to16(const double* ext, double* out, const double* A, int ni,
                                     int nj, int nk, int nb, int FDn, const double* cx,
                                     const double* cy, const double* cz, double c0) {
  calc_laplacian_extended_packed_16to16(ext, out, A, ni, nj, nk, nb, FDn, cx, cy, cz, c0);
}
SKREF_EXPORT void ref_stencil_16to32_scalar(const double* ext, double* out, const double* A,
                                            int ni, int nj, int nk, int nb, int FDn,
                                            const double* cx, const double* cy,
                                            const double* cz, double c0) {
  calc_laplacian_extended_packed_16to32_scalar(ext, out, A, ni, nj, nk, nb, FDn, cx, cy, cz,
                                               c0);
}
