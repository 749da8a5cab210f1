// Ozaki split-precision path (declarations used by the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "skg_runtime.h"

namespace skg {

int ozaki_gemm_packed(int64_t M, int64_t N, int64_t K, const double* Ap, const double* Bp,
                      double* D, int64_t ldd, double alpha, double gamma,
                      skgemm_options_t* opts, cudaStream_t s);
int ozaki_syrk_packed(int64_t K, int64_t M, const double* Ap, double* C, int64_t ldc,
                      double alpha, double beta, skgemm_options_t* opts, cudaStream_t s);
int ozaki_subspace(int64_t K, int64_t M, const double* Psi, const double* HPsi, double* S,
                   int64_t lds, double alpha_s, double beta_s, double* Hs, int64_t ldh,
                   double alpha_h, double gamma_h, skgemm_options_t* opts, cudaStream_t s);
// A grid-packed, or band-packed when a_band (read K-major by the conversion).
int ozaki_rot(int64_t Nd, int64_t nb, const double* A, const double* Q, double* D,
              skgemm_options_t* opts, cudaStream_t s, bool a_band = false);
int ozaki_consume_error(DeviceState* dev, cudaStream_t s);
// Estimated device time (s) of an Ozaki call (op = SKGEMM_OP_*), < 0 if the
// shape is not eligible.
double ozaki_time_estimate(int op, int64_t M, int64_t N, int64_t K, int slices);
// Estimated device time (s) of ozaki_subspace on (K, M), < 0 if not eligible.
double ozaki_pair_time_estimate(int64_t K, int64_t M, int slices);
int igemm_s8(int64_t M, int64_t N, int64_t K, const int8_t* A, int64_t lda, const int8_t* B,
             int64_t ldb, int32_t* C, int64_t ldc, cudaStream_t s);
int probe_i8_peak(DeviceState* dev, double* tops);
int ozaki_scratch_bytes(DeviceState* dev, int op, int64_t M, int64_t N, int64_t K, int slices,
                        size_t* bytes);
int ozaki_reserve(DeviceState* dev, cudaStream_t s, int64_t Nd, int64_t nb, int slices);
size_t ozaki_stream_bytes(DeviceState* dev, cudaStream_t s);
int ozaki_release_stream(DeviceState* dev, cudaStream_t s);

}  // namespace skg
