// Header-compatible C++ front end of libskgemm.
//
// Declares the same class templates and static entry points as the
// reference's kernel headers, forwarding to the C ABI in skgemm.h, so a
// driver written against the reference links unchanged against libskgemm.so:
//
//   gemm<double>::compute_test / compute_packed / compute_streamk_packed
//       (gemm_opt.cpp:314-392, gemm_crsp.cpp:316-385)
//   gemm<double>::pack_A / pack_B  (gemm_opt.cpp:342-371; host-side packing,
//       ceil(M/16) / ceil(N/32) panels with zero padding)
//   sme_syrk<double>::compute      (include/sme_syrk.hpp:137, syrk_crsp.cpp:306)
//   sme_gemm_trp_3d<double>::compute, sme_gemm_trp<double>
//                                  (include/sme_trp_3d.hpp:194, :218-220)
//
// Like the reference these return void; a failing call throws
// skgemm::error (the reference has no error channel at all). Define
// SKGEMM_NO_EXCEPTIONS to get std::abort() with a message instead.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "skgemm.h"

namespace skgemm {

struct error : std::runtime_error {
  int code;
  error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int status) {
  if (status == SKGEMM_OK) return;
#ifdef SKGEMM_NO_EXCEPTIONS
  std::fprintf(stderr, "skgemm error %d: %s\n", status, skgemm_last_error());
  std::abort();
#else
  throw error(status, skgemm_last_error());
#endif
}

}  // namespace skgemm

template <typename T>
class gemm {
  static_assert(std::is_same<T, double>::value, "libskgemm implements the FP64 path");

 public:
  static constexpr int ZA_TILE_M = 16;  // packed-A panel width
  static constexpr int ZA_TILE_N = 32;  // packed-B panel width

  static void compute_packed(const int M, const int N, const int K, const T* A_packed,
                             const T* B_packed, T* D, const T alpha, const T gamma) {
    skgemm::check(skgemm_dgemm_packed(M, N, K, A_packed, B_packed, D, alpha, gamma));
  }
  static void compute_streamk_packed(const int M, const int N, const int K, const T* A_packed,
                                     const T* B_packed, T* D, const T alpha, const T gamma) {
    compute_packed(M, N, K, A_packed, B_packed, D, alpha, gamma);
  }
  static void compute_test(const int M, const int N, const int K, const T* A_colmajor,
                           const T* B_rowmajor, T* D, const T alpha, const T gamma) {
    skgemm::check(skgemm_dgemm(M, N, K, A_colmajor, B_rowmajor, D, alpha, gamma));
  }
  // Packs into ceil(M/16) (resp. ceil(N/32)) panels; the destination must hold
  // that many panels (the reference's pack_A drops the M % 16 remainder).
  static void pack_A(const int M, const int K, const T* A_colmajor, T* A_packed) {
    const int64_t tiles = (M + ZA_TILE_M - 1) / ZA_TILE_M;
    for (int64_t tm = 0; tm < tiles; ++tm)
      for (int64_t k = 0; k < K; ++k)
        for (int i = 0; i < ZA_TILE_M; ++i) {
          const int64_t m = tm * ZA_TILE_M + i;
          A_packed[(tm * K + k) * ZA_TILE_M + i] = m < M ? A_colmajor[m + k * (int64_t)M] : T(0);
        }
  }
  static void pack_B(const int N, const int K, const T* B_rowmajor, T* B_packed) {
    const int64_t tiles = (N + ZA_TILE_N - 1) / ZA_TILE_N;
    for (int64_t tn = 0; tn < tiles; ++tn)
      for (int64_t k = 0; k < K; ++k)
        for (int j = 0; j < ZA_TILE_N; ++j) {
          const int64_t n = tn * ZA_TILE_N + j;
          B_packed[(tn * K + k) * ZA_TILE_N + j] = n < N ? B_rowmajor[k * (int64_t)N + n] : T(0);
        }
  }
};

template <typename T>
class sme_syrk {
  static_assert(std::is_same<T, double>::value, "libskgemm implements the FP64 path");

 public:
  static constexpr int TILE_M = 16;
  static void compute(const int K, const int M, const T* A_packed, T* C, const T alpha,
                      const T beta) {
    skgemm::check(skgemm_dsyrk_packed(K, M, A_packed, C, alpha, beta));
  }
};

template <typename T>
class sme_gemm_trp_3d {
  static_assert(std::is_same<T, double>::value, "libskgemm implements the FP64 path");

 public:
  static constexpr int TILE_G = 16;
  static void compute(const int Nd, const int nb, const T* A, const T* B, T* D) {
    skgemm::check(skgemm_drot(Nd, nb, A, B, D));
  }
};

template <typename T>
using sme_gemm_trp = sme_gemm_trp_3d<T>;
