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
//   sme_pack<double>::pack_c16 / pack_r16 / unpack_c16 / unpack_r16 /
//       band_to_grid_tile / grid_to_band_tile (include/sme_pack.hpp:85-313;
//       host-side layout converters)
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

inline void require(bool ok, const char* msg) {
  if (ok) return;
#ifdef SKGEMM_NO_EXCEPTIONS
  std::fprintf(stderr, "skgemm error %d: %s\n", SKGEMM_ERR_INVALID_ARG, msg);
  std::abort();
#else
  throw error(SKGEMM_ERR_INVALID_ARG, msg);
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

// The reference's host-side layout converters (sme_pack<double>,
// include/sme_pack.hpp:30-313) under the same names, as plain loops; the
// device forms are skgemm_{pack,unpack}_{c16,r16}_dev and
// skgemm_band_to_grid_dev / skgemm_grid_to_band_dev. Grid point g, band b:
//   column-major [Nd, nb] (= row-major [nb, Nd]): X[g + b*Nd]
//   grid-packed [Nd/16][nb][16]:                 P[(g/16)*nb*16 + b*16 + g%16]
//   band-packed [nb/16][Nd][16]:                 B[(b/16)*Nd*16 + g*16 + b%16]
// Nd (and nb for the band form) must be multiples of 16: the reference drops
// the remainder tiles, these throw skgemm::error.
template <typename T>
class sme_pack {
 public:
  static constexpr int PACK_G = 16;

  static void pack_c16(const int Nd, const int nb, const T* src, T* dst) {
    skgemm::require(Nd >= 0 && nb >= 0 && Nd % 16 == 0, "pack_c16: Nd must be a multiple of 16");
    for (int gt = 0; gt < Nd / 16; ++gt)
      for (int b = 0; b < nb; ++b)
        for (int i = 0; i < 16; ++i)
          dst[((int64_t)gt * nb + b) * 16 + i] = src[gt * 16 + i + (int64_t)b * Nd];
  }
  static void pack_r16(const int Nd, const int nb, const T* src, T* dst) {
    pack_c16(Nd, nb, src, dst);  // row-major [nb, Nd] is the same bytes
  }
  static void unpack_c16(const int Nd, const int nb, const T* src, T* dst) {
    skgemm::require(Nd >= 0 && nb >= 0 && Nd % 16 == 0, "unpack_c16: Nd must be a multiple of 16");
    for (int gt = 0; gt < Nd / 16; ++gt)
      for (int b = 0; b < nb; ++b)
        for (int i = 0; i < 16; ++i)
          dst[gt * 16 + i + (int64_t)b * Nd] = src[((int64_t)gt * nb + b) * 16 + i];
  }
  static void unpack_r16(const int Nd, const int nb, const T* src, T* dst) {
    unpack_c16(Nd, nb, src, dst);
  }
  static void band_to_grid_tile(const int Nd, const int nb, const T* src, T* dst) {
    skgemm::require(Nd >= 0 && nb >= 0 && Nd % 16 == 0 && nb % 16 == 0,
                    "band_to_grid_tile: Nd and nb must be multiples of 16");
    for (int gt = 0; gt < Nd / 16; ++gt)
      for (int b = 0; b < nb; ++b)
        for (int i = 0; i < 16; ++i)
          dst[((int64_t)gt * nb + b) * 16 + i] =
              src[((int64_t)(b / 16) * Nd + gt * 16 + i) * 16 + b % 16];
  }
  static void grid_to_band_tile(const int Nd, const int nb, const T* src, T* dst) {
    skgemm::require(Nd >= 0 && nb >= 0 && Nd % 16 == 0 && nb % 16 == 0,
                    "grid_to_band_tile: Nd and nb must be multiples of 16");
    for (int bt = 0; bt < nb / 16; ++bt)
      for (int g = 0; g < Nd; ++g)
        for (int i = 0; i < 16; ++i)
          dst[((int64_t)bt * Nd + g) * 16 + i] =
              src[((int64_t)(g / 16) * nb + bt * 16 + i) * 16 + g % 16];
  }
};
