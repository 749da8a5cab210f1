// Scalar emulation of the subset of the Arm SME/SVE ACLE that the reference's
// FP64 kernels use, so that those kernels (gemm_opt.cpp, gemm_crsp.cpp,
// syrk_crsp.cpp, include/sme_syrk.hpp, include/sme_trp_3d.hpp,
// include/sme_pack.hpp) compile and run unchanged on an x86-64 host.
//
// TEST INFRASTRUCTURE ONLY: this header is part of the oracle. It lets the
// reference's own kernels produce the golden outputs the CUDA path is checked
// against; nothing in the product links it.
//
// Semantics follow the published ACLE / Arm ARM definitions:
//  * a vector holds SVL/sizeof(T) lanes; SVL is the streaming vector length in
//    bytes (the reference fixes SVL=64, i.e. 8 doubles per vector);
//  * ZA holds SVL/8 = 8 64-bit tiles of 8x8 doubles (and 4 32-bit tiles of
//    16x16 floats); each OpenMP thread has its own ZA, as each core has its own
//    ZA storage in hardware, so the storage is thread_local;
//  * FMOPA (non-widening) is a fused multiply-add per element:
//    ZA[i][j] = fma(zn[i], zm[j], ZA[i][j]) where both predicates are active;
//  * predicated loads zero inactive lanes (_z forms zero inactive lanes too);
//    _m reads keep the inactive lanes of the merge operand.
#ifndef SKGEMM_ORACLE_ARM_SME_SHIM_H
#define SKGEMM_ORACLE_ARM_SME_SHIM_H

#include <cmath>
#include <cstdint>
#include <cstring>

#ifndef SVL
#define SVL 64
#endif

// SME function-type attributes have no meaning on the host.
#define __arm_streaming
#define __arm_locally_streaming
#define __arm_streaming_compatible
#define __arm_inout(...)
#define __arm_in(...)
#define __arm_out(...)
#define __arm_new(...)

namespace skgemm_sme_emul {
constexpr int kLanesD = SVL / 8;
constexpr int kLanesS = SVL / 4;
}  // namespace skgemm_sme_emul

struct svfloat64_t {
  double v[skgemm_sme_emul::kLanesD];
};
struct svfloat32_t {
  float v[skgemm_sme_emul::kLanesS];
};
// One flag per byte lane, as in the architecture (a 64-bit element is active
// when the flag of its lowest byte is set).
struct svbool_t {
  uint8_t p[SVL];
};

typedef double float64_t;
typedef float float32_t;

namespace skgemm_sme_emul {
inline bool act_d(const svbool_t& pg, int i) { return pg.p[i * 8] != 0; }
inline bool act_s(const svbool_t& pg, int i) { return pg.p[i * 4] != 0; }
// ZA storage per thread: 8 x (8x8) f64 tiles, 4 x (16x16) f32 tiles.
inline double (&za_d())[kLanesD][kLanesD][kLanesD] {
  static thread_local double za[kLanesD][kLanesD][kLanesD];
  return za;
}
inline float (&za_s())[4][kLanesS][kLanesS] {
  static thread_local float za[4][kLanesS][kLanesS];
  return za;
}
}  // namespace skgemm_sme_emul

// ---------------------------------------------------------------- predicates
inline svbool_t svptrue_b64() {
  svbool_t r;
  std::memset(r.p, 0, sizeof(r.p));
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i) r.p[i * 8] = 1;
  return r;
}
inline svbool_t svptrue_b32() {
  svbool_t r;
  std::memset(r.p, 0, sizeof(r.p));
  for (int i = 0; i < skgemm_sme_emul::kLanesS; ++i) r.p[i * 4] = 1;
  return r;
}

// ---------------------------------------------------------------- f64 vectors
inline svfloat64_t svdup_f64(double x) {
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i) r.v[i] = x;
  return r;
}
inline svfloat32_t svdup_f32(float x) {
  svfloat32_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesS; ++i) r.v[i] = x;
  return r;
}
inline svfloat64_t svld1(svbool_t pg, const double* p) {
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i)
    r.v[i] = skgemm_sme_emul::act_d(pg, i) ? p[i] : 0.0;
  return r;
}
inline svfloat64_t svld1_f64(svbool_t pg, const double* p) { return svld1(pg, p); }
inline svfloat64_t svld1_vnum(svbool_t pg, const double* p, int64_t vnum) {
  return svld1(pg, p + vnum * skgemm_sme_emul::kLanesD);
}
inline void svst1(svbool_t pg, double* p, svfloat64_t v) {
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i)
    if (skgemm_sme_emul::act_d(pg, i)) p[i] = v.v[i];
}
inline void svst1_f64(svbool_t pg, double* p, svfloat64_t v) { svst1(pg, p, v); }
inline void svst1_vnum(svbool_t pg, double* p, int64_t vnum, svfloat64_t v) {
  svst1(pg, p + vnum * skgemm_sme_emul::kLanesD, v);
}

// Arithmetic. _z: inactive lanes become zero. _x: inactive lanes unspecified
// (computed like active ones here). Scalar second operands are the _n forms.
inline svfloat64_t svmul_z(svbool_t pg, svfloat64_t a, svfloat64_t b) {
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i)
    r.v[i] = skgemm_sme_emul::act_d(pg, i) ? a.v[i] * b.v[i] : 0.0;
  return r;
}
inline svfloat64_t svmul_z(svbool_t pg, svfloat64_t a, double b) {
  return svmul_z(pg, a, svdup_f64(b));
}
// FMULX differs from FMUL only for 0 * inf (gives +-2); the kernels never
// produce that case, so it is an ordinary product here.
inline svfloat64_t svmulx_z(svbool_t pg, svfloat64_t a, svfloat64_t b) {
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i) {
    double x = a.v[i], y = b.v[i];
    double prod = ((x == 0.0 && std::isinf(y)) || (std::isinf(x) && y == 0.0))
                      ? std::copysign(2.0, x) * std::copysign(1.0, y)
                      : x * y;
    r.v[i] = skgemm_sme_emul::act_d(pg, i) ? prod : 0.0;
  }
  return r;
}
inline svfloat64_t svmulx_z(svbool_t pg, svfloat64_t a, double b) {
  return svmulx_z(pg, a, svdup_f64(b));
}
inline svfloat64_t svadd_z(svbool_t pg, svfloat64_t a, svfloat64_t b) {
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i)
    r.v[i] = skgemm_sme_emul::act_d(pg, i) ? a.v[i] + b.v[i] : 0.0;
  return r;
}
inline svfloat64_t svadd_z(svbool_t pg, svfloat64_t a, double b) {
  return svadd_z(pg, a, svdup_f64(b));
}
inline svfloat64_t svadd_f64_x(svbool_t pg, svfloat64_t a, svfloat64_t b) {
  (void)pg;
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i) r.v[i] = a.v[i] + b.v[i];
  return r;
}
// FMLA: acc + a * b with a single rounding.
inline svfloat64_t svmla_f64_x(svbool_t pg, svfloat64_t acc, svfloat64_t a,
                               svfloat64_t b) {
  (void)pg;
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i)
    r.v[i] = std::fma(a.v[i], b.v[i], acc.v[i]);
  return r;
}
// The overloaded (type-generic) names of the same operations.
inline svfloat64_t svadd_x(svbool_t pg, svfloat64_t a, svfloat64_t b) {
  return svadd_f64_x(pg, a, b);
}
inline svfloat64_t svmul_x(svbool_t pg, svfloat64_t a, svfloat64_t b) {
  (void)pg;
  svfloat64_t r;
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i) r.v[i] = a.v[i] * b.v[i];
  return r;
}
inline svfloat64_t svmla_x(svbool_t pg, svfloat64_t acc, svfloat64_t a, svfloat64_t b) {
  return svmla_f64_x(pg, acc, a, b);
}
// WHILELT: 64-bit lane i active while a + i < b.
inline svbool_t svwhilelt_b64(uint64_t a, uint64_t b) {
  svbool_t r;
  std::memset(r.p, 0, sizeof(r.p));
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i) r.p[i * 8] = (a + (uint64_t)i < b) ? 1 : 0;
  return r;
}

// ---------------------------------------------------------------- ZA (f64)
inline void svzero_za() {
  std::memset(&skgemm_sme_emul::za_d(), 0, sizeof(skgemm_sme_emul::za_d()));
  std::memset(&skgemm_sme_emul::za_s(), 0, sizeof(skgemm_sme_emul::za_s()));
}
inline void svmopa_za64_f64_m(uint64_t tile, svbool_t pn, svbool_t pm,
                              svfloat64_t zn, svfloat64_t zm) {
  auto& t = skgemm_sme_emul::za_d()[tile];
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i) {
    if (!skgemm_sme_emul::act_d(pn, i)) continue;
    for (int j = 0; j < skgemm_sme_emul::kLanesD; ++j)
      if (skgemm_sme_emul::act_d(pm, j)) t[i][j] = std::fma(zn.v[i], zm.v[j], t[i][j]);
  }
}
inline svfloat64_t svread_hor_za64_f64_m(svfloat64_t zd, svbool_t pg,
                                         uint64_t tile, uint32_t slice) {
  const auto& t = skgemm_sme_emul::za_d()[tile];
  for (int j = 0; j < skgemm_sme_emul::kLanesD; ++j)
    if (skgemm_sme_emul::act_d(pg, j)) zd.v[j] = t[slice][j];
  return zd;
}
inline svfloat64_t svread_ver_za64_f64_m(svfloat64_t zd, svbool_t pg,
                                         uint64_t tile, uint32_t slice) {
  const auto& t = skgemm_sme_emul::za_d()[tile];
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i)
    if (skgemm_sme_emul::act_d(pg, i)) zd.v[i] = t[i][slice];
  return zd;
}
inline void svwrite_hor_za64_f64_m(uint64_t tile, uint32_t slice, svbool_t pg,
                                   svfloat64_t zn) {
  auto& t = skgemm_sme_emul::za_d()[tile];
  for (int j = 0; j < skgemm_sme_emul::kLanesD; ++j)
    if (skgemm_sme_emul::act_d(pg, j)) t[slice][j] = zn.v[j];
}
inline void svwrite_ver_za64_f64_m(uint64_t tile, uint32_t slice, svbool_t pg,
                                   svfloat64_t zn) {
  auto& t = skgemm_sme_emul::za_d()[tile];
  for (int i = 0; i < skgemm_sme_emul::kLanesD; ++i)
    if (skgemm_sme_emul::act_d(pg, i)) t[i][slice] = zn.v[i];
}
inline void svld1_hor_za64(uint64_t tile, uint32_t slice, svbool_t pg,
                           const void* ptr) {
  auto& t = skgemm_sme_emul::za_d()[tile];
  const double* p = static_cast<const double*>(ptr);
  for (int j = 0; j < skgemm_sme_emul::kLanesD; ++j)
    t[slice][j] = skgemm_sme_emul::act_d(pg, j) ? p[j] : 0.0;
}
inline void svst1_hor_za64(uint64_t tile, uint32_t slice, svbool_t pg, void* ptr) {
  const auto& t = skgemm_sme_emul::za_d()[tile];
  double* p = static_cast<double*>(ptr);
  for (int j = 0; j < skgemm_sme_emul::kLanesD; ++j)
    if (skgemm_sme_emul::act_d(pg, j)) p[j] = t[slice][j];
}

// ---------------------------------------------------------------- ZA (f32)
// Declared because utils.hpp names them inside templates; the FP64 path never
// instantiates them.
inline void svmopa_za32_f32_m(uint64_t tile, svbool_t pn, svbool_t pm,
                              svfloat32_t zn, svfloat32_t zm) {
  auto& t = skgemm_sme_emul::za_s()[tile];
  for (int i = 0; i < skgemm_sme_emul::kLanesS; ++i) {
    if (!skgemm_sme_emul::act_s(pn, i)) continue;
    for (int j = 0; j < skgemm_sme_emul::kLanesS; ++j)
      if (skgemm_sme_emul::act_s(pm, j)) t[i][j] = std::fma(zn.v[i], zm.v[j], t[i][j]);
  }
}
inline svfloat32_t svread_hor_za32_f32_m(svfloat32_t zd, svbool_t pg,
                                         uint64_t tile, uint32_t slice) {
  const auto& t = skgemm_sme_emul::za_s()[tile];
  for (int j = 0; j < skgemm_sme_emul::kLanesS; ++j)
    if (skgemm_sme_emul::act_s(pg, j)) zd.v[j] = t[slice][j];
  return zd;
}
inline void svld1_hor_za32(uint64_t tile, uint32_t slice, svbool_t pg,
                           const void* ptr) {
  auto& t = skgemm_sme_emul::za_s()[tile];
  const float* p = static_cast<const float*>(ptr);
  for (int j = 0; j < skgemm_sme_emul::kLanesS; ++j)
    t[slice][j] = skgemm_sme_emul::act_s(pg, j) ? p[j] : 0.0f;
}
inline void svst1_hor_za32(uint64_t tile, uint32_t slice, svbool_t pg, void* ptr) {
  const auto& t = skgemm_sme_emul::za_s()[tile];
  float* p = static_cast<float*>(ptr);
  for (int j = 0; j < skgemm_sme_emul::kLanesS; ++j)
    if (skgemm_sme_emul::act_s(pg, j)) p[j] = t[slice][j];
}

#endif  // SKGEMM_ORACLE_ARM_SME_SHIM_H
