// Ozaki scheme II on sm_100a: FP64-accurate GEMM / SYRK / rotation from exact
// INT8 tensor-core products (Ozaki, Uchino, Imamura, "Ozaki Scheme II: A
// GEMM-oriented emulation of floating-point matrix multiplication using an
// integer modular technique", 2025).
//
// For C = A B (A: rows i, B: columns j, inner dimension k):
//  1. Scaling. Row i of A is scaled by 2^mu_i, column j of B by 2^nu_j, with
//     mu_i = gamma - ceil(log2 ||A_i||_2), so ||A_i 2^mu_i||_2 <= 2^gamma, and
//     rounded to integers A', B'. By Cauchy-Schwarz |(A'B')_ij| <= 2^(2 gamma)
//     (up to rounding slack), chosen below M/4 where M = m_0 ... m_{L-1}.
//  2. Residues. A' and B' are reduced modulo L pairwise-coprime moduli
//     m_l <= 256 into symmetric residues that fit int8.
//  3. Products. For every l, C_l = A'_l B'_l is computed exactly on tcgen05
//     kind::i8 (INT32 accumulation, k-segments short enough to be exact).
//  4. Reconstruction. C' = CRT(C_l mod m_l) in [-M/2, M/2] is evaluated in
//     FP64 with split constants: W_l = (M/m_l) * ((M/m_l)^-1 mod m_l) is
//     stored as Wh_l + Wl_l where Wh_l has at most 40 significant bits on a
//     common grid 2^e (so sum_l r_l Wh_l is exact in FP64) and Wl_l < 2^e;
//     q = rint(s / M), C' = (S_hi - q Mh) + (S_lo - q Ml). Finally
//     C = 2^(-mu_i - nu_j) C'.
// The error is that of rounding A and B to gamma bits (about
// sqrt(k/12) * 2^-gamma relative to ||A_i|| ||B_j|| per element); the
// reconstruction itself adds ~2^-70 relative.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "skg_i8gemm2_kernel.cuh"
#include "skg_i8gemm_kernel.cuh"
#include "skg_ozaki.h"

namespace skg {

namespace {

// Pairwise-coprime moduli <= 256, largest first: 2^8, 3*5*17, 11*23, 251,
// 13*19, 241, 239, 233, 229, 227, 223, 7*31, 211, 199, 197, 193.
constexpr uint32_t kModuli[kI8MaxModuli] = {256, 255, 253, 251, 247, 241, 239, 233,
                                            229, 227, 223, 217, 211, 199, 197, 193};
constexpr int kMinModuli = 6;
// k-blocks (128 k) per INT32-exact segment: s8 x s8 products are <= 2^14.
constexpr int kSegKbCapSigned = 1023;   // 1023 * 128 * 2^14 < 2^31
// BF16 residues: FP32 tile sums exact for <= 1024 products (16 k-blocks of
// 64), int32 slots for <= 127 such sub-segments.
constexpr int kSubKbCapBf16 = 16;
constexpr int kSegKbCapBf16 = 127 * kSubKbCapBf16;

// Residue constants for one moduli count L (gamma depends on L). The scaled
// integer X = rint(v 2^mu) (int64, |X| <= 2^gamma + 1/2) is cut into digits
// X = d0 + d1 2^12 + d2 2^24 + d3 2^36 + d4 2^48, d0..d3 in [0, 4096) (the low
// 48 bits of X) and d4 = floor(X / 2^48) signed (|d4| <= 2^12 for gamma <=
// 60), so X = S (mod m) with S = d0 + sum_j d_j c_j, c_j = 2^(12 j) mod m. In
// FP32 every product is below 2^20 and |S| < 2^22: all exact. For odd m,
// q = rint(S fl(1/m)) equals rint(S / m): |S| |fl(1/m) - 1/m| < 2^22 2^-31 =
// 2^-9 < 1/(2m), the least distance of S/m from a half-integer. Then
// r = S - q m in [-(m-1)/2, (m-1)/2] is the symmetric residue, a signed byte,
// read from the low mantissa byte of r + 1.5 2^23. m = 256: the low byte of X.
// Residue digit sets: for L <= kShortDigitsMaxL moduli (|X| <= 2^57) three
// unsigned 14-bit digits and a signed X >> 42 with symmetric constants
// (|c| <= 127), so |S| < 2^23 with one FMA fewer per modulus; for L = 16
// (|X| <= 2^61) four unsigned 12-bit digits and a signed X >> 48.
constexpr int kShortDigitsMaxL = 15;

struct ResidueConsts {
  int gamma_bits;
  float c[4][kI8MaxModuli];  // 2^(12 (j+1)) mod m
  float cs[3][kI8MaxModuli]; // 2^(14 (j+1)) mod m, symmetric representative
  float inv[kI8MaxModuli];   // fl(1/m)
  float m[kI8MaxModuli];
  uint32_t mi[kI8MaxModuli];
  // The same constants as {x, x} pairs for the packed FP32x2 pipe: pc[j] is
  // cs[j] (L <= kShortDigitsMaxL) or c[j]; pinv = inv, pnm = -m.
  float2 pc[4][kI8MaxModuli];
  float2 pinv[kI8MaxModuli];
  float2 pnm[kI8MaxModuli];
};

struct CrtConsts {  // for one moduli count L
  double wh[kI8MaxModuli];
  double wl[kI8MaxModuli];
  double mh, ml, inv_m;
};

__constant__ ResidueConsts c_res[kI8MaxModuli + 1];
__constant__ CrtConsts c_crt[kI8MaxModuli + 1];
__constant__ double c_inv_mod[kI8MaxModuli];  // fl(1 / m_l) of the moduli

typedef unsigned __int128 u128;

int bitlen(u128 x) {
  int b = 0;
  while (x) {
    x >>= 1;
    ++b;
  }
  return b;
}

double u128_to_double(u128 x) { return (double)x; }

// Host constants for L moduli (the first L of kModuli).
CrtConsts make_crt(int L, double* log2M_out) {
  CrtConsts c;
  memset(&c, 0, sizeof(c));
  u128 M = 1;
  for (int l = 0; l < L; ++l) M *= kModuli[l];
  const int e = bitlen(M) - 40;
  for (int l = 0; l < L; ++l) {
    const uint32_t m = kModuli[l];
    const u128 Ml = M / m;
    const uint32_t r = (uint32_t)(Ml % m);
    uint32_t y = 0;
    for (uint32_t t = 1; t < m; ++t)
      if ((uint64_t)r * t % m == 1) {
        y = t;
        break;
      }
    const u128 W = (Ml * y) % M;
    const u128 Wh = (W >> e) << e;
    c.wh[l] = ldexp((double)(uint64_t)(W >> e), e);
    c.wl[l] = u128_to_double(W - Wh);
  }
  const u128 Mh = (M >> e) << e;
  c.mh = ldexp((double)(uint64_t)(M >> e), e);
  c.ml = u128_to_double(M - Mh);
  c.inv_m = 1.0 / u128_to_double(M);
  if (log2M_out) *log2M_out = log2(u128_to_double(M));
  return c;
}

// Largest gamma with (2^gamma)^2 < M / 4.2 (Cauchy-Schwarz bound of A'B').
int gamma_for(int L) {
  double lg = 0;
  make_crt(L, &lg);
  return (int)floor((lg - 2.1) / 2.0);
}

// ------------------------------------------------------------ device math
__device__ __forceinline__ int ceil_log2_pos(double x) {
  int e;
  const double f = frexp(x, &e);  // x = f 2^e, f in [0.5, 1)
  return f == 0.5 ? e - 1 : e;
}

__device__ __forceinline__ int row_exponent(double sumsq, int gamma_bits) {
  if (!(sumsq > 0.0)) return 0;  // zero (or empty) row: any scale
  return gamma_bits - ceil_log2_pos(sqrt(sumsq));
}

// s1 * s2 = 2^mu exactly, each factor a normal double for |mu| < 2044.
__device__ __forceinline__ void pow2_pair(int mu, double& s1, double& s2) {
  const int h = mu / 2;
  s1 = ldexp(1.0, h);
  s2 = ldexp(1.0, mu - h);
}

// Shared-memory staging of a [128 k][16 rows] block as tileT[r][k'] with row
// pitch 129 doubles and k' = k ^ ((k >> 3) & 7): the transposing stores
// (consecutive r) and the reads of 8 consecutive k per thread (consecutive
// threads 8 k apart) are at most 2-way bank-conflicted.
constexpr int kTilePitch = 129;
__device__ __forceinline__ int swz_k(int k) { return k ^ ((k >> 3) & 7); }

template <int T>
__device__ __forceinline__ void stage_tile(double* tileT, const double* src, int64_t ks,
                                           int64_t k0, int64_t K, int rows_valid) {
  for (int i = threadIdx.x; i < 128 * T; i += blockDim.x) {
    const int kk = i / T, r = i % T;
    const int64_t k = k0 + kk;
    tileT[r * kTilePitch + swz_k(kk)] = (k < K && r < rows_valid) ? src[k * ks + r] : 0.0;
  }
}

__device__ __forceinline__ uint32_t pack4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  return __byte_perm(__byte_perm(a, b, 0x0040), __byte_perm(c, d, 0x0040), 0x5410);
}

constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: integers below 2^22 sit in the low mantissa

// Exact FP32 value of a 12-bit field (the bits 0x4B000000 | x are 2^23 + x).
__device__ __forceinline__ float field12(uint32_t x) {
  return __uint_as_float(0x4B000000u | (x & 0xFFFu)) - 8388608.0f;
}

// Exact FP32 value of a 14-bit field.
__device__ __forceinline__ float field14(uint32_t x) {
  return __uint_as_float(0x4B000000u | (x & 0x3FFFu)) - 8388608.0f;
}

// The digits of X = rint((v s1) s2) as exact floats, and X's low word.
struct Digits {
  float f0, f1, f2, f3, f4;
  uint32_t lo;
};
template <int L>
__device__ __forceinline__ Digits digits_of(double v, double s1, double s2) {
  const long long X = __double2ll_rn((v * s1) * s2);
  const uint32_t lo = (uint32_t)X, hi = (uint32_t)((unsigned long long)X >> 32);
  Digits d;
  d.lo = lo;  // m = 256: its low byte
  if constexpr (L <= kShortDigitsMaxL) {
    d.f0 = field14(lo);
    d.f1 = field14(lo >> 14);
    d.f2 = field14(__funnelshift_r(lo, hi, 28));
    d.f3 = __int_as_float(0x4B400000 + ((int)hi >> 10)) - kMagic;  // signed X >> 42
    d.f4 = 0.0f;
  } else {
    d.f0 = field12(lo);
    d.f1 = field12(lo >> 12);
    d.f2 = field12(__funnelshift_r(lo, hi, 24));
    d.f3 = field12(hi >> 4);
    d.f4 = __int_as_float(0x4B400000 + ((int)hi >> 16)) - kMagic;  // signed X >> 48
  }
  return d;
}

// BF16 bits of residue 0, X mod 256 as a signed byte. Integers of magnitude
// <= 128 are exact in BF16: the top half of the FP32.
__device__ __forceinline__ uint32_t low_byte_bf16(const Digits& d) {
  return __float_as_uint((float)((int)(d.lo << 24) >> 24)) >> 16;
}

__device__ __forceinline__ uint32_t pack2(uint32_t a, uint32_t b) { return a | (b << 16); }

// Symmetric residues modulo odd kModuli[l] of two elements a (x) and b (y),
// as exact floats (|r| <= 127): S = d0 + sum_j d_j c_j, q = rint(S fl(1/m))
// through the 1.5 2^23 shift, r = S - q m. Computed on the packed FP32x2
// pipe (__ffma2_rn / __fadd2_rn: each lane rounds to nearest like fmaf), two
// elements per issue slot — the conversion is issue-bound.
template <int L>
__device__ __forceinline__ float2 residue_float2(const Digits& a, const Digits& b, int l) {
  const ResidueConsts& rc = c_res[L];
  float2 S = __ffma2_rn(make_float2(a.f1, b.f1), rc.pc[0][l], make_float2(a.f0, b.f0));
  S = __ffma2_rn(make_float2(a.f2, b.f2), rc.pc[1][l], S);
  S = __ffma2_rn(make_float2(a.f3, b.f3), rc.pc[2][l], S);
  if constexpr (L > kShortDigitsMaxL) S = __ffma2_rn(make_float2(a.f4, b.f4), rc.pc[3][l], S);
  const float2 q = __fadd2_rn(__ffma2_rn(S, rc.pinv[l], make_float2(kMagic, kMagic)),
                              make_float2(-kMagic, -kMagic));
  return __ffma2_rn(q, rc.pnm[l], S);
}

// The residues of two elements as the low bytes of the returned words.
template <int L>
__device__ __forceinline__ uint2 residue_byte2(const Digits& a, const Digits& b, int l) {
  const float2 r = __fadd2_rn(residue_float2<L>(a, b, l), make_float2(kMagic, kMagic));
  return make_uint2(__float_as_uint(r.x), __float_as_uint(r.y));
}

// BF16 bits of the residues l >= 1 of two elements, packed into one word (a
// in the low half): the top halves of the two FP32 residues.
template <int L>
__device__ __forceinline__ uint32_t residue_bf16x2(const Digits& a, const Digits& b, int l) {
  const float2 r = residue_float2<L>(a, b, l);
  return __byte_perm(__float_as_uint(r.x), __float_as_uint(r.y), 0x7632);
}

// ------------------------------------------------- packed-T operand prep
// Partial sums of squares of each row of a packed-T operand
// ([ceil(R/T)][K][T]): part[(p*C + c)*T + r] over k-chunk c.
template <int T, bool KM = false>
__global__ void __launch_bounds__(256) norm_partials_kernel(int64_t R, int64_t K,
                                                           const double* __restrict__ X,
                                                           int C, double* __restrict__ part) {
  __shared__ double red[256];
  const int p = blockIdx.x, c = blockIdx.y;
  // KM: thread (kl = tid % 16, r = tid / 16), so that a warp reads two rows'
  // whole 128-byte k-blocks; each (r, kl) sum is the packed layout's, and
  // red[] is indexed as there, so the result is the same bit for bit.
  const int r = KM ? (int)threadIdx.x / 16 : (int)threadIdx.x % T;
  const int kl = KM ? (int)threadIdx.x % 16 : (int)threadIdx.x / T;
  const int slot = kl * T + r;  // = threadIdx.x for the packed layout
  constexpr int KL = 256 / T;
  const int64_t k0 = (int64_t)c * K / C, k1 = (int64_t)(c + 1) * K / C;
  const double* src = X + (int64_t)p * K * T;
  // KM (T = 16): a K-major [K/16][R][16] operand, row p*16 + r read at
  // X[(k/16)*R*16 + (p*16 + r)*16 + k%16]; the same sums in the same order.
  const int64_t row_r = (int64_t)p * T + r;
  double acc = 0.0;
  // Unrolled so that loads run ahead of the (unchanged) fma chain.
#pragma unroll 8
  for (int64_t k = k0 + kl; k < k1; k += KL) {
    double v;
    if constexpr (KM)
      v = row_r < R ? X[(k >> 4) * R * 16 + row_r * 16 + (k & 15)] : 0.0;
    else
      v = src[k * T + r];
    acc = fma(v, v, acc);
  }
  red[slot] = acc;
  __syncthreads();
  if (threadIdx.x < T) {
    double s = 0.0;
    for (int j = 0; j < KL; ++j) s += red[j * T + threadIdx.x];
    const int64_t row = (int64_t)p * T + threadIdx.x;
    part[((int64_t)p * C + c) * T + threadIdx.x] = row < R ? s : 0.0;
  }
}

// Row exponents mu[row] (row < Rpad) of a packed-T operand from its norm
// partials; rows past R (padding) get 0.
template <int T>
__global__ void row_exponents_kernel(int64_t R, int64_t Rpad, int C, const double* __restrict__ part,
                                     int gamma_bits, int* __restrict__ mu) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= Rpad) return;
  int m = 0;
  if (row < R) {
    const int64_t p = row / T;
    const int rin = (int)(row - p * T);
    double sq = 0.0;
    for (int c = 0; c < C; ++c) sq += part[(p * C + c) * T + rin];
    m = row_exponent(sq, gamma_bits);
  }
  mu[row] = m;
}

// Residues of a packed-T operand -> res[l][Rpad][KP] (K-major bytes).
// Every warp runs its own pipeline over a contiguous range of tiles of 16
// rows x 32 k (group g = 16-row group, kb = 32-k block, g-major): a TMA box
// {16 rows, 32 k} of the operand lands as [32 k][16 rows] doubles in one of
// the warp's three 4 KB stages (zero-filled past K and past the operand's
// panels), the tile two ahead already in flight. INT8: lanes 2r and 2r + 1
// convert k = 0 .. 15 and 16 .. 31 of row r, so that each residue leaves as
// one 16-byte store per lane whose quarter-warp phases (8 lanes) fill the
// whole 32-byte sectors of 4 rows (8 rows of half sectors in lane order
// r + 16 h took twice the L1 store wavefronts); the stage is 128B-swizzled so
// that the two k-rows a half-warp reads fall on disjoint banks. BF16 (64-byte
// rows): lane r + 16 h, unswizzled stage. No CTA-wide barrier. Row exponents
// mu[row] are read from the exponent pass.
constexpr int kConvStages = 3;
constexpr int kConvWarps = 8;
constexpr int kConvTile = 16 * 32;  // doubles per warp tile
constexpr int kConvSmem = kConvWarps * (kConvStages * kConvTile * 8 + kConvStages * 8);

// BF16 residues of one staged 16-row x 32-k tile (BF16 stages: packed16
// [32 k][16 rows] unswizzled, K-major as for INT8) for lane (r = lane % 16,
// h = lane / 16). BF16 rows take 64 bytes per 32-k block: lane h converts
// k = 8 h .. 8 h + 7 and 16 + 8 h .. 16 + 8 h + 7, so that each of its two
// 16-byte stores and the other half-lane's together fill one whole 32-byte
// sector. row: the residue row's first byte of this k-block (plane 0).
template <int L, bool KM>
__device__ __forceinline__ void convert_stage_bf16(const double* stage, int r, int h, double s1,
                                                   double s2, uint8_t* row, int64_t lstride) {
  auto at = [&](int k) {  // element (k, r) of the stage
    if constexpr (KM)
      return stage[(16 * (k >> 4) + r) * 16 + (((((k & 15) >> 1) ^ (r & 7))) << 1) + (k & 1)];
    else
      return stage[k * 16 + r];
  };
  Digits d[16];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    d[j] = digits_of<L>(at(8 * h + j), s1, s2);
    d[8 + j] = digits_of<L>(at(16 + 8 * h + j), s1, s2);
  }
#pragma unroll
  for (int l = 0; l < L; ++l) {
    uint32_t w[8];  // w[i]: elements 2i, 2i + 1
#pragma unroll
    for (int i = 0; i < 8; ++i)
      w[i] = l == 0 ? pack2(low_byte_bf16(d[2 * i]), low_byte_bf16(d[2 * i + 1]))
                    : residue_bf16x2<L>(d[2 * i], d[2 * i + 1], l);
    uint8_t* base = row + l * lstride;
    *reinterpret_cast<uint4*>(base + 16 * h) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4*>(base + 32 + 16 * h) = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

// INT8 residues of one staged 16-row x 32-k tile (conversion kernels' stage
// layout) for lane (r = lane / 2, h = lane % 2): k = 16 h .. 16 h + 15 of row
// r, one 16-byte store per residue plane at dst + l lstride.
template <int L, bool KM>
__device__ __forceinline__ void convert_stage_i8(const double* stage, int r, int h, double s1,
                                                 double s2, uint8_t* dst, int64_t lstride) {
  // Swizzled stage: 16-byte chunk c of k-row k at c ^ (k % 8). At step j
  // lane (r, h) reads k = 16 h + (j ^ 4 h), whose chunk (r / 2) ^ (j % 8)
  // ^ 4 h differs from the other half-lane's in bit 2, so a half-warp
  // touches 8 distinct chunks (all 32 banks once). d[j] then holds
  // k = 16 h + (j ^ 4 h): for h = 1 the packed words are in the order
  // 1, 0, 3, 2, and put() swaps them back.
  // KM: lane h = 1 walks its k in the order j ^ 1 instead, so that the
  // half-warp's two k-blocks read opposite halves of each 16-byte unit
  // (conflict-free); its pairs come out swapped, which the byte-permute
  // selector of pk() undoes, and put() keeps the word order.
  const int z = KM ? 256 * h + 16 * r + ((r & 7) << 1) + h
                   : 320 * h | (((r >> 1) ^ (4 * h)) << 1) | (r & 1);
  Digits d[16];
#pragma unroll
  for (int j = 0; j < 16; ++j)
    d[j] = digits_of<L>(stage[(KM ? j : ((j << 4) | ((j & 7) << 1))) ^ z], s1, s2);
  const uint32_t sel = (KM && h) ? 0x0004u : 0x0040u;
  auto pk = [&](uint32_t a, uint32_t b, uint32_t c, uint32_t e) {
    return __byte_perm(__byte_perm(a, b, sel), __byte_perm(c, e, sel), 0x5410);
  };
  auto put = [&](uint8_t* p, uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3) {
    *reinterpret_cast<uint4*>(p) =
        (!KM && h) ? make_uint4(w1, w0, w3, w2) : make_uint4(w0, w1, w2, w3);
  };
  put(dst, pk(d[0].lo, d[1].lo, d[2].lo, d[3].lo), pk(d[4].lo, d[5].lo, d[6].lo, d[7].lo),
      pk(d[8].lo, d[9].lo, d[10].lo, d[11].lo), pk(d[12].lo, d[13].lo, d[14].lo, d[15].lo));
#pragma unroll
  for (int l = 1; l < L; ++l) {
    uint32_t b[16];
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
      const uint2 v = residue_byte2<L>(d[j], d[j + 1], l);
      b[j] = v.x;
      b[j + 1] = v.y;
    }
    put(dst + l * lstride, pk(b[0], b[1], b[2], b[3]), pk(b[4], b[5], b[6], b[7]),
        pk(b[8], b[9], b[10], b[11]), pk(b[12], b[13], b[14], b[15]));
  }
}

// KM: the operand is K-major, [K/16][R][16] (band-packed Psi as the
// rotation's A: the band -> grid transposition happens here, in the reads).
// Its box {16 k, 16 rows, 2 k-blocks} lands as [2][16 rows][16 k], 128B-
// swizzled per 128-byte row: element (k, r) at row R = 16 (k / 16) + r, unit
// ((k % 16) / 2) ^ (R % 8), half k % 2.
template <int T, int L, bool BF, bool KM = false>
__global__ void __launch_bounds__(256, 2) convert_tma_kernel(
    const __grid_constant__ CUtensorMap map, int64_t KP, int64_t Rpad,
    const int* __restrict__ mu, uint8_t* __restrict__ res, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* buf = reinterpret_cast<double*>(sm) + warp * kConvStages * kConvTile;
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kConvWarps * kConvStages * kConvTile * 8) +
                  warp * kConvStages;
  const int64_t KB = KP / 32;
  const int64_t ntiles = (Rpad / 16) * KB;
  // Warp gw takes tiles gw, gw + nw, gw + 2 nw, ...: at any moment the
  // machine converts one contiguous window of tiles, so the stores of all
  // warps land in a narrow band of each residue plane (page-local writes)
  // and the loads stream one contiguous span.
  const int64_t gw = (int64_t)blockIdx.x * kConvWarps + warp, nw = (int64_t)gridDim.x * kConvWarps;
  if (gw >= ntiles) return;
  const int64_t nmine = (ntiles - gw + nw - 1) / nw;  // tiles of this warp
  const int64_t dq = nw / KB, dr = nw % KB;           // stride nw as (groups, k-blocks)
  if (lane == 0) {
    for (int st = 0; st < kConvStages; ++st) mbar_init(&bar[st], 1);
    fence_mbar_init();
  }
  __syncwarp();
  // Tile (g, kb): rows 16 g .. +16 = panel g / (T/16), rows 16 (g % (T/16)) ..
  // of that panel.
  auto issue = [&](int64_t g, int64_t kb, int st) {
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(&bar[st], kConvTile * 8);
    if constexpr (KM)
      tma_load_3d(buf + st * kConvTile, &map, &bar[st], 0, (int)(16 * g), (int)(2 * kb));
    else
      tma_load_3d(buf + st * kConvTile, &map, &bar[st], (int)(16 * (g % (T / 16))),
                  (int)(kb * 32), (int)(g / (T / 16)));
  };
  auto advance = [&](int64_t& g, int64_t& kb) {
    g += dq;
    kb += dr;
    if (kb >= KB) {
      kb -= KB;
      ++g;
    }
  };
  int64_t g = gw / KB, kb = gw % KB;
  // Counters of the next tile to issue.
  int64_t gi = g, ki = kb;
  if (lane == 0) tma_prefetch_desc(&map);
  for (int st = 0; st < kConvStages - 1; ++st) {
    if (lane == 0 && st < nmine) issue(gi, ki, st);
    advance(gi, ki);
  }
  const int r = BF ? (lane & 15) : (lane >> 1), h = BF ? (lane >> 4) : (lane & 1);
  double s1 = 1.0, s2 = 1.0;
  int64_t cur_g = -1;
  uint32_t phase = 0;  // bit s: parity of stage s's next completion
  int s = 0;
  for (int64_t n = 0; n < nmine; ++n) {
    if (lane == 0 && n + kConvStages - 1 < nmine) issue(gi, ki, (s + kConvStages - 1) % kConvStages);
    advance(gi, ki);
    if (g != cur_g) {
      pow2_pair(mu[g * 16 + r], s1, s2);
      cur_g = g;
    }
    const bool ok = mbar_wait(&bar[s], (phase >> s) & 1u, err);
    phase ^= 1u << s;
    constexpr int ES = BF ? 2 : 1;  // bytes per residue
    uint8_t* dst = res + ((g * 16 + r) * KP + kb * 32 + 16 * h) * ES;
    const int64_t lstride = Rpad * KP * ES;
    if (ok && BF) {
      uint8_t* row = res + ((g * 16 + r) * KP + kb * 32) * 2;
      convert_stage_bf16<L, KM>(buf + s * kConvTile, r, h, s1, s2, row, lstride);
    } else if (ok) {
      convert_stage_i8<L, KM>(buf + s * kConvTile, r, h, s1, s2, dst, lstride);
    } else {
#pragma unroll
      for (int l = 0; l < L; ++l)
#pragma unroll
        for (int e = 0; e < ES; ++e)
          reinterpret_cast<uint4*>(dst + l * lstride)[e] = make_uint4(0, 0, 0, 0);
    }
    __syncwarp();  // stage s consumed by every lane before it is refilled
    s = (s + 1) % kConvStages;
    advance(g, kb);
  }
}

// Element (k, r) (k < 32) of a conversion stage: packed16 stages are
// [32 k][16 rows] with 16-byte chunk c of k-row k at c ^ (k % 8); K-major
// stages are [2][16 rows][16 k], 128-byte row 16 (k / 16) + r with chunk c
// at c ^ (r % 8).
template <bool KM, bool BF = false>
__device__ __forceinline__ double stage_elem(const double* st, int k, int r) {
  if constexpr (KM)
    return st[(16 * (k >> 4) + r) * 16 + ((((k & 15) >> 1) ^ (r & 7)) << 1) + (k & 1)];
  else if constexpr (BF)
    return st[k * 16 + r];  // BF16 packed16 stages are not swizzled
  else
    return st[k * 16 + (((r >> 1) ^ (k & 7)) << 1) + (r & 1)];
}

// One pass for packed16 operands with short rows (K <= 512: grid-packed Psi
// as the rotation's A, rows = grid points, k = bands). A persistent CTA of
// four warps (three per SM, so that some load while others convert) takes
// one 16-row group at a time: its KP/32 boxes of 16 rows x 32 k (the
// conversion kernels' stage layout) land in shared memory by TMA together;
// the rows' sums of squares are taken there, then each warp converts its
// boxes with the conversion kernels' tile code. HBM reads the operand once
// instead of twice. The sums follow the two-pass path exactly when that path
// uses one k-chunk (ceil(R/16) >= 600): partial (r, kl) of 256 (two per
// thread) adds v*v by fma over k = kl, kl + 16, ..., and row r adds its 16
// partials in kl order. So the exponents, and the residues, equal that
// path's bit for bit. KM: the K-major form [K/16][R][16] (band-packed Psi),
// staged as the conversion kernel's K-major boxes; same sums, same bits.
constexpr int kShortKbMax = 16;   // KP <= 512
constexpr int kShortThreads = 128;  // 4 warps; three CTAs per SM
constexpr int kShortSmem = kShortKbMax * kConvTile * 8 + 256 * 8 + 32 * 8 + 64 + 1024;

template <int L, bool KM, bool BF>
__global__ void __launch_bounds__(kShortThreads, 3) convert_short_kernel(
    const __grid_constant__ CUtensorMap map, int64_t R, int64_t K, int64_t KP, int64_t Rpad,
    int gamma_bits, int* __restrict__ mu, uint8_t* __restrict__ res, uint32_t* __restrict__ err) {
  extern __shared__ uint8_t ssm[];
  double* tiles =  // [16 boxes][32 k][16 rows]
      reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(ssm) + 1023) & ~uintptr_t(1023));
  double* red = tiles + kShortKbMax * kConvTile;  // [16 kl][16 rows]
  double* sc = red + 256;                         // s1 [16], s2 [16]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sc + 32);
  const int KB = (int)(KP / 32);
  const int64_t G = Rpad / 16;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    tma_prefetch_desc(&map);
  }
  __syncthreads();
  uint32_t phase = 0;
  for (int64_t g = blockIdx.x; g < G; g += gridDim.x) {
    if (threadIdx.x == 0) {
      fence_proxy_async_smem();  // the previous group's reads of the tiles are done
      mbar_arrive_expect_tx(bar, (uint32_t)(KB * kConvTile * 8));
      for (int kb = 0; kb < KB; ++kb) {
        if constexpr (KM)
          tma_load_3d(tiles + kb * kConvTile, &map, bar, 0, (int)(16 * g), 2 * kb);
        else
          tma_load_3d(tiles + kb * kConvTile, &map, bar, 0, kb * 32, (int)g);
      }
    }
    const bool ok = mbar_wait(bar, phase, err);
    phase ^= 1;
    for (int t = threadIdx.x; t < 256; t += kShortThreads) {  // partial (r, kl) = t
      const int r = t & 15, kl = t >> 4;
      double acc = 0.0;
      for (int64_t k = kl; k < K; k += 16) {
        const double v = stage_elem<KM, BF>(tiles + (k >> 5) * kConvTile, (int)(k & 31), r);
        acc = fma(v, v, acc);
      }
      red[kl * 16 + r] = acc;
    }
    __syncthreads();
    if (threadIdx.x < 16) {
      double part = 0.0;
      for (int j = 0; j < 16; ++j) part += red[j * 16 + threadIdx.x];
      const int64_t row = g * 16 + threadIdx.x;
      double sq = 0.0;
      sq += row < R ? part : 0.0;
      const int m = row < R ? row_exponent(sq, gamma_bits) : 0;
      mu[row] = m;
      double s1v, s2v;
      pow2_pair(m, s1v, s2v);
      sc[threadIdx.x] = s1v;
      sc[16 + threadIdx.x] = s2v;
    }
    __syncthreads();
    const int r = BF ? (lane & 15) : (lane >> 1), h = BF ? (lane >> 4) : (lane & 1);
    const double s1 = sc[r], s2 = sc[16 + r];
    constexpr int ES = BF ? 2 : 1;  // bytes per residue
    const int64_t lstride = Rpad * KP * ES;
    for (int kb = warp; kb < KB; kb += kShortThreads / 32) {
      uint8_t* row = res + ((g * 16 + r) * KP + kb * 32) * ES;
      if (ok && BF) {
        convert_stage_bf16<L, KM>(tiles + kb * kConvTile, r, h, s1, s2, row, lstride);
      } else if (ok) {
        convert_stage_i8<L, KM>(tiles + kb * kConvTile, r, h, s1, s2, row + 16 * h, lstride);
      } else {
        for (int l = 0; l < L; ++l)
          for (int e = 0; e < ES; ++e)
            reinterpret_cast<uint4*>(row + 16 * h * ES + l * lstride)[e] = make_uint4(0, 0, 0, 0);
      }
    }
    __syncthreads();  // the tiles (and sc, red) are consumed before the next group
  }
}

// Residues of 16-row panels whose rows are scaled over their full (short)
// k range, one CTA per panel: element (k, r) of panel p at
// src[p * panel_stride + k * ks + r]. Used for the rotation's A (grid-packed
// Psi, rows = grid points, k = bands: panel_stride nb*16, ks 16) and B
// (Q row-major, rows = columns of Q, k = rows of Q: panel_stride 16, ks nb).
template <int L, bool BF>
__global__ void __launch_bounds__(256) convert_local_kernel(
    int64_t R, int64_t K, int64_t KP, int64_t Rpad, const double* __restrict__ src,
    int64_t panel_stride, int64_t ks, uint8_t* __restrict__ res, int* __restrict__ mu_out) {
  __shared__ double tileT[16 * kTilePitch];
  __shared__ double red[256];
  __shared__ double s1[16], s2[16];
  const int64_t p = blockIdx.x;
  const int64_t rem = R - p * 16;
  const int rows_valid = rem <= 0 ? 0 : (int)(rem < 16 ? rem : 16);
  const double* base = src + p * panel_stride;
  {
    const int r = threadIdx.x & 15, kl = threadIdx.x >> 4;
    double acc = 0.0;
    if (r < rows_valid)
      for (int64_t k = kl; k < K; k += 16) {
        const double v = base[k * ks + r];
        acc = fma(v, v, acc);
      }
    red[threadIdx.x] = acc;
  }
  __syncthreads();
  if (threadIdx.x < 16) {
    double sq = 0.0;
    for (int j = 0; j < 16; ++j) sq += red[j * 16 + threadIdx.x];
    const int m = threadIdx.x < rows_valid ? row_exponent(sq, c_res[L].gamma_bits) : 0;
    pow2_pair(m, s1[threadIdx.x], s2[threadIdx.x]);
    if (p * 16 + threadIdx.x < Rpad) mu_out[p * 16 + threadIdx.x] = m;
  }
  const int kk = threadIdx.x & 15, r = threadIdx.x >> 4;
  for (int64_t k0 = 0; k0 < KP; k0 += 128) {
    __syncthreads();
    stage_tile<16>(tileT, base, ks, k0, K, rows_valid);
    __syncthreads();
    Digits d[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      d[j] = digits_of<L>(tileT[r * kTilePitch + swz_k(8 * kk + j)], s1[r], s2[r]);
    if (BF) {
      uint8_t* dst = res + ((p * 16 + r) * KP + k0 + 8 * kk) * 2;
#pragma unroll
      for (int l = 0; l < L; ++l) {
        uint32_t w[4];  // w[i]: elements 2i, 2i + 1
#pragma unroll
        for (int i = 0; i < 4; ++i)
          w[i] = l == 0 ? pack2(low_byte_bf16(d[2 * i]), low_byte_bf16(d[2 * i + 1]))
                        : residue_bf16x2<L>(d[2 * i], d[2 * i + 1], l);
        *reinterpret_cast<uint4*>(dst + (int64_t)l * Rpad * KP * 2) =
            make_uint4(w[0], w[1], w[2], w[3]);
      }
      continue;
    }
    uint8_t* dst = res + (p * 16 + r) * KP + k0 + 8 * kk;
    *reinterpret_cast<uint2*>(dst) = make_uint2(pack4(d[0].lo, d[1].lo, d[2].lo, d[3].lo),
                                                pack4(d[4].lo, d[5].lo, d[6].lo, d[7].lo));
#pragma unroll
    for (int l = 1; l < L; ++l) {
      uint32_t b[8];
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        const uint2 v = residue_byte2<L>(d[j], d[j + 1], l);
        b[j] = v.x;
        b[j + 1] = v.y;
      }
      *reinterpret_cast<uint2*>(dst + (int64_t)l * Rpad * KP) =
          make_uint2(pack4(b[0], b[1], b[2], b[3]), pack4(b[4], b[5], b[6], b[7]));
    }
  }
}

// ------------------------------------------------------- reconstruction
// r[] holds the L non-negative residues (entries >= L are ignored).
__device__ __forceinline__ double crt_value(const uint32_t (&r)[kI8MaxModuli], int L) {
  const CrtConsts& c = c_crt[L];
  double sh = 0.0, sl = 0.0;
#pragma unroll
  for (int l = 0; l < kI8MaxModuli; ++l) {
    if (l < L) {
      const double rd = (double)r[l];
      sh = fma(rd, c.wh[l], sh);  // exact: 8-bit x 40-bit on a common grid
      sl = fma(rd, c.wl[l], sl);
    }
  }
  const double q = rint((sh + sl) * c.inv_m);
  return fma(-q, c.mh, sh) + fma(-q, c.ml, sl);
}

__device__ __forceinline__ double pow2i(int e) {  // 2^e, e in [-1022, 1023]
  return __longlong_as_double((long long)(e + 1023) << 52);
}

// GEMM / SYRK: out(i, j) from the int32 partial slabs of the lane schedule.
// mode 0: D[i*ldd + j] = alpha*v + gamma; mode 1 (SYRK, i <= j only):
// C[i + j*ldd] = alpha*v + beta*C (beta_zero: no read).
__global__ void __launch_bounds__(256) crt_partials_kernel(
    int M, int N, int L, const int32_t* __restrict__ partials, int T,
    const int* __restrict__ tile_index, int tiles_n, const int* __restrict__ mod_slot_off,
    const int* __restrict__ mod_slots, const int* __restrict__ mu, const int* __restrict__ nu,
    int mode, double* __restrict__ D, int64_t ldd, double alpha, double gamma, int beta_zero) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)M * N) return;
  const int i = (int)(idx / N), j = (int)(idx % N);
  if (mode == 1 && i > j) return;
  const int t = tile_index[(i / kI8BM) * tiles_n + j / kI8BN];
  const int64_t off = (int64_t)(i % kI8BM) * kI8BN + (j % kI8BN);
  uint32_t r[kI8MaxModuli];
#pragma unroll
  for (int l = 0; l < kI8MaxModuli; ++l) {
    r[l] = 0;
    if (l < L) {
      int64_t s = 0;
      for (int q = mod_slot_off[l]; q < mod_slot_off[l + 1]; ++q)
        s += partials[((int64_t)mod_slots[q] * T + t) * (kI8BM * kI8BN) + off];
      // s mod m without an integer division: |s| < 2^31 * (slots) is exact in
      // a double, floor(s * fl(1/m)) is the true quotient or one off (the
      // product's error is below 2^-20), and one correction step each way
      // makes the remainder exact.
      const int64_t m = c_res[L].mi[l];
      const int64_t q = (int64_t)floor((double)s * c_inv_mod[l]);
      int64_t rr = s - q * m;
      rr += rr < 0 ? m : 0;
      rr -= rr >= m ? m : 0;
      r[l] = (uint32_t)rr;
    }
  }
  const double x = crt_value(r, L);
  const int ex = -(mu[i] + nu[j]);
  const double v = (ex >= -1022 && ex <= 1023) ? x * pow2i(ex) : ldexp(ldexp(x, -mu[i]), -nu[j]);
  if (mode == 0) {
    D[(int64_t)i * ldd + j] = alpha * v + gamma;
  } else {
    double* c = D + i + (int64_t)j * ldd;
    *c = beta_zero ? alpha * v : alpha * v + gamma * (*c);
  }
}

// Rotation: Psi'(g, b) band-packed from the residue bytes res[l][g][ldr].
// Thread (g, c): the 16 states of chunk c at grid point g. All L 16-byte
// residue loads are issued before any arithmetic (the kernel is bound by
// their latency otherwise); bytes widen to doubles exactly (2^52 + r - 2^52).
// The scale 2^-(mu[g] + nu[b]) is built from exponent bits (four 16-byte
// loads of nu per thread).

template <int L>
__global__ void __launch_bounds__(128) crt_residues_band_kernel(
    int64_t Nd, int64_t nb, const uint8_t* __restrict__ res, int64_t ldr,
    const int* __restrict__ mu, const int* __restrict__ nu, double* __restrict__ Dband) {
  // Thread (g, c, hf): states 16 c + 8 hf .. + 8 at grid point g (hf fastest:
  // a lane pair writes one whole 128-byte line of the band-packed output).
  const int64_t halves = nb / 8;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= Nd * halves) return;
  const int64_t g = idx / halves, hc = idx % halves;
  const int64_t c = hc >> 1, hf = hc & 1;
  const CrtConsts& cc = c_crt[L];
  uint2 v[L];
#pragma unroll
  for (int l = 0; l < L; ++l)
    v[l] = __ldcs(reinterpret_cast<const uint2*>(res + ((int64_t)l * Nd + g) * ldr + hc * 8));
  int e[8];
  {
    const int4* n4 = reinterpret_cast<const int4*>(nu + hc * 8);
    const int4 t0 = __ldg(n4), t1 = __ldg(n4 + 1);
    e[0] = t0.x; e[1] = t0.y; e[2] = t0.z; e[3] = t0.w;
    e[4] = t1.x; e[5] = t1.y; e[6] = t1.z; e[7] = t1.w;
  }
  const int mg = mu[g];
  double out[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    double sh = 0.0, sl = 0.0;
#pragma unroll
    for (int l = 0; l < L; ++l) {
      const uint32_t w = t < 4 ? v[l].x : v[l].y;
      const double d =
          __hiloint2double(0x43300000, (int)((w >> (8 * (t & 3))) & 0xFFu)) - 4503599627370496.0;
      sh = fma(d, cc.wh[l], sh);  // exact: 8-bit x 40-bit on a common grid
      sl = fma(d, cc.wl[l], sl);
    }
    const double q = rint((sh + sl) * cc.inv_m);
    const double x = fma(-q, cc.mh, sh) + fma(-q, cc.ml, sl);
    const int ex = -(mg + e[t]);
    out[t] = (ex >= -1022 && ex <= 1023) ? x * pow2i(ex) : ldexp(ldexp(x, -mg), -e[t]);
  }
  double2* dst = reinterpret_cast<double2*>(Dband + (c * Nd + g) * 16 + hf * 8);
#pragma unroll
  for (int t = 0; t < 4; ++t) __stcs(dst + t, make_double2(out[2 * t], out[2 * t + 1]));
}

template <int L>
int launch_crt_band(int64_t Nd, int64_t nb, const uint8_t* res, const int* mu, const int* nu,
                    double* D, cudaStream_t s) {
  const int64_t n = Nd * (nb / 8);
  KernelTimer kt_(s, "crt_residues_band_kernel");
  crt_residues_band_kernel<L><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(Nd, nb, res, nb, mu,
                                                                          nu, D);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

// Exact INT8 GEMM output: C[i*ldc + j] = sum over slots of the partial slabs.
__global__ void __launch_bounds__(256) sum_partials_kernel(
    int M, int N, const int32_t* __restrict__ partials, int T, const int* __restrict__ tile_index,
    int tiles_n, const int* __restrict__ mod_slot_off, const int* __restrict__ mod_slots,
    int32_t* __restrict__ C, int64_t ldc) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)M * N) return;
  const int i = (int)(idx / N), j = (int)(idx % N);
  const int t = tile_index[(i / kI8BM) * tiles_n + j / kI8BN];
  const int64_t off = (int64_t)(i % kI8BM) * kI8BN + (j % kI8BN);
  int64_t s = 0;
  for (int q = mod_slot_off[0]; q < mod_slot_off[1]; ++q)
    s += partials[((int64_t)mod_slots[q] * T + t) * (kI8BM * kI8BN) + off];
  C[(int64_t)i * ldc + j] = (int32_t)s;
}

// ------------------------------------------------------------- host side
struct LanePlan {
  int T = 0, T1 = 0, Q = 0, slots = 0, L = 0, KB = 0, tiles_m = 0, tiles_n = 0;
  int T2 = 0;              // CTA-pair plans: pair tiles (0: one-CTA plan)
  int4* pairs = nullptr;   // [T2] {tm_lo, tn, t_lo, t_hi}
  // tiles | lane_seg_off | segs | tile_index | mod_slot_off | mod_slots | tile_index2
  DeviceBuffer buf;
  int2* tiles = nullptr;
  int* lane_seg_off = nullptr;
  I8Segment* segs = nullptr;
  int* tile_index = nullptr;
  int* tile_index2 = nullptr;  // fused pair: the GEMM's tiles (t >= T1)
  int* mod_slot_off = nullptr;
  int* mod_slots = nullptr;
};

struct OzakiStream {
  DeviceBuffer res_a, res_b, part_a, part_b, mu_a, mu_b, partials, rbytes;
  cudaEvent_t fork2 = nullptr, join2 = nullptr;
  // Helper stream forked from the caller's stream: the norm pass of B runs
  // there while A is converted (the conversion leaves HBM bandwidth idle).
  cudaStream_t aux = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};

struct OzakiDevice {
  bool consts_ready = false;
  std::map<std::tuple<int, int, int, int, int>, LanePlan*> plans;  // (M, N, KB, L, syrk)
  std::map<cudaStream_t, OzakiStream*> streams;
};

std::mutex g_oz_mu;
OzakiDevice g_oz[64];
I8ModConsts g_modc;
bool g_modc_ready = false;


int ensure_consts(DeviceState* dev) {
  OzakiDevice& od = g_oz[dev->device];
  if (od.consts_ready) return SKGEMM_OK;
  ResidueConsts rc[kI8MaxModuli + 1];
  memset(rc, 0, sizeof(rc));
  for (int L = kMinModuli; L <= kI8MaxModuli; ++L) {
    rc[L].gamma_bits = gamma_for(L);
    for (int l = 0; l < kI8MaxModuli; ++l) {
      const uint64_t m = kModuli[l];
      uint64_t pj = 1;
      for (int j = 0; j < 4; ++j) {
        pj = (pj * 4096) % m;
        rc[L].c[j][l] = (float)pj;  // 2^(12 (j+1)) mod m
      }
      uint64_t p14 = 1;
      for (int j = 0; j < 3; ++j) {
        p14 = (p14 * 16384) % m;
        const int64_t sym = p14 > m / 2 ? (int64_t)p14 - (int64_t)m : (int64_t)p14;
        rc[L].cs[j][l] = (float)sym;  // 2^(14 (j+1)) mod m in (-m/2, m/2]
      }
      rc[L].inv[l] = 1.0f / (float)m;
      rc[L].m[l] = (float)m;
      rc[L].mi[l] = (uint32_t)m;
      for (int j = 0; j < 4; ++j) {
        const float c = L <= kShortDigitsMaxL ? (j < 3 ? rc[L].cs[j][l] : 0.0f) : rc[L].c[j][l];
        rc[L].pc[j][l] = make_float2(c, c);
      }
      rc[L].pinv[l] = make_float2(rc[L].inv[l], rc[L].inv[l]);
      rc[L].pnm[l] = make_float2(-rc[L].m[l], -rc[L].m[l]);
    }
  }
  for (int l = 0; l < kI8MaxModuli; ++l) {
    g_modc.m[l] = kModuli[l];
    g_modc.magic[l] = (uint32_t)((1ull << 37) / kModuli[l] + 1);
    g_modc.offset[l] = (uint32_t)((((1u << 25) + kModuli[l] - 1) / kModuli[l]) * kModuli[l]);
    const uint32_t acc24 = 512u * 127u * 127u;  // |acc| bound for K <= 512, odd m
    g_modc.magic24[l] = (uint32_t)(((1ull << 32) + kModuli[l] - 1) / kModuli[l]);
    g_modc.offset24[l] = (uint32_t)((acc24 + kModuli[l] - 1) / kModuli[l] * kModuli[l]);
  }
  g_modc_ready = true;
  SKG_CUDA(cudaMemcpyToSymbol(c_i8mod, &g_modc, sizeof(g_modc)));
  CrtConsts cc[kI8MaxModuli + 1];
  memset(cc, 0, sizeof(cc));
  for (int L = kMinModuli; L <= kI8MaxModuli; ++L) cc[L] = make_crt(L, nullptr);
  SKG_CUDA(cudaMemcpyToSymbol(c_res, rc, sizeof(rc)));
  SKG_CUDA(cudaMemcpyToSymbol(c_crt, cc, sizeof(cc)));
  double inv_mod[kI8MaxModuli];
  for (int l = 0; l < kI8MaxModuli; ++l) inv_mod[l] = 1.0 / (double)kModuli[l];
  SKG_CUDA(cudaMemcpyToSymbol(c_inv_mod, inv_mod, sizeof(inv_mod)));
  od.consts_ready = true;
  return SKGEMM_OK;
}

OzakiStream* ozaki_stream(DeviceState* dev, cudaStream_t s) {
  OzakiStream*& o = g_oz[dev->device].streams[s];
  if (!o) o = new OzakiStream();
  if (debug_fill_enabled())  // the call's scratch starts as 0xFF bytes
    for (DeviceBuffer* b : {&o->res_a, &o->res_b, &o->part_a, &o->part_b, &o->mu_a, &o->mu_b,
                            &o->partials, &o->rbytes})
      debug_poison(b->ptr, b->bytes, s);
  return o;
}

// Lanes per tile for T tiles over a (modulus, k-block) space of W blocks on
// `sms` persistent CTAs: the T x Q equal items take ceil(T Q / sms) waves of
// W / Q blocks each, so Q minimises ceil(T Q / sms) / Q; among Q within 2%
// of the best the smallest (fewer slabs) wins. A lane keeps >= 64 k-blocks.
int lanes_for(int sms, int T, int64_t W) {
  const int qmax = (int)std::max<int64_t>(1, std::min<int64_t>(64, W / 64));
  double best = 1e300;
  for (int Q = 1; Q <= qmax; ++Q)
    best = std::min(best, (double)(((int64_t)T * Q + sms - 1) / sms) / Q);
  for (int Q = 1; Q <= qmax; ++Q)
    if ((double)(((int64_t)T * Q + sms - 1) / sms) / Q <= best * 1.02) return Q;
  return 1;
}

// Lane schedule: T tiles x Q lanes, each lane a contiguous range of the
// (modulus, k-block) space, cut into segments at modulus boundaries and at
// seg_cap k-blocks (INT32 exactness).
// With `pair` (M == N) the tile list is the SYRK's upper tiles (t < T1,
// tile_index) followed by all tiles of the GEMM (tile_index2): one launch
// computes S = A^T A and Hs = A^T B from the same A panels.
// With `units` > 0 the plan is for the CTA-pair kernel (i8_gemm2_kernel) on
// `units` co-resident clusters: the tile set is closed under pairing
// (tiles 2p and 2p + 1 of a column), the pair list is built, and the lanes
// are sized for the clusters.
int get_lane_plan(DeviceState* dev, int M, int N, int KB, int L, bool syrk, int seg_cap,
                  LanePlan** out, int sub_cap = 0, bool pair = false, int units = 0) {
  OzakiDevice& od = g_oz[dev->device];
  auto key = std::make_tuple(M, N, KB, (L * 4096 + seg_cap) * 64 + sub_cap,
                             (syrk ? 1 : 0) + (pair ? 2 : 0) + units * 4);
  auto itp = od.plans.find(key);
  if (itp != od.plans.end()) {
    *out = itp->second;
    return SKGEMM_OK;
  }
  LanePlan* pl = new LanePlan();
  pl->L = L;
  pl->KB = KB;
  pl->tiles_m = (M + kI8BM - 1) / kI8BM;
  pl->tiles_n = (N + kI8BN - 1) / kI8BN;
  std::vector<int2> tiles;
  std::vector<int4> pairs;
  std::vector<int> tile_index(pl->tiles_m * pl->tiles_n, -1), tile_index2;
  // Rows of tile tm: 128 tm ..; residue planes are padded to 256 rows, so a
  // pair plan may use tile row tiles_m (padding) as the partner of the last.
  const int tm_span = units > 0 ? (pl->tiles_m + 1) / 2 * 2 : pl->tiles_m;
  auto add_set = [&](bool upper, std::vector<int>& index) {
    if (units == 0) {  // one-CTA plan: row-major tile order
      for (int tm = 0; tm < pl->tiles_m; ++tm)
        for (int tn = 0; tn < pl->tiles_n; ++tn) {
          if (upper && tm * kI8BM > tn * kI8BN + kI8BN - 1) continue;  // strictly lower
          index[tm * pl->tiles_n + tn] = (int)tiles.size();
          tiles.push_back(make_int2(tm, tn));
        }
      return;
    }
    for (int tn = 0; tn < pl->tiles_n; ++tn)
      for (int tm2 = 0; tm2 < tm_span; tm2 += 2) {
        const int span = 2;
        bool need = false;
        for (int h = 0; h < span; ++h) {
          const int tm = tm2 + h;
          if (tm < pl->tiles_m && !(upper && tm * kI8BM > tn * kI8BN + kI8BN - 1)) need = true;
        }
        if (!need) continue;
        int t[2] = {-1, -1};
        for (int h = 0; h < span; ++h) {
          const int tm = tm2 + h;
          t[h] = (int)tiles.size();
          if (tm < pl->tiles_m) index[tm * pl->tiles_n + tn] = t[h];
          tiles.push_back(make_int2(tm, tn));
        }
        pairs.push_back(make_int4(tm2, tn, t[0], t[1]));
      }
  };
  add_set(syrk || pair, tile_index);
  pl->T1 = 0;
  if (pair) {
    pl->T1 = (int)tiles.size();
    tile_index2.assign(pl->tiles_m * pl->tiles_n, -1);
    add_set(false, tile_index2);
  }
  pl->T = (int)tiles.size();
  pl->T2 = (int)pairs.size();
  const int64_t W = (int64_t)L * KB;
  pl->Q = units > 0 ? lanes_for(units, pl->T2, W) : lanes_for(dev->num_sms, pl->T, W);
  std::vector<int> lane_off(pl->Q + 1, 0);
  std::vector<I8Segment> segs;
  int nslots = 0;
  std::vector<std::vector<int>> by_mod(L);
  for (int q = 0; q < pl->Q; ++q) {
    lane_off[q] = (int)segs.size();
    int64_t it = (int64_t)q * W / pl->Q, end = (int64_t)(q + 1) * W / pl->Q;
    while (it < end) {
      const int l = (int)(it / KB);
      int64_t stop = std::min<int64_t>(end, (int64_t)(l + 1) * KB);
      stop = std::min<int64_t>(stop, it + seg_cap);
      // One slot per segment; with sub_cap > 0 the segment is issued as
      // sub-segments of <= sub_cap k-blocks that accumulate into that slot.
      const int slot = nslots++;
      const int step = sub_cap > 0 ? sub_cap : (int)(stop - it);
      for (int64_t a = it; a < stop; a += step) {
        I8Segment sg;
        sg.l = l;
        sg.kb0 = (int)(a - (int64_t)l * KB);
        sg.kb1 = (int)(std::min<int64_t>(stop, a + step) - (int64_t)l * KB);
        sg.slot = slot;
        segs.push_back(sg);
      }
      by_mod[l].push_back(slot);
      it = stop;
    }
  }
  lane_off[pl->Q] = (int)segs.size();
  pl->slots = nslots;
  std::vector<int> mod_off(L + 1, 0), mod_slots;
  for (int l = 0; l < L; ++l) {
    mod_off[l] = (int)mod_slots.size();
    mod_slots.insert(mod_slots.end(), by_mod[l].begin(), by_mod[l].end());
  }
  mod_off[L] = (int)mod_slots.size();
  // one device buffer, 16-byte aligned sections
  auto al = [](size_t x) { return (x + 15) / 16 * 16; };
  const size_t s0 = al(tiles.size() * sizeof(int2)), s1 = al(lane_off.size() * sizeof(int)),
               s2 = al(segs.size() * sizeof(I8Segment)), s3 = al(tile_index.size() * sizeof(int)),
               s4 = al(mod_off.size() * sizeof(int)), s5 = al(mod_slots.size() * sizeof(int) + 4),
               s6 = al(tile_index2.size() * sizeof(int) + 4),
               s7 = al(pairs.size() * sizeof(int4) + 16);
  int st;
  if ((st = pl->buf.ensure(s0 + s1 + s2 + s3 + s4 + s5 + s6 + s7)) != SKGEMM_OK) {
    delete pl;
    return st;
  }
  uint8_t* b = static_cast<uint8_t*>(pl->buf.ptr);
  std::vector<uint8_t> host(s0 + s1 + s2 + s3 + s4 + s5 + s6 + s7, 0);
  if (!pairs.empty())
    memcpy(host.data() + s0 + s1 + s2 + s3 + s4 + s5 + s6, pairs.data(),
           pairs.size() * sizeof(int4));
  if (!tile_index2.empty())
    memcpy(host.data() + s0 + s1 + s2 + s3 + s4 + s5, tile_index2.data(),
           tile_index2.size() * sizeof(int));
  memcpy(host.data(), tiles.data(), tiles.size() * sizeof(int2));
  memcpy(host.data() + s0, lane_off.data(), lane_off.size() * sizeof(int));
  memcpy(host.data() + s0 + s1, segs.data(), segs.size() * sizeof(I8Segment));
  memcpy(host.data() + s0 + s1 + s2, tile_index.data(), tile_index.size() * sizeof(int));
  memcpy(host.data() + s0 + s1 + s2 + s3, mod_off.data(), mod_off.size() * sizeof(int));
  memcpy(host.data() + s0 + s1 + s2 + s3 + s4, mod_slots.data(), mod_slots.size() * sizeof(int));
  SKG_CUDA(cudaMemcpy(b, host.data(), host.size(), cudaMemcpyHostToDevice));
  pl->tiles = reinterpret_cast<int2*>(b);
  pl->lane_seg_off = reinterpret_cast<int*>(b + s0);
  pl->segs = reinterpret_cast<I8Segment*>(b + s0 + s1);
  pl->tile_index = reinterpret_cast<int*>(b + s0 + s1 + s2);
  pl->mod_slot_off = reinterpret_cast<int*>(b + s0 + s1 + s2 + s3);
  pl->mod_slots = reinterpret_cast<int*>(b + s0 + s1 + s2 + s3 + s4);
  pl->tile_index2 = pair ? reinterpret_cast<int*>(b + s0 + s1 + s2 + s3 + s4 + s5) : nullptr;
  pl->pairs = units > 0 ? reinterpret_cast<int4*>(b + s0 + s1 + s2 + s3 + s4 + s5 + s6) : nullptr;
  od.plans[key] = pl;
  *out = pl;
  return SKGEMM_OK;
}

int make_res_map(CUtensorMap* map, const void* base, int64_t KP, int64_t Rpad, int L,
                 int box_rows) {
  uint64_t dims[3] = {(uint64_t)KP, (uint64_t)Rpad, (uint64_t)L};
  uint64_t strides[2] = {(uint64_t)KP, (uint64_t)(KP * Rpad)};
  uint32_t box[3] = {128, (uint32_t)box_rows, 1};
  return encode_tiled(map, 3, base, dims, strides, box, CU_TENSOR_MAP_DATA_TYPE_UINT8,
                      CU_TENSOR_MAP_SWIZZLE_128B);
}

template <bool BF>
int launch_i8_t(DeviceState* dev, const CUtensorMap& mA, const CUtensorMap& mB,
                const CUtensorMap& mB2, const I8Params& p, int grid, cudaStream_t s) {
  static bool attr_done[64] = {false};
  if (!attr_done[dev->device]) {
    SKG_CUDA(cudaFuncSetAttribute(i8_gemm_kernel<BF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kI8SmemBytes));
    attr_done[dev->device] = true;
  }
  KernelTimer kt_(s, "i8_gemm_kernel");
  i8_gemm_kernel<BF><<<grid, kI8Threads, kI8SmemBytes, s>>>(mA, mB, mB2, p);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

// CTA-pair lanes kernel: on unless SKGEMM_LANES_PAIR=0 selects the one-CTA
// kernel (same slabs, same results bit for bit; kept for comparison).
bool lanes_pair_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("SKGEMM_LANES_PAIR");
    v = (e && e[0] == '0') ? 0 : 1;
  }
  return v == 1;
}

cudaLaunchConfig_t pair_config(int grid, cudaStream_t s, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kI8Threads);
  cfg.dynamicSmemBytes = kI8P2SmemBytes;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <bool BF>
int pair_setup(DeviceState* dev, int* clusters) {
  static int ncl[64] = {0};
  if (!ncl[dev->device]) {
    SKG_CUDA(cudaFuncSetAttribute(i8_gemm2_kernel<BF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kI8P2SmemBytes));
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t cfg = pair_config(2 * (dev->num_sms / 2), nullptr, attr);
    int n = 0;
    SKG_CUDA(cudaOccupancyMaxActiveClusters(&n, (const void*)i8_gemm2_kernel<BF>, &cfg));
    if (n < 1) return fail(SKGEMM_ERR_CUDA, "INT8 pair kernel: no cluster of two fits");
    ncl[dev->device] = n;
  }
  *clusters = ncl[dev->device];
  return SKGEMM_OK;
}

// Co-resident clusters of the pair kernel on this device (0: pair kernel off).
int lanes_pair_units(DeviceState* dev, bool bf) {
  if (!lanes_pair_enabled()) return 0;
  int n = 0;
  if ((bf ? pair_setup<true>(dev, &n) : pair_setup<false>(dev, &n)) != SKGEMM_OK) return 0;
  return n;
}

template <bool BF>
int launch_i8_pair_t(const CUtensorMap& mA, const CUtensorMap& mB, const CUtensorMap& mB2,
                     const I8Params& p, int clusters, cudaStream_t s) {
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = pair_config(2 * clusters, s, attr);
  KernelTimer kt_(s, "i8_gemm2_kernel");
  SKG_CUDA(cudaLaunchKernelEx(&cfg, i8_gemm2_kernel<BF>, mA, mB, mB2, p));
  return SKGEMM_OK;
}

// INT8 (bf = false) or BF16 (bf = true) residue products.
int launch_i8(DeviceState* dev, const CUtensorMap& mA, const CUtensorMap& mB, const I8Params& p,
              int grid, cudaStream_t s, bool bf = false, const CUtensorMap* mB2 = nullptr) {
  const CUtensorMap& b2 = mB2 ? *mB2 : mB;
  return bf ? launch_i8_t<true>(dev, mA, mB, b2, p, grid, s)
            : launch_i8_t<false>(dev, mA, mB, b2, p, grid, s);
}

// The lanes products of plan `pl`: the CTA-pair kernel when the plan was
// built for it (B boxes of 128 rows), the one-CTA kernel otherwise (B boxes
// of 256 rows). `p` holds everything but the plan's tile / pair fields.
int launch_lanes(DeviceState* dev, const LanePlan* pl, const void* resA, int64_t KPb, int64_t RA,
                 const void* resB, int64_t RB, const void* resB2, I8Params p, cudaStream_t s,
                 bool bf) {
  int st;
  const bool pair_k = pl->T2 > 0;
  CUtensorMap mA, mB, mB2;
  if ((st = make_res_map(&mA, resA, KPb, RA, p.L, kI8BM))) return st;
  if ((st = make_res_map(&mB, resB, KPb, RB, p.L, pair_k ? 128 : kI8BN))) return st;
  if (resB2 && (st = make_res_map(&mB2, resB2, KPb, RB, p.L, pair_k ? 128 : kI8BN))) return st;
  p.T = pl->T;
  p.T1 = pl->T1;
  p.Q = pl->Q;
  p.tiles = pl->tiles;
  p.lane_seg_off = pl->lane_seg_off;
  p.segs = pl->segs;
  p.T2 = pl->T2;
  p.pairs = pl->pairs;
  if (!pair_k)
    return launch_i8(dev, mA, mB, p, std::min(dev->num_sms, pl->T * pl->Q), s, bf,
                     resB2 ? &mB2 : nullptr);
  int ncl = 0;
  if ((st = bf ? pair_setup<true>(dev, &ncl) : pair_setup<false>(dev, &ncl))) return st;
  ncl = std::min(ncl, pl->T2 * pl->Q);
  const CUtensorMap& b2 = resB2 ? mB2 : mB;
  return bf ? launch_i8_pair_t<true>(mA, mB, b2, p, ncl, s)
            : launch_i8_pair_t<false>(mA, mB, b2, p, ncl, s);
}

int launch_i8_rot(DeviceState* dev, const CUtensorMap& mA, const CUtensorMap& mB,
                  const CUtensorMap& mR, const I8RotParams& p, int grid, cudaStream_t s) {
  static bool attr_done[64] = {false};
  if (!attr_done[dev->device]) {
    SKG_CUDA(cudaFuncSetAttribute(i8_rot_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  kI8RotSmemBytes));
    attr_done[dev->device] = true;
  }
  KernelTimer kt_(s, "i8_rot_kernel");
  i8_rot_kernel<<<grid, kI8Threads, kI8RotSmemBytes, s>>>(mA, mB, mR, p);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

bool is_bf16(const skgemm_options_t* opts) {
  return opts && opts->precision == SKGEMM_PREC_OZAKI_BF16;
}

int choose_L(const skgemm_options_t* opts, int64_t K, int* L_out, int* gamma_out) {
  if (opts && opts->precision != SKGEMM_PREC_OZAKI_I8 && opts->precision != SKGEMM_PREC_OZAKI_BF16)
    return fail(SKGEMM_ERR_INVALID_ARG, "precision must be native, Ozaki INT8 or Ozaki BF16");
  int L = opts ? opts->slices : 0;
  if (L == 0) {
    // Smallest L whose error estimate for random-sign data,
    // sqrt(K/12) * 2^(1-gamma) relative, stays below 3e-14 (a factor of three
    // under the 1e-13 gate).
    L = kMinModuli;
    while (L < kI8MaxModuli &&
           std::sqrt((double)K / 12.0) * std::ldexp(2.0, -gamma_for(L)) > 3e-14)
      ++L;
  }
  if (L < kMinModuli || L > kI8MaxModuli)
    return fail(SKGEMM_ERR_INVALID_ARG, "Ozaki moduli count must be in [6, 16]");
  *L_out = L;
  *gamma_out = gamma_for(L);
  return SKGEMM_OK;
}

void report(skgemm_options_t* opts, int L, int gamma_bits, int64_t K) {
  if (!opts) return;
  opts->slices_used_out = L;
  opts->err_bound_out = 2.0 * std::sqrt((double)K / 12.0) * std::ldexp(1.0, -gamma_bits);
}

// L-dispatch of a launcher template (L in [kMinModuli, 16]).
#define SKG_DISPATCH_L(L, CALL)                                                  \
  switch (L) {                                                                   \
    case 6: { constexpr int LL = 6; return CALL; }                               \
    case 7: { constexpr int LL = 7; return CALL; }                               \
    case 8: { constexpr int LL = 8; return CALL; }                               \
    case 9: { constexpr int LL = 9; return CALL; }                               \
    case 10: { constexpr int LL = 10; return CALL; }                             \
    case 11: { constexpr int LL = 11; return CALL; }                             \
    case 12: { constexpr int LL = 12; return CALL; }                             \
    case 13: { constexpr int LL = 13; return CALL; }                             \
    case 14: { constexpr int LL = 14; return CALL; }                             \
    case 15: { constexpr int LL = 15; return CALL; }                             \
    case 16: { constexpr int LL = 16; return CALL; }                             \
    default: return fail(SKGEMM_ERR_INVALID_ARG, "moduli count out of range");   \
  }

template <int T, int L, bool BF, bool KM = false>
int launch_convert(DeviceState* dev, const CUtensorMap& map, int64_t KP, int64_t Rpad,
                   const int* mu, uint8_t* res, uint32_t* err, cudaStream_t s) {
  static int occ[64] = {0};
  if (!occ[dev->device]) {
    SKG_CUDA(cudaFuncSetAttribute(convert_tma_kernel<T, L, BF, KM>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, kConvSmem));
    int n = 0;
    SKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, convert_tma_kernel<T, L, BF, KM>,
                                                           256, kConvSmem));
    occ[dev->device] = n > 0 ? n : 1;
  }
  const int64_t ntiles = (Rpad / 16) * (KP / 32);
  const int64_t blocks = std::min<int64_t>((ntiles + kConvWarps - 1) / kConvWarps,
                                           (int64_t)dev->num_sms * occ[dev->device]);
  // (every warp of the grid gets at least one tile only if ntiles >= warps;
  // warps without a tile return at once)
  KernelTimer kt_(s, "convert_tma_kernel");
  convert_tma_kernel<T, L, BF, KM><<<(unsigned)blocks, 256, kConvSmem, s>>>(map, KP, Rpad, mu,
                                                                            res, err);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

// Residues of a packed-T operand (rows R, reduction K) into res[L][Rpad][KP]
// plus row exponents, in two steps: prep_norms (norm partials, then the row
// exponents) and prep_convert (the TMA-fed conversion). The steps may run on
// different streams with an event between them.
template <int L, bool KM, bool BF>
int launch_short_L(DeviceState* dev, const CUtensorMap& map, int64_t R, int64_t K, int64_t KP,
                   int64_t Rpad, int* mu, uint8_t* res, uint32_t* err, cudaStream_t s) {
  static bool attr_done[64] = {false};
  if (!attr_done[dev->device]) {
    SKG_CUDA(cudaFuncSetAttribute(convert_short_kernel<L, KM, BF>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, kShortSmem));
    attr_done[dev->device] = true;
  }
  const int64_t G = Rpad / 16;
  const int64_t grid = std::min<int64_t>(G, 3 * (int64_t)dev->num_sms);  // three CTAs per SM
  KernelTimer kt_(s, "convert_short_kernel");
  convert_short_kernel<L, KM, BF><<<(unsigned)grid, kShortThreads, kShortSmem, s>>>(map, R, K, KP, Rpad,
                                                                  gamma_for(L), mu, res, err);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

template <int T>
int prep_norms(int64_t R, int64_t K, int64_t KP, int64_t Rpad, const double* X, int L,
               DeviceBuffer& res, DeviceBuffer& part, DeviceBuffer& mu, cudaStream_t s,
               bool bf = false, bool km = false) {
  if ((reinterpret_cast<uintptr_t>(X) & 15) != 0)
    return fail(SKGEMM_ERR_INVALID_ARG, "operand base must be 16-byte aligned");
  if (K > ((int64_t)1 << 31) - 128) return fail(SKGEMM_ERR_INVALID_ARG, "K too large");
  const int64_t P_in = (R + T - 1) / T;
  const int C = (int)std::max<int64_t>(1, std::min<int64_t>(64, (600 + P_in - 1) / P_in));
  int st;
  if ((st = res.ensure((size_t)L * Rpad * KP * (bf ? 2 : 1))) != SKGEMM_OK) return st;
  if ((st = part.ensure((size_t)P_in * C * T * sizeof(double))) != SKGEMM_OK) return st;
  if ((st = mu.ensure((size_t)Rpad * sizeof(int))) != SKGEMM_OK) return st;
  if (km && T != 16) return fail(SKGEMM_ERR_INVALID_ARG, "K-major operand with 32-wide panels");
  {
    KernelTimer kt_(s, "norm_partials_kernel");
    if (km)
      norm_partials_kernel<16, true><<<dim3((unsigned)P_in, C), 256, 0, s>>>(R, K, X, C,
                                                                            (double*)part.ptr);
    else
      norm_partials_kernel<T><<<dim3((unsigned)P_in, C), 256, 0, s>>>(R, K, X, C,
                                                                      (double*)part.ptr);
  }
  SKG_CUDA(cudaGetLastError());
  KernelTimer kt_(s, "row_exponents_kernel");
  row_exponents_kernel<T><<<(unsigned)((Rpad + 255) / 256), 256, 0, s>>>(
      R, Rpad, C, (const double*)part.ptr, gamma_for(L), (int*)mu.ptr);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

template <int T>
int prep_convert(DeviceState* dev, int64_t R, int64_t K, int64_t KP, int64_t Rpad,
                 const double* X, int L, DeviceBuffer& res, DeviceBuffer& mu, uint32_t* err,
                 cudaStream_t s, bool bf = false, bool km = false) {
  CUtensorMap map;
  const int* mp = (const int*)mu.ptr;
  uint8_t* rp = (uint8_t*)res.ptr;
  if (km) {
    // K-major [K/16][R][16] (T = 16, K % 16 == 0): boxes {16 k, 16 rows, 2
    // k-blocks}, zero fill past R and past the last k-block.
    if (T != 16 || K % 16) return fail(SKGEMM_ERR_INVALID_ARG, "K-major operand layout");
    const uint64_t dims[3] = {16, (uint64_t)R, (uint64_t)(K / 16)};
    const uint64_t strides[2] = {16 * 8, (uint64_t)R * 16 * 8};
    const uint32_t box[3] = {16, 16, 2};
    int st;
    if ((st = encode_tiled(&map, 3, X, dims, strides, box, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                           CU_TENSOR_MAP_SWIZZLE_128B)))
      return st;
    if (bf) {
      SKG_DISPATCH_L(L, (launch_convert<16, LL, true, true>(dev, map, KP, Rpad, mp, rp, err, s)))
    }
    SKG_DISPATCH_L(L, (launch_convert<16, LL, false, true>(dev, map, KP, Rpad, mp, rp, err, s)))
  }
  // [P_in][K][T] doubles; boxes of 16 rows x 32 k (zero fill past K / P_in).
  const int64_t P_in = (R + T - 1) / T;
  const uint64_t dims[3] = {(uint64_t)T, (uint64_t)K, (uint64_t)P_in};
  const uint64_t strides[2] = {(uint64_t)T * 8, (uint64_t)K * T * 8};
  const uint32_t box[3] = {16, 32, 1};
  int st;
  if ((st = encode_tiled(&map, 3, X, dims, strides, box, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         bf ? CU_TENSOR_MAP_SWIZZLE_NONE : CU_TENSOR_MAP_SWIZZLE_128B)))
    return st;
  if (bf) {
    SKG_DISPATCH_L(L, (launch_convert<T, LL, true>(dev, map, KP, Rpad, mp, rp, err, s)))
  }
  SKG_DISPATCH_L(L, (launch_convert<T, LL, false>(dev, map, KP, Rpad, mp, rp, err, s)))
}

template <int T>
int prep_packed(DeviceState* dev, int64_t R, int64_t K, int64_t KP, int64_t Rpad,
                const double* X, int L, DeviceBuffer& res, DeviceBuffer& part, DeviceBuffer& mu,
                uint32_t* err, cudaStream_t s, bool bf = false, bool km = false) {
  int st;
  // Short rows (K <= 512) and a one-chunk norm pass (ceil(R/16) >= 600): one
  // pass, convert_short_kernel (same exponents and residues bit for bit),
  // for the packed16 layout and its K-major form.
  if (T == 16 && KP <= 32 * kShortKbMax && (R + 15) / 16 >= 600 && (!km || K % 16 == 0)) {
    if ((reinterpret_cast<uintptr_t>(X) & 15) != 0)
      return fail(SKGEMM_ERR_INVALID_ARG, "operand base must be 16-byte aligned");
    if ((st = res.ensure((size_t)L * Rpad * KP * (bf ? 2 : 1)))) return st;
    if ((st = mu.ensure((size_t)Rpad * sizeof(int)))) return st;
    CUtensorMap map;
    if (km) {
      // [K/16][R][16]: boxes {16 k, 16 rows, 2 k-blocks} (the conversion
      // kernel's K-major stage).
      const uint64_t dims[3] = {16, (uint64_t)R, (uint64_t)(K / 16)};
      const uint64_t strides[2] = {16 * 8, (uint64_t)R * 16 * 8};
      const uint32_t box[3] = {16, 16, 2};
      if ((st = encode_tiled(&map, 3, X, dims, strides, box, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                             CU_TENSOR_MAP_SWIZZLE_128B)))
        return st;
      if (bf) {
        SKG_DISPATCH_L(L, (launch_short_L<LL, true, true>(dev, map, R, K, KP, Rpad, (int*)mu.ptr,
                                                          (uint8_t*)res.ptr, err, s)))
      }
      SKG_DISPATCH_L(L, (launch_short_L<LL, true, false>(dev, map, R, K, KP, Rpad, (int*)mu.ptr,
                                                         (uint8_t*)res.ptr, err, s)))
    }
    const int64_t P_in = (R + 15) / 16;
    const uint64_t dims[3] = {16, (uint64_t)K, (uint64_t)P_in};
    const uint64_t strides[2] = {16 * 8, (uint64_t)K * 16 * 8};
    const uint32_t box[3] = {16, 32, 1};
    if ((st = encode_tiled(&map, 3, X, dims, strides, box, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                           bf ? CU_TENSOR_MAP_SWIZZLE_NONE : CU_TENSOR_MAP_SWIZZLE_128B)))
      return st;
    if (bf) {
      SKG_DISPATCH_L(L, (launch_short_L<LL, false, true>(dev, map, R, K, KP, Rpad, (int*)mu.ptr,
                                                         (uint8_t*)res.ptr, err, s)))
    }
    SKG_DISPATCH_L(L, (launch_short_L<LL, false, false>(dev, map, R, K, KP, Rpad, (int*)mu.ptr,
                                                        (uint8_t*)res.ptr, err, s)))
  }
  if ((st = prep_norms<T>(R, K, KP, Rpad, X, L, res, part, mu, s, bf, km))) return st;
  return prep_convert<T>(dev, R, K, KP, Rpad, X, L, res, mu, err, s, bf, km);
}

template <int L, bool BF>
int launch_local_L(int64_t R, int64_t K, int64_t KP, int64_t Rpad, const double* src,
                   int64_t panel_stride, int64_t ks, uint8_t* res, int* mu, cudaStream_t s) {
  KernelTimer kt_(s, "convert_local_kernel");
  convert_local_kernel<L, BF><<<(unsigned)(Rpad / 16), 256, 0, s>>>(R, K, KP, Rpad, src,
                                                                    panel_stride, ks, res, mu);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int launch_local(int64_t R, int64_t K, int64_t KP, int64_t Rpad, const double* src,
                 int64_t panel_stride, int64_t ks, int L, uint8_t* res, int* mu, cudaStream_t s,
                 bool bf = false) {
  if (bf) {
    SKG_DISPATCH_L(L, (launch_local_L<LL, true>(R, K, KP, Rpad, src, panel_stride, ks, res, mu,
                                                s)))
  }
  SKG_DISPATCH_L(L, (launch_local_L<LL, false>(R, K, KP, Rpad, src, panel_stride, ks, res, mu, s)))
}

// Lane-scheduled INT8 (or BF16) products of prepared residues (A: os->res_a / mu_a,
// B: resB / muB) and their reconstruction into D: SYRK (upper triangle of
// the column-major M x M C = alpha A^T A + beta C) or GEMM (row-major
// D = alpha A B + gamma).
int lanes_product(DeviceState* dev, OzakiStream* os, StreamWorkspace* ws, int64_t M, int64_t N,
                  int64_t KP, int L, bool syrk, const DeviceBuffer* resB, const DeviceBuffer* muB,
                  double* D, int64_t ldd, double alpha, double gamma, cudaStream_t s,
                  bool bf = false) {
  int st;
  // Residue rows are KP * es bytes; a k-block is 128 bytes (128 INT8 or 64
  // BF16 values). BF16: sub-segments of 16 k-blocks (1024 products, exact in
  // FP32), 127 of them per int32 slot.
  const int64_t KPb = KP * (bf ? 2 : 1);
  const int KB = (int)(KPb / 128);
  const int64_t RA = (M + kI8BN - 1) / kI8BN * kI8BN;
  const int64_t RB = (N + kI8BN - 1) / kI8BN * kI8BN;
  DeviceBuffer& part = os->partials;
  LanePlan* pl = nullptr;
  if ((st = get_lane_plan(dev, (int)M, (int)N, KB, L, syrk,
                          bf ? kSegKbCapBf16 : kSegKbCapSigned, &pl,
                          bf ? kSubKbCapBf16 : 0, false, lanes_pair_units(dev, bf))) != SKGEMM_OK)
    return st;
  if ((st = part.ensure((size_t)pl->slots * pl->T * kI8BM * kI8BN * sizeof(int32_t)))) return st;
  I8Params p;
  memset(&p, 0, sizeof(p));
  p.sched = kSchedLanes;
  p.is_signed = 1;
  p.L = L;
  p.KB = KB;
  p.M = (int)M;
  p.N = (int)N;
  p.partials = (int32_t*)part.ptr;
  p.err = ws->err;
  if ((st = launch_lanes(dev, pl, os->res_a.ptr, KPb, RA, resB->ptr, syrk ? RA : RB, nullptr, p,
                         s, bf)))
    return st;
  const int64_t n = M * N;
  KernelTimer kt_(s, "crt_partials_kernel");
  crt_partials_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      (int)M, (int)N, L, (const int32_t*)part.ptr, pl->T, pl->tile_index, pl->tiles_n,
      pl->mod_slot_off, pl->mod_slots, (const int*)os->mu_a.ptr, (const int*)muB->ptr,
      syrk ? 1 : 0, D, ldd, alpha, gamma, (syrk && gamma == 0.0) ? 1 : 0);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

// Fused subspace pair products: one lane-scheduled launch over S's upper
// tiles (B = A's residues) and Hs's tiles (B = os->res_b), so each A panel
// is read once for both; then the two reconstructions from the shared slabs,
// S's on the helper stream.
int pair_product(DeviceState* dev, OzakiStream* os, StreamWorkspace* ws, int64_t M, int64_t KP,
                 int L, double* S, int64_t lds, double alpha_s, double beta_s, double* Hs,
                 int64_t ldh, double alpha_h, double gamma_h, cudaStream_t s, bool bf) {
  int st;
  const int64_t KPb = KP * (bf ? 2 : 1);
  const int KB = (int)(KPb / 128);
  const int64_t RA = (M + kI8BN - 1) / kI8BN * kI8BN;
  LanePlan* pl = nullptr;
  if ((st = get_lane_plan(dev, (int)M, (int)M, KB, L, false,
                          bf ? kSegKbCapBf16 : kSegKbCapSigned, &pl, bf ? kSubKbCapBf16 : 0,
                          true, lanes_pair_units(dev, bf))) != SKGEMM_OK)
    return st;
  DeviceBuffer& part = os->partials;
  if ((st = part.ensure((size_t)pl->slots * pl->T * kI8BM * kI8BN * sizeof(int32_t)))) return st;
  I8Params p;
  memset(&p, 0, sizeof(p));
  p.sched = kSchedLanes;
  p.is_signed = 1;
  p.L = L;
  p.KB = KB;
  p.M = (int)M;
  p.N = (int)M;
  p.partials = (int32_t*)part.ptr;
  p.err = ws->err;
  if ((st = launch_lanes(dev, pl, os->res_a.ptr, KPb, RA, os->res_a.ptr, RA, os->res_b.ptr, p, s,
                         bf)))
    return st;
  SKG_CUDA(cudaEventRecord(os->fork2, s));
  SKG_CUDA(cudaStreamWaitEvent(os->aux, os->fork2, 0));
  const int64_t n = M * M;
  const unsigned blocks = (unsigned)((n + 255) / 256);
  {
    KernelTimer kt_(os->aux, "crt_partials_kernel");
    crt_partials_kernel<<<blocks, 256, 0, os->aux>>>(
        (int)M, (int)M, L, (const int32_t*)part.ptr, pl->T, pl->tile_index, pl->tiles_n,
        pl->mod_slot_off, pl->mod_slots, (const int*)os->mu_a.ptr, (const int*)os->mu_a.ptr, 1, S,
        lds, alpha_s, beta_s, beta_s == 0.0 ? 1 : 0);
  }
  const cudaError_t e1 = cudaGetLastError();
  SKG_CUDA(cudaEventRecord(os->join2, os->aux));
  if (e1 != cudaSuccess) return cuda_fail(e1, "crt_partials_kernel");
  KernelTimer kt_(s, "crt_partials_kernel");
  crt_partials_kernel<<<blocks, 256, 0, s>>>(
      (int)M, (int)M, L, (const int32_t*)part.ptr, pl->T, pl->tile_index2, pl->tiles_n,
      pl->mod_slot_off, pl->mod_slots, (const int*)os->mu_a.ptr, (const int*)os->mu_b.ptr, 0, Hs,
      ldh, alpha_h, gamma_h, 0);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

// Residues of A (packed16, M rows) into os->res_a and, unless Bp is null, of
// B (packed32, N rows) into os->res_b: norms(A) | norms(B) on the helper
// stream, convert(A), join, convert(B).
int prep_pair(DeviceState* dev, OzakiStream* os, StreamWorkspace* ws, int64_t M, int64_t N,
              int64_t K, int L, const double* Ap, const double* Bp, cudaStream_t s,
              bool bf = false) {
  int st;
  const int64_t KP = (K + 127) / 128 * 128;
  const int64_t RA = (M + kI8BN - 1) / kI8BN * kI8BN;  // 256-multiples serve both box heights
  const int64_t RB = (N + kI8BN - 1) / kI8BN * kI8BN;
  if (!Bp)
    return prep_packed<16>(dev, M, K, KP, RA, Ap, L, os->res_a, os->part_a, os->mu_a, ws->err, s,
                           bf);
  if (!os->aux) {
    SKG_CUDA(cudaStreamCreateWithFlags(&os->aux, cudaStreamNonBlocking));
    SKG_CUDA(cudaEventCreateWithFlags(&os->fork, cudaEventDisableTiming));
    SKG_CUDA(cudaEventCreateWithFlags(&os->join, cudaEventDisableTiming));
  }
  SKG_CUDA(cudaEventRecord(os->fork, s));
  SKG_CUDA(cudaStreamWaitEvent(os->aux, os->fork, 0));
  const int st_b =
      prep_norms<32>(N, K, KP, RB, Bp, L, os->res_b, os->part_b, os->mu_b, os->aux, bf);
  SKG_CUDA(cudaEventRecord(os->join, os->aux));  // join even when the B step failed
  if (st_b) return st_b;
  if ((st = prep_packed<16>(dev, M, K, KP, RA, Ap, L, os->res_a, os->part_a, os->mu_a, ws->err,
                            s, bf)))
    return st;
  SKG_CUDA(cudaStreamWaitEvent(s, os->join, 0));
  return prep_convert<32>(dev, N, K, KP, RB, Bp, L, os->res_b, os->mu_b, ws->err, s, bf);
}

// Shared body of the Ozaki GEMM and SYRK: residues of A (packed16) and B
// (packed32 for GEMM; the SYRK reuses A's), lane-scheduled INT8 products,
// reconstruction.
int ozaki_lanes(int64_t M, int64_t N, int64_t K, const double* Ap, const double* Bp, bool syrk,
                double* D, int64_t ldd, double alpha, double gamma, skgemm_options_t* opts,
                cudaStream_t s) {
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (M == 0 || N == 0) return SKGEMM_OK;
  if (!Ap || !Bp || !D) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  if (K == 0) return fail(SKGEMM_ERR_UNSUPPORTED, "Ozaki path needs K > 0");
  if (M > (1 << 20) || N > (1 << 20)) return fail(SKGEMM_ERR_INVALID_ARG, "dimension too large");
  int L, gb;
  if ((st = choose_L(opts, K, &L, &gb)) != SKGEMM_OK) return st;
  std::lock_guard<std::mutex> lk(g_oz_mu);
  if ((st = ensure_consts(dev)) != SKGEMM_OK) return st;
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  OzakiStream* os = ozaki_stream(dev, s);
  const int64_t KP = (K + 127) / 128 * 128;
  const bool bf = is_bf16(opts);
  if ((st = prep_pair(dev, os, ws, M, N, K, L, Ap, syrk ? nullptr : Bp, s, bf))) return st;
  const DeviceBuffer* resB = syrk ? &os->res_a : &os->res_b;
  const DeviceBuffer* muB = syrk ? &os->mu_a : &os->mu_b;
  if ((st = lanes_product(dev, os, ws, M, N, KP, L, syrk, resB, muB, D, ldd, alpha, gamma, s,
                          bf)))
    return st;
  report(opts, L, gb, K);
  return SKGEMM_OK;
}

// Subspace pair S = alpha_s Psi^T Psi + beta_s S (upper, column-major) and
// Hs = alpha_h Psi^T HPsi + gamma_h (row-major) sharing Psi's residues.
int subspace_impl(int64_t K, int64_t M, const double* Psi, const double* HPsi, double* S,
                   int64_t lds, double alpha_s, double beta_s, double* Hs, int64_t ldh,
                   double alpha_h, double gamma_h, skgemm_options_t* opts, cudaStream_t s) {
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (M == 0) return SKGEMM_OK;
  if (!Psi || !HPsi || !S || !Hs) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  if (K == 0) return fail(SKGEMM_ERR_UNSUPPORTED, "Ozaki path needs K > 0");
  if (M > (1 << 20)) return fail(SKGEMM_ERR_INVALID_ARG, "dimension too large");
  int L, gb;
  if ((st = choose_L(opts, K, &L, &gb)) != SKGEMM_OK) return st;
  std::lock_guard<std::mutex> lk(g_oz_mu);
  if ((st = ensure_consts(dev)) != SKGEMM_OK) return st;
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  OzakiStream* os = ozaki_stream(dev, s);
  const int64_t KP = (K + 127) / 128 * 128;
  const bool bf = is_bf16(opts);
  if (!os->aux) {
    SKG_CUDA(cudaStreamCreateWithFlags(&os->aux, cudaStreamNonBlocking));
    SKG_CUDA(cudaEventCreateWithFlags(&os->fork, cudaEventDisableTiming));
    SKG_CUDA(cudaEventCreateWithFlags(&os->join, cudaEventDisableTiming));
  }
  if (!os->fork2) {
    SKG_CUDA(cudaEventCreateWithFlags(&os->fork2, cudaEventDisableTiming));
    SKG_CUDA(cudaEventCreateWithFlags(&os->join2, cudaEventDisableTiming));
  }
  // Two streams (none of these kernels waits on another CTA, so they may
  // share the machine in any proportion):
  //   s:   norms(Psi) -> convert(Psi) -- wait(join) -> products(S, Hs) -> CRT(Hs)
  //   aux: norms(HPsi) -> convert(HPsi) -> [join] -- wait(fork2) -> CRT(S) -> [join2]
  // HPsi's norm pass and conversion overlap Psi's; one INT8 launch computes
  // the products of both (pair_product); the two reconstructions overlap.
  const int64_t RA = (M + kI8BN - 1) / kI8BN * kI8BN;
  SKG_CUDA(cudaEventRecord(os->fork, s));
  SKG_CUDA(cudaStreamWaitEvent(os->aux, os->fork, 0));
  int st_b = prep_norms<32>(M, K, KP, RA, HPsi, L, os->res_b, os->part_b, os->mu_b, os->aux, bf);
  if (!st_b)
    st_b = prep_convert<32>(dev, M, K, KP, RA, HPsi, L, os->res_b, os->mu_b, ws->err, os->aux, bf);
  SKG_CUDA(cudaEventRecord(os->join, os->aux));  // recorded even when a B step failed
  if (st_b) {
    SKG_CUDA(cudaStreamWaitEvent(s, os->join, 0));
    return st_b;
  }
  if ((st = prep_packed<16>(dev, M, K, KP, RA, Psi, L, os->res_a, os->part_a, os->mu_a, ws->err,
                            s, bf))) {
    SKG_CUDA(cudaStreamWaitEvent(s, os->join, 0));
    return st;
  }
  SKG_CUDA(cudaStreamWaitEvent(s, os->join, 0));
  st = pair_product(dev, os, ws, M, KP, L, S, lds, alpha_s, beta_s, Hs, ldh, alpha_h, gamma_h, s,
                    bf);
  SKG_CUDA(cudaStreamWaitEvent(s, os->join2, 0));
  if (st) return st;
  report(opts, L, gb, K);
  return SKGEMM_OK;
}

}  // namespace

namespace {

// Scratch of one stream's Ozaki calls, per buffer of OzakiStream.
struct OzakiNeed {
  size_t res_a = 0, res_b = 0, part_a = 0, part_b = 0, mu_a = 0, mu_b = 0, partials = 0,
         rbytes = 0;
  void max_with(const OzakiNeed& o) {
    res_a = std::max(res_a, o.res_a);
    res_b = std::max(res_b, o.res_b);
    part_a = std::max(part_a, o.part_a);
    part_b = std::max(part_b, o.part_b);
    mu_a = std::max(mu_a, o.mu_a);
    mu_b = std::max(mu_b, o.mu_b);
    partials = std::max(partials, o.partials);
    rbytes = std::max(rbytes, o.rbytes);
  }
  size_t total() const {
    return res_a + res_b + part_a + part_b + mu_a + mu_b + partials + rbytes;
  }
};

size_t norm_part_bytes(int64_t R, int T) {
  const int64_t P_in = (R + T - 1) / T;
  const int64_t C = std::max<int64_t>(1, std::min<int64_t>(64, (600 + P_in - 1) / P_in));
  return (size_t)P_in * C * T * sizeof(double);
}

// Tiles and segment slots of the lane plan of (M, N, KB, L) (the counting
// part of get_lane_plan).
void lane_counts(int num_sms, int M, int N, int KB, int L, bool syrk, int seg_cap, int* T_out,
                 int* slots_out, bool pair = false) {
  const int tiles_m = (M + kI8BM - 1) / kI8BM, tiles_n = (N + kI8BN - 1) / kI8BN;
  int T = 0;
  for (int tm = 0; tm < tiles_m; ++tm)
    for (int tn = 0; tn < tiles_n; ++tn)
      if (!((syrk || pair) && tm * kI8BM > tn * kI8BN + kI8BN - 1)) ++T;
  if (pair) T += tiles_m * tiles_n;
  const int64_t W = (int64_t)L * KB;
  const int Q = lanes_for(num_sms, T, W);
  int slots = 0;
  for (int q = 0; q < Q; ++q) {
    int64_t it = (int64_t)q * W / Q, end = (int64_t)(q + 1) * W / Q;
    while (it < end) {
      const int l = (int)(it / KB);
      int64_t stop = std::min<int64_t>(end, (int64_t)(l + 1) * KB);
      stop = std::min<int64_t>(stop, it + seg_cap);
      ++slots;
      it = stop;
    }
  }
  *T_out = T;
  *slots_out = slots;
}

OzakiNeed need_lanes(DeviceState* dev, int64_t M, int64_t N, int64_t K, int L, bool syrk,
                     bool pair = false) {
  OzakiNeed n;
  const int64_t KP = (K + 127) / 128 * 128;
  const int KB = (int)(KP / 128);
  const int64_t RA = (M + kI8BN - 1) / kI8BN * kI8BN;
  const int64_t RB = (N + kI8BN - 1) / kI8BN * kI8BN;
  n.res_a = (size_t)L * RA * KP;
  n.part_a = norm_part_bytes(M, 16);
  n.mu_a = (size_t)RA * sizeof(int);
  if (!syrk) {
    n.res_b = (size_t)L * RB * KP;
    n.part_b = norm_part_bytes(N, 32);
    n.mu_b = (size_t)RB * sizeof(int);
  }
  int T = 0, slots = 0;
  lane_counts(dev->num_sms, (int)M, (int)N, KB, L, syrk, kSegKbCapSigned, &T, &slots, pair);
  n.partials = (size_t)slots * T * kI8BM * kI8BN * sizeof(int32_t);
  return n;
}

OzakiNeed need_rot(int64_t Nd, int64_t nb, int L) {
  OzakiNeed n;
  const int64_t KP = (nb + 127) / 128 * 128;
  const int64_t RA = (Nd + kI8BM - 1) / kI8BM * kI8BM;
  const int64_t RB = (nb + kI8BN - 1) / kI8BN * kI8BN;
  n.res_a = (size_t)L * RA * KP;
  n.res_b = (size_t)L * RB * KP;
  n.part_a = norm_part_bytes(Nd, 16);
  n.mu_a = (size_t)RA * sizeof(int);
  n.mu_b = (size_t)RB * sizeof(int);
  n.rbytes = (size_t)L * Nd * nb;
  return n;
}

}  // namespace

// Scratch a stream needs for Ozaki calls of `op` (SKGEMM_OP_*) on the given
// shape (GEMM: M, N, K; SYRK: M, K; rotation: Nd = M, nb = N) with `slices`
// moduli (0 = the automatic choice).
int ozaki_scratch_bytes(DeviceState* dev, int op, int64_t M, int64_t N, int64_t K, int slices,
                        size_t* bytes) {
  skgemm_options_t o;
  memset(&o, 0, sizeof(o));
  o.precision = SKGEMM_PREC_OZAKI_I8;
  o.slices = slices;
  int L, gb, st;
  OzakiNeed n;
  if (op == SKGEMM_OP_ROT) {
    if ((st = choose_L(&o, N, &L, &gb))) return st;
    n = need_rot(M, N, L);
  } else {
    if ((st = choose_L(&o, K, &L, &gb))) return st;
    n = need_lanes(dev, M, op == SKGEMM_OP_SYRK_PACKED ? M : N, K, L,
                   op == SKGEMM_OP_SYRK_PACKED);
  }
  *bytes = n.total();
  return SKGEMM_OK;
}

// Grows stream `s`'s Ozaki scratch to serve every call of the three ops and
// of the subspace pair on shapes up to (Nd, nb) with `slices` moduli without
// allocating later.
int ozaki_reserve(DeviceState* dev, cudaStream_t s, int64_t Nd, int64_t nb, int slices) {
  skgemm_options_t o;
  memset(&o, 0, sizeof(o));
  o.precision = SKGEMM_PREC_OZAKI_I8;
  o.slices = slices;
  int Lk, Lr, gb, st;
  if ((st = choose_L(&o, Nd, &Lk, &gb))) return st;
  if ((st = choose_L(&o, nb, &Lr, &gb))) return st;
  OzakiNeed n = need_lanes(dev, nb, nb, Nd, Lk, false);
  n.max_with(need_lanes(dev, nb, nb, Nd, Lk, true));
  n.max_with(need_lanes(dev, nb, nb, Nd, Lk, false, true));  // the fused subspace pair
  n.max_with(need_rot(Nd, nb, Lr));
  std::lock_guard<std::mutex> lk(g_oz_mu);
  if ((st = ensure_consts(dev))) return st;
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  OzakiStream* os = ozaki_stream(dev, s);
  if ((st = os->res_a.ensure(n.res_a)) || (st = os->res_b.ensure(n.res_b)) ||
      (st = os->part_a.ensure(n.part_a)) || (st = os->part_b.ensure(n.part_b)) ||
      (st = os->mu_a.ensure(n.mu_a)) || (st = os->mu_b.ensure(n.mu_b)) ||
      (st = os->partials.ensure(n.partials)) ||
      (st = os->rbytes.ensure(n.rbytes)))
    return st;
  return SKGEMM_OK;
}

// Frees stream `s`'s Ozaki buffers (the stream has been synchronised).
int ozaki_release_stream(DeviceState* dev, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_oz_mu);
  auto& m = g_oz[dev->device].streams;
  auto it = m.find(s);
  if (it == m.end()) return SKGEMM_OK;
  OzakiStream* os = it->second;
  if (os->aux) {
    cudaStreamSynchronize(os->aux);
    cudaStreamDestroy(os->aux);
    cudaEventDestroy(os->fork);
    cudaEventDestroy(os->join);
  }
  if (os->fork2) {
    cudaEventDestroy(os->fork2);
    cudaEventDestroy(os->join2);
  }
  for (DeviceBuffer* b : {&os->res_a, &os->res_b, &os->part_a, &os->part_b, &os->mu_a, &os->mu_b,
                          &os->partials, &os->rbytes})
    b->release();
  delete os;
  m.erase(it);
  return SKGEMM_OK;
}

// Bytes of device scratch stream `s` holds for the Ozaki path.
size_t ozaki_stream_bytes(DeviceState* dev, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_oz_mu);
  auto it = g_oz[dev->device].streams.find(s);
  if (it == g_oz[dev->device].streams.end()) return 0;
  const OzakiStream* os = it->second;
  return os->res_a.bytes + os->res_b.bytes + os->part_a.bytes + os->part_b.bytes +
         os->mu_a.bytes + os->mu_b.bytes + os->partials.bytes +
         os->rbytes.bytes;
}

int ozaki_subspace(int64_t K, int64_t M, const double* Psi, const double* HPsi, double* S,
                   int64_t lds, double alpha_s, double beta_s, double* Hs, int64_t ldh,
                   double alpha_h, double gamma_h, skgemm_options_t* opts, cudaStream_t s) {
  return subspace_impl(K, M, Psi, HPsi, S, lds, alpha_s, beta_s, Hs, ldh, alpha_h, gamma_h, opts,
                       s);
}

// Estimated device time (s) of one Ozaki call on this shape, from the
// measured rates of its kernels on B200: conversion 0.38 ps per element and
// modulus, the norm pass at 6 TB/s, INT8 products at 2.5 POP/s on the issued
// (128 x 256-tile, 128-k padded) MACs of the lanes schedule or 1.4 POP/s on
// the rotation's units schedule, reconstruction 15 ps per output and modulus
// (lanes) or 4.4 ps per output (rotation band CRT), plus ~40 us of launches.
// Negative when the Ozaki path does not take the shape (empty product,
// nb > 2048 for the rotation). Batched plans use it to choose precision.
double ozaki_time_estimate(int op, int64_t M, int64_t N, int64_t K, int slices) {
  skgemm_options_t o;
  memset(&o, 0, sizeof(o));
  o.precision = SKGEMM_PREC_OZAKI_I8;
  o.slices = slices;
  int L, gb;
  const double tile = (double)kI8BM * kI8BN;
  if (op == SKGEMM_OP_ROT) {
    if (N <= 0 || N > 2048 || M <= 0 || M > ((int64_t)1 << 30)) return -1.0;
    if (choose_L(&o, N, &L, &gb)) return -1.0;
    const double el = (double)M * N;
    const double tiles = (double)((M + kI8BM - 1) / kI8BM) * ((N + kI8BN - 1) / kI8BN);
    const double kp = (double)((N + 127) / 128 * 128);
    return el * L * 0.38e-12 + el * 8 / 6e12 + 2.0 * tiles * tile * kp * L / 1.4e15 +
           el * 4.4e-12 + 40e-6;
  }
  if (K <= 0 || M <= 0 || N <= 0 || M > (1 << 20) || N > (1 << 20)) return -1.0;
  if (choose_L(&o, K, &L, &gb)) return -1.0;
  const bool syrk = (op == SKGEMM_OP_SYRK_PACKED);
  const int64_t tm = (M + kI8BM - 1) / kI8BM, tn = (N + kI8BN - 1) / kI8BN;
  double tiles = 0.0;
  if (syrk) {
    for (int64_t j = 0; j < tn; ++j)
      tiles += (double)std::min<int64_t>(tm, (j * kI8BN + kI8BN - 1) / kI8BM + 1);
  } else {
    tiles = (double)tm * tn;
  }
  const double el = (double)K * (syrk ? M : M + N);
  const double kp = (double)((K + 127) / 128 * 128);
  return el * L * 0.38e-12 + el * 8 / 6e12 + 2.0 * tiles * tile * kp * L / 2.5e15 +
         (double)M * N * L * 15e-12 + 40e-6;
}

// Estimated device time (s) of ozaki_subspace (S and Hs from one split of
// Psi): the SYRK and GEMM estimates less the conversion and norm pass of Psi
// that the pair shares. Negative when the shape is not eligible.
double ozaki_pair_time_estimate(int64_t K, int64_t M, int slices) {
  const double ts = ozaki_time_estimate(SKGEMM_OP_SYRK_PACKED, M, M, K, slices);
  const double tg = ozaki_time_estimate(SKGEMM_OP_GEMM_PACKED, M, M, K, slices);
  if (ts < 0.0 || tg < 0.0) return -1.0;
  skgemm_options_t o;
  memset(&o, 0, sizeof(o));
  o.precision = SKGEMM_PREC_OZAKI_I8;
  o.slices = slices;
  int L, gb;
  if (choose_L(&o, K, &L, &gb)) return -1.0;
  const double el = (double)K * M;
  return ts + tg - (el * L * 0.38e-12 + el * 8 / 6e12);
}

int ozaki_gemm_packed(int64_t M, int64_t N, int64_t K, const double* Ap, const double* Bp,
                      double* D, int64_t ldd, double alpha, double gamma,
                      skgemm_options_t* opts, cudaStream_t s) {
  return ozaki_lanes(M, N, K, Ap, Bp, false, D, ldd, alpha, gamma, opts, s);
}

int ozaki_syrk_packed(int64_t K, int64_t M, const double* Ap, double* C, int64_t ldc,
                      double alpha, double beta, skgemm_options_t* opts, cudaStream_t s) {
  return ozaki_lanes(M, M, K, Ap, Ap, true, C, ldc, alpha, beta, opts, s);
}

int ozaki_rot(int64_t Nd, int64_t nb, const double* A, const double* Q, double* D,
              skgemm_options_t* opts, cudaStream_t s, bool a_band) {
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (Nd == 0 || nb == 0) return SKGEMM_OK;
  if (!A || !Q || !D) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  if (nb > 2048) return fail(SKGEMM_ERR_UNSUPPORTED, "Ozaki rotation supports nb <= 2048");
  const bool bf = is_bf16(opts);
  // BF16: one FP32 accumulation over K = nb must stay exact (<= 1024 products).
  if (bf && nb > 1024)
    return fail(SKGEMM_ERR_UNSUPPORTED, "Ozaki BF16 rotation supports nb <= 1024");
  if (Nd > ((int64_t)1 << 30)) return fail(SKGEMM_ERR_INVALID_ARG, "Nd too large");
  int L, gb;
  if ((st = choose_L(opts, nb, &L, &gb)) != SKGEMM_OK) return st;
  std::lock_guard<std::mutex> lk(g_oz_mu);
  if ((st = ensure_consts(dev)) != SKGEMM_OK) return st;
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  OzakiStream* os = ozaki_stream(dev, s);
  const int64_t KP = (nb + 127) / 128 * 128;
  const int64_t RA = (Nd + kI8BM - 1) / kI8BM * kI8BM;
  const int64_t RB = (nb + kI8BN - 1) / kI8BN * kI8BN;
  const int64_t KPb = KP * (bf ? 2 : 1);
  if ((st = os->res_b.ensure((size_t)L * RB * KPb))) return st;
  if ((st = os->mu_b.ensure((size_t)RB * sizeof(int)))) return st;
  if ((st = os->rbytes.ensure((size_t)L * Nd * nb))) return st;
  // Grid-packed Psi is a packed16 operand with rows = grid points, K = bands;
  // band-packed Psi (a_band) the K-major form of the same operand.
  if ((st = prep_packed<16>(dev, Nd, nb, KP, RA, A, L, os->res_a, os->part_a, os->mu_a, ws->err,
                            s, bf, a_band)))
    return st;
  if ((st = launch_local(nb, nb, KP, RB, Q, 16, nb, L, (uint8_t*)os->res_b.ptr,
                         (int*)os->mu_b.ptr, s, bf)))
    return st;
  CUtensorMap mA, mB;
  if ((st = make_res_map(&mA, os->res_a.ptr, KPb, RA, L, kI8BM))) return st;
  if ((st = make_res_map(&mB, os->res_b.ptr, KPb, RB, L, kI8BN))) return st;
  if (!bf && KP / 128 <= kI8RotKbMax && nb % 16 == 0 && nb >= 128 && Nd >= 128) {
    // B_l[tn] fits in shared memory: the B-resident schedule, residue bytes
    // [L][Nd][nb] written by 32 x 128-byte TMA store boxes.
    CUtensorMap mR;
    {
      uint64_t dims[3] = {(uint64_t)nb, (uint64_t)Nd, (uint64_t)L};
      uint64_t strides[2] = {(uint64_t)nb, (uint64_t)(Nd * nb)};
      uint32_t box[3] = {128, 32, 1};
      if ((st = encode_tiled(&mR, 3, os->rbytes.ptr, dims, strides, box,
                             CU_TENSOR_MAP_DATA_TYPE_UINT8, CU_TENSOR_MAP_SWIZZLE_128B)))
        return st;
    }
    I8RotParams p;
    memset(&p, 0, sizeof(p));
    p.L = L;
    p.KB = (int)(KP / 128);
    p.M = (int)Nd;
    p.N = (int)nb;
    p.tiles_m = (int)(RA / kI8BM);
    p.tiles_n = (int)(RB / kI8BN);
    const int64_t V = (int64_t)L * p.tiles_m;
    p.groups = (int)std::max<int64_t>(1, std::min<int64_t>(dev->num_sms / p.tiles_n, V));
    p.err = ws->err;
    if ((st = launch_i8_rot(dev, mA, mB, mR, p, p.groups * p.tiles_n, s))) return st;
  } else {
    I8Params p;
    memset(&p, 0, sizeof(p));
    p.sched = kSchedUnits;
    p.is_signed = 1;
    p.L = L;
    p.KB = (int)(KPb / 128);
    p.M = (int)Nd;
    p.N = (int)nb;
    p.tiles_m = (int)(RA / kI8BM);
    p.tiles_n = (int)(RB / kI8BN);
    p.residues = (uint8_t*)os->rbytes.ptr;
    p.ldr = nb;
    p.err = ws->err;
    const int64_t units = (int64_t)p.tiles_m * L * p.tiles_n;
    const int grid = (int)std::min<int64_t>(dev->num_sms, units);
    if ((st = launch_i8(dev, mA, mB, p, grid, s, bf))) return st;
  }
  {
    const uint8_t* rb = (const uint8_t*)os->rbytes.ptr;
    const int* mua = (const int*)os->mu_a.ptr;
    const int* mub = (const int*)os->mu_b.ptr;
    auto crt = [&]() -> int {
      SKG_DISPATCH_L(L, (launch_crt_band<LL>(Nd, nb, rb, mua, mub, D, s)))
    };
    if ((st = crt())) return st;
  }
  report(opts, L, gb, nb);
  return SKGEMM_OK;
}

int ozaki_consume_error(DeviceState*, cudaStream_t) { return SKGEMM_OK; }

// Exact INT8 GEMM (public): C[M][N] int32 = A[M][K] . B[N][K]^T with K-major
// int8 operands (row strides lda, ldb bytes). The operands are staged into
// the padded residue layout (one "modulus") and run on the lane schedule.
int igemm_s8(int64_t M, int64_t N, int64_t K, const int8_t* A, int64_t lda, const int8_t* B,
             int64_t ldb, int32_t* C, int64_t ldc, cudaStream_t s) {
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (M < 0 || N < 0 || K < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative dimension");
  if (lda < K || ldb < K || ldc < N) return fail(SKGEMM_ERR_INVALID_ARG, "leading dimension");
  if (M == 0 || N == 0) return SKGEMM_OK;
  if (M > (1 << 20) || N > (1 << 20)) return fail(SKGEMM_ERR_INVALID_ARG, "dimension too large");
  std::lock_guard<std::mutex> lk(g_oz_mu);
  if ((st = ensure_consts(dev)) != SKGEMM_OK) return st;
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  OzakiStream* os = ozaki_stream(dev, s);
  const int64_t KP = std::max<int64_t>(128, (K + 127) / 128 * 128);
  const int KB = (int)(KP / 128);
  const int64_t RA = (M + kI8BN - 1) / kI8BN * kI8BN;
  const int64_t RB = (N + kI8BN - 1) / kI8BN * kI8BN;
  if ((st = os->res_a.ensure((size_t)RA * KP))) return st;
  if ((st = os->res_b.ensure((size_t)RB * KP))) return st;
  SKG_CUDA(cudaMemsetAsync(os->res_a.ptr, 0, (size_t)RA * KP, s));
  SKG_CUDA(cudaMemsetAsync(os->res_b.ptr, 0, (size_t)RB * KP, s));
  if (K > 0) {
    SKG_CUDA(cudaMemcpy2DAsync(os->res_a.ptr, KP, A, lda, K, M, cudaMemcpyDeviceToDevice, s));
    SKG_CUDA(cudaMemcpy2DAsync(os->res_b.ptr, KP, B, ldb, K, N, cudaMemcpyDeviceToDevice, s));
  }
  LanePlan* pl = nullptr;
  if ((st = get_lane_plan(dev, (int)M, (int)N, KB, 1, false, kSegKbCapSigned, &pl, 0, false,
                          lanes_pair_units(dev, false))) != SKGEMM_OK)
    return st;
  if ((st = os->partials.ensure((size_t)pl->slots * pl->T * kI8BM * kI8BN * sizeof(int32_t))))
    return st;
  I8Params p;
  memset(&p, 0, sizeof(p));
  p.sched = kSchedLanes;
  p.is_signed = 1;
  p.L = 1;
  p.KB = KB;
  p.M = (int)M;
  p.N = (int)N;
  p.partials = (int32_t*)os->partials.ptr;
  p.err = ws->err;
  if ((st = launch_lanes(dev, pl, os->res_a.ptr, KP, RA, os->res_b.ptr, RB, nullptr, p, s,
                         false)))
    return st;
  const int64_t n = M * N;
  KernelTimer kt_(s, "sum_partials_kernel");
  sum_partials_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      (int)M, (int)N, (const int32_t*)os->partials.ptr, pl->T, pl->tile_index, pl->tiles_n,
      pl->mod_slot_off, pl->mod_slots, C, ldc);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int probe_i8_peak(DeviceState* dev, double* tops) {
  uint32_t* sink = nullptr;
  SKG_CUDA(cudaMalloc(&sink, 2 * sizeof(uint32_t)));
  SKG_CUDA(cudaMemset(sink, 0, 2 * sizeof(uint32_t)));
  // More shared memory than two CTAs can share: one CTA (one 512-column TMEM
  // allocation) per SM.
  const int smem = 160 * 1024;
  SKG_CUDA(cudaFuncSetAttribute(i8_peak_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  cudaEvent_t e0, e1;
  SKG_CUDA(cudaEventCreate(&e0));
  SKG_CUDA(cudaEventCreate(&e1));
  const int iters = 20000;
  i8_peak_kernel<<<dev->num_sms, 128, smem>>>(iters / 10, sink);
  SKG_CUDA(cudaEventRecord(e0));
  i8_peak_kernel<<<dev->num_sms, 128, smem>>>(iters, sink);
  SKG_CUDA(cudaEventRecord(e1));
  SKG_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  SKG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  uint32_t h[2] = {0, 0};
  SKG_CUDA(cudaMemcpy(h, sink, sizeof(h), cudaMemcpyDeviceToHost));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (h[1] != 0) return fail(SKGEMM_ERR_DEVICE_TIMEOUT, "INT8 peak probe wait ran out");
  const double ops = 2.0 * kI8BM * kI8BN * kI8BK * (double)iters * dev->num_sms;
  *tops = ops / (ms * 1e-3) / 1e12;
  return SKGEMM_OK;
}

}  // namespace skg
