// The H Psi producer of a CheFSI step on device: the 6th-order finite-
// difference stencil on extended (halo-padded) band-packed Psi, output in the
// 32-band-packed layout that the GEMM reads as B (Hs = Psi^T H Psi) or in the
// 16-band-packed layout (calc_laplacian_extended_packed_16to32 / _16to16,
// include/stencil_extended_packed.hpp:47-181, :276-), and the single-rank
// periodic halo that extends band-packed Psi (copy_interior_to_extended_packed,
// include/halo_packed.hpp:93-124, and the no-MPI wrap of :350-393).
//
// Per grid point g = i + j ni + k ni nj (extended index g_ex, offset FDn on
// each axis) and band b:
//   res = psi(g_ex) (A[g] + c0)
//   for r = 1 .. 6: res = fma(psi(g_ex + r) + psi(g_ex - r), cx[r], res), then
//                   the same along y (stride ni_ex) and z (ni_ex nj_ex)
// in the reference SVE kernels' order (x, y, z for each r; FMLA is fused),
// so the results equal those kernels bit for bit.
#include <algorithm>

#include "skg_common.cuh"
#include "skg_runtime.h"

namespace skg {

namespace {

constexpr int kFDn = 6;
constexpr int kZq = 2 * kFDn + 1;  // planes k - 6 .. k + 6

struct StencilCoef {
  double cx[kFDn + 1], cy[kFDn + 1], cz[kFDn + 1];
  double c0;
};

// CTA = one 4-band slab (bands 4 q ..
// 4 q + 3: one 32-byte sector per point) of a 16 x 16 column tile, marching
// k through [k0, k1). A producer warp streams, by TMA, one stage per k step
// into a ring of kStRing shared-memory stages, kStRing - 1 steps ahead:
//   the tile's plane k with its x / y halo, 28 x 28 points x 4 bands;
//   the tile's 16 x 16 points of plane k + 6 (the z queue's new entry);
//   A[g] of the tile's 16 x 16 points of plane k: one 2-D box when ni is
//   even (A viewed as [nj nk][ni]: 16-byte row strides), else one 18-double
//   box per row from an even index, in a 256-byte slot.
// Consumer thread = two columns (i, j) and (i, j + 1) and a band pair: a
// quarter-warp reads 4 consecutive points (128 contiguous bytes); the 14
// staged values j - 6 .. j + 7 serve the y neighbours of both columns; the
// 12 z neighbours come from the columns' 13-slot register queues (slot of
// plane k + d at step u of a 13-step period: (u + d + 6) mod 13). No global
// load waits inside the k loop. Same arithmetic in the same order as the
// reference kernels: the output equals theirs bit for bit. Every wait is
// bounded; on expiry the CTA records the error and skips the remaining waits.
constexpr int kStI = 16;                 // columns per CTA along x
constexpr int kStJ = 16;                 // columns per CTA along y
constexpr int kSlab = 4;                 // bands per CTA
constexpr int kStHI = kStI + 2 * kFDn;   // staged points along x
constexpr int kStHJ = kStJ + 2 * kFDn;   // staged points along y
constexpr int kStARow = 18;              // doubles per A box (from an even index)
constexpr int kStAPitch = 32;            // doubles between staged A rows (TMA
                                         // destinations are 128-byte aligned)
constexpr int kStPlane = kStHI * kStHJ * kSlab;  // doubles: halo plane
constexpr int kStCenter = kStI * kStJ * kSlab;   // doubles: plane k + 6
constexpr int kStStage = kStPlane + kStCenter + kStJ * kStAPitch;  // doubles per stage
constexpr int kStRing = 4;
constexpr int kStConsumerWarps = kStJ / 2;
constexpr int kStThreads = (kStConsumerWarps + 1) * 32;
constexpr int kStTxBytes2d = (kStPlane + kStCenter + kStJ * kStI) * 8;
constexpr int kStTxBytesRows = (kStPlane + kStCenter + kStJ * kStARow) * 8;
constexpr int kStSmem = kStRing * kStStage * 8 + 2 * kStRing * 8 + 16 + 128;
static_assert((kStPlane * 8) % 128 == 0 && (kStCenter * 8) % 128 == 0, "stage alignment");
static_assert((kStStage * 8) % 128 == 0 && (kStAPitch * 8) % 128 == 0, "stage alignment");
static_assert((kStARow * 8) % 16 == 0 && kStARow <= kStAPitch, "A box");
static_assert(kStSmem <= 232448, "stencil stages exceed 227 KB of shared memory");

template <int OT>
__global__ void __launch_bounds__(kStThreads, 1) stencil_staged_kernel(
    const __grid_constant__ CUtensorMap mapP, const __grid_constant__ CUtensorMap mapC,
    const __grid_constant__ CUtensorMap mapA, bool a2d, int ni, int nj, int nk, int nb, int kc,
    const double* __restrict__ ext, const __grid_constant__ StencilCoef cf,
    double* __restrict__ out, uint32_t* __restrict__ err) {
  extern __shared__ uint8_t sraw[];
  double* stages =
      reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(sraw) + 127) & ~uintptr_t(127));
  uint64_t* full = reinterpret_cast<uint64_t*>(stages + kStRing * kStStage);
  uint64_t* empty = full + kStRing;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty + kStRing);
  const int itiles = (ni + kStI - 1) / kStI;
  const int i0 = (int)(blockIdx.x % itiles) * kStI, j0 = (int)(blockIdx.x / itiles) * kStJ;
  const int q = blockIdx.y;  // slab: bands 4 q .. 4 q + 3
  const int t = q / (16 / kSlab), sl = q % (16 / kSlab);
  const int k0 = blockIdx.z * kc;
  const int k1 = min(nk, k0 + kc);
  if (q * kSlab >= nb || k0 >= k1) return;
  const int nsteps = k1 - k0;
  const int64_t nix = ni + 2 * kFDn, njx = nj + 2 * kFDn, nkx = nk + 2 * kFDn;
  const int64_t plane_pts = (int64_t)ni * nj;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int b = 0; b < kStRing; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], kStConsumerWarps);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == kStConsumerWarps) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      tma_prefetch_desc(&mapP);
      tma_prefetch_desc(&mapC);
      tma_prefetch_desc(&mapA);
      int issued = 0;
      for (int u = 0; u < nsteps; ++u) {
        const int b = u % kStRing;
        if (u >= kStRing) {
          if (*abort_flag || !mbar_wait(&empty[b], ((u / kStRing) - 1) & 1, err)) {
            *abort_flag = 1;
            break;
          }
        }
        const int k = k0 + u;
        double* st = stages + b * kStStage;
        mbar_arrive_expect_tx(&full[b], a2d ? kStTxBytes2d : kStTxBytesRows);
        tma_load_4d(st, &mapP, &full[b], sl * kSlab, i0, j0, (int)(t * nkx + k + kFDn));
        tma_load_4d(st + kStPlane, &mapC, &full[b], sl * kSlab, i0 + kFDn, j0 + kFDn,
                    (int)(t * nkx + k + 2 * kFDn));
        if (a2d) {
          tma_load_2d(st + kStPlane + kStCenter, &mapA, &full[b], i0, j0 + k * nj);
        } else {
          for (int jj = 0; jj < kStJ; ++jj) {
            const int64_t g = (int64_t)i0 + (int64_t)(j0 + jj) * ni + (int64_t)k * plane_pts;
            tma_load_1d(st + kStPlane + kStCenter + jj * kStAPitch, &mapA, &full[b],
                        (int)(g & ~1LL));
          }
        }
        ++issued;
      }
      // The CTA leaves only after its last loads have landed (immediate on
      // the normal path: the consumers waited for every one of them).
      for (int u = issued - 1; u >= 0 && u >= issued - kStRing; --u)
        mbar_wait(&full[u % kStRing], (u / kStRing) & 1, err);
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  const int bp = lane & 1;
  const int il = lane >> 1;
  const int jA = 2 * warp;  // tile rows jA, jA + 1
  const int i = i0 + il, j = j0 + jA;
  const int b = q * kSlab + 2 * bp;
  const bool actA = i < ni && j < nj && b < nb;
  const bool actB = i < ni && j + 1 < nj && b < nb;
  const int64_t sk = nix * njx * 8;  // z stride in lane pairs
  const int64_t K = plane_pts * nk;
  const double2* baseA =
      reinterpret_cast<const double2*>(ext) +
      ((int64_t)t * nix * njx * nkx + (i + kFDn) + (int64_t)(j + kFDn) * nix) * 8 + sl * 2 + bp;
  const double2* baseB = baseA + nix * 8;
  double2 zqA[kZq], zqB[kZq];
#pragma unroll
  for (int d = -kFDn; d < kFDn; ++d) {  // prologue: planes k0 - 6 .. k0 + 5
    zqA[d + kFDn] = actA ? __ldg(baseA + (int64_t)(k0 + d + kFDn) * sk) : make_double2(0.0, 0.0);
    zqB[d + kFDn] = actB ? __ldg(baseB + (int64_t)(k0 + d + kFDn) * sk) : make_double2(0.0, 0.0);
  }
  // Lane pair (il, row) offsets in a stage, in double2 units.
  const int pA = ((jA + kFDn) * kStHI + il + kFDn) * 2 + bp;  // halo plane, row jA
  const int yA = (jA * kStHI + il + kFDn) * 2 + bp;            // halo plane, row jA - 6
  const int cA = ((jA * kStI) + il) * 2 + bp;                   // center box, row jA
  for (int kb = k0; kb < k1; kb += kZq) {
#pragma unroll
    for (int u = 0; u < kZq; ++u) {
      const int k = kb + u;
      if (k >= k1) break;
      const int step = k - k0, buf = step % kStRing;
      if (!*abort_flag && !mbar_wait(&full[buf], (step / kStRing) & 1, err)) *abort_flag = 1;
      const double* st = stages + buf * kStStage;
      const double2* P = reinterpret_cast<const double2*>(st);
      const double2* C = reinterpret_cast<const double2*>(st + kStPlane);
      const double* As = st + kStPlane + kStCenter;
      zqA[(u + 2 * kFDn) % kZq] = C[cA];
      zqB[(u + 2 * kFDn) % kZq] = C[cA + kStI * 2];
      if (actA) {
        const int64_t g = (int64_t)i + (int64_t)j * ni + (int64_t)k * plane_pts;
        const int64_t gr = g - il;  // row start
        const int64_t grB = gr + ni;
        const double aA = (a2d ? As[jA * kStI + il] : As[jA * kStAPitch + (int)(gr & 1) + il]) +
                          cf.c0;
        const double aB = (a2d ? As[(jA + 1) * kStI + il]
                               : As[(jA + 1) * kStAPitch + (int)(grB & 1) + il]) + cf.c0;
        double2 Y[2 * kFDn + 2];  // rows jA - 6 .. jA + 7
#pragma unroll
        for (int d = 0; d < 2 * kFDn + 2; ++d) Y[d] = P[yA + d * kStHI * 2];
        const double2 ca = zqA[(u + kFDn) % kZq], cb = zqB[(u + kFDn) % kZq];
        double a0 = ca.x * aA, a1 = ca.y * aA;
        double b0 = cb.x * aB, b1 = cb.y * aB;
#pragma unroll
        for (int r = 1; r <= kFDn; ++r) {
          const double2 xpA = P[pA + 2 * r], xmA = P[pA - 2 * r];
          const double2 xpB = P[pA + 2 * kStHI + 2 * r], xmB = P[pA + 2 * kStHI - 2 * r];
          a0 = fma(xpA.x + xmA.x, cf.cx[r], a0);
          a1 = fma(xpA.y + xmA.y, cf.cx[r], a1);
          b0 = fma(xpB.x + xmB.x, cf.cx[r], b0);
          b1 = fma(xpB.y + xmB.y, cf.cx[r], b1);
          a0 = fma(Y[kFDn + r].x + Y[kFDn - r].x, cf.cy[r], a0);
          a1 = fma(Y[kFDn + r].y + Y[kFDn - r].y, cf.cy[r], a1);
          b0 = fma(Y[kFDn + 1 + r].x + Y[kFDn + 1 - r].x, cf.cy[r], b0);
          b1 = fma(Y[kFDn + 1 + r].y + Y[kFDn + 1 - r].y, cf.cy[r], b1);
          const double2 zpA = zqA[(u + kFDn + r) % kZq], zmA = zqA[(u + kFDn - r + kZq) % kZq];
          const double2 zpB = zqB[(u + kFDn + r) % kZq], zmB = zqB[(u + kFDn - r + kZq) % kZq];
          a0 = fma(zpA.x + zmA.x, cf.cz[r], a0);
          a1 = fma(zpA.y + zmA.y, cf.cz[r], a1);
          b0 = fma(zpB.x + zmB.x, cf.cz[r], b0);
          b1 = fma(zpB.y + zmB.y, cf.cz[r], b1);
        }
        double* o = out + ((int64_t)(b / OT) * K + g) * OT + b % OT;
        if (b + 1 < nb)
          *reinterpret_cast<double2*>(o) = make_double2(a0, a1);
        else
          o[0] = a0;  // lane b + 1 is padding: left untouched
        if (actB) {
          double* o2 = o + (int64_t)ni * OT;
          if (b + 1 < nb)
            *reinterpret_cast<double2*>(o2) = make_double2(b0, b1);
          else
            o2[0] = b0;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[buf]);
    }
  }
}

// One CTA per extended row (tile t, k_ex, j_ex): ext[(t K_ex + g_ex) 16 + l] =
// local[(t K + g) 16 + l], g the periodic image of g_ex's interior point;
// 16-byte lane pairs (the copy is bound by its index arithmetic).
__global__ void __launch_bounds__(256) halo_periodic_kernel(int ni, int nj, int nk, int FDn,
                                                            const double* __restrict__ local,
                                                            double* __restrict__ ext) {
  const int64_t nix = ni + 2 * FDn, njx = nj + 2 * FDn, nkx = nk + 2 * FDn;
  const int64_t row = blockIdx.x;  // (t * nkx + kx) * njx + jx
  const int64_t jx = row % njx, kx = (row / njx) % nkx, t = row / (njx * nkx);
  int jl = (int)jx - FDn, kl = (int)kx - FDn;
  jl += jl < 0 ? nj : (jl >= nj ? -nj : 0);
  kl += kl < 0 ? nk : (kl >= nk ? -nk : 0);
  const int64_t K = (int64_t)ni * nj * nk;
  const double2* src = reinterpret_cast<const double2*>(local) +
                       (t * K + (int64_t)jl * ni + (int64_t)kl * ni * nj) * 8;
  double2* dst = reinterpret_cast<double2*>(ext) + row * nix * 8;
  for (int e = threadIdx.x; e < (int)nix * 8; e += blockDim.x) {
    int il = (e >> 3) - FDn;
    il += il < 0 ? ni : (il >= ni ? -ni : 0);
    dst[e] = src[il * 8 + (e & 7)];
  }
}

}  // namespace

namespace {

template <int OT>
int launch_staged(const CUtensorMap& mapP, const CUtensorMap& mapC, const CUtensorMap& mapA,
                  bool a2d, int ni, int nj, int nk, int nb, int kc, dim3 grid, const double* ext,
                  const StencilCoef& cf, double* out, uint32_t* err, cudaStream_t s) {
  static bool attr_set[64] = {};  // function attributes are per device
  int d = 0;
  SKG_CUDA(cudaGetDevice(&d));
  if (d < 0 || d >= 64) return fail(SKGEMM_ERR_INVALID_ARG, "device index");
  if (!attr_set[d]) {
    SKG_CUDA(cudaFuncSetAttribute(stencil_staged_kernel<OT>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, kStSmem));
    attr_set[d] = true;
  }
  KernelTimer kt_(s, "stencil_staged_kernel");
  stencil_staged_kernel<OT><<<grid, kStThreads, kStSmem, s>>>(mapP, mapC, mapA, a2d, ni, nj, nk,
                                                              nb, kc, ext, cf, out, err);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

}  // namespace

int launch_stencil_ext(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                       const double* ext, const double* A, const double* cx, const double* cy,
                       const double* cz, double c0, double* out, int out_tile, int num_sms,
                       uint32_t* err, cudaStream_t s) {
  if (ni < 0 || nj < 0 || nk < 0 || nb < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative extent");
  if (FDn != kFDn)
    return fail(SKGEMM_ERR_UNSUPPORTED, "stencil radius FDn must be 6 (the reference's kernels)");
  if (out_tile != 16 && out_tile != 32) return fail(SKGEMM_ERR_INVALID_ARG, "out_tile must be 16 or 32");
  if (ni == 0 || nj == 0 || nk == 0 || nb == 0) return SKGEMM_OK;
  if (!ext || !A || !cx || !cy || !cz || !out) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  if (ni > (1 << 20) || nj > (1 << 20) || nk > (1 << 20) || ni * nj * nk > ((int64_t)1 << 40))
    return fail(SKGEMM_ERR_INVALID_ARG, "grid too large");
  StencilCoef cf;
  for (int r = 0; r <= kFDn; ++r) {
    cf.cx[r] = cx[r];
    cf.cy[r] = cy[r];
    cf.cz[r] = cz[r];
  }
  cf.c0 = c0;
  if ((reinterpret_cast<uintptr_t>(ext) | reinterpret_cast<uintptr_t>(out)) & 15)
    return fail(SKGEMM_ERR_INVALID_ARG, "stencil arrays must be 16-byte aligned");
  if ((reinterpret_cast<uintptr_t>(A) & 15) != 0)
    return fail(SKGEMM_ERR_INVALID_ARG, "stencil A_diag must be 16-byte aligned");
  const int64_t cols = ((ni + kStI - 1) / kStI) * ((nj + kStJ - 1) / kStJ);
  const int64_t tiles = (nb + 15) / 16;
  const int64_t slabs = tiles * (16 / kSlab);
  if (cols > INT32_MAX || slabs > 65535) return fail(SKGEMM_ERR_INVALID_ARG, "grid too large");
  const int64_t nix = ni + 2 * kFDn, njx = nj + 2 * kFDn, nkx = nk + 2 * kFDn;
  if (tiles * nkx > INT32_MAX || ni * nj * nk + 2 >= INT32_MAX)
    return fail(SKGEMM_ERR_INVALID_ARG, "grid too large");
  // Extended Psi as a 4-D tensor [tiles * nkx][njx][nix][16 lanes]: boxes of
  // 4 lanes x 28 x 28 points (halo planes) and 4 lanes x 16 x 16 points (z
  // entries); A as a 1-D tensor, boxes of 18 doubles. Zero fill outside.
  CUtensorMap mapP, mapC, mapA;
  const uint64_t dims[4] = {16, (uint64_t)nix, (uint64_t)njx, (uint64_t)(tiles * nkx)};
  const uint64_t strides[3] = {16 * 8, (uint64_t)nix * 16 * 8, (uint64_t)(nix * njx) * 16 * 8};
  const uint32_t boxP[4] = {(uint32_t)kSlab, (uint32_t)kStHI, (uint32_t)kStHJ, 1};
  const uint32_t boxC[4] = {(uint32_t)kSlab, (uint32_t)kStI, (uint32_t)kStJ, 1};
  // A: [nj nk][ni] with 16 x 16 boxes when its rows are 16-byte strided,
  // else 1-D with 18-double boxes.
  const bool a2d = ni % 2 == 0;
  const uint64_t dimsA[2] = {a2d ? (uint64_t)ni : (uint64_t)(ni * nj * nk), (uint64_t)(nj * nk)};
  const uint64_t stridesA[1] = {(uint64_t)ni * 8};
  const uint32_t boxA[2] = {a2d ? (uint32_t)kStI : (uint32_t)kStARow, (uint32_t)kStJ};
  int st;
  if ((st = encode_tiled(&mapP, 4, ext, dims, strides, boxP, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         CU_TENSOR_MAP_SWIZZLE_NONE)) ||
      (st = encode_tiled(&mapC, 4, ext, dims, strides, boxC, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         CU_TENSOR_MAP_SWIZZLE_NONE)) ||
      (st = encode_tiled(&mapA, a2d ? 2 : 1, A, dimsA, stridesA, boxA, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                         CU_TENSOR_MAP_SWIZZLE_NONE)))
    return st;
  // Split k only when the column tiles and slabs alone give fewer than four
  // CTAs per SM; each chunk reloads 12 planes per column.
  int64_t chunks = 1;
  while (cols * slabs * chunks < 4LL * num_sms && nk / (chunks * 2) >= 16) chunks *= 2;
  const int kc = (int)((nk + chunks - 1) / chunks);
  const dim3 grid((unsigned)cols, (unsigned)slabs, (unsigned)((nk + kc - 1) / kc));
  if (out_tile == 32)
    return launch_staged<32>(mapP, mapC, mapA, a2d, (int)ni, (int)nj, (int)nk, (int)nb, kc, grid, ext,
                             cf, out, err, s);
  return launch_staged<16>(mapP, mapC, mapA, a2d, (int)ni, (int)nj, (int)nk, (int)nb, kc, grid, ext,
                           cf, out, err, s);
}

int launch_halo_periodic(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                         const double* local, double* ext, cudaStream_t s) {
  if (ni < 0 || nj < 0 || nk < 0 || nb < 0 || FDn < 0)
    return fail(SKGEMM_ERR_INVALID_ARG, "negative extent");
  if (ni == 0 || nj == 0 || nk == 0 || nb == 0) return SKGEMM_OK;
  if (FDn > ni || FDn > nj || FDn > nk)
    return fail(SKGEMM_ERR_INVALID_ARG, "periodic halo wider than the domain");
  if (!local || !ext) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  if ((reinterpret_cast<uintptr_t>(local) | reinterpret_cast<uintptr_t>(ext)) & 15)
    return fail(SKGEMM_ERR_INVALID_ARG, "halo arrays must be 16-byte aligned");
  if (ni > (1 << 20) || nj > (1 << 20) || nk > (1 << 20))
    return fail(SKGEMM_ERR_INVALID_ARG, "grid too large");
  const int64_t rows = ((nb + 15) / 16) * (nk + 2 * FDn) * (nj + 2 * FDn);
  if (rows > INT32_MAX) return fail(SKGEMM_ERR_INVALID_ARG, "grid too large");
  KernelTimer kt_(s, "halo_periodic_kernel");
  halo_periodic_kernel<<<(unsigned)rows, 256, 0, s>>>((int)ni, (int)nj, (int)nk, FDn, local, ext);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

}  // namespace skg
