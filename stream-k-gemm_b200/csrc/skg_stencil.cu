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

// Thread = (two band lanes 2h, 2h + 1, read as one 16-byte load; one (i, j)
// column): 8 lane pairs x 8 i x 4 j per 256-thread CTA. It marches k through
// [k0, k1) keeping the column's planes k - 6 .. k + 6 in a 13-slot register
// queue (slot of plane k + d at step u of a 13-step period: (u + d + 6) mod
// 13), so a step loads one new plane and the 24 x and y neighbours: 25 loads
// per output pair instead of 74, and the CTA's own rows serve most y
// neighbours from L1 (8 x 4 columns: 5.5 rows of the plane per output row
// come from L2). Measured alternatives: one lane per thread on 4 x 4 columns
// 0.73 ms, two i per thread on 16 x 2 columns 0.95 ms, against 0.66 ms here
// (48^3 points x 512 bands).
template <int OT>
__global__ void __launch_bounds__(256, 2) stencil_ext_kernel(
    int ni, int nj, int nk, int nb, int kc, const double* __restrict__ ext,
    const double* __restrict__ A, const __grid_constant__ StencilCoef cf,
    double* __restrict__ out) {
  const int h = threadIdx.x & 7;
  const int it = (threadIdx.x >> 3) & 7;
  const int jt = threadIdx.x >> 6;
  const int itiles = (ni + 7) / 8;
  const int i = (blockIdx.x % itiles) * 8 + it;
  const int j = (blockIdx.x / itiles) * 4 + jt;
  const int t = blockIdx.y;
  const int b = t * 16 + 2 * h;
  const int k0 = blockIdx.z * kc;
  const int k1 = min(nk, k0 + kc);
  if (i >= ni || j >= nj || b >= nb) return;
  const int64_t nix = ni + 2 * kFDn, njx = nj + 2 * kFDn, nkx = nk + 2 * kFDn;
  const int64_t sj = nix * 8, sk = nix * njx * 8;  // y / z strides in lane pairs
  const int64_t K = (int64_t)ni * nj * nk;
  // Lane pair h of extended point (i, j, k): base + (k + F) * sk.
  const double2* base = reinterpret_cast<const double2*>(ext) +
                        ((int64_t)t * nix * njx * nkx + (i + kFDn) + (int64_t)(j + kFDn) * nix) * 8 +
                        h;
  double2 zq[kZq];
#pragma unroll
  for (int d = -kFDn; d < kFDn; ++d)  // prologue: planes k0 - 6 .. k0 + 5
    zq[d + kFDn] = __ldg(base + (int64_t)(k0 + d + kFDn) * sk);
  for (int kb = k0; kb < k1; kb += kZq) {
#pragma unroll
    for (int u = 0; u < kZq; ++u) {
      const int k = kb + u;
      if (k >= k1) break;
      const double2* pk = base + (int64_t)(k + kFDn) * sk;
      zq[(u + 2 * kFDn) % kZq] = __ldg(pk + kFDn * sk);
      const int64_t g = (int64_t)i + (int64_t)j * ni + (int64_t)k * ni * nj;
      const double a = __ldg(A + g) + cf.c0;
      const double2 c = zq[(u + kFDn) % kZq];
      double r0 = c.x * a, r1 = c.y * a;
#pragma unroll
      for (int r = 1; r <= kFDn; ++r) {
        const double2 xp = __ldg(pk + r * 8), xm = __ldg(pk - r * 8);
        r0 = fma(xp.x + xm.x, cf.cx[r], r0);
        r1 = fma(xp.y + xm.y, cf.cx[r], r1);
        const double2 yp = __ldg(pk + r * sj), ym = __ldg(pk - r * sj);
        r0 = fma(yp.x + ym.x, cf.cy[r], r0);
        r1 = fma(yp.y + ym.y, cf.cy[r], r1);
        const double2 zp = zq[(u + kFDn + r) % kZq], zm = zq[(u + kFDn - r + kZq) % kZq];
        r0 = fma(zp.x + zm.x, cf.cz[r], r0);
        r1 = fma(zp.y + zm.y, cf.cz[r], r1);
      }
      double* o = out + ((int64_t)(b / OT) * K + g) * OT + b % OT;
      if (b + 1 < nb)
        *reinterpret_cast<double2*>(o) = make_double2(r0, r1);
      else
        o[0] = r0;  // lane b + 1 is padding: left untouched
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

int launch_stencil_ext(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                       const double* ext, const double* A, const double* cx, const double* cy,
                       const double* cz, double c0, double* out, int out_tile, int num_sms,
                       cudaStream_t s) {
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
  const int64_t cols = ((ni + 7) / 8) * ((nj + 3) / 4);
  const int64_t tiles = (nb + 15) / 16;
  if (cols > INT32_MAX || tiles > 65535) return fail(SKGEMM_ERR_INVALID_ARG, "grid too large");
  // Split k only when the columns alone give fewer than two waves of CTAs
  // (2 per SM); each chunk reloads 12 planes per column.
  int64_t chunks = 1;
  while (cols * tiles * chunks < 4LL * num_sms && nk / (chunks * 2) >= 16) chunks *= 2;
  const int kc = (int)((nk + chunks - 1) / chunks);
  dim3 grid((unsigned)cols, (unsigned)tiles, (unsigned)((nk + kc - 1) / kc));
  if (out_tile == 32)
    stencil_ext_kernel<32><<<grid, 256, 0, s>>>((int)ni, (int)nj, (int)nk, (int)nb, kc, ext, A, cf,
                                                out);
  else
    stencil_ext_kernel<16><<<grid, 256, 0, s>>>((int)ni, (int)nj, (int)nk, (int)nb, kc, ext, A, cf,
                                                out);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
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
  halo_periodic_kernel<<<(unsigned)rows, 256, 0, s>>>((int)ni, (int)nj, (int)nk, FDn, local, ext);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

}  // namespace skg
