// HBM-bound layout kernels: strided dense -> packed-T panels (the device
// counterpart of gemm<double>::pack_A / pack_B, gemm_opt.cpp:342-371) and the
// band-packed <-> grid-packed transposition of a block of states
// (sme_pack<double>::band_to_grid_tile / grid_to_band_tile,
// include/sme_pack.hpp:232-313).
#include <algorithm>

#include "skg_common.cuh"
#include "skg_runtime.h"

namespace skg {

namespace {

// Packs X(r, k) = X[r*sr + k*sk] into out[(r/T)*K*T + k*T + r%T] through a
// 32 (r) x 32 (k) shared-memory tile, so that reads are coalesced along
// whichever of r / k is contiguous and writes are coalesced along r%T, k.
template <int T>
__global__ void __launch_bounds__(256) pack_kernel(int64_t R, int64_t K, const double* __restrict__ X,
                                                   int64_t sr, int64_t sk,
                                                   double* __restrict__ out) {
  __shared__ double tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const bool r_contig = (sr == 1);
  for (int i = ty; i < 32; i += 8) {
    // Read with the contiguous index on tx.
    int64_t r = r_contig ? r0 + tx : r0 + i;
    int64_t k = r_contig ? k0 + i : k0 + tx;
    double v = 0.0;
    if (r < R && k < K) v = X[r * sr + k * sk];
    if (r_contig)
      tile[i][tx] = v;  // [k][r]
    else
      tile[tx][i] = v;  // [k][r]
  }
  __syncthreads();
  // Write: each output row (fixed k) of a T-panel is T contiguous doubles.
  const int64_t Rpad = ((R + T - 1) / T) * T;
  for (int i = ty; i < 32; i += 8) {
    int64_t k = k0 + i, r = r0 + tx;
    if (k < K && r < Rpad) out[(r / T) * K * T + k * T + (r % T)] = tile[i][tx];
  }
}

// The inverse of pack_kernel: X[r*sr + k*sk] = Xp[(r/T)*K*T + k*T + r%T] for
// r < R. Reads are coalesced along r%T (T contiguous doubles per panel row),
// writes along whichever of r / k is contiguous in X.
template <int T>
__global__ void __launch_bounds__(256) unpack_kernel(int64_t R, int64_t K,
                                                     const double* __restrict__ Xp,
                                                     double* __restrict__ X, int64_t sr,
                                                     int64_t sk) {
  __shared__ double tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int i = ty; i < 32; i += 8) {
    const int64_t k = k0 + i, r = r0 + tx;
    tile[i][tx] = (k < K && r < R) ? Xp[(r / T) * K * T + k * T + (r % T)] : 0.0;  // [k][r]
  }
  __syncthreads();
  const bool r_contig = (sr == 1);
  for (int i = ty; i < 32; i += 8) {
    const int64_t r = r_contig ? r0 + tx : r0 + i;
    const int64_t k = r_contig ? k0 + i : k0 + tx;
    if (r < R && k < K) X[r * sr + k * sk] = r_contig ? tile[i][tx] : tile[tx][i];
  }
}

// One 16 x 16 block per warp-pair: src[(b/16)*Nd*16 + g*16 + b%16] (band) ->
// dst[(g/16)*nb*16 + b*16 + g%16] (grid), or the reverse.
template <bool kBandToGrid>
__global__ void __launch_bounds__(256) band_grid_kernel(int64_t Nd, int64_t nb,
                                                        const double* __restrict__ src,
                                                        double* __restrict__ dst) {
  __shared__ double tile[4][16][17];
  const int sub = threadIdx.x >> 6;  // 4 blocks of 16x16 per CTA
  const int lt = threadIdx.x & 63;
  const int64_t blk = (int64_t)blockIdx.x * 4 + sub;
  const int64_t gtiles = Nd / 16, btiles = nb / 16;
  const bool live = blk < gtiles * btiles;
  const int64_t gt = live ? blk % gtiles : 0, bt = live ? blk / gtiles : 0;
  // Source rows are 16 contiguous doubles; 64 threads read 4 rows per pass.
  for (int pass = 0; pass < 4; ++pass) {
    int row = pass * 4 + (lt >> 4), col = lt & 15;
    double v = 0.0;
    if (live) {
      if (kBandToGrid)  // row = g_local, col = b_local
        v = src[bt * Nd * 16 + (gt * 16 + row) * 16 + col];
      else  // row = b_local, col = g_local
        v = src[gt * nb * 16 + (bt * 16 + row) * 16 + col];
    }
    tile[sub][row][col] = v;
  }
  __syncthreads();
  if (!live) return;
  for (int pass = 0; pass < 4; ++pass) {
    int row = pass * 4 + (lt >> 4), col = lt & 15;
    if (kBandToGrid)  // dst row = b_local, col = g_local
      dst[gt * nb * 16 + (bt * 16 + row) * 16 + col] = tile[sub][col][row];
    else  // dst row = g_local, col = b_local
      dst[bt * Nd * 16 + (gt * 16 + row) * 16 + col] = tile[sub][col][row];
  }
}

// out[i] = gamma + sum over p < nparts of parts[p * n + i] (out may be parts).
__global__ void __launch_bounds__(256) sum_parts_kernel(const double* parts, int nparts, int64_t n,
                                                        double gamma, double* out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double v = parts[i];
    for (int p = 1; p < nparts; ++p) v += parts[p * n + i];
    out[i] = v + gamma;
  }
}

}  // namespace

// Sum of `nparts` partial outputs of n doubles each plus gamma (the K-chunked
// host GEMM's combine step).
int launch_sum_parts(const double* parts, int nparts, int64_t n, double gamma, double* out,
                     cudaStream_t s) {
  if (n <= 0) return SKGEMM_OK;
  const int64_t blocks = std::min<int64_t>((n + 255) / 256, 148 * 8);
  sum_parts_kernel<<<(unsigned)blocks, 256, 0, s>>>(parts, nparts, n, gamma, out);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int launch_pack(int64_t R, int64_t K, const double* X, int64_t sr, int64_t sk, int T,
                double* Xp, cudaStream_t s) {
  if (R < 0 || K < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative pack extent");
  if (R == 0 || K == 0) return SKGEMM_OK;
  if (!X || !Xp) return fail(SKGEMM_ERR_INVALID_ARG, "null pack pointer");
  const int64_t Rpad = T == 16 ? (R + 15) / 16 * 16 : (R + 31) / 32 * 32;
  dim3 grid((unsigned)((Rpad + 31) / 32), (unsigned)((K + 31) / 32));
  if (grid.y > 65535u) return fail(SKGEMM_ERR_INVALID_ARG, "pack: K too large for one launch");
  if (T == 16)
    pack_kernel<16><<<grid, 256, 0, s>>>(R, K, X, sr, sk, Xp);
  else if (T == 32)
    pack_kernel<32><<<grid, 256, 0, s>>>(R, K, X, sr, sk, Xp);
  else
    return fail(SKGEMM_ERR_INVALID_ARG, "pack width must be 16 or 32");
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int launch_unpack(int64_t R, int64_t K, const double* Xp, int T, double* X, int64_t sr,
                  int64_t sk, cudaStream_t s) {
  if (R < 0 || K < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative unpack extent");
  if (R == 0 || K == 0) return SKGEMM_OK;
  if (!X || !Xp) return fail(SKGEMM_ERR_INVALID_ARG, "null unpack pointer");
  dim3 grid((unsigned)((R + 31) / 32), (unsigned)((K + 31) / 32));
  if (grid.y > 65535u) return fail(SKGEMM_ERR_INVALID_ARG, "unpack: K too large for one launch");
  if (T == 16)
    unpack_kernel<16><<<grid, 256, 0, s>>>(R, K, Xp, X, sr, sk);
  else if (T == 32)
    unpack_kernel<32><<<grid, 256, 0, s>>>(R, K, Xp, X, sr, sk);
  else
    return fail(SKGEMM_ERR_INVALID_ARG, "pack width must be 16 or 32");
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int launch_band_to_grid(int64_t Nd, int64_t nb, const double* src, double* dst,
                        cudaStream_t s) {
  if (Nd < 0 || nb < 0 || Nd % 16 || nb % 16)
    return fail(SKGEMM_ERR_INVALID_ARG, "band/grid packing needs Nd, nb multiples of 16");
  if (Nd == 0 || nb == 0) return SKGEMM_OK;
  int64_t blocks = (Nd / 16) * (nb / 16);
  band_grid_kernel<true><<<(unsigned)((blocks + 3) / 4), 256, 0, s>>>(Nd, nb, src, dst);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int launch_grid_to_band(int64_t Nd, int64_t nb, const double* src, double* dst,
                        cudaStream_t s) {
  if (Nd < 0 || nb < 0 || Nd % 16 || nb % 16)
    return fail(SKGEMM_ERR_INVALID_ARG, "band/grid packing needs Nd, nb multiples of 16");
  if (Nd == 0 || nb == 0) return SKGEMM_OK;
  int64_t blocks = (Nd / 16) * (nb / 16);
  band_grid_kernel<false><<<(unsigned)((blocks + 3) / 4), 256, 0, s>>>(Nd, nb, src, dst);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

}  // namespace skg
