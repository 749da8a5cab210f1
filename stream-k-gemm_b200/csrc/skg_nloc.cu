// The nonlocal part of H on device: Hamiltonian::nloc_project_vectors_packed
// (16-band-packed Psi -> 32-band-packed H Psi) and _16to16
// (include/nloc_packed_opt2.hpp:226-445). Per projector p (grid rows
// index_p, coefficients chi_p column-major nrow x ncol, coefficient block at
// offsets[p], shared by the projectors of one atom's periodic images):
//   C_p[j, b] = C_p + dv * sum_r chi_p[r, j] psi[index_p[r], b]  (gather + chi^T psi)
//   C_p *= gamma_p per column, on every change of atom index in projector order
//   out[index_p[r], b] += sum_j chi_p[r, j] C_p[j, b]             (chi C + scatter)
// The single-rank all-reduce of the coefficients is the identity here.
//
// Three kernels, no atomics, the reference's loop and rounding order (as its
// C++ compiles: the forward dot products unfused, the block update fused, the
// back-projection sums fused), so results equal it bit for bit:
//  * nloc_forward_kernel: CTA per (block, 32 bands, 16 columns) — for each of
//    the block's projectors in order, gathered psi rows staged in shared
//    memory (double-buffered asynchronous copies), each (column, band) thread
//    summing them in row order; then the block's gamma scalings in order;
//  * nloc_chi_c_kernel: the back-projection rows chi_p C_p of every projector
//    (spans of 64-row tiles x 64 bands, C and chi staged in shared memory),
//    into a scratch of total rows x nb;
//  * nloc_backward_kernel: thread per (touched grid point, band pair) — walks
//    the point's (projector, row) entries in projector order (an inverse index
//    built at creation, each entry stored as its scratch row), so the
//    scatter-adds keep the reference's order.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "skg_common.cuh"
#include "skg_runtime.h"

struct skgemm_nloc {
  int device = 0;
  int64_t P = 0, K = 0, nblk = 0, ntouch = 0, total_cols = 0;
  // device arrays
  uint32_t *d_nrow = nullptr, *d_ncol = nullptr, *d_index = nullptr;
  int64_t *d_row_off = nullptr, *d_chi_off = nullptr;
  double *d_chi = nullptr, *d_gamma = nullptr;
  // blocks: column base, width, projectors (CSR), gamma scalings (CSR)
  int64_t* d_blk = nullptr;  // [nblk][4]: col base, ncol, proj begin, scale begin
  int64_t* d_blk_end = nullptr;  // [nblk][2]: proj end, scale end
  int32_t* d_blk_proj = nullptr;
  int64_t* d_blk_scale = nullptr;  // gamma offsets
  int64_t* d_proj_blk_col = nullptr;  // per projector: its block's column base
  // touched points: grid index, entries (CSR of (projector, row))
  uint32_t* d_touch = nullptr;
  int64_t* d_touch_off = nullptr;
  int64_t* d_ent_off = nullptr;  // per entry: its temp row (projector's row_off + row)
  // back-projection row tiles (projector, first row)
  int64_t ntiles = 0;
  int64_t *d_tile_proj = nullptr, *d_tile_r0 = nullptr;
  int64_t total_rows = 0, max_cols = 0;
  // scratch: the coefficient blocks ([column][band], total_cols x nb), then
  // the back-projection rows (total_rows x nb)
  double* d_coef = nullptr;
  int64_t coef_cap = 0;
  bool chi_c_smem_set = false;  // the chi*C kernel's shared-memory attribute
  std::vector<int64_t> blk_width;  // host copy of each block's ncol
  std::mutex mu;
};

namespace skg {

namespace {

// Forward CTA: (block q, 32 bands, 16 columns); thread (band bl = tid % 32,
// columns 4 jq .. 4 jq + 3, jq = tid / 32). The CTA walks the block's
// projectors in order and each projector's rows in chunks of 32: per chunk,
// 32 gathered rows x 32 bands of psi and the matching 32 rows x 16 columns
// of chi land in shared memory by asynchronous copies, double-buffered (24 KB
// a CTA, so that all CTAs of the apply are resident at once; the
// next chunk's gathers are in flight while the current one is summed). Every
// thread adds its four columns' products over a chunk's rows in row order —
// the reference's order, so the sums are exact to it — and folds each
// projector's sum into the block coefficient with fma(dv, sum, C).
// Coefficients stored [column][band].
constexpr int kNlocBands = 32;
constexpr int kNlocCols = 16;
constexpr int kNlocRows = 32;
constexpr int kNlocThreads = kNlocBands * kNlocCols / 4;

__global__ void __launch_bounds__(kNlocThreads) nloc_forward_kernel(
    int64_t nb, int64_t K, double dv, const int64_t* __restrict__ blk,
    const int64_t* __restrict__ blk_end, const int32_t* __restrict__ blk_proj,
    const int64_t* __restrict__ blk_scale, const uint32_t* __restrict__ nrow,
    const int64_t* __restrict__ row_off, const int64_t* __restrict__ chi_off,
    const uint32_t* __restrict__ index, const double* __restrict__ chi,
    const double* __restrict__ gamma, const double* __restrict__ psi16,
    double* __restrict__ coef) {
  __shared__ __align__(16) double rows[2][kNlocRows][kNlocBands];
  __shared__ __align__(16) double xs[2][kNlocCols][kNlocRows];
  const int64_t q = blockIdx.x;
  const int64_t b0 = (int64_t)blockIdx.y * kNlocBands;
  const int64_t jb = (int64_t)blockIdx.z * kNlocCols;  // the CTA's first column
  const int bl = threadIdx.x % kNlocBands;
  const int jq = threadIdx.x / kNlocBands;
  const int64_t col0 = blk[4 * q], nc = blk[4 * q + 1];
  if (jb >= nc) return;  // the whole CTA past the block
  const int ncc = (int)min((int64_t)kNlocCols, nc - jb);  // columns of this CTA
  const int64_t b = b0 + bl;
  const int64_t e_begin = blk[4 * q + 2], e_end = blk_end[2 * q];
  // Issue the copies of chunk r0 of projector entry e into buffer buf.
  auto issue = [&](int64_t e, int64_t r0, int buf) {
    const int p = blk_proj[e];
    const int64_t nr = nrow[p];
    const int nrr = (int)min((int64_t)kNlocRows, nr - r0);
    const uint32_t* idx = index + row_off[p];
    // psi rows: 64 rows x 2 band tiles x 8 pieces of 16 bytes (two bands).
#pragma unroll
    for (int i = threadIdx.x; i < kNlocRows * kNlocBands / 2; i += kNlocThreads) {
      const int rr = i / (kNlocBands / 2), cb = 2 * (i % (kNlocBands / 2));
      const int64_t bb = b0 + cb;
      const bool ok = rr < nrr && bb < nb;
      const double* src = psi16;
      if (ok) src = psi16 + ((bb / 16) * K + (int64_t)__ldg(idx + r0 + rr)) * 16 + (bb % 16);
      cp_async16(&rows[buf][rr][cb], src, ok ? 16u : 0u);
    }
    const double* x = chi + chi_off[p] + jb * nr;
#pragma unroll
    for (int i = threadIdx.x; i < kNlocCols * kNlocRows; i += kNlocThreads) {
      const int jj = i / kNlocRows, rr = i % kNlocRows;
      const bool ok = jj < ncc && rr < nrr;
      cp_async8(&xs[buf][jj][rr], ok ? x + jj * nr + r0 + rr : chi, ok ? 8u : 0u);
    }
  };
  // Chunk cursor over (projector entry, first row); advance returns false at
  // the block's end.
  auto advance = [&](int64_t& e, int64_t& r0) -> bool {
    r0 += kNlocRows;
    while (e < e_end && r0 >= (int64_t)nrow[blk_proj[e]]) {
      ++e;
      r0 = 0;
    }
    return e < e_end;
  };
  int64_t e = e_begin, r0 = 0;
  // Skip leading projectors without rows.
  while (e < e_end && nrow[blk_proj[e]] == 0) ++e;
  double acc[4] = {};
  double sum[4] = {};
  if (e < e_end) {
    issue(e, r0, 0);
    cp_async_commit();
  }
  int buf = 0;
  int64_t done_e = e_begin;  // projectors before this one are folded into acc
  while (e < e_end) {
    int64_t ne = e, nr0 = r0;
    const bool more = advance(ne, nr0);
    if (more) issue(ne, nr0, buf ^ 1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const int p = blk_proj[e];
    const int nrr = (int)min((int64_t)kNlocRows, (int64_t)nrow[p] - r0);
    for (int rr = 0; rr < nrr; ++rr) {
      const double v = rows[buf][rr][bl];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        sum[jj] = __dadd_rn(sum[jj], __dmul_rn(xs[buf][4 * jq + jj][rr], v));
    }
    // Projector e ends with this chunk: fold its sum; projectors without
    // rows between e and the next chunk's contribute zero sums.
    if (!more || ne != e) {
      for (int64_t f = done_e; f <= e; ++f) {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[jj] = fma(dv, f == e ? sum[jj] : 0.0, acc[jj]);
      }
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) sum[jj] = 0.0;
      done_e = e + 1;
    }
    __syncthreads();  // buffer buf consumed before the next issue refills it
    buf ^= 1;
    e = ne;
    r0 = nr0;
  }
  // Trailing projectors without rows.
  for (int64_t f = done_e; f < e_end; ++f) {
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) acc[jj] = fma(dv, 0.0, acc[jj]);
  }
  if (b >= nb) return;
#pragma unroll
  for (int jj = 0; jj < 4; ++jj) {
    const int64_t j = jb + 4 * jq + jj;
    if (j >= nc) break;
    double a = acc[jj];
    for (int64_t f = blk[4 * q + 3]; f < blk_end[2 * q + 1]; ++f)
      a = __dmul_rn(a, __ldg(gamma + blk_scale[f] + j));
    coef[(col0 + j) * nb + b] = a;
  }
}

// Back-projection, step 1: temp_p[r, b] = sum_k chi_p[r, k] C_p[k, b] (fused,
// k ascending: the reference's gemm_ab order) for every projector row, into
// temp[(row_off_p + r) * nb + b]. CTA = (a span of up to kNlocSpan row tiles
// of 64 rows of one projector, 64 bands): C's columns for the 64 bands are
// staged in shared memory once, then each row tile's chi rows are staged and
// its 64 x 64 outputs written.
constexpr int kNlocTileR = 64;
constexpr int kNlocTileB = 64;
constexpr int kNlocMaxCols = 64;
constexpr int kNlocSpan = 4;

__global__ void __launch_bounds__(256) nloc_chi_c_kernel(
    int64_t nb, int max_cols, const int64_t* __restrict__ tile_proj,
    const int64_t* __restrict__ tile_r0,
    const uint32_t* __restrict__ nrow, const uint32_t* __restrict__ ncol,
    const int64_t* __restrict__ row_off, const int64_t* __restrict__ chi_off,
    const int64_t* __restrict__ proj_col, const double* __restrict__ chi,
    const double* __restrict__ coef, double* __restrict__ temp) {
  extern __shared__ double nsm[];
  double* cs = nsm;                     // [max_cols][kNlocTileB]
  double* xs = nsm + max_cols * kNlocTileB;  // [kNlocTileR][nc + 1]
  const int64_t tile = blockIdx.x;
  const int p = (int)tile_proj[tile];
  const int64_t span0 = tile_r0[tile];
  const int64_t nr = nrow[p], nc = ncol[p];
  const int64_t b0 = (int64_t)blockIdx.y * kNlocTileB;
  const double* c = coef + proj_col[p] * nb;
  for (int i = threadIdx.x; i < nc * kNlocTileB; i += blockDim.x) {
    const int k = i / kNlocTileB, bb = i % kNlocTileB;
    cs[k * kNlocTileB + bb] = (b0 + bb < nb) ? c[k * nb + b0 + bb] : 0.0;
  }
  // Thread: band pairs 2 q4, 2 q4 + 1 and 32 + 2 q4, 33 + 2 q4 of the tile
  // (q4 = tid % 16; 16-byte loads and stores, consecutive lanes on
  // consecutive pairs) and rows rg, rg + 16, rg + 32, rg + 48 (rg = tid / 16):
  // per column, four chi and four C values feed 16 multiply-adds, each
  // output's sum over the columns in order.
  const int q4 = threadIdx.x % 16, rg = threadIdx.x / 16;
  for (int t = 0; t < kNlocSpan; ++t) {
    const int64_t r0 = span0 + (int64_t)t * kNlocTileR;
    if (r0 >= nr) break;
    const int nrr = (int)min((int64_t)kNlocTileR, nr - r0);
    if (t > 0) __syncthreads();  // the previous tile's chi rows are consumed
    const double* x = chi + chi_off[p] + r0;
    for (int i = threadIdx.x; i < nc * kNlocTileR; i += blockDim.x) {
      const int k = i / kNlocTileR, rr = i % kNlocTileR;
      xs[rr * (nc + 1) + k] = rr < nrr ? x[k * nr + rr] : 0.0;
    }
    __syncthreads();
    double tt[4][4] = {};
    for (int k = 0; k < nc; ++k) {
      double cv[4], xv[4];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) cv[jj] = cs[k * kNlocTileB + 32 * (jj >> 1) + 2 * q4 + (jj & 1)];
#pragma unroll
      for (int i = 0; i < 4; ++i) xv[i] = xs[(rg + 16 * i) * (nc + 1) + k];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) tt[i][jj] = fma(xv[i], cv[jj], tt[i][jj]);
    }
    double* out = temp + (row_off[p] + r0) * nb + b0 + 2 * q4;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int rr = rg + 16 * i;
      if (rr >= nrr) break;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        double* o = out + (int64_t)rr * nb + 32 * h;
        const int64_t bb = b0 + 32 * h + 2 * q4;
        if (bb + 1 < nb && ((reinterpret_cast<uintptr_t>(o) & 15) == 0)) {
          *reinterpret_cast<double2*>(o) = make_double2(tt[i][2 * h], tt[i][2 * h + 1]);
        } else {
          if (bb < nb) o[0] = tt[i][2 * h];
          if (bb + 1 < nb) o[1] = tt[i][2 * h + 1];
        }
      }
    }
  }
}

// Back-projection, step 2: thread per (touched grid point, band pair): the
// point's (projector, row) entries added to out in projector order.
template <int OT>
__global__ void __launch_bounds__(256) nloc_backward_kernel(
    int64_t ntouch, int64_t nb, int64_t K, const uint32_t* __restrict__ touch,
    const int64_t* __restrict__ touch_off, const int64_t* __restrict__ ent_off,
    const double* __restrict__ temp, double* __restrict__ out) {
  const int64_t nbp = (nb + 1) / 2;  // band pairs
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntouch * nbp) return;
  const int64_t b = 2 * (t % nbp), s = t / nbp;
  const bool two = b + 1 < nb;
  const int64_t g = touch[s];
  double* o = out + ((b / OT) * K + g) * OT + (b % OT);  // b + 1 in the same tile (OT even)
  double v0 = o[0], v1 = two ? o[1] : 0.0;
  for (int64_t e = touch_off[s]; e < touch_off[s + 1]; ++e) {
    const double* tr = temp + __ldg(ent_off + e) * nb + b;
    v0 = __dadd_rn(v0, __ldg(tr));
    if (two) v1 = __dadd_rn(v1, __ldg(tr + 1));
  }
  o[0] = v0;
  if (two) o[1] = v1;
}

template <typename T>
int upload(T** dst, const std::vector<T>& v) {
  if (v.empty()) return SKGEMM_OK;
  SKG_CUDA(cudaMalloc(dst, v.size() * sizeof(T)));
  SKG_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return SKGEMM_OK;
}

void release(skgemm_nloc* h) {
  void* ptrs[] = {h->d_nrow, h->d_ncol, h->d_index, h->d_row_off, h->d_chi_off, h->d_chi,
                  h->d_gamma, h->d_blk, h->d_blk_end, h->d_blk_proj, h->d_blk_scale,
                  h->d_proj_blk_col, h->d_touch, h->d_touch_off, h->d_ent_off,
                  h->d_tile_proj, h->d_tile_r0, h->d_coef};
  for (void* p : ptrs)
    if (p) cudaFree(p);
}

}  // namespace

// Builds the device form of a projector set (see skgemm_nloc_create).
int nloc_create(int64_t P, const uint32_t* nrow, const uint32_t* ncol, const int32_t* atom,
                const uint32_t* offsets, const uint32_t* index, const double* chi,
                const double* gamma, int64_t K, skgemm_nloc** out) {
  if (!out) return fail(SKGEMM_ERR_INVALID_ARG, "null handle pointer");
  *out = nullptr;
  if (P < 0 || P > INT32_MAX || K <= 0 || K > ((int64_t)1 << 32))
    return fail(SKGEMM_ERR_INVALID_ARG, "projector count or grid size out of range");
  if (P > 0 && (!nrow || !ncol || !atom || !offsets))
    return fail(SKGEMM_ERR_INVALID_ARG, "null projector array");
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  std::vector<int64_t> row_off(P), chi_off(P);
  int64_t rows = 0, chis = 0, gams = 0;
  std::vector<int64_t> gam_off(P);
  const int64_t total = P > 0 ? offsets[P] : 0;
  for (int64_t p = 0; p < P; ++p) {
    row_off[p] = rows;
    chi_off[p] = chis;
    gam_off[p] = gams;
    rows += nrow[p];
    chis += (int64_t)nrow[p] * ncol[p];
    gams += ncol[p];
    if ((int64_t)offsets[p] + ncol[p] > total)
      return fail(SKGEMM_ERR_INVALID_ARG, "projector block past the total column count");
    if (ncol[p] > kNlocMaxCols)
      return fail(SKGEMM_ERR_UNSUPPORTED, "projectors of more than 64 columns");
  }
  if (rows > 0 && !index) return fail(SKGEMM_ERR_INVALID_ARG, "null index array");
  if ((chis > 0 && !chi) || (gams > 0 && !gamma))
    return fail(SKGEMM_ERR_INVALID_ARG, "null coefficient array");
  for (int64_t i = 0; i < rows; ++i)
    if (index[i] >= (uint64_t)K) return fail(SKGEMM_ERR_INVALID_ARG, "grid index out of range");
  // Blocks by offset, in order of first use; projectors sharing one must
  // share its width, and distinct blocks must not overlap.
  std::map<uint32_t, int64_t> blk_of;
  std::vector<int64_t> bcol, bnc;
  std::vector<std::vector<int32_t>> bproj;
  std::vector<std::vector<int64_t>> bscale;
  std::vector<int64_t> proj_col(P);
  for (int64_t p = 0; p < P; ++p) {
    auto it = blk_of.find(offsets[p]);
    int64_t q;
    if (it == blk_of.end()) {
      q = (int64_t)bcol.size();
      blk_of[offsets[p]] = q;
      bcol.push_back(offsets[p]);
      bnc.push_back(ncol[p]);
      bproj.emplace_back();
      bscale.emplace_back();
    } else {
      q = it->second;
      if (bnc[q] != ncol[p])
        return fail(SKGEMM_ERR_INVALID_ARG, "projectors sharing a block differ in width");
    }
    proj_col[p] = offsets[p];
    if (nrow[p] > 0 && ncol[p] > 0) bproj[q].push_back((int32_t)p);
  }
  {
    int64_t end = 0;
    for (const auto& kv : blk_of) {
      const int64_t q = kv.second;
      if (bcol[q] < end) return fail(SKGEMM_ERR_INVALID_ARG, "projector blocks overlap");
      end = bcol[q] + bnc[q];
    }
  }
  if (P > 0) {  // gamma on each change of atom index, in projector order
    int32_t a = atom[0] - 1;
    for (int64_t p = 0; p < P; ++p) {
      if (a == atom[p]) continue;
      a = atom[p];
      bscale[blk_of[offsets[p]]].push_back(gam_off[p]);
    }
  }
  // Inverse index: grid point -> (projector, row) in projector order.
  std::map<uint32_t, std::vector<std::pair<int32_t, uint32_t>>> inv;
  for (int64_t p = 0; p < P; ++p) {
    if (nrow[p] == 0 || ncol[p] == 0) continue;
    for (uint32_t r = 0; r < nrow[p]; ++r) inv[index[row_off[p] + r]].push_back({(int32_t)p, r});
  }
  auto* h = new skgemm_nloc();
  h->device = dev->device;
  h->P = P;
  h->K = K;
  h->nblk = (int64_t)bcol.size();
  h->total_cols = total;
  h->blk_width = bnc;
  std::vector<int64_t> blk(4 * h->nblk), blk_end(2 * h->nblk);
  std::vector<int32_t> blk_proj;
  std::vector<int64_t> blk_scale;
  for (int64_t q = 0; q < h->nblk; ++q) {
    blk[4 * q] = bcol[q];
    blk[4 * q + 1] = bnc[q];
    blk[4 * q + 2] = (int64_t)blk_proj.size();
    blk[4 * q + 3] = (int64_t)blk_scale.size();
    blk_proj.insert(blk_proj.end(), bproj[q].begin(), bproj[q].end());
    blk_scale.insert(blk_scale.end(), bscale[q].begin(), bscale[q].end());
    blk_end[2 * q] = (int64_t)blk_proj.size();
    blk_end[2 * q + 1] = (int64_t)blk_scale.size();
  }
  std::vector<uint32_t> touch;
  std::vector<int64_t> touch_off{0};
  std::vector<int64_t> ent_off;
  for (const auto& kv : inv) {
    touch.push_back(kv.first);
    for (const auto& e : kv.second) ent_off.push_back(row_off[e.first] + e.second);
    touch_off.push_back((int64_t)ent_off.size());
  }
  h->ntouch = (int64_t)touch.size();
  h->total_rows = rows;
  std::vector<int64_t> tile_proj, tile_r0;
  for (int64_t p = 0; p < P; ++p) {
    if (nrow[p] == 0 || ncol[p] == 0) continue;
    h->max_cols = std::max<int64_t>(h->max_cols, ncol[p]);
    for (int64_t r0 = 0; r0 < nrow[p]; r0 += kNlocTileR * kNlocSpan) {
      tile_proj.push_back(p);
      tile_r0.push_back(r0);
    }
  }
  h->ntiles = (int64_t)tile_proj.size();
  std::vector<uint32_t> vnrow(nrow, nrow + P), vncol(ncol, ncol + P);
  std::vector<uint32_t> vindex(index, index + rows);
  std::vector<double> vchi(chi, chi + chis), vgam(gamma, gamma + gams);
  if ((st = upload(&h->d_nrow, vnrow)) || (st = upload(&h->d_ncol, vncol)) ||
      (st = upload(&h->d_index, vindex)) || (st = upload(&h->d_row_off, row_off)) ||
      (st = upload(&h->d_chi_off, chi_off)) || (st = upload(&h->d_chi, vchi)) ||
      (st = upload(&h->d_gamma, vgam)) || (st = upload(&h->d_blk, blk)) ||
      (st = upload(&h->d_blk_end, blk_end)) || (st = upload(&h->d_blk_proj, blk_proj)) ||
      (st = upload(&h->d_blk_scale, blk_scale)) || (st = upload(&h->d_proj_blk_col, proj_col)) ||
      (st = upload(&h->d_touch, touch)) || (st = upload(&h->d_touch_off, touch_off)) ||
      (st = upload(&h->d_ent_off, ent_off)) ||
      (st = upload(&h->d_tile_proj, tile_proj)) || (st = upload(&h->d_tile_r0, tile_r0))) {
    release(h);
    delete h;
    return st;
  }
  *out = h;
  return SKGEMM_OK;
}

int nloc_apply(skgemm_nloc* h, int64_t nb, double dv, const double* psi16, double* out,
               int out_tile, cudaStream_t s) {
  if (!h) return fail(SKGEMM_ERR_INVALID_ARG, "null projector handle");
  if (nb < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative band count");
  if (out_tile != 16 && out_tile != 32) return fail(SKGEMM_ERR_INVALID_ARG, "out_tile must be 16 or 32");
  if (nb == 0 || h->nblk == 0 || h->total_cols == 0) return SKGEMM_OK;
  if (!psi16 || !out) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (dev->device != h->device) return fail(SKGEMM_ERR_INVALID_ARG, "handle of another device");
  std::lock_guard<std::mutex> lk(h->mu);
  // Scratch: coefficients (total columns x nb), then back-projection rows
  // (total rows x nb); grown on demand.
  const int64_t need = (h->total_cols + h->total_rows) * nb;
  if (need > h->coef_cap) {
    if (h->d_coef) {
      SKG_CUDA(cudaStreamSynchronize(s));
      cudaFree(h->d_coef);
      h->d_coef = nullptr;
      h->coef_cap = 0;
    }
    SKG_CUDA(cudaMalloc(&h->d_coef, need * sizeof(double)));
    h->coef_cap = need;
  }
  // Debug mode: the coefficient and scratch rows start as 0xFF bytes.
  if ((st = debug_poison(h->d_coef, (size_t)h->coef_cap * sizeof(double), s))) return st;
  const int64_t maxw = *std::max_element(h->blk_width.begin(), h->blk_width.end());
  if (maxw > 0) {
    dim3 grid((unsigned)h->nblk, (unsigned)((nb + kNlocBands - 1) / kNlocBands),
              (unsigned)((maxw + kNlocCols - 1) / kNlocCols));
    if (grid.y > 65535u || grid.z > 65535u)
      return fail(SKGEMM_ERR_INVALID_ARG, "too many bands or projector columns");
    KernelTimer kt_(s, "nloc_forward_kernel");
    nloc_forward_kernel<<<grid, kNlocThreads, 0, s>>>(
        nb, h->K, dv, h->d_blk, h->d_blk_end, h->d_blk_proj, h->d_blk_scale, h->d_nrow,
        h->d_row_off, h->d_chi_off, h->d_index, h->d_chi, h->d_gamma, psi16, h->d_coef);
    SKG_CUDA(cudaGetLastError());
  }
  double* temp = h->d_coef + h->total_cols * nb;
  if (h->ntiles > 0) {
    dim3 grid((unsigned)h->ntiles, (unsigned)((nb + kNlocTileB - 1) / kNlocTileB));
    if (h->ntiles > INT32_MAX || grid.y > 65535u)
      return fail(SKGEMM_ERR_INVALID_ARG, "too many projector rows or bands");
    // Shared memory for the set's widest projector (C columns and chi rows).
    const int mc = (int)h->max_cols;
    const size_t smem = ((size_t)mc * kNlocTileB + kNlocTileR * (size_t)(mc + 1)) * 8;
    if (!h->chi_c_smem_set) {  // per handle: a handle belongs to one device
      const size_t smem_max = (kNlocMaxCols * kNlocTileB + kNlocTileR * (kNlocMaxCols + 1)) * 8;
      SKG_CUDA(cudaFuncSetAttribute(nloc_chi_c_kernel,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max));
      h->chi_c_smem_set = true;
    }
    KernelTimer kt_(s, "nloc_chi_c_kernel");
    nloc_chi_c_kernel<<<grid, 256, smem, s>>>(nb, mc, h->d_tile_proj, h->d_tile_r0, h->d_nrow,
                                              h->d_ncol, h->d_row_off, h->d_chi_off,
                                              h->d_proj_blk_col, h->d_chi, h->d_coef, temp);
    SKG_CUDA(cudaGetLastError());
  }
  const int64_t nbk = h->ntouch * ((nb + 1) / 2);  // threads: (touched point, band pair)
  if (nbk > 0) {
    if ((nbk + 255) / 256 > INT32_MAX)
      return fail(SKGEMM_ERR_INVALID_ARG, "too many touched points x bands");
    KernelTimer kt_(s, "nloc_backward_kernel");
    if (out_tile == 32)
      nloc_backward_kernel<32><<<(unsigned)((nbk + 255) / 256), 256, 0, s>>>(
          h->ntouch, nb, h->K, h->d_touch, h->d_touch_off, h->d_ent_off, temp, out);
    else
      nloc_backward_kernel<16><<<(unsigned)((nbk + 255) / 256), 256, 0, s>>>(
          h->ntouch, nb, h->K, h->d_touch, h->d_touch_off, h->d_ent_off, temp, out);
    SKG_CUDA(cudaGetLastError());
  }
  return SKGEMM_OK;
}

void nloc_destroy(skgemm_nloc* h) {
  if (!h) return;
  release(h);
  delete h;
}

}  // namespace skg
