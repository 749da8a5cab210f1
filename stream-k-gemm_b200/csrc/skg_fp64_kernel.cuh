// Persistent Stream-K FP64 GEMM kernel for sm_100a (native-precision path).
//
// Computes, over a set of BM x BN output tiles, acc(m,n) = sum_k A(m,k) B(k,n)
// and applies one of three epilogues:
//   kOutRowMajor  D[m*ldd + n]                     = alpha*acc + gamma
//                 (gemm<double>::compute_packed, gemm_opt.cpp:314; gamma is a
//                  scalar added to every element, gemm_opt.cpp:201-204)
//   kOutSyrkUpper C[m + n*ldd], m <= n only        = alpha*acc + beta*C
//                 (sme_syrk<double>::compute, sme_syrk.hpp:137; upper triangle of
//                  a column-major M x M matrix)
//   kOutBand16    D[(n/16)*M*16 + m*16 + n%16]     = acc
//                 (sme_gemm_trp_3d<double>::compute, sme_trp_3d.hpp:194; the
//                  rotation writes band-packed output, no scaling)
//
// Work decomposition (Stream-K): the MAC-loop iterations of all tiles
// (tiles * ceil(K/BK)) are split evenly over the persistent CTAs. A CTA whose
// range starts inside a tile stores its partial accumulator to a workspace slot
// and publishes a flag; the CTA that owns the tile's k = 0 segment waits (with
// a time budget) for those flags, adds the partials in ascending-k order and
// runs the epilogue. The reduction order is a pure function of the schedule,
// so results are bitwise reproducible run to run.
//
// Data movement: one producer warp issues TMA tile loads (128B-swizzled boxes
// of 16 doubles x BK rows) into an NSTAGE ring; 8 consumer warps run FP64 DMMA
// (m16n8k8) from shared memory. Every operand tile in shared memory is a set of
// "chunks" [BK][16] doubles (16 rows/columns of the output, k-major rows of
// 128 B), which is exactly the reference's packed panel layout
// ([tiles][K][16], gemm_opt.cpp:342-354) restricted to a BK slice.
//
// Fragment mapping: lane (g = lane/4, t = lane%4) reads one 16-byte unit per
// (chunk, k-row) with ld.shared.v2.f64. MMA row r maps to chunk row 2r (r<8)
// or 2(r-8)+1, MMA column c of the even/odd n8 block of a pair maps to chunk
// column 2c / 2c+1, and MMA k index t / t+4 maps to k-row 2t / 2t+1 of the k8
// step. With the 128B swizzle (16B unit ^= k-row mod 8) every quarter-warp hits
// eight distinct bank groups, so fragment loads are conflict-free.
#pragma once

#include "skg_common.cuh"

#include "skg_fp64_types.h"

namespace skg {

// Tile index -> (tm, tn). kTilesAll: row-major over (tm, tn) so that
// consecutive tiles of one CTA share the A panel (L2 reuse). kTilesUpper:
// row-major over the upper triangle tm <= tn.
__device__ __forceinline__ void tile_coords(const Fp64Params& p, int tile, int& tm, int& tn) {
  if (p.tile_order == kTilesAll) {
    tm = tile / p.tiles_n;
    tn = tile - tm * p.tiles_n;
  } else {
    int T = p.tiles_n;
    int r = 0, rem = tile;
    while (rem >= T - r) {
      rem -= T - r;
      ++r;
    }
    tm = r;
    tn = r + rem;
  }
}

__device__ __forceinline__ void load_operand(int kind, const CUtensorMap* map, uint8_t* dst,
                                             uint64_t* bar, int tile_idx, int rows_per_tile,
                                             int k0) {
  if (kind == kOpPacked16) {
    tma_load_3d(dst, map, bar, 0, k0, tile_idx * (rows_per_tile / 16));
  } else if (kind == kOpPacked32) {
    const int per = rows_per_tile / 32;
    tma_load_3d(dst, map, bar, 0, k0, tile_idx * per);
    tma_load_3d(dst + per * kChunkBytes, map, bar, 16, k0, tile_idx * per);
  } else {
#pragma unroll 1
    for (int c = 0; c < rows_per_tile / 16; ++c)
      tma_load_2d(dst + c * kChunkBytes, map, bar, tile_idx * rows_per_tile + c * 16, k0);
  }
}

__device__ __forceinline__ void store_row4(const Fp64Params& p, int64_t m, int64_t n, double v0,
                                           double v1, double v2, double v3) {
  // Four consecutive columns n..n+3 of output row m.
  if (m >= p.M) return;
  double v[4] = {v0, v1, v2, v3};
  if (p.out_kind == kOutRowMajor) {
    double* row = p.D + m * p.ldd;
    bool vec_ok = (n + 3 < p.N) && ((((uintptr_t)(row + n)) & 15) == 0);
    if (vec_ok) {
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = p.alpha * v[i] + p.gamma;
      *reinterpret_cast<double2*>(row + n) = make_double2(v[0], v[1]);
      *reinterpret_cast<double2*>(row + n + 2) = make_double2(v[2], v[3]);
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (n + i < p.N) row[n + i] = p.alpha * v[i] + p.gamma;
    }
  } else if (p.out_kind == kOutSyrkUpper) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int64_t col = n + i;
      if (col < p.N && m <= col) {
        double* c = p.D + m + col * p.ldd;
        double r = p.alpha * v[i];
        if (!p.beta_zero) r += p.gamma * (*c);
        *c = r;
      }
    }
  } else {  // kOutBand16
    double* dst = p.D + (n >> 4) * (p.M * 16) + m * 16 + (n & 15);
    if (n + 3 < p.N) {
      *reinterpret_cast<double2*>(dst) = make_double2(v[0], v[1]);
      *reinterpret_cast<double2*>(dst + 2) = make_double2(v[2], v[3]);
    } else {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (n + i < p.N) dst[i] = v[i];
    }
  }
}

__global__ void __launch_bounds__(kThreads, 1)
    fp64_streamk_kernel(const __grid_constant__ CUtensorMap mapA,
                        const __grid_constant__ CUtensorMap mapB, const Fp64Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty_bar = full_bar + kStages;
  volatile int* abort_flag = reinterpret_cast<volatile int*>(empty_bar + kStages);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int cta = blockIdx.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], kConsumerWarps);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();

  const int64_t it_begin = (int64_t)cta * p.total_iters / p.grid;
  const int64_t it_end = (int64_t)(cta + 1) * p.total_iters / p.grid;
  const int ipt = p.iters_per_tile;

  if (warp == kConsumerWarps) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      tma_prefetch_desc(&mapA);
      tma_prefetch_desc(&mapB);
      int stage = 0;
      uint32_t phase = 0;
      for (int64_t it = it_begin; it < it_end;) {
        int tile = (int)(it / ipt);
        int kb = (int)(it - (int64_t)tile * ipt);
        int ke = (int)((int64_t)ipt < kb + (it_end - it) ? (int64_t)ipt : kb + (it_end - it));
        int tm, tn;
        tile_coords(p, tile, tm, tn);
        for (int k = kb; k < ke; ++k) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1, p.err)) *abort_flag = 1;
          if (*abort_flag) break;
          uint8_t* sa = smem + stage * kStageBytes;
          uint8_t* sb = sa + kTileABytes;
          mbar_arrive_expect_tx(&full_bar[stage], kStageBytes);
          load_operand(p.a_kind, &mapA, sa, &full_bar[stage], tm, kBM, k * kBK);
          load_operand(p.b_kind, &mapB, sb, &full_bar[stage], tn, kBN, k * kBK);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (*abort_flag) break;
        it += ke - kb;
      }
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  const int wm = warp >> 2;  // 0..1 : rows wm*64 .. +64
  const int wn = warp & 3;   // 0..3 : cols wn*32 .. +32
  const int g = lane >> 2;
  const int t = lane & 3;
  // Byte offsets inside a chunk of the two k-rows this lane reads per k8 step.
  // Row 2t holds MMA k index t, row 2t+1 holds MMA k index t+4; the 16-byte
  // unit g is XOR-swizzled with the row index (TMA SWIZZLE_128B).
  const uint32_t off_r0 = (2 * t) * 128 + ((g ^ (2 * t)) << 4);
  const uint32_t off_r1 = (2 * t + 1) * 128 + ((g ^ (2 * t + 1)) << 4);
  const uint32_t smem_base = smem_u32(smem);
  // Shared-memory chunk of this warp's two B column chunks (logical 2*wn+q).
  // A packed32 operand lands as [half][tile][BK][16]: logical chunk c sits at
  // (c % 2) * (BN/32) + c / 2.
  uint32_t b_chunk[2];
#pragma unroll
  for (int q = 0; q < 2; ++q)
    b_chunk[q] = (p.b_kind == kOpPacked32) ? (q * (kBN / 32) + wn) : (2 * wn + q);
  __shared__ int fixup_ok;

  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

  int stage = 0;
  uint32_t phase = 0;
  bool aborted = false;

  for (int64_t it = it_begin; it < it_end;) {
    const int tile = (int)(it / ipt);
    const int kb = (int)(it - (int64_t)tile * ipt);
    const int ke = (int)((int64_t)ipt < kb + (it_end - it) ? (int64_t)ipt : kb + (it_end - it));
    int tm, tn;
    tile_coords(p, tile, tm, tn);

    for (int k = kb; k < ke && !aborted; ++k) {
      if (!mbar_wait(&full_bar[stage], phase, p.err)) {
        aborted = true;
        *abort_flag = 1;
        break;
      }
      const uint32_t sa = smem_base + stage * kStageBytes + (wm * 4) * kChunkBytes;
      const uint32_t sb = smem_base + stage * kStageBytes + kTileABytes;
#pragma unroll
      for (int s = 0; s < kBK / 8; ++s) {
        const uint32_t ks = s * 8 * 128;  // k8 step = 8 rows of 128 B
        double2 a_lo[4], a_hi[4], b_lo[2], b_hi[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          a_lo[i] = lds128(sa + i * kChunkBytes + ks + off_r0);
          a_hi[i] = lds128(sa + i * kChunkBytes + ks + off_r1);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          b_lo[q] = lds128(sb + b_chunk[q] * kChunkBytes + ks + off_r0);
          b_hi[q] = lds128(sb + b_chunk[q] * kChunkBytes + ks + off_r1);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            dmma_16x8x8(acc[i][2 * q], a_lo[i].x, a_lo[i].y, a_hi[i].x, a_hi[i].y, b_lo[q].x,
                        b_hi[q].x);
            dmma_16x8x8(acc[i][2 * q + 1], a_lo[i].x, a_lo[i].y, a_hi[i].x, a_hi[i].y,
                        b_lo[q].y, b_hi[q].y);
          }
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty_bar[stage]);
      if (++stage == kStages) {
        stage = 0;
        phase ^= 1;
      }
    }
    if (aborted) break;

    // ---------------------------------------------------------- epilogue
    const bool owner = (kb == 0);
    const bool complete = owner && (ke == ipt);
    const int ctid = threadIdx.x;  // 0..255
    if (!owner) {
      // Publish this CTA's partial tile (layout [reg][thread], coalesced).
      double* slot = p.workspace + (int64_t)cta * (kBM * kBN);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int r = 0; r < 4; ++r)
            __stcg(slot + ((i * 4 + j) * 4 + r) * kConsumerThreads + ctid, acc[i][j][r]);
      __threadfence();
      asm volatile("bar.sync 1, %0;" ::"n"(kConsumerThreads));
      if (ctid == 0) st_release_gpu(p.flags + cta, p.epoch);
    } else {
      if (!complete) {
        // Add the partials of the later CTAs that cover the rest of this tile,
        // in ascending k order. A flag that does not arrive within the budget
        // is recorded in the error word and its partial is skipped; the CTA
        // keeps consuming its pipeline so no copy is left in flight.
        const int64_t tile_end = (int64_t)(tile + 1) * ipt;
        for (int c2 = cta + 1; c2 < p.grid; ++c2) {
          const int64_t s2 = (int64_t)c2 * p.total_iters / p.grid;
          if (s2 >= tile_end) break;
          if (ctid == 0) {
            const uint64_t t0 = globaltimer_ns();
            uint32_t spins = 0;
            int ok = 1;
            while (ld_acquire_gpu(p.flags + c2) != p.epoch) {
              __nanosleep(128);
              if (++spins > kFixupSpinCap || globaltimer_ns() - t0 > kFixupBudgetNs) {
                atomicOr(p.err, kDevErrFixupTimeout);
                ok = 0;
                break;
              }
            }
            fixup_ok = ok;
          }
          asm volatile("bar.sync 1, %0;" ::"n"(kConsumerThreads));
          const bool have = fixup_ok != 0;
          asm volatile("bar.sync 1, %0;" ::"n"(kConsumerThreads));
          if (!have) continue;
          const double* slot = p.workspace + (int64_t)c2 * (kBM * kBN);
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
              for (int r = 0; r < 4; ++r)
                acc[i][j][r] += __ldcg(slot + ((i * 4 + j) * 4 + r) * kConsumerThreads + ctid);
        }
      }
      // Final epilogue for tile (tm, tn).
      const int64_t mbase = (int64_t)tm * kBM + wm * 64;
      const int64_t nbase = (int64_t)tn * kBN + wn * 32;
      const bool syrk_skip = (p.out_kind == kOutSyrkUpper) && (mbase > nbase + 31);
      if (!syrk_skip) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int64_t m0 = mbase + i * 16 + 2 * g;
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int64_t n0 = nbase + q * 16 + 4 * t;
            store_row4(p, m0, n0, acc[i][2 * q][0], acc[i][2 * q + 1][0], acc[i][2 * q][1],
                       acc[i][2 * q + 1][1]);
            store_row4(p, m0 + 1, n0, acc[i][2 * q][2], acc[i][2 * q + 1][2], acc[i][2 * q][3],
                       acc[i][2 * q + 1][3]);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
    it += ke - kb;
  }
}

}  // namespace skg
