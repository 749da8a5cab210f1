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
// The same body serves one problem (fp64_streamk_kernel, BM = BN = 128, or
// fp64_streamk_kernel64, BM = BN = 64) and a
// group of problems in one launch (fp64_grouped_kernel<TileShape>, the
// batched path: iterations of all problems concatenated, see Fp64Group).
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
  } else if (kind == kOpBandK) {
    tma_load_3d(dst, map, bar, 0, tile_idx * rows_per_tile, k0 / 16);
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

// One problem: its parameters and tensor maps are kernel parameters; flags
// carry the host-side epoch of the launch.
struct SingleSched {
  const Fp64Params& p;
  const CUtensorMap* mA;
  const CUtensorMap* mB;
  __device__ __forceinline__ int64_t total() const { return p.total_iters; }
  __device__ __forceinline__ int grid() const { return p.grid; }
  __device__ __forceinline__ const Fp64Params& prob(int) const { return p; }
  __device__ __forceinline__ const CUtensorMap* map_a(int) const { return mA; }
  __device__ __forceinline__ const CUtensorMap* map_b(int) const { return mB; }
  __device__ __forceinline__ int64_t begin(int) const { return 0; }
  __device__ __forceinline__ int locate(int64_t, int) const { return 0; }
  __device__ __forceinline__ double* workspace() const { return p.workspace; }
  __device__ __forceinline__ uint32_t* flags() const { return p.flags; }
  __device__ __forceinline__ uint32_t* err() const { return p.err; }
  __device__ __forceinline__ uint32_t pub() const { return p.epoch; }
};

// A group of problems: descriptors and tensor maps in global memory.
struct GroupSched {
  const Fp64Group& g;
  __device__ __forceinline__ int64_t total() const { return g.total_iters; }
  __device__ __forceinline__ int grid() const { return g.grid; }
  __device__ __forceinline__ const Fp64Params& prob(int i) const { return g.probs[i]; }
  __device__ __forceinline__ const CUtensorMap* map_a(int i) const { return g.maps + 2 * i; }
  __device__ __forceinline__ const CUtensorMap* map_b(int i) const { return g.maps + 2 * i + 1; }
  __device__ __forceinline__ int64_t begin(int i) const { return g.iter_begin[i]; }
  // Problem containing iteration `it`; `hint` is a problem at or before it.
  __device__ __forceinline__ int locate(int64_t it, int hint) const {
    int i = hint;
    if (g.iter_begin[i + 1] <= it) {
      int lo = i + 1, hi = g.num_problems - 1;  // invariant: answer in [lo, hi]
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (g.iter_begin[mid] <= it) lo = mid; else hi = mid - 1;
      }
      i = lo;
    }
    return i;
  }
  __device__ __forceinline__ double* workspace() const { return g.workspace; }
  __device__ __forceinline__ uint32_t* flags() const { return g.flags; }
  __device__ __forceinline__ uint32_t* err() const { return g.err; }
  __device__ __forceinline__ uint32_t pub() const { return 1u; }
};

// Where iteration `it` (< it_end) falls: problem, tile, k-block range of this
// CTA inside the tile and the tile coordinates.
struct Seg {
  int pid, tile, kb, ke, tm, tn;
};

template <class Sched>
__device__ __forceinline__ Seg locate_seg(const Sched& S, int64_t it, int64_t it_end, int hint) {
  Seg sg;
  sg.pid = S.locate(it, hint);
  const Fp64Params& q = S.prob(sg.pid);
  const int ipt = q.iters_per_tile;
  const int64_t local = it - S.begin(sg.pid);
  sg.tile = (int)(local / ipt);
  sg.kb = (int)(local - (int64_t)sg.tile * ipt);
  sg.ke = (int)((int64_t)ipt < sg.kb + (it_end - it) ? (int64_t)ipt : sg.kb + (it_end - it));
  tile_coords(q, sg.tile, sg.tm, sg.tn);
  return sg;
}

template <class TS, bool AKM = false, class Sched>
__device__ __forceinline__ void streamk_body(const Sched& S) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + kStages * TS::kStage);
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

  const int64_t it_begin = (int64_t)cta * S.total() / S.grid();
  const int64_t it_end = (int64_t)(cta + 1) * S.total() / S.grid();

  if (warp == kConsumerWarps) {
    // ------------------------------------------------------------ producer
    if (lane == 0) {
      int stage = 0;
      uint32_t phase = 0;
      int hint = S.locate(it_begin < it_end ? it_begin : 0, 0);
      int prefetched = -1;
      for (int64_t it = it_begin; it < it_end;) {
        const Seg sg = locate_seg(S, it, it_end, hint);
        hint = sg.pid;
        const Fp64Params& q = S.prob(sg.pid);
        const CUtensorMap* mA = S.map_a(sg.pid);
        const CUtensorMap* mB = S.map_b(sg.pid);
        if (prefetched != sg.pid) {
          tma_prefetch_desc(mA);
          tma_prefetch_desc(mB);
          prefetched = sg.pid;
        }
        for (int k = sg.kb; k < sg.ke; ++k) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1, S.err())) *abort_flag = 1;
          if (*abort_flag) break;
          uint8_t* sa = smem + stage * TS::kStage;
          uint8_t* sb = sa + TS::kABytes;
          mbar_arrive_expect_tx(&full_bar[stage], TS::kStage);
          load_operand(q.a_kind, mA, sa, &full_bar[stage], sg.tm, TS::BM, k * kBK);
          load_operand(q.b_kind, mB, sb, &full_bar[stage], sg.tn, TS::BN, k * kBK);
          if (++stage == kStages) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (*abort_flag) break;
        it += sg.ke - sg.kb;
      }
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  constexpr int MI = TS::MI, NJ = TS::NJ, NQ = TS::NQ;
  const int wm = warp >> 2;  // 0..1 : rows wm*BM/2 ..
  const int wn = warp & 3;   // 0..3 : cols wn*BN/4 ..
  const int g = lane >> 2;
  const int t = lane & 3;
  // Byte offsets inside a chunk of the two k-rows this lane reads per k8 step.
  // Row 2t holds MMA k index t, row 2t+1 holds MMA k index t+4; the 16-byte
  // unit g is XOR-swizzled with the row index (TMA SWIZZLE_128B).
  const uint32_t off_r0 = (2 * t) * 128 + ((g ^ (2 * t)) << 4);
  const uint32_t off_r1 = (2 * t + 1) * 128 + ((g ^ (2 * t + 1)) << 4);
  // K-major A (AKM): output row r holds its 16 k in one 128-byte row, the
  // 16-byte unit u at u ^ (r mod 8). MMA rows g and g + 8 are fed from tile
  // rows q(g) and 8 + q(g), q(g) = 4 (g % 2) + g / 2 (the epilogue stores
  // them there): the two g of a quarter-warp then differ in bit 2 of the
  // swizzle, so its 16-byte loads of unit 4s + t (k = 8s + 2t, 8s + 2t + 1)
  // hit 8 distinct units (conflict-free). Each load holds (a0, a2) or
  // (a1, a3) of the fragment and is transposed into its order. Step s's
  // unit is step 0's with bit 2 flipped: offset ^ (s << 6).
  const int qg = 4 * (g & 1) + (g >> 1);
  const uint32_t offk0 = qg * 128 + ((t ^ qg) << 4);
  const uint32_t smem_base = smem_u32(smem);
  __shared__ int fixup_ok;

  double acc[MI][NJ][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

  int stage = 0;
  uint32_t phase = 0;
  bool aborted = false;
  int hint = S.locate(it_begin < it_end ? it_begin : 0, 0);
  const uint32_t pubval = S.pub();

  for (int64_t it = it_begin; it < it_end;) {
    const Seg sg = locate_seg(S, it, it_end, hint);
    hint = sg.pid;
    const Fp64Params& q = S.prob(sg.pid);
    // Shared-memory chunk of this warp's B column chunks (logical wn*NQ+qq).
    // A packed32 operand lands as [half][tile32][BK][16]: logical chunk c
    // sits at (c % 2) * (BN/32) + c / 2.
    uint32_t b_chunk[NQ];
    const bool b32 = !AKM && (q.b_kind == kOpPacked32);  // AKM: B never packed32
#pragma unroll
    for (int qq = 0; qq < NQ; ++qq) {
      const int c = wn * NQ + qq;
      b_chunk[qq] = b32 ? (uint32_t)((c & 1) * (TS::BN / 32) + (c >> 1)) : (uint32_t)c;
    }

    for (int k = sg.kb; k < sg.ke && !aborted; ++k) {
      if (!mbar_wait(&full_bar[stage], phase, S.err())) {
        aborted = true;
        *abort_flag = 1;
        break;
      }
      const uint32_t sa = smem_base + stage * TS::kStage + (wm * MI) * kChunkBytes;
      const uint32_t sb = smem_base + stage * TS::kStage + TS::kABytes;
#pragma unroll
      for (int s = 0; s < kBK / 8; ++s) {
        const uint32_t ks = s * 8 * 128;  // k8 step = 8 rows of 128 B
        double2 a_lo[MI], a_hi[MI], b_lo[NQ], b_hi[NQ];
#pragma unroll
        for (int i = 0; i < MI; ++i) {
          if constexpr (AKM) {
            const uint32_t o = sa + i * kChunkBytes + (offk0 ^ (s << 6));
            const double2 r0 = lds128(o), r1 = lds128(o + 8 * 128);
            a_lo[i] = make_double2(r0.x, r1.x);
            a_hi[i] = make_double2(r0.y, r1.y);
          } else {
            a_lo[i] = lds128(sa + i * kChunkBytes + ks + off_r0);
            a_hi[i] = lds128(sa + i * kChunkBytes + ks + off_r1);
          }
        }
#pragma unroll
        for (int qq = 0; qq < NQ; ++qq) {
          b_lo[qq] = lds128(sb + b_chunk[qq] * kChunkBytes + ks + off_r0);
          b_hi[qq] = lds128(sb + b_chunk[qq] * kChunkBytes + ks + off_r1);
        }
#pragma unroll
        for (int i = 0; i < MI; ++i) {
#pragma unroll
          for (int qq = 0; qq < NQ; ++qq) {
            dmma_16x8x8(acc[i][2 * qq], a_lo[i].x, a_lo[i].y, a_hi[i].x, a_hi[i].y, b_lo[qq].x,
                        b_hi[qq].x);
            dmma_16x8x8(acc[i][2 * qq + 1], a_lo[i].x, a_lo[i].y, a_hi[i].x, a_hi[i].y,
                        b_lo[qq].y, b_hi[qq].y);
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
    const bool owner = (sg.kb == 0);
    const bool complete = owner && (sg.ke == q.iters_per_tile);
    const int ctid = threadIdx.x;  // 0..255
    constexpr int kSlot = TS::BM * TS::BN;
    if (!owner) {
      // Publish this CTA's partial tile (layout [reg][thread], coalesced).
      double* slot = S.workspace() + (int64_t)cta * kSlot;
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j)
#pragma unroll
          for (int r = 0; r < 4; ++r)
            __stcg(slot + ((i * NJ + j) * 4 + r) * kConsumerThreads + ctid, acc[i][j][r]);
      __threadfence();
      asm volatile("bar.sync 1, %0;" ::"n"(kConsumerThreads));
      if (ctid == 0) st_release_gpu(S.flags() + cta, pubval);
    } else {
      if (!complete) {
        // Add the partials of the later CTAs that cover the rest of this tile,
        // in ascending k order. A flag that does not arrive within the budget
        // is recorded in the error word and its partial is skipped; the CTA
        // keeps consuming its pipeline so no copy is left in flight.
        const int64_t tile_end = S.begin(sg.pid) + (int64_t)(sg.tile + 1) * q.iters_per_tile;
        for (int c2 = cta + 1; c2 < S.grid(); ++c2) {
          const int64_t s2 = (int64_t)c2 * S.total() / S.grid();
          if (s2 >= tile_end) break;
          if (ctid == 0)
            fixup_ok = fixup_flag_wait(S.flags() + c2, pubval, S.err(), kFixupBudgetNs) ? 1 : 0;
          asm volatile("bar.sync 1, %0;" ::"n"(kConsumerThreads));
          const bool have = fixup_ok != 0;
          asm volatile("bar.sync 1, %0;" ::"n"(kConsumerThreads));
          if (!have) continue;
          const double* slot = S.workspace() + (int64_t)c2 * kSlot;
#pragma unroll
          for (int i = 0; i < MI; ++i)
#pragma unroll
            for (int j = 0; j < NJ; ++j)
#pragma unroll
              for (int r = 0; r < 4; ++r)
                acc[i][j][r] += __ldcg(slot + ((i * NJ + j) * 4 + r) * kConsumerThreads + ctid);
        }
      }
      // Final epilogue for tile (tm, tn).
      const int64_t mbase = (int64_t)sg.tm * TS::BM + wm * (TS::BM / 2);
      const int64_t nbase = (int64_t)sg.tn * TS::BN + wn * (TS::BN / 4);
      const bool syrk_skip = (q.out_kind == kOutSyrkUpper) && (mbase > nbase + TS::BN / 4 - 1);
      if (!syrk_skip) {
#pragma unroll
        for (int i = 0; i < MI; ++i) {
          // MMA rows g, g + 8 sit at tile rows 2g, 2g + 1 (AKM: q(g), 8 + q(g)).
          const int64_t m0 = mbase + i * 16 + (AKM ? qg : 2 * g);
          const int64_t m1 = m0 + (AKM ? 8 : 1);
#pragma unroll
          for (int qq = 0; qq < NQ; ++qq) {
            const int64_t n0 = nbase + qq * 16 + 4 * t;
            store_row4(q, m0, n0, acc[i][2 * qq][0], acc[i][2 * qq + 1][0], acc[i][2 * qq][1],
                       acc[i][2 * qq + 1][1]);
            store_row4(q, m1, n0, acc[i][2 * qq][2], acc[i][2 * qq + 1][2],
                       acc[i][2 * qq][3], acc[i][2 * qq + 1][3]);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
    it += sg.ke - sg.kb;
  }
}

__global__ void __launch_bounds__(kThreads, 1)
    fp64_streamk_kernel(const __grid_constant__ CUtensorMap mapA,
                        const __grid_constant__ CUtensorMap mapB,
                        const __grid_constant__ Fp64Params p) {
  const SingleSched S{p, &mapA, &mapB};
  streamk_body<Tile128>(S);
}

// One problem on 64 x 64 tiles, two CTAs per SM.
__global__ void __launch_bounds__(kThreads, Tile64::kMinBlocks)
    fp64_streamk_kernel64(const __grid_constant__ CUtensorMap mapA,
                          const __grid_constant__ CUtensorMap mapB,
                          const __grid_constant__ Fp64Params p) {
  const SingleSched S{p, &mapA, &mapB};
  streamk_body<Tile64>(S);
}

// The same two kernels on a K-major A (kOpBandK: the rotation reading
// band-packed Psi, the band -> grid transposition folded into the loads).
__global__ void __launch_bounds__(kThreads, 1)
    fp64_streamk_kernel_ak(const __grid_constant__ CUtensorMap mapA,
                           const __grid_constant__ CUtensorMap mapB,
                           const __grid_constant__ Fp64Params p) {
  const SingleSched S{p, &mapA, &mapB};
  streamk_body<Tile128, true>(S);
}

__global__ void __launch_bounds__(kThreads, Tile64::kMinBlocks)
    fp64_streamk_kernel64_ak(const __grid_constant__ CUtensorMap mapA,
                             const __grid_constant__ CUtensorMap mapB,
                             const __grid_constant__ Fp64Params p) {
  const SingleSched S{p, &mapA, &mapB};
  streamk_body<Tile64, true>(S);
}

template <class TS>
__global__ void __launch_bounds__(kThreads, TS::kMinBlocks)
    fp64_grouped_kernel(const __grid_constant__ Fp64Group g) {
  const GroupSched S{g};
  streamk_body<TS>(S);
}

}  // namespace skg
