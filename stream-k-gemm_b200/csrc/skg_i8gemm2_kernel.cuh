// Lane-scheduled INT8 (or BF16) residue products on CTA pairs (tcgen05
// .cta_group::2): the S = Psi^T Psi / Hs = Psi^T H Psi products of the Ozaki
// path, the kSchedLanes schedule of skg_i8gemm_kernel.cuh on 256 x 256 tiles
// computed by a cluster of two CTAs on two SMs.
//
// Why: a 128 x 256 tile of the one-CTA kernel needs 48 KB of operands per
// 128-byte k-block (16 KB A + 32 KB B) for 4.2 M MACs, and its four-stage
// ring keeps about 144 KB in flight, short of what the L2 latency needs at
// the tensor pipe's rate (~72% busy). Here each CTA holds its 128 rows of A
// and its 128 rows (N / 2) of B: 32 KB per k-block for the same 4.2 M MACs
// per SM, and six stages in flight.
//
// Roles per CTA (320 threads): warp 0 TMA producer (both CTAs load their own
// halves; completions are counted on rank 0's full barrier), warp 1 MMA
// issuer (rank 0 only; both ranks' warp 1 allocate and free TMEM together),
// warps 2-9 epilogue (each CTA drains its own TMEM: rows 128 r .. +127 of the
// pair tile, all 256 columns) into the int32 partial slabs of its 128 x 256
// tile, exactly the slabs the one-CTA kernel writes, so the reconstruction
// is unchanged and the results are the same bit for bit.
//
// Barriers: full[s] (rank 0: one arrival with the byte count of both CTAs'
// loads), empty[s] and tfull[a] (each CTA: one arrival from rank 0's
// multicast commit), tempty[a] (rank 0: one arrival per epilogue warp of
// both CTAs; the peer's arrive remotely). Every wait is bounded; on expiry a
// CTA records the timeout and stops issuing work, the peer's waits then run
// out as well, and both CTAs meet at the final cluster barrier.
#pragma once

#include "skg_i8gemm_kernel.cuh"

namespace skg {

constexpr int kI8P2Stages = 6;
constexpr int kI8P2TileBytes = 128 * kI8BK;  // 16 KB: 128 rows x one k-block
constexpr int kI8P2StageBytes = 2 * kI8P2TileBytes;
constexpr int kI8P2SmemBytes = kI8P2Stages * kI8P2StageBytes + 1024 + 256;
static_assert(kI8P2SmemBytes <= 232448, "pair kernel exceeds 227 KB of shared memory");
static_assert((2 * kI8P2Stages + 4) * 8 + 8 <= 256, "pair kernel barrier area");

// Item of a cluster: pair tile t2 = w mod T2, lane q = w / T2 for
// w = cluster + j * clusters; this CTA's half is `rank`.
__device__ __forceinline__ bool i8p2_next_item(const I8Params& p, int cl, int ncl, int rank,
                                               I8Cursor& cur, I8Item& it) {
  const int total = p.T2 * p.Q;
  for (;;) {
    const int w = cl + cur.item * ncl;
    if (w >= total) return false;
    const int q = w / p.T2, t2 = w - q * p.T2;
    const int idx = p.lane_seg_off[q] + cur.seg;
    if (idx >= p.lane_seg_off[q + 1]) {
      ++cur.item;
      cur.seg = 0;
      continue;
    }
    const I8Segment s = p.segs[idx];
    const int4 pr = p.pairs[t2];
    it.l = s.l;
    it.kb0 = s.kb0;
    it.kb1 = s.kb1;
    it.t = rank ? pr.w : pr.z;
    it.slot = s.slot * p.T + it.t;
    it.tm = pr.x + rank;  // this CTA's 128-row tile
    it.tn = pr.y;
    ++cur.seg;
    return true;
  }
}

template <bool BF>
__global__ void __launch_bounds__(kI8Threads, 1)
    i8_gemm2_kernel(const __grid_constant__ CUtensorMap mapA,
                    const __grid_constant__ CUtensorMap mapB,
                    const __grid_constant__ CUtensorMap mapB2, const I8Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + kI8P2Stages * kI8P2StageBytes);
  uint64_t* empty_bar = full_bar + kI8P2Stages;
  uint64_t* tfull_bar = empty_bar + kI8P2Stages;
  uint64_t* tempty_bar = tfull_bar + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty_bar + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int rank = (int)cluster_ctarank();
  const int cl = blockIdx.x >> 1, ncl = gridDim.x >> 1;

  // Clusters with no work leave together (both ranks see the same items).
  {
    I8Cursor cur;
    I8Item probe;
    if (!i8p2_next_item(p, cl, ncl, rank, cur, probe)) return;
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < kI8P2Stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull_bar[a], 1);
      mbar_init(&tempty_bar[a], 2 * kI8EpiWarps);  // both CTAs' epilogue warps
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc_pair(tmem_slot, kI8TmemCols);
    tmem_relinquish_pair();
  }
  tc_fence_before();
  // Barriers initialised and TMEM allocated in both CTAs before any remote
  // arrival or pair MMA.
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  const uint32_t full0 = mapa_shared(smem_u32(full_bar), 0);     // rank 0's full[0]
  const uint32_t tempty0 = mapa_shared(smem_u32(tempty_bar), 0);  // rank 0's tempty[0]

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    if (lane == 0) {
      tma_prefetch_desc(&mapA);
      tma_prefetch_desc(&mapB);
      if (p.T1 > 0) tma_prefetch_desc(&mapB2);
      int stage = 0;
      uint32_t phase = 0;
      I8Cursor cur;
      int64_t issued = 0;
      I8Item it;
      while (!*abort_flag && i8p2_next_item(p, cl, ncl, rank, cur, it)) {
        const CUtensorMap* mb = (p.T1 > 0 && it.t >= p.T1) ? &mapB2 : &mapB;
        for (int kb = it.kb0; kb < it.kb1; ++kb) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1, p.err)) {
            *abort_flag = 1;
            break;
          }
          ++issued;
          uint8_t* sa = smem + stage * kI8P2StageBytes;
          if (rank == 0) mbar_arrive_expect_tx(&full_bar[stage], 2 * kI8P2StageBytes);
          const uint32_t fb = full0 + stage * 8;
          tma_load_3d_pair(sa, &mapA, fb, kb * kI8BK, it.tm * kI8BM, it.l);
          tma_load_3d_pair(sa + kI8P2TileBytes, mb, fb, kb * kI8BK, it.tn * kI8BN + 128 * rank,
                           it.l);
          if (++stage == kI8P2Stages) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      // Drain: the CTA may exit only after its last loads have landed. Rank
      // 0 sees them on its full barriers; rank 1's loads are complete once
      // the MMAs that read them have released the stage (empty barrier).
      for (int j = 1; j <= kI8P2Stages && j <= issued; ++j) {
        int s2 = stage - j;
        uint32_t ph = phase;
        if (s2 < 0) {
          s2 += kI8P2Stages;
          ph ^= 1;
        }
        if (rank == 0)
          mbar_wait(&full_bar[s2], ph, p.err);
        else
          mbar_wait(&empty_bar[s2], ph, p.err);
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------- MMA issuer
    if (lane == 0 && rank == 0) {
      const uint32_t idesc = BF ? umma_idesc_bf16(2 * kI8BM, kI8BN)
                                : umma_idesc_i8(2 * kI8BM, kI8BN, p.is_signed);
      const uint32_t smem_base = smem_u32(smem);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      I8Cursor cur;
      I8Item it;
      while (!*abort_flag && i8p2_next_item(p, cl, ncl, rank, cur, it)) {
        if (!mbar_wait(&tempty_bar[acc], acc_phase ^ 1, p.err)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t tmem_d = tmem_base + (uint32_t)(acc * kI8BN);
        for (int kb = it.kb0; kb < it.kb1; ++kb) {
          if (!mbar_wait(&full_bar[stage], phase, p.err)) {
            *abort_flag = 1;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_base + stage * kI8P2StageBytes;
          const uint64_t adesc = umma_desc_kmajor_sw128(sa);
          const uint64_t bdesc = umma_desc_kmajor_sw128(sa + kI8P2TileBytes);
#pragma unroll
          for (int kk = 0; kk < kI8BK / kI8UmmaK; ++kk) {
            const uint32_t accum = (kb > it.kb0 || kk > 0) ? 1u : 0u;
            if (BF)
              umma_bf16_pair(tmem_d, adesc + (uint64_t)(kk * 2), bdesc + (uint64_t)(kk * 2),
                             idesc, accum);
            else
              umma_i8_pair(tmem_d, adesc + (uint64_t)(kk * 2), bdesc + (uint64_t)(kk * 2), idesc,
                           accum);
          }
          umma_commit_pair(&empty_bar[stage], 0x3);  // frees the stage in both CTAs
          if (++stage == kI8P2Stages) {
            stage = 0;
            phase ^= 1;
          }
        }
        umma_commit_pair(&tfull_bar[acc], 0x3);  // both halves of the accumulator ready
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int quarter = warp & 3;
    const int row_in_tile = quarter * 32 + lane;
    const int c_begin = ((warp - 2) >> 2) * (kI8BN / 64);
    int acc = 0;
    uint32_t acc_phase = 0;
    I8Cursor cur;
    I8Item it;
    int32_t run[BF ? 128 : 1];
#pragma unroll
    for (int j = 0; j < (BF ? 128 : 1); ++j) run[j] = 0;
    while (i8p2_next_item(p, cl, ncl, rank, cur, it)) {
      if (*abort_flag || !mbar_wait(&tfull_bar[acc], acc_phase, p.err)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kI8BN);
      int32_t* dst = p.partials + ((int64_t)it.slot * kI8BM + row_in_tile) * kI8BN;
      if (BF) {
#pragma unroll
        for (int cc = 0; cc < 8; ++cc) {
          uint32_t v[16];
          tmem_ld_32x32b_x16(taddr + c_begin * 32 + cc * 16, v);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 16; ++j)
            run[(BF ? cc * 16 + j : 0)] += __float2int_rn(__uint_as_float(v[j]));
        }
      } else {
#pragma unroll 1
        for (int c = c_begin; c < c_begin + kI8BN / 64; ++c) {
          uint32_t v[32];
          tmem_ld_32x32b_x32(taddr + c * 32, v);
          tmem_ld_wait();
          int4* d4 = reinterpret_cast<int4*>(dst + c * 32);
#pragma unroll
          for (int j = 0; j < 8; ++j)
            d4[j] = make_int4((int)v[4 * j], (int)v[4 * j + 1], (int)v[4 * j + 2], (int)v[4 * j + 3]);
        }
      }
      // The accumulator is free as soon as it has been read: one arrival per
      // warp on rank 0's tempty barrier (remote for rank 1).
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cluster(tempty0 + acc * 8);
      if (BF) {
        I8Item nx;
        I8Cursor peek = cur;
        if (!i8p2_next_item(p, cl, ncl, rank, peek, nx) || nx.slot != it.slot) {
#pragma unroll
          for (int cc = 0; cc < 4; ++cc) {
            int4* d4 = reinterpret_cast<int4*>(dst + (c_begin + cc) * 32);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const int b = BF ? cc * 32 + 4 * j : 0;
              d4[j] = make_int4(run[b], run[(BF ? b + 1 : 0)], run[(BF ? b + 2 : 0)],
                                run[(BF ? b + 3 : 0)]);
            }
          }
#pragma unroll
          for (int j = 0; j < (BF ? 128 : 1); ++j) run[j] = 0;
        }
      }
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
  }

  // Teardown: every role's loop is bounded, so every thread of both CTAs
  // arrives here; neither CTA frees TMEM or exits while the other may still
  // arrive on its barriers or be read by a pair MMA.
  tc_fence_before();
  cluster_sync_all();
  tc_fence_after();
  if (warp == 1) tmem_dealloc_pair(tmem_base, kI8TmemCols);
}

}  // namespace skg
