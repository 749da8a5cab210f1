// 8-bit x 8-bit -> INT32 GEMM on tcgen05 tensor cores (sm_100a), the engine of
// the Ozaki split-precision path. Exact: operands are signed bytes (s8 x s8,
// products <= 2^14: symmetric residues and the public integer GEMM; an
// unsigned u8 x u8 mode exists for callers with byte data); the host cuts the
// k range into segments short enough that a 32-bit accumulator cannot
// overflow.
//
// Operands are per-modulus residue matrices, K-major bytes:
//   A_res[l][RA][KP], B_res[l][RB][KP]   (row r, k contiguous; zero padding)
// loaded by TMA boxes {128 B of k, 128 (A) / 256 (B) rows, 1 modulus} with the
// 128-byte swizzle, which is the canonical K-major SW128 UMMA layout.
//
// CTA: 320 threads = warp 0 TMA producer, warp 1 MMA issuer (one thread) and
// TMEM owner, warps 2-9 epilogue (warp w reads TMEM lanes 32*(w%4)..+31 and
// columns 128*((w-2)/4)..+127: two epilogue warps per TMEM lane quarter keep
// the epilogue's latency hidden).
// Tile 128 x 256 (UMMA M=128, N=256, K=32), 4-stage smem ring (48 KB/stage),
// two 256-column TMEM accumulators so the epilogue of one work item overlaps
// the MMAs of the next.
//
// BF16 variant (template BF): the same residues stored as BF16 (|r| <= 128
// is exact in BF16), kind::f16 MMAs with FP32 accumulators, 64 k per 128-byte
// k-block. A sum of at most 1024 products of magnitude <= 2^14 is an integer
// of magnitude <= 2^24, which FP32 holds exactly, so the host cuts the k range
// into sub-segments of <= 16 k-blocks; the lanes epilogue converts each
// sub-segment's FP32 tile to int32 and adds it into registers until the
// slot changes (<= 127 sub-segments per slot keeps |sum| < 2^31), then writes
// the slab. Results equal the INT8 path's bit for bit.
//
// Schedules:
//  kSchedLanes   (huge K, small M x N: S = Psi^T Psi, Hs = Psi^T H Psi)
//     T x Q items (tile t, lane q), persistent: CTA c takes items
//     c, c + grid, ... with t = item mod T, q = item / T. Lane q owns a
//     contiguous range of the (modulus, k-block) space; the T CTAs working on
//     one lane at a time walk the same range in lockstep, so each
//     (modulus, k-range) panel of A and B is read from HBM about once and
//     served to the other tiles from L2. The host picks Q so that T x Q items
//     fill whole waves of the grid (lanes_for). Each
//     segment (one modulus, <= seg_kb_cap k-blocks) ends in an int32 partial
//     slab written to `partials[seg_slot][t]` (plan-built slot table).
//  kSchedUnits   (huge M, small K: Psi' = Psi Q)
//     work units (tm, l, tn) with the full K, round-robin over CTAs; the
//     epilogue writes (acc mod m_l) as one byte per element to
//     `residues[l][row][col]`.
#pragma once

#include "skg_common.cuh"
#include "skg_tcgen05.cuh"

namespace skg {

constexpr int kI8BM = 128;
constexpr int kI8BN = 256;
constexpr int kI8BK = 128;  // bytes of k per stage
constexpr int kI8UmmaK = 32;
constexpr int kI8Stages = 4;
constexpr int kI8EpiWarps = 8;
constexpr int kI8Threads = 64 + 32 * kI8EpiWarps;
constexpr int kI8TileABytes = kI8BM * kI8BK;  // 16 KB
constexpr int kI8TileBBytes = kI8BN * kI8BK;  // 32 KB
constexpr int kI8StageBytes = kI8TileABytes + kI8TileBBytes;
constexpr int kI8SmemBytes = kI8Stages * kI8StageBytes + 1024 + 256;
constexpr int kI8TmemCols = 512;
constexpr int kI8MaxModuli = 16;

enum I8Sched : int { kSchedLanes = 0, kSchedUnits = 1 };

// One k-segment of a lane: modulus l, k-blocks [kb0, kb1), partial slot.
struct I8Segment {
  int l, kb0, kb1, slot;
};

struct I8Params {
  int sched;
  int is_signed;     // 1: s8 x s8, 0: u8 x u8
  int L;             // moduli
  int KB;            // k-blocks of the padded K (KP / 128)
  int M, N;          // output extent (bounds of stores)
  // kSchedLanes
  int T;             // tiles
  int T1;            // tiles t >= T1 (T1 > 0) take B from mapB2 (fused subspace pair)
  int Q;             // lanes
  const int2* tiles;            // [T] (tm, tn)
  const int* lane_seg_off;      // [Q+1] offsets into segs
  const I8Segment* segs;        // segments of all lanes
  int32_t* partials;            // [slots][T][128][256]
  // kSchedUnits
  int tiles_m, tiles_n;
  uint8_t* residues;            // [L][M][ldr]
  int64_t ldr;
  uint32_t* err;
  // kSchedLanes on CTA pairs (i8_gemm2_kernel): T2 pair tiles, each two
  // vertically adjacent 128 x 256 tiles {tm_lo, tn, t_lo, t_hi} (t_* index
  // `tiles`, which then holds both halves of every pair).
  int T2;
  const int4* pairs;
};

// Moduli and the constants of an exact remainder by multiply-high: with
// magic = floor(2^37 / m) + 1, q = umulhi(u, magic) >> 5 equals floor(u / m)
// for every 0 <= u < 2^29 and m <= 256 (the rounding excess u * (magic -
// 2^37/m) / 2^37 stays below 2^-8 <= 1/m). `offset` is a multiple of m
// >= 2^25 that makes a signed accumulator (|acc| < 2^25, K <= 2048)
// non-negative.
// For K <= 512 and symmetric residues of an odd modulus (|r| <= 127, so
// |acc| <= 512 * 127^2 = 8258048) the rotation kernel uses a shorter form:
// offset24 = the smallest multiple of m >= 8258048 puts u = acc + offset24
// in [0, 2^24), where q = umulhi(u, magic24 = ceil(2^32 / m)) is already
// floor(u / m) (excess below u / 2^32 < 2^-8 < 1/m), with no shift. For
// m = 256 the residue is the accumulator's low byte.
struct I8ModConsts {
  uint32_t m[kI8MaxModuli];
  uint32_t magic[kI8MaxModuli];
  uint32_t offset[kI8MaxModuli];
  uint32_t magic24[kI8MaxModuli];
  uint32_t offset24[kI8MaxModuli];
};

// Moduli of the residue epilogue (constant memory: indexed by the work item's
// modulus, uniform across the warp).
__constant__ I8ModConsts c_i8mod;

__device__ __forceinline__ uint32_t mod_exact29(uint32_t u, uint32_t m, uint32_t magic) {
  const uint32_t q = __umulhi(u, magic) >> 5;
  return u - q * m;
}

__device__ __forceinline__ uint32_t mod_exact24(uint32_t u, uint32_t m, uint32_t magic24) {
  return u - __umulhi(u, magic24) * m;
}

// Work item seen by all roles.
struct I8Item {
  int l, tm, tn, kb0, kb1, slot, t;
};

// Position of one role in the CTA's item sequence: the persistent item
// (lanes: (tile, lane) pair; units: work unit) and, for lanes, the segment
// within that lane.
struct I8Cursor {
  int item = 0;
  int seg = 0;
};

__device__ __forceinline__ bool i8_next_item(const I8Params& p, int cta, I8Cursor& cur,
                                             I8Item& it) {
  if (p.sched == kSchedLanes) {
    // Persistent over the T x Q items w = cta + j * grid (tile t = w mod T,
    // lane q = w / T): consecutive CTAs take the tiles of one lane, which
    // read the same (modulus, k) panels at the same time.
    const int total = p.T * p.Q;
    for (;;) {
      const int w = cta + cur.item * (int)gridDim.x;
      if (w >= total) return false;
      const int q = w / p.T, t = w - q * p.T;
      const int idx = p.lane_seg_off[q] + cur.seg;
      if (idx >= p.lane_seg_off[q + 1]) {
        ++cur.item;
        cur.seg = 0;
        continue;
      }
      const I8Segment s = p.segs[idx];
      const int2 tt = p.tiles[t];
      it.l = s.l;
      it.kb0 = s.kb0;
      it.kb1 = s.kb1;
      it.slot = s.slot * p.T + t;
      it.t = t;
      it.tm = tt.x;
      it.tn = tt.y;
      ++cur.seg;
      return true;
    }
  }
  // kSchedUnits: u = cta + item * grid, order (tm, l, tn)
  const int64_t u = (int64_t)cta + (int64_t)cur.item * gridDim.x;
  const int64_t total = (int64_t)p.tiles_m * p.L * p.tiles_n;
  if (u >= total) return false;
  const int tn = (int)(u % p.tiles_n);
  const int64_t r = u / p.tiles_n;
  it.l = (int)(r % p.L);
  it.tm = (int)(r / p.L);
  it.tn = tn;
  it.kb0 = 0;
  it.kb1 = p.KB;
  it.slot = 0;
  it.t = 0;
  ++cur.item;
  return true;
}

// Residue epilogue of one 128 x 256 work item (modulus it.l): this thread's
// row `row` of the tile, TMEM column chunks [c_begin, c_end) of 32, written
// as (acc mod m_l) bytes to residues[l][row][col] (row stride ldr).
// s8 x s8 accumulators: |acc| <= K 2^14 < 2^25 (K <= 2048); acc + offset is
// non-negative and below 2^29.
template <bool BF>
__device__ __forceinline__ void i8_residue_epilogue(uint32_t taddr, int c_begin, int c_end,
                                                    const I8Item& it, int row, int M, int N,
                                                    uint8_t* residues, int64_t ldr) {
  const uint32_t m = c_i8mod.m[it.l], magic = c_i8mod.magic[it.l];
  const uint32_t off = c_i8mod.offset[it.l];
  const bool row_ok = row < M;
  uint8_t* dst = residues + ((int64_t)it.l * M + row) * ldr;
#pragma unroll 1
  for (int c = c_begin; c < c_end; ++c) {
    uint32_t v[32];
    tmem_ld_32x32b_x32(taddr + c * 32, v);
    tmem_ld_wait();
    if (BF) {
      // FP32 accumulators hold exact integers (K <= 1024): back to int32.
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = (uint32_t)__float2int_rn(__uint_as_float(v[j]));
    }
    const int col0 = it.tn * kI8BN + c * 32;
    if (row_ok && col0 < N) {
      uint32_t w[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t b0 = mod_exact29(v[4 * j] + off, m, magic);
        const uint32_t b1 = mod_exact29(v[4 * j + 1] + off, m, magic);
        const uint32_t b2 = mod_exact29(v[4 * j + 2] + off, m, magic);
        const uint32_t b3 = mod_exact29(v[4 * j + 3] + off, m, magic);
        w[j] = __byte_perm(__byte_perm(b0, b1, 0x0040), __byte_perm(b2, b3, 0x0040), 0x5410);
      }
      if (col0 + 32 <= N) {
        uint4* d4 = reinterpret_cast<uint4*>(dst + col0);
        d4[0] = make_uint4(w[0], w[1], w[2], w[3]);
        d4[1] = make_uint4(w[4], w[5], w[6], w[7]);
      } else {
        for (int j = 0; j < 32 && col0 + j < N; ++j)
          dst[col0 + j] = (uint8_t)(w[j >> 2] >> (8 * (j & 3)));
      }
    }
  }
}

template <bool BF>
__global__ void __launch_bounds__(kI8Threads, 1)
    i8_gemm_kernel(const __grid_constant__ CUtensorMap mapA,
                   const __grid_constant__ CUtensorMap mapB,
                   const __grid_constant__ CUtensorMap mapB2, const I8Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + kI8Stages * kI8StageBytes);
  uint64_t* empty_bar = full_bar + kI8Stages;
  uint64_t* tfull_bar = empty_bar + kI8Stages;
  uint64_t* tempty_bar = tfull_bar + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty_bar + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int cta = blockIdx.x;

  // Idle CTAs (no work at all) leave before touching TMEM.
  {
    I8Cursor cur;
    I8Item probe;
    if (!i8_next_item(p, cta, cur, probe)) return;
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < kI8Stages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull_bar[a], 1);
      mbar_init(&tempty_bar[a], kI8EpiWarps);  // one arrival per epilogue warp
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, kI8TmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

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
      while (!*abort_flag && i8_next_item(p, cta, cur, it)) {
        const CUtensorMap* mb = (p.T1 > 0 && it.t >= p.T1) ? &mapB2 : &mapB;
        for (int kb = it.kb0; kb < it.kb1; ++kb) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1, p.err)) {
            *abort_flag = 1;
            break;
          }
          ++issued;
          uint8_t* sa = smem + stage * kI8StageBytes;
          mbar_arrive_expect_tx(&full_bar[stage], kI8StageBytes);
          tma_load_3d(sa, &mapA, &full_bar[stage], kb * kI8BK, it.tm * kI8BM, it.l);
          tma_load_3d(sa + kI8TileABytes, mb, &full_bar[stage], kb * kI8BK, it.tn * kI8BN, it.l);
          if (++stage == kI8Stages) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      // Drain: the last (up to kI8Stages) loads issued have landed before the
      // CTA may exit (immediate on the normal path, where the MMA issuer has
      // already consumed them; bounded on an abort path).
      for (int j = 1; j <= kI8Stages && j <= issued; ++j) {
        int s2 = stage - j;
        uint32_t ph = phase;
        if (s2 < 0) {
          s2 += kI8Stages;
          ph ^= 1;
        }
        mbar_wait(&full_bar[s2], ph, p.err);
      }
    }
  } else if (warp == 1) {
    // --------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc =
          BF ? umma_idesc_bf16(kI8BM, kI8BN) : umma_idesc_i8(kI8BM, kI8BN, p.is_signed);
      const uint32_t smem_base = smem_u32(smem);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      I8Cursor cur;
      I8Item it;
      while (!*abort_flag && i8_next_item(p, cta, cur, it)) {
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
          const uint32_t sa = smem_base + stage * kI8StageBytes;
          const uint64_t adesc = umma_desc_kmajor_sw128(sa);
          const uint64_t bdesc = umma_desc_kmajor_sw128(sa + kI8TileABytes);
#pragma unroll
          for (int kk = 0; kk < kI8BK / kI8UmmaK; ++kk) {
            // advance 32 bytes of k inside the 128-byte swizzle atom (32 INT8
            // or 16 BF16 values: one MMA's K either way)
            const uint32_t accum = (kb > it.kb0 || kk > 0) ? 1u : 0u;
            if (BF)
              umma_bf16(tmem_d, adesc + (uint64_t)(kk * 2), bdesc + (uint64_t)(kk * 2), idesc,
                        accum);
            else
              umma_i8(tmem_d, adesc + (uint64_t)(kk * 2), bdesc + (uint64_t)(kk * 2), idesc,
                      accum);
          }
          umma_commit(&empty_bar[stage]);  // frees the smem stage when these MMAs finish
          if (++stage == kI8Stages) {
            stage = 0;
            phase ^= 1;
          }
        }
        umma_commit(&tfull_bar[acc]);  // accumulator ready for the epilogue
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int quarter = warp & 3;  // TMEM lanes 32*quarter .. +31
    const int row_in_tile = quarter * 32 + lane;
    const int c_begin = ((warp - 2) >> 2) * (kI8BN / 64), c_end = c_begin + kI8BN / 64;
    int acc = 0;
    uint32_t acc_phase = 0;
    I8Cursor cur;
    I8Item it;
    int32_t run[BF ? 128 : 1];  // BF16 lanes: int32 sums of this slot's sub-segments
#pragma unroll
    for (int j = 0; j < (BF ? 128 : 1); ++j) run[j] = 0;
    while (i8_next_item(p, cta, cur, it)) {
      if (*abort_flag || !mbar_wait(&tfull_bar[acc], acc_phase, p.err)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * kI8BN);
      const int row = it.tm * kI8BM + row_in_tile;
      bool released = false;
      if (p.sched == kSchedLanes) {
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
          // The accumulator is free as soon as it has been read.
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty_bar[acc]);
          released = true;
          I8Item nx;
          I8Cursor peek = cur;
          if (!i8_next_item(p, cta, peek, nx) || nx.slot != it.slot) {
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
        } else {
#pragma unroll 1
          for (int c = c_begin; c < c_end; ++c) {
            uint32_t v[32];
            tmem_ld_32x32b_x32(taddr + c * 32, v);
            tmem_ld_wait();
            int4* d4 = reinterpret_cast<int4*>(dst + c * 32);
#pragma unroll
            for (int j = 0; j < 8; ++j)
              d4[j] = make_int4((int)v[4 * j], (int)v[4 * j + 1], (int)v[4 * j + 2], (int)v[4 * j + 3]);
          }
        }
      } else {
        i8_residue_epilogue<BF>(taddr, c_begin, c_end, it, row, p.M, p.N, p.residues, p.ldr);
      }
      if (!released) {
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty_bar[acc]);
      }
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
  }

  // Teardown: every role's loop is bounded, so all threads arrive here.
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, kI8TmemCols);
}


// ---------------------------------------------------------------------------
// Rotation kernel with B resident in shared memory (Psi' = Psi Q, K = nb
// <= 512). Work units (l, tm, tn) as in kSchedUnits, but CTA c belongs to
// group q = c / tiles_n and fixed column tile tn = c % tiles_n; group q walks
// the contiguous range [q V / G, (q+1) V / G) of the V = L * tiles_m units
// (l, tm) (l major). The CTA keeps B_l[tn] (256 rows x KP bytes, all k
// blocks) in shared memory while l stays the same and streams only A tiles,
// so the per-unit shared-memory fill is 128 x KP bytes instead of 384 x KP;
// the tiles_n CTAs of a group read the same A tiles at the same time, so HBM
// serves each A tile about once and L2 the rest.
//
// Epilogue: each epilogue warp owns a 32-row x 128-column box of the tile;
// it writes the box's residue bytes to shared memory in the TMA 128-byte
// swizzle (conflict-free: 4 wavefronts per 16-byte store) and one lane issues
// a TMA store of the box, so global writes go out as whole 128-byte lines
// instead of 32 scattered 16-byte pieces per store instruction.
//
// Shared memory: B region (kI8RotKbMax x 32 KB) | A ring (kI8RotStages x
// 16 KB) | 8 store boxes (4 KB each) | barriers. B reloads wait for the MMAs
// that read the old B (bempty, committed by the MMA issuer when l changes).
constexpr int kI8RotKbMax = 4;  // KP <= 512
constexpr int kI8RotStages = 4;
constexpr int kI8RotBBytes = kI8RotKbMax * kI8TileBBytes;
constexpr int kI8RotBoxBytes = 32 * 128;
constexpr int kI8RotSmemBytes = kI8RotBBytes + kI8RotStages * kI8TileABytes +
                                kI8EpiWarps * kI8RotBoxBytes + 1024 + 256;
static_assert(kI8RotSmemBytes <= 232448, "rotation kernel exceeds 227 KB of shared memory");
static_assert((2 * kI8RotStages + 6) * 8 + 8 <= 256, "rotation kernel barrier area");

struct I8RotParams {
  int L, KB;            // moduli, k-blocks of KP (KB <= kI8RotKbMax)
  int M, N;             // output extent (Nd, nb); residues [L][M][N] through mapR
  int tiles_m, tiles_n;
  int groups;           // grid = groups * tiles_n
  uint32_t* err;
};

__device__ __forceinline__ bool rot_next_item(const I8RotParams& p, int cta, int& cursor,
                                              I8Item& it) {
  const int q = cta / p.tiles_n;
  if (q >= p.groups) return false;
  const int64_t V = (int64_t)p.L * p.tiles_m;
  const int64_t b = V * q / p.groups, e = V * (q + 1) / p.groups;
  const int64_t v = b + cursor;
  if (v >= e) return false;
  it.l = (int)(v / p.tiles_m);
  it.tm = (int)(v - (int64_t)it.l * p.tiles_m);
  it.tn = cta - q * p.tiles_n;
  it.kb0 = 0;
  it.kb1 = p.KB;
  it.slot = 0;
  ++cursor;
  return true;
}

__global__ void __launch_bounds__(kI8Threads, 1)
    i8_rot_kernel(const __grid_constant__ CUtensorMap mapA,
                  const __grid_constant__ CUtensorMap mapB,
                  const __grid_constant__ CUtensorMap mapR, const I8RotParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint8_t* sB = smem;
  uint8_t* sA = smem + kI8RotBBytes;
  uint8_t* sR = sA + kI8RotStages * kI8TileABytes;
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(sR + kI8EpiWarps * kI8RotBoxBytes);
  uint64_t* empty_bar = full_bar + kI8RotStages;
  uint64_t* bfull = empty_bar + kI8RotStages;
  uint64_t* bempty = bfull + 1;
  uint64_t* tfull_bar = bempty + 1;
  uint64_t* tempty_bar = tfull_bar + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty_bar + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int cta = blockIdx.x;

  // Idle CTAs and shapes outside the B region leave before touching TMEM.
  if (p.KB < 1 || p.KB > kI8RotKbMax) return;
  {
    int cur = 0;
    I8Item probe;
    if (!rot_next_item(p, cta, cur, probe)) return;
  }

  if (threadIdx.x == 0) {
    for (int s = 0; s < kI8RotStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(bfull, 1);
    mbar_init(bempty, 1);
    for (int a = 0; a < 2; ++a) {
      mbar_init(&tfull_bar[a], 1);
      mbar_init(&tempty_bar[a], kI8EpiWarps);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, kI8TmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    if (lane == 0) {
      tma_prefetch_desc(&mapA);
      tma_prefetch_desc(&mapB);
      tma_prefetch_desc(&mapR);
      int stage = 0;
      uint32_t phase = 0;
      int cur = 0;
      int64_t issued = 0;
      int cur_l = -1;
      uint32_t bempty_ph = 0;
      int b_loads = 0;
      I8Item it;
      while (!*abort_flag && rot_next_item(p, cta, cur, it)) {
        if (it.l != cur_l) {
          // B_l[tn] for the next run of units: all k blocks, one barrier.
          if (cur_l >= 0) {
            if (!mbar_wait(bempty, bempty_ph, p.err)) {
              *abort_flag = 1;
              break;
            }
            bempty_ph ^= 1;
          }
          mbar_arrive_expect_tx(bfull, (uint32_t)(p.KB * kI8TileBBytes));
          for (int kb = 0; kb < p.KB; ++kb)
            tma_load_3d(sB + kb * kI8TileBBytes, &mapB, bfull, kb * kI8BK, it.tn * kI8BN, it.l);
          ++b_loads;
          cur_l = it.l;
        }
        for (int kb = 0; kb < p.KB; ++kb) {
          if (!mbar_wait(&empty_bar[stage], phase ^ 1, p.err)) {
            *abort_flag = 1;
            break;
          }
          ++issued;
          mbar_arrive_expect_tx(&full_bar[stage], kI8TileABytes);
          tma_load_3d(sA + stage * kI8TileABytes, &mapA, &full_bar[stage], kb * kI8BK,
                      it.tm * kI8BM, it.l);
          if (++stage == kI8RotStages) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      // Drain: the last A loads and the last B load have landed before the
      // CTA may exit (immediate on the normal path; bounded on an abort path).
      for (int j = 1; j <= kI8RotStages && j <= issued; ++j) {
        int s2 = stage - j;
        uint32_t ph = phase;
        if (s2 < 0) {
          s2 += kI8RotStages;
          ph ^= 1;
        }
        mbar_wait(&full_bar[s2], ph, p.err);
      }
      if (b_loads > 0) mbar_wait(bfull, (uint32_t)((b_loads - 1) & 1), p.err);
    }
  } else if (warp == 1) {
    // --------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_i8(kI8BM, kI8BN, 1);
      const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
      int stage = 0;
      uint32_t phase = 0;
      int acc = 0;
      uint32_t acc_phase = 0;
      int cur = 0;
      int cur_l = -1;
      uint32_t bfull_ph = 0;
      I8Item it;
      while (!*abort_flag && rot_next_item(p, cta, cur, it)) {
        if (it.l != cur_l) {
          // Every MMA issued so far read the old B: release it once they finish.
          if (cur_l >= 0) umma_commit(bempty);
          if (!mbar_wait(bfull, bfull_ph, p.err)) {
            *abort_flag = 1;
            break;
          }
          bfull_ph ^= 1;
          cur_l = it.l;
        }
        if (!mbar_wait(&tempty_bar[acc], acc_phase ^ 1, p.err)) {
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t tmem_d = tmem_base + (uint32_t)(acc * kI8BN);
        for (int kb = 0; kb < p.KB; ++kb) {
          if (!mbar_wait(&full_bar[stage], phase, p.err)) {
            *abort_flag = 1;
            break;
          }
          tc_fence_after();
          const uint64_t adesc = umma_desc_kmajor_sw128(a_base + stage * kI8TileABytes);
          const uint64_t bdesc = umma_desc_kmajor_sw128(b_base + kb * kI8TileBBytes);
#pragma unroll
          for (int kk = 0; kk < kI8BK / kI8UmmaK; ++kk)
            umma_i8(tmem_d, adesc + (uint64_t)(kk * 2), bdesc + (uint64_t)(kk * 2), idesc,
                    (kb > 0 || kk > 0) ? 1u : 0u);
          umma_commit(&empty_bar[stage]);
          if (++stage == kI8RotStages) {
            stage = 0;
            phase ^= 1;
          }
        }
        umma_commit(&tfull_bar[acc]);
        if (++acc == 2) {
          acc = 0;
          acc_phase ^= 1;
        }
      }
    }
  } else {
    // ---------------------------------------------------------- epilogue
    const int quarter = warp & 3;                  // TMEM lanes / tile rows 32*quarter..+31
    const int half = (warp - 2) >> 2;              // tile columns 128*half..+127
    uint8_t* box = sR + (warp - 2) * kI8RotBoxBytes;
    uint8_t* my_row = box + lane * 128;
    const int sw = lane & 7;                       // 128-byte swizzle of this box row
    int acc = 0;
    uint32_t acc_phase = 0;
    int cur = 0;
    I8Item it;
    while (rot_next_item(p, cta, cur, it)) {
      if (*abort_flag || !mbar_wait(&tfull_bar[acc], acc_phase, p.err)) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) +
                             (uint32_t)(acc * kI8BN + half * 128);
      // The box is free once the previous unit's store has read it.
      if (lane == 0) bulk_wait_read_all();
      __syncwarp();
      // K <= 512: the 24-bit remainder (no shift); m = 256 keeps the low
      // byte of the accumulator as it is.
      const uint32_t m = c_i8mod.m[it.l], magic = c_i8mod.magic24[it.l];
      const uint32_t off = c_i8mod.offset24[it.l];
      const bool pow2 = (m == 256u);
#pragma unroll 1
      for (int c = 0; c < 4; c += 2) {
        uint32_t v0[32], v1[32];
        tmem_ld_32x32b_x32(taddr + c * 32, v0);
        tmem_ld_32x32b_x32(taddr + c * 32 + 32, v1);
        tmem_ld_wait();
        if (!pow2) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            v0[j] = mod_exact24(v0[j] + off, m, magic);
            v1[j] = mod_exact24(v1[j] + off, m, magic);
          }
        }
        uint32_t w[16];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          w[j] = __byte_perm(__byte_perm(v0[4 * j], v0[4 * j + 1], 0x0040),
                             __byte_perm(v0[4 * j + 2], v0[4 * j + 3], 0x0040), 0x5410);
          w[8 + j] = __byte_perm(__byte_perm(v1[4 * j], v1[4 * j + 1], 0x0040),
                                 __byte_perm(v1[4 * j + 2], v1[4 * j + 3], 0x0040), 0x5410);
        }
#pragma unroll
        for (int h = 0; h < 4; ++h)
          *reinterpret_cast<uint4*>(my_row + (((2 * c + h) ^ sw) << 4)) =
              make_uint4(w[4 * h], w[4 * h + 1], w[4 * h + 2], w[4 * h + 3]);
      }
      // TMEM reads done: hand the accumulator back before the store.
      tc_fence_before();
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&tempty_bar[acc]);
        const int x = it.tn * kI8BN + half * 128, y = it.tm * kI8BM + quarter * 32;
        if (x < p.N && y < p.M) {
          tma_store_3d(&mapR, box, x, y, it.l);
          bulk_commit_group();
        }
      }
      if (++acc == 2) {
        acc = 0;
        acc_phase ^= 1;
      }
    }
    if (lane == 0) bulk_wait_all();
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, kI8TmemCols);
}

// INT8 tensor-core peak probe: MMAs on one resident smem stage (no TMA),
// accumulating into TMEM; used only to measure the kind::i8 throughput.
__global__ void __launch_bounds__(128, 1) i8_peak_kernel(int iters, uint32_t* sink) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~uintptr_t(1023));
  uint64_t* done = reinterpret_cast<uint64_t*>(smem + kI8StageBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  for (int i = threadIdx.x; i < kI8StageBytes / 4; i += blockDim.x)
    reinterpret_cast<uint32_t*>(smem)[i] = 0x01010101u * (uint32_t)(i & 3);
  if (threadIdx.x == 0) {
    mbar_init(done, 1);
    fence_mbar_init();
  }
  fence_proxy_async_smem();
  if ((threadIdx.x >> 5) == 0) {
    tmem_alloc(tmem_slot, kI8TmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;
  if (threadIdx.x == 0) {
    const uint32_t idesc = umma_idesc_i8(kI8BM, kI8BN, 1);
    const uint32_t sa = smem_u32(smem);
    const uint64_t adesc = umma_desc_kmajor_sw128(sa);
    const uint64_t bdesc = umma_desc_kmajor_sw128(sa + kI8TileABytes);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        umma_i8(tmem_base + (uint32_t)((it & 1) * kI8BN), adesc + kk * 2, bdesc + kk * 2, idesc,
                it > 1 ? 1u : 0u);
    }
    umma_commit(done);
  }
  __syncwarp();
  if (threadIdx.x < 32) {  // warp 0, converged: tcgen05.ld is warp-collective
    const bool ok = mbar_wait(done, 0, sink + 1);
    tc_fence_after();
    uint32_t v[32];
    tmem_ld_32x32b_x32(tmem_base, v);
    tmem_ld_wait();
    if (ok && v[0] == 0xFFFFFFFFu) sink[0] = v[1];  // keeps the MMAs live
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if ((threadIdx.x >> 5) == 0) tmem_dealloc(tmem_base, kI8TmemCols);
}

}  // namespace skg
