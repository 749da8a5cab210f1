// Constants, enums and launch parameters of the native FP64 Stream-K kernel,
// shared by the kernel and its host-side users.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace skg {

constexpr int kBM = 128;
constexpr int kBN = 128;
constexpr int kBK = 16;
constexpr int kStages = 6;
constexpr int kConsumerWarps = 8;
constexpr int kConsumerThreads = kConsumerWarps * 32;
constexpr int kThreads = kConsumerThreads + 32;  // + one producer warp
constexpr int kChunkBytes = kBK * 16 * 8;           // [BK][16] doubles = 2 KB
constexpr int kTileABytes = (kBM / 16) * kChunkBytes;  // 16 KB
constexpr int kTileBBytes = (kBN / 16) * kChunkBytes;  // 16 KB
constexpr int kStageBytes = kTileABytes + kTileBBytes;
constexpr int kAccPerThread = 64;  // warp tile 64x32 -> 64 doubles per lane
constexpr int kSmemBytes = kStages * kStageBytes + 1024 /*align*/ + 256 /*barriers*/;

// Output-tile shape of one kernel instantiation. Eight consumer warps in a
// 2 x 4 grid: a warp owns (BM/2) x (BN/4) outputs = MI m16 blocks x NJ n8
// blocks, fed by MI A chunks and NQ = NJ/2 B chunks of 16 columns.
template <int BM_, int BN_>
struct TileShape {
  static constexpr int BM = BM_;
  static constexpr int BN = BN_;
  static constexpr int MI = BM / 32;
  static constexpr int NJ = BN / 32;
  static constexpr int NQ = NJ / 2;
  static constexpr int kABytes = (BM / 16) * kChunkBytes;
  static constexpr int kBBytes = (BN / 16) * kChunkBytes;
  static constexpr int kStage = kABytes + kBBytes;
  static constexpr int kSmem = kStages * kStage + 1024 /*align*/ + 256 /*barriers*/;
  static constexpr int kAcc = MI * NJ * 4;  // doubles per consumer thread
  // CTAs per SM the launch bounds ask for: one 197 KB ring for 128 x 128,
  // two 97 KB rings for 64 x 64.
  static constexpr int kMinBlocks = BM * BN >= 128 * 128 ? 1 : 2;
};
using Tile128 = TileShape<128, 128>;
using Tile64 = TileShape<64, 64>;
static_assert(Tile128::kStage == kStageBytes && Tile128::kSmem == kSmemBytes, "tile constants");

enum OperandKind : int {
  kOpPacked16 = 0,  // [ceil(R/16)][K][16]; 3-D map {16, K, tiles}, one box per stage
  kOpPacked32 = 1,  // [ceil(R/32)][K][32]; 3-D map {32, K, tiles}, two half-width boxes
                    // per stage -> shared memory [half][tile][BK][16]
  kOpDense = 2,     // R contiguous, k stride ld; 2-D map {R, K}, one box per 16-chunk
  kOpBandK = 3,     // K-major [K/16][R][16] (band-packed Psi as the rotation's A:
                    // element (r, k) at (k/16)*R*16 + r*16 + k%16); 3-D map
                    // {16, R, K/16}, one box {16, BM, 1} per stage (BK = 16) ->
                    // shared memory [BM][16 k]; A operand of the single-problem
                    // kernels only, K % 16 == 0
};

enum OutKind : int { kOutRowMajor = 0, kOutSyrkUpper = 1, kOutBand16 = 2 };

enum TileOrder : int { kTilesAll = 0, kTilesUpper = 1 };

struct Fp64Params {
  int64_t M, N, K;
  int tiles_m, tiles_n;
  int num_tiles;
  int iters_per_tile;  // ceil(K / BK)
  int64_t total_iters;
  int grid;
  int a_kind, b_kind;
  int tile_order;
  int out_kind;
  double* D;
  int64_t ldd;  // row stride (row-major) / column stride (SYRK); unused for band16
  double alpha;
  double gamma;  // GEMM: added scalar; SYRK: beta
  int beta_zero;
  double* workspace;  // grid * BM*BN doubles (partial tiles)
  uint32_t* flags;    // grid flags
  uint32_t epoch;     // value a published flag carries for this launch
  uint32_t* err;      // device error word
};

// Grouped launch: many independent problems in one persistent Stream-K
// launch. Their MAC-loop iterations are concatenated (problem p owns
// [iter_begin[p], iter_begin[p+1])) and split evenly over the CTAs; a CTA's
// range may cross tile and problem boundaries. Per-problem fields of
// Fp64Params used: M, N, K, tiles_m, tiles_n, num_tiles, iters_per_tile,
// a_kind, b_kind, tile_order, out_kind, D, ldd, alpha, gamma, beta_zero.
// Flags are cleared by the launcher before every launch (a memset in the same
// stream or graph) and published as 1, so the pair can be replayed from a
// CUDA graph.
struct Fp64Group {
  const Fp64Params* probs;
  const CUtensorMap* maps;     // 2 per problem (A, B), 64-byte aligned
  const int64_t* iter_begin;   // num_problems + 1 entries
  int num_problems;
  int64_t total_iters;
  int grid;
  double* workspace;  // grid * BM*BN doubles
  uint32_t* flags;    // grid flags, zero at launch
  uint32_t* err;
};

}  // namespace skg
