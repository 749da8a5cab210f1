// Constants, enums and launch parameters of the native FP64 Stream-K kernel,
// shared by the kernel and its host-side users.
#pragma once

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

enum OperandKind : int {
  kOpPacked16 = 0,  // [ceil(R/16)][K][16]; 3-D map {16, K, tiles}, one box per stage
  kOpPacked32 = 1,  // [ceil(R/32)][K][32]; 3-D map {32, K, tiles}, two half-width boxes
                    // per stage -> shared memory [half][tile][BK][16]
  kOpDense = 2,     // R contiguous, k stride ld; 2-D map {R, K}, one box per 16-chunk
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

}  // namespace skg
