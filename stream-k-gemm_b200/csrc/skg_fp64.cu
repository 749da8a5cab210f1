// Host launcher of the native FP64 Stream-K kernel: operand descriptors ->
// TMA tensor maps, Stream-K schedule, cooperative persistent launch.
#include <algorithm>

#include "skg_fp64_kernel.cuh"
#include "skg_runtime.h"

namespace skg {

int make_operand_map(CUtensorMap* map, const Fp64Operand& op, int64_t K, int rows_per_tile) {
  if (op.ptr == nullptr) return fail(SKGEMM_ERR_INVALID_ARG, "null operand pointer");
  if ((reinterpret_cast<uintptr_t>(op.ptr) & 15) != 0)
    return fail(SKGEMM_ERR_INVALID_ARG, "operand base must be 16-byte aligned");
  const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  const CUtensorMapSwizzle sw = CU_TENSOR_MAP_SWIZZLE_128B;
  if (op.kind == kOpPacked16) {
    uint64_t dims[3] = {16, (uint64_t)K, (uint64_t)((op.rows + 15) / 16)};
    uint64_t strides[2] = {16 * 8, (uint64_t)K * 16 * 8};
    uint32_t box[3] = {16, (uint32_t)kBK, (uint32_t)(rows_per_tile / 16)};
    return encode_tiled(map, 3, op.ptr, dims, strides, box, dt, sw);
  }
  if (op.kind == kOpPacked32) {
    uint64_t dims[3] = {32, (uint64_t)K, (uint64_t)((op.rows + 31) / 32)};
    uint64_t strides[2] = {32 * 8, (uint64_t)K * 32 * 8};
    uint32_t box[3] = {16, (uint32_t)kBK, (uint32_t)(rows_per_tile / 32)};
    return encode_tiled(map, 3, op.ptr, dims, strides, box, dt, sw);
  }
  if (op.kind == kOpBandK) {
    if (K % 16) return fail(SKGEMM_ERR_INVALID_ARG, "K-major operand needs K a multiple of 16");
    uint64_t dims[3] = {16, (uint64_t)op.rows, (uint64_t)(K / 16)};
    uint64_t strides[2] = {16 * 8, (uint64_t)op.rows * 16 * 8};
    uint32_t box[3] = {16, (uint32_t)rows_per_tile, 1};
    return encode_tiled(map, 3, op.ptr, dims, strides, box, dt, sw);
  }
  if (op.kind == kOpDense) {
    if (op.ld < op.rows || ((op.ld * 8) % 16) != 0)
      return fail(SKGEMM_ERR_INVALID_ARG, "dense operand leading dimension must be even and >= rows");
    uint64_t dims[2] = {(uint64_t)op.rows, (uint64_t)K};
    uint64_t strides[1] = {(uint64_t)op.ld * 8};
    uint32_t box[2] = {16, (uint32_t)kBK};
    return encode_tiled(map, 2, op.ptr, dims, strides, box, dt, sw);
  }
  return fail(SKGEMM_ERR_INVALID_ARG, "unknown operand kind");
}

namespace {

struct Schedule {
  int tiles_m, tiles_n, num_tiles, ipt;
  int64_t total;
  int grid;
};

Schedule make_schedule(DeviceState* dev, const Fp64Problem& prob, int tile, int per_sm) {
  Schedule sc;
  sc.tiles_m = (int)((prob.M + tile - 1) / tile);
  sc.tiles_n = (int)((prob.N + tile - 1) / tile);
  sc.num_tiles = prob.tile_order == kTilesUpper ? sc.tiles_n * (sc.tiles_n + 1) / 2
                                                : sc.tiles_m * sc.tiles_n;
  sc.ipt = (int)((prob.K + kBK - 1) / kBK);
  sc.total = (int64_t)sc.num_tiles * sc.ipt;
  sc.grid = (int)std::min<int64_t>((int64_t)dev->num_sms * per_sm, sc.total);
  return sc;
}

// Issued MACs (padding included) of `prob` on tile x tile outputs.
double issued_macs(const Fp64Problem& prob, int tile) {
  const double tm = (double)((prob.M + tile - 1) / tile), tn = (double)((prob.N + tile - 1) / tile);
  const double tiles = prob.tile_order == kTilesUpper ? tn * (tn + 1) / 2 : tm * tn;
  return tiles * tile * tile * (double)((prob.K + kBK - 1) / kBK * kBK);
}

// Tile of a single-problem launch: 64 x 64 when it issues fewer MACs than
// 128 x 128 (triangles, ragged edges) or when the output has so many
// 128 x 128 tiles (>= 4 per SM) that two CTAs per SM pay off; 128 x 128
// otherwise. Measured on B200 with 110592 x 512 operands: SYRK 0.95 ms on
// 64 x 64 vs 1.08 ms on 128 x 128, rotation 1.72 vs 1.77 ms, GEMM
// (M = N = 512, 16 tiles) 1.68 vs 1.67 ms.
int single_tile(DeviceState* dev, const Fp64Problem& prob) {
  const double i64 = issued_macs(prob, 64), i128 = issued_macs(prob, 128);
  if (i64 < i128) return 64;
  const double t128 = i128 / (128.0 * 128.0 * (double)((prob.K + kBK - 1) / kBK * kBK));
  return (i64 == i128 && t128 >= 4.0 * dev->num_sms) ? 64 : 128;
}

// CTAs per SM of the single-problem kernel of `tile` and A layout (its
// shared-memory attribute set once per device).
template <class TS>
int single_setup(int device, const void* kernel, bool akm, int* per_sm) {
  static int occ[2][2][64] = {};
  int& o = occ[TS::BM == 64 ? 1 : 0][akm ? 1 : 0][device];
  if (!o) {
    SKG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  TS::kSmem));
    int n = 0;
    SKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, kThreads, TS::kSmem));
    if (n < 1) return fail(SKGEMM_ERR_CUDA, "FP64 kernel does not fit on an SM");
    o = std::min(n, TS::kMinBlocks);
  }
  *per_sm = o;
  return SKGEMM_OK;
}

}  // namespace

int fp64_preload(DeviceState* dev) {
  int per_sm = 0;
  return single_setup<Tile128>(dev->device, (const void*)fp64_streamk_kernel, false, &per_sm);
}

int fp64_grid_for(DeviceState* dev, const Fp64Problem& prob) {
  if (prob.M <= 0 || prob.N <= 0 || prob.K <= 0) return 0;
  return make_schedule(dev, prob, 128, 1).grid;
}

int launch_fp64(DeviceState* dev, const Fp64Problem& prob, cudaStream_t s,
                StreamWorkspace* ws_override, int tile) {
  if (prob.M < 0 || prob.N < 0 || prob.K < 0)
    return fail(SKGEMM_ERR_INVALID_ARG, "negative dimension");
  if (prob.tile_order == kTilesUpper && prob.M != prob.N)
    return fail(SKGEMM_ERR_INVALID_ARG, "SYRK tiles need a square output");
  if (prob.K > (int64_t)INT32_MAX - kBK || prob.M > ((int64_t)1 << 31) ||
      prob.N > ((int64_t)1 << 31))
    return fail(SKGEMM_ERR_INVALID_ARG, "dimension too large");
  if (prob.M == 0 || prob.N == 0) return SKGEMM_OK;
  if (prob.D == nullptr) return fail(SKGEMM_ERR_INVALID_ARG, "null output pointer");
  if (prob.K == 0) {
    // Empty reduction: D = gamma (GEMM), C = beta*C (SYRK), D = 0 (rotation).
    return fail(SKGEMM_ERR_UNSUPPORTED, "K == 0 is handled by the caller");
  }
  if (tile == 0) tile = single_tile(dev, prob);
  if (tile != 128 && tile != 64) return fail(SKGEMM_ERR_INVALID_ARG, "tile must be 128 or 64");
  const bool akm = prob.a.kind == kOpBandK;
  if (prob.b.kind == kOpBandK || (akm && prob.b.kind == kOpPacked32))
    return fail(SKGEMM_ERR_INVALID_ARG, "operand layouts not supported together");
  const void* kernel = tile == 64 ? (akm ? (const void*)fp64_streamk_kernel64_ak
                                         : (const void*)fp64_streamk_kernel64)
                                  : (akm ? (const void*)fp64_streamk_kernel_ak
                                         : (const void*)fp64_streamk_kernel);
  int per_sm = 1, st = SKGEMM_OK;
  if ((st = tile == 64 ? single_setup<Tile64>(dev->device, kernel, akm, &per_sm)
                       : single_setup<Tile128>(dev->device, kernel, akm, &per_sm)))
    return st;
  Schedule sc = make_schedule(dev, prob, tile, per_sm);
  if ((int64_t)sc.num_tiles * sc.ipt > ((int64_t)1 << 40))
    return fail(SKGEMM_ERR_INVALID_ARG, "problem too large");

  StreamWorkspace* ws = ws_override ? ws_override : stream_workspace(dev, s, sc.grid, &st);
  if (!ws) return st;
  if ((int)ws->partial_slots < sc.grid)
    return fail(SKGEMM_ERR_INVALID_ARG, "workspace has fewer partial slots than the grid");

  CUtensorMap mapA, mapB;
  if ((st = make_operand_map(&mapA, prob.a, prob.K, tile)) != SKGEMM_OK) return st;
  if ((st = make_operand_map(&mapB, prob.b, prob.K, tile)) != SKGEMM_OK) return st;

  Fp64Params p;
  p.M = prob.M;
  p.N = prob.N;
  p.K = prob.K;
  p.tiles_m = sc.tiles_m;
  p.tiles_n = sc.tiles_n;
  p.num_tiles = sc.num_tiles;
  p.iters_per_tile = sc.ipt;
  p.total_iters = sc.total;
  p.grid = sc.grid;
  p.a_kind = prob.a.kind;
  p.b_kind = prob.b.kind;
  p.tile_order = prob.tile_order;
  p.out_kind = prob.out_kind;
  p.D = prob.D;
  p.ldd = prob.ldd;
  p.alpha = prob.alpha;
  p.gamma = prob.gamma;
  p.beta_zero = prob.beta_zero ? 1 : 0;
  p.workspace = ws->partials;
  p.flags = ws->flags;
  p.epoch = ++ws->epoch;
  if (p.epoch == 0) p.epoch = ++ws->epoch;  // 0 is the value of a fresh flag
  p.err = ws->err;

  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sc.grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = tile == 64 ? Tile64::kSmem : Tile128::kSmem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  KernelTimer kt_(s, tile == 64 ? (akm ? "fp64_streamk_kernel64_ak" : "fp64_streamk_kernel64")
                                 : (akm ? "fp64_streamk_kernel_ak" : "fp64_streamk_kernel"));
  if (tile == 64)
    SKG_CUDA(cudaLaunchKernelEx(&cfg, akm ? fp64_streamk_kernel64_ak : fp64_streamk_kernel64,
                                mapA, mapB, p));
  else
    SKG_CUDA(cudaLaunchKernelEx(&cfg, akm ? fp64_streamk_kernel_ak : fp64_streamk_kernel, mapA,
                                mapB, p));
  return SKGEMM_OK;
}

}  // namespace skg

// ------------------------------------------------------------ grouped launch
namespace skg {

namespace {

template <class TS>
int grouped_setup(int device, int* blocks_per_sm) {
  static int occ[64] = {0};
  if (device < 0 || device >= 64) return fail(SKGEMM_ERR_INVALID_ARG, "device index");
  if (!occ[device]) {
    SKG_CUDA(cudaFuncSetAttribute(fp64_grouped_kernel<TS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, TS::kSmem));
    int n = 0;
    SKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fp64_grouped_kernel<TS>,
                                                           kThreads, TS::kSmem));
    if (n < 1) return fail(SKGEMM_ERR_UNSUPPORTED, "grouped kernel does not fit on an SM");
    occ[device] = n;
  }
  *blocks_per_sm = occ[device];
  return SKGEMM_OK;
}

template <class TS>
int grouped_launch(const Fp64Group& g, cudaStream_t s) {
  // Flags start at zero for every launch (a stream-ordered memset, captured
  // together with the kernel when the pair is recorded into a graph).
  SKG_CUDA(cudaMemsetAsync(g.flags, 0, (size_t)g.grid * sizeof(uint32_t), s));
  fp64_grouped_kernel<TS><<<g.grid, kThreads, TS::kSmem, s>>>(g);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

}  // namespace

int fp64_group_occupancy(DeviceState* dev, int tile, int* blocks_per_sm) {
  if (tile == 128) return grouped_setup<Tile128>(dev->device, blocks_per_sm);
  if (tile == 64) return grouped_setup<Tile64>(dev->device, blocks_per_sm);
  return fail(SKGEMM_ERR_INVALID_ARG, "tile must be 128 or 64");
}

int launch_fp64_group(int tile, const Fp64Group& g, cudaStream_t s) {
  if (g.grid <= 0 || g.total_iters <= 0) return SKGEMM_OK;
  if (tile == 128) return grouped_launch<Tile128>(g, s);
  if (tile == 64) return grouped_launch<Tile64>(g, s);
  return fail(SKGEMM_ERR_INVALID_ARG, "tile must be 128 or 64");
}

}  // namespace skg
