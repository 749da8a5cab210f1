// Internal host-side runtime shared by the C ABI and the kernels' launchers:
// per-device state, per-stream Stream-K workspaces, device buffers and the
// status plumbing. Not part of the public ABI (include/skgemm.h is).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "skgemm.h"

namespace skg {

// NVTX range over one C-ABI call (named after the entry point), so that a
// profiler's timeline shows the library's calls around their kernels; a push
// and a pop through the NVTX injection hooks, nearly free without a tool.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Records a message for skgemm_last_error() and returns `code`.
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define SKG_CUDA(call)                                        \
  do {                                                        \
    cudaError_t skg_e_ = (call);                              \
    if (skg_e_ != cudaSuccess) return ::skg::cuda_fail(skg_e_, #call); \
  } while (0)

// Grow-only device buffer.
// Debug mode (environment SKGEMM_DEBUG_FILL=1, read once): every scratch
// buffer is filled with 0xFF bytes when it is allocated and again, on the
// call's stream, at the start of each call that uses it (an FP64 NaN, an
// int8 residue of -1), so that a kernel reading scratch it did not write
// first shows in its results. Results are unchanged when the kernels are
// right (tests/test_debug_fill_gpu.py); the fills cost time.
bool debug_fill_enabled();
int debug_poison(void* p, size_t bytes, cudaStream_t s);

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  int ensure(size_t need);
  void release();
};

// State of one stream's Stream-K launches: partial-tile slots, flags, the
// epoch the flags of the next launch will carry, and the device error word.
struct StreamWorkspace {
  double* partials = nullptr;
  size_t partial_slots = 0;
  uint32_t* flags = nullptr;
  uint32_t* err = nullptr;  // device error word
  uint32_t epoch = 0;
  int ensure(int slots);
};

struct DeviceState {
  int device = -1;
  int num_sms = 0;
  int cc_major = 0, cc_minor = 0;
  char name[96] = {0};  // the device's product name (keys of persisted tuning)
  std::mutex mu;
  std::map<cudaStream_t, StreamWorkspace*> ws;
  // Staging buffers of the blocking host-pointer entry points (guarded by
  // host_mu: host-pointer calls on one device are serialised).
  std::mutex host_mu;
  DeviceBuffer stage[4];
  cudaStream_t host_stream = nullptr;
  // Copy streams of the pipelined host-pointer rotation (H2D and D2H run
  // concurrently with each other and with the compute on host_stream).
  cudaStream_t host_h2d = nullptr, host_d2h = nullptr;
};

// Current device's state (initialises on first use). Returns nullptr and
// records an error when no sm_100 device is usable.
DeviceState* current_device(int* status);
StreamWorkspace* stream_workspace(DeviceState* dev, cudaStream_t s, int slots, int* status);

// Encodes a tiled TMA descriptor through the driver entry point.
int encode_tiled(CUtensorMap* map, int rank, const void* base, const uint64_t* dims,
                 const uint64_t* strides_bytes /*rank-1*/, const uint32_t* box,
                 CUtensorMapDataType dtype, CUtensorMapSwizzle swizzle);

// ----------------------------------------------------------------- FP64
struct Fp64Operand {
  const double* ptr;
  int kind;    // skg::OperandKind
  int64_t rows;  // extent of the M (or N) dimension
  int64_t ld;    // k stride for kOpDense
};

struct Fp64Problem {
  Fp64Operand a, b;
  int64_t M, N, K;
  int tile_order;  // skg::TileOrder
  int out_kind;    // skg::OutKind
  double* D;
  int64_t ldd;
  double alpha;
  double gamma;  // GEMM gamma / SYRK beta
  bool beta_zero;
};

// Enqueues the native FP64 Stream-K kernel on `s`. `ws_override` (optional)
// supplies caller-owned partial slots/flags/err instead of the stream cache.
// `tile` 128 or 64 fixes the output tile; 0 lets the cost model choose.
int launch_fp64(DeviceState* dev, const Fp64Problem& prob, cudaStream_t s,
                StreamWorkspace* ws_override = nullptr, int tile = 0);
// Number of Stream-K partial slots the 128 x 128-tile launch of `prob` uses
// (= its grid).
int fp64_grid_for(DeviceState* dev, const Fp64Problem& prob);
// Loads the 128 x 128 single-problem kernel's code on the current device and
// sets its shared-memory attribute, without launching it (with lazy module
// loading the code would otherwise be loaded, and its memory taken, at the
// first launch).
int fp64_preload(DeviceState* dev);
// Grouped launch (batched path): CTAs per SM the grouped kernel of `tile`
// (128 or 64) fits, and the launch itself (flag reset + kernel, no cooperative
// attribute so that the pair can be captured into a CUDA graph; the grid must
// not exceed SMs x blocks_per_sm so that every CTA can be resident).
struct Fp64Group;
int fp64_group_occupancy(DeviceState* dev, int tile, int* blocks_per_sm);
int launch_fp64_group(int tile, const Fp64Group& g, cudaStream_t s);
// TMA descriptor of one operand for tiles of `rows_per_tile` rows.
int make_operand_map(CUtensorMap* map, const Fp64Operand& op, int64_t K, int rows_per_tile);

// Problem descriptors of the three entry points (contracts of
// skgemm_dgemm_packed_dev, skgemm_dsyrk_packed_dev, skgemm_drot_dev).
Fp64Problem gemm_packed_problem(int64_t M, int64_t N, int64_t K, const double* Ap,
                                const double* Bp, double* D, int64_t ldd, double alpha,
                                double gamma);
Fp64Problem syrk_problem(int64_t K, int64_t M, const double* Ap, double* C, int64_t ldc,
                         double alpha, double beta);
// a_band: A band-packed (read K-major), else grid-packed.
Fp64Problem rot_problem(int64_t Nd, int64_t nb, const double* A, const double* Q, double* D,
                        bool a_band = false);
// Result of an empty reduction (K == 0): D = gamma (GEMM), C = beta*C (SYRK).
int run_k0(int mode, int64_t M, int64_t N, double* D, int64_t ld, double gamma, bool beta_zero,
           cudaStream_t s);

// Layout kernels.
int launch_sum_parts(const double* parts, int nparts, int64_t n, double gamma, double* out,
                     cudaStream_t s);
int launch_pack(int64_t R, int64_t K, const double* X, int64_t sr, int64_t sk, int T,
                double* Xp, cudaStream_t s);
int launch_unpack(int64_t R, int64_t K, const double* Xp, int T, double* X, int64_t sr,
                  int64_t sk, cudaStream_t s);
// H Psi stencil on extended band-packed Psi (skg_stencil.cu) and the
// single-rank periodic halo that builds that extended array.
int launch_stencil_ext(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                       const double* ext, const double* A, const double* cx, const double* cy,
                       const double* cz, double c0, double* out, int out_tile, int num_sms,
                       uint32_t* err, cudaStream_t s);
int launch_halo_periodic(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                         const double* local, double* ext, cudaStream_t s);
// Nonlocal projector set on the device (skg_nloc.cu).
int nloc_create(int64_t P, const uint32_t* nrow, const uint32_t* ncol, const int32_t* atom,
                const uint32_t* offsets, const uint32_t* index, const double* chi,
                const double* gamma, int64_t K, skgemm_nloc** out);
int nloc_apply(skgemm_nloc* h, int64_t nb, double dv, const double* psi16, double* out,
               int out_tile, cudaStream_t s);
void nloc_destroy(skgemm_nloc* h);
int launch_band_to_grid(int64_t Nd, int64_t nb, const double* src, double* dst,
                        cudaStream_t s);
int launch_grid_to_band(int64_t Nd, int64_t nb, const double* src, double* dst,
                        cudaStream_t s);

// Peak probe.
int probe_fp64_peak(DeviceState* dev, double* tflops);
// Diagnostic: one bounded device wait that runs out after budget_ms
// (recorded in stream s's device error word).
int expire_wait(DeviceState* dev, double budget_ms, cudaStream_t s);
int expire_fixup_wait(DeviceState* dev, double budget_ms, cudaStream_t s);

// Device-side failures of one-shot batched launches on `s` (read and cleared;
// `s` already synchronised).
int batch_consume_error(DeviceState* dev, cudaStream_t s);

// Reads and clears the error word of `ws` (synchronises `s`).
int consume_device_error(StreamWorkspace* ws, cudaStream_t s);

// Per-kernel timing (off by default; skgemm_kernel_timing). While it is on,
// a KernelTimer around a launch records a CUDA event before and after it on
// the launch's stream, under the kernel's name; skgemm_kernel_timing_report
// sums the elapsed times per name. While it is off a KernelTimer only reads
// one flag.
extern bool g_ktimer_on;
void ktimer_record(cudaStream_t s, const char* name, bool start);
struct KernelTimer {
  cudaStream_t s;
  const char* name;
  KernelTimer(cudaStream_t s_, const char* n) : s(s_), name(n) {
    if (g_ktimer_on) ktimer_record(s, name, true);
  }
  ~KernelTimer() {
    if (g_ktimer_on) ktimer_record(s, name, false);
  }
};

}  // namespace skg
