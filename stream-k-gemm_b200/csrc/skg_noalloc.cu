// Allocation-free form of the packed Stream-K GEMM (skgemm_dgemm_packed_dev).
//
// Who needs it: callers that cannot allocate device memory when they call
// the GEMM — an application that reserves the device's memory up front in its
// own pool (a DFT code sizing its wave-function blocks to fill HBM), code
// whose device footprint must not grow after start-up (admission under a
// fixed HBM budget), or loops that cannot accept the implicit device-wide
// synchronisation of cudaFree / the stalls of cudaMalloc. The regular entry
// point allocates a Stream-K workspace (19 MB) the first time it sees a
// stream; this one never calls cudaMalloc, cudaFree or any allocating routine.
//
// Its scratch (one partial-tile slot per persistent CTA, the CTAs' fixup
// flags and a device error word) is the file-scope array below: 148 slots of
// 128 x 128 doubles plus flags, 19.4 MB in all. With CUDA's lazy module
// loading (the default) the array, like the kernel code it feeds, takes its
// device memory when this file's module is first used on a device, not when
// the library is loaded: the first call on a device — an empty call with
// M = 0 or N = 0 will do — loads both, and should come before the caller
// reserves the rest of the device's memory. From then on the array stays
// allocated on that device until the process exits.
//
// The array's name in host code is only a host-side stand-in, not a device
// address, so the first call on a device (with that device current) looks up
// the real address once with cudaGetSymbolAddress and passes it to the
// kernel.
//
// Every call uses the same array and finds the previous call's contents in
// it. The flags carry a per-call epoch, so stale flags never match; the error
// word is cleared at the start of each call; partial slots are written before
// they are read. Two calls running on the same GPU at the same time would
// race on the slots and flags, so calls on one device are serialised by that
// device's lock and a call returns only after its kernel has finished (it
// synchronises `stream`; it therefore cannot be issued under stream capture).
#include <cstdio>
#include <mutex>

#include "skg_fp64_types.h"
#include "skg_runtime.h"

namespace skg {

namespace {

constexpr int kNoAllocSlots = 148;  // partial-tile slots = largest grid served
constexpr size_t kNoAllocPartialBytes = (size_t)kNoAllocSlots * kBM * kBN * sizeof(double);
constexpr size_t kNoAllocFlagBytes = 1024;  // kNoAllocSlots 32-bit flags, padded
constexpr size_t kNoAllocBytes = kNoAllocPartialBytes + kNoAllocFlagBytes + 256;  // + error word
static_assert(kNoAllocSlots * sizeof(uint32_t) <= kNoAllocFlagBytes, "flag area too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocDevices = 64;

struct NoAllocDevice {
  std::mutex mu;  // serialises the calls on this device (they share its array)
  bool ready = false;
  StreamWorkspace ws;  // views into g_noalloc_scratch; never allocates
};

NoAllocDevice g_noalloc_dev[kNoAllocDevices];

// Once per device, with that device current (caller holds d.mu): the
// array's device address, and the GEMM kernel's code loaded.
int noalloc_setup(DeviceState* dev, NoAllocDevice& d) {
  if (d.ready) return SKGEMM_OK;
  if (int st = fp64_preload(dev)) return st;
  void* base = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&base, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
  unsigned char* b = static_cast<unsigned char*>(base);
  d.ws.partials = reinterpret_cast<double*>(b);
  d.ws.partial_slots = kNoAllocSlots;
  d.ws.flags = reinterpret_cast<uint32_t*>(b + kNoAllocPartialBytes);
  d.ws.err = reinterpret_cast<uint32_t*>(b + kNoAllocPartialBytes + kNoAllocFlagBytes);
  d.ws.epoch = 0;  // the array starts zeroed: first epoch used is 1
  d.ready = true;
  return SKGEMM_OK;
}

}  // namespace
}  // namespace skg

using namespace skg;

extern "C" __attribute__((visibility("default"))) int skgemm_dgemm_packed_dev_noalloc(
    int64_t M, int64_t N, int64_t K, const double* A_packed16, const double* B_packed32,
    double* D, int64_t ldd, double alpha, double gamma, void* stream) {
  if (M < 0 || N < 0 || K < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative dimension");
  if (ldd < N) return fail(SKGEMM_ERR_INVALID_ARG, "ldd < N");
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (dev->device < 0 || dev->device >= kNoAllocDevices)
    return fail(SKGEMM_ERR_UNSUPPORTED, "no-alloc GEMM: device ordinal beyond 63");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

  NoAllocDevice& nd = g_noalloc_dev[dev->device];
  std::lock_guard<std::mutex> lk(nd.mu);
  // Set-up before the empty-shape return, so that an empty call loads the
  // array and the kernel on this device ahead of the caller's own pool.
  if ((st = noalloc_setup(dev, nd)) != SKGEMM_OK) return st;
  if (M == 0 || N == 0) return SKGEMM_OK;
  if (!D) return fail(SKGEMM_ERR_INVALID_ARG, "null output pointer");

  if (K == 0) {  // empty reduction: D = alpha * 0 + gamma
    if ((st = run_k0(kOutRowMajor, M, N, D, ldd, gamma, false, s)) != SKGEMM_OK) return st;
    SKG_CUDA(cudaStreamSynchronize(s));
    return SKGEMM_OK;
  }

  Fp64Problem p;
  p.a = {A_packed16, kOpPacked16, M, 0};
  p.b = {B_packed32, kOpPacked32, N, 0};
  p.M = M;
  p.N = N;
  p.K = K;
  p.tile_order = kTilesAll;
  p.out_kind = kOutRowMajor;
  p.D = D;
  p.ldd = ldd;
  p.alpha = alpha;
  p.gamma = gamma;
  p.beta_zero = false;
  const int grid = fp64_grid_for(dev, p);
  if (grid > kNoAllocSlots) {
    char buf[200];
    snprintf(buf, sizeof(buf),
             "no-alloc GEMM: this launch needs %d partial-tile slots but the static scratch "
             "holds %d (19.4 MB); use skgemm_dgemm_packed_dev",
             grid, kNoAllocSlots);
    return fail(SKGEMM_ERR_INVALID_ARG, buf);
  }
  SKG_CUDA(cudaMemsetAsync(nd.ws.err, 0, sizeof(uint32_t), s));
  // 128 x 128 tiles: the static scratch holds that launch's slots.
  if ((st = launch_fp64(dev, p, s, &nd.ws, 128)) != SKGEMM_OK) return st;
  SKG_CUDA(cudaStreamSynchronize(s));
  uint32_t word = 0;
  SKG_CUDA(cudaMemcpy(&word, nd.ws.err, sizeof(word), cudaMemcpyDeviceToHost));
  if (word != 0) {
    char buf[120];
    snprintf(buf, sizeof(buf), "device-side wait ran past its budget (error word 0x%x)", word);
    return fail(SKGEMM_ERR_DEVICE_TIMEOUT, buf);
  }
  return SKGEMM_OK;
}
