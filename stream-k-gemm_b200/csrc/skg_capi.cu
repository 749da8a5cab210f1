// C ABI of libskgemm (declared in include/skgemm.h) and the host runtime it
// rests on: per-device state, per-stream Stream-K workspaces, staging of the
// blocking host-pointer entry points, TMA descriptor encoding, status strings.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "skg_batch.h"
#include "skg_common.cuh"
#include "skg_fp64_types.h"
#include "skg_ozaki.h"
#include "skg_runtime.h"

namespace skg {

// ------------------------------------------------------------------ status
static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return fail(SKGEMM_ERR_OOM, m);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
    return fail(SKGEMM_ERR_NO_DEVICE, m);
  return fail(SKGEMM_ERR_CUDA, m);
}

// ----------------------------------------------------------------- buffers
bool debug_fill_enabled() {
  static const bool on = [] {
    const char* e = getenv("SKGEMM_DEBUG_FILL");
    return e && e[0] == '1';
  }();
  return on;
}

int debug_poison(void* p, size_t bytes, cudaStream_t s) {
  if (!debug_fill_enabled() || !p || !bytes) return SKGEMM_OK;
  SKG_CUDA(cudaMemsetAsync(p, 0xFF, bytes, s));
  return SKGEMM_OK;
}

int DeviceBuffer::ensure(size_t need) {
  if (need <= bytes) return SKGEMM_OK;
  release();
  SKG_CUDA(cudaMalloc(&ptr, need));
  bytes = need;
  if (debug_fill_enabled()) SKG_CUDA(cudaMemset(ptr, 0xFF, need));
  return SKGEMM_OK;
}

void DeviceBuffer::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

int StreamWorkspace::ensure(int slots) {
  if ((size_t)slots <= partial_slots && err) return SKGEMM_OK;
  if (partials) cudaFree(partials);
  if (flags) cudaFree(flags);
  partials = nullptr;
  flags = nullptr;
  partial_slots = 0;
  SKG_CUDA(cudaMalloc(&partials, (size_t)slots * kBM * kBN * sizeof(double)));
  if (debug_fill_enabled())
    SKG_CUDA(cudaMemset(partials, 0xFF, (size_t)slots * kBM * kBN * sizeof(double)));
  SKG_CUDA(cudaMalloc(&flags, (size_t)slots * sizeof(uint32_t)));
  SKG_CUDA(cudaMemset(flags, 0, (size_t)slots * sizeof(uint32_t)));
  if (!err) {
    SKG_CUDA(cudaMalloc(&err, sizeof(uint32_t)));
    SKG_CUDA(cudaMemset(err, 0, sizeof(uint32_t)));
  }
  partial_slots = slots;
  epoch = 0;
  return SKGEMM_OK;
}

// ------------------------------------------------------------------ device
static DeviceState g_dev[64];
static std::mutex g_dev_mu;

DeviceState* current_device(int* status) {
  int d = -1;
  cudaError_t e = cudaGetDevice(&d);
  if (e != cudaSuccess || d < 0 || d >= 64) {
    *status = cuda_fail(e == cudaSuccess ? cudaErrorNoDevice : e, "cudaGetDevice");
    return nullptr;
  }
  DeviceState* dev = &g_dev[d];
  std::lock_guard<std::mutex> lk(g_dev_mu);
  if (dev->device < 0) {
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, d);
    if (e != cudaSuccess) {
      *status = cuda_fail(e, "cudaGetDeviceProperties");
      return nullptr;
    }
    if (prop.major != 10) {
      *status = fail(SKGEMM_ERR_NO_DEVICE, "skgemm requires an sm_100 (B200-class) device");
      return nullptr;
    }
    dev->num_sms = prop.multiProcessorCount;
    snprintf(dev->name, sizeof(dev->name), "%s", prop.name);
    for (char* c = dev->name; *c; ++c)
      if (*c == '"' || *c == '\\' || *c == '|') *c = '_';  // safe inside a JSON string and a key
    dev->cc_major = prop.major;
    dev->cc_minor = prop.minor;
    dev->device = d;
  }
  *status = SKGEMM_OK;
  return dev;
}

StreamWorkspace* stream_workspace(DeviceState* dev, cudaStream_t s, int slots, int* status) {
  std::lock_guard<std::mutex> lk(dev->mu);
  StreamWorkspace*& ws = dev->ws[s];
  if (!ws) ws = new StreamWorkspace();
  *status = ws->ensure(slots);
  if (*status == SKGEMM_OK)
    *status = debug_poison(ws->partials, ws->partial_slots * kBM * kBN * sizeof(double), s);
  return *status == SKGEMM_OK ? ws : nullptr;
}

int consume_device_error(StreamWorkspace* ws, cudaStream_t s) {
  SKG_CUDA(cudaStreamSynchronize(s));
  if (!ws || !ws->err) return SKGEMM_OK;
  uint32_t word = 0;
  SKG_CUDA(cudaMemcpy(&word, ws->err, sizeof(word), cudaMemcpyDeviceToHost));
  if (word == 0) return SKGEMM_OK;
  SKG_CUDA(cudaMemset(ws->err, 0, sizeof(uint32_t)));
  char buf[160];
  snprintf(buf, sizeof(buf), "device-side wait ran past its budget (error word 0x%x)", word);
  return fail(SKGEMM_ERR_DEVICE_TIMEOUT, buf);
}

// ------------------------------------------------------- kernel timing
bool g_ktimer_on = false;
namespace {
struct KtRecord {
  const char* name;
  cudaEvent_t start, stop;
};
std::mutex g_kt_mu;
std::vector<KtRecord> g_kt_records;
std::vector<cudaEvent_t> g_kt_pool;
std::map<cudaStream_t, std::pair<const char*, cudaEvent_t>> g_kt_open;

cudaEvent_t kt_event() {
  if (!g_kt_pool.empty()) {
    cudaEvent_t e = g_kt_pool.back();
    g_kt_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}
}  // namespace

void ktimer_record(cudaStream_t s, const char* name, bool start) {
  std::lock_guard<std::mutex> lk(g_kt_mu);
  cudaEvent_t e = kt_event();
  if (!e) return;
  if (cudaEventRecord(e, s) != cudaSuccess) {
    g_kt_pool.push_back(e);
    return;
  }
  if (start) {
    auto it = g_kt_open.find(s);
    if (it != g_kt_open.end()) g_kt_pool.push_back(it->second.second);  // unmatched start
    g_kt_open[s] = {name, e};
    return;
  }
  auto it = g_kt_open.find(s);
  if (it == g_kt_open.end()) {
    g_kt_pool.push_back(e);
    return;
  }
  g_kt_records.push_back({name, it->second.second, e});
  g_kt_open.erase(it);
}

// ------------------------------------------------------------------- TMA
int encode_tiled(CUtensorMap* map, int rank, const void* base, const uint64_t* dims,
                 const uint64_t* strides_bytes, const uint32_t* box, CUtensorMapDataType dtype,
                 CUtensorMapSwizzle swizzle) {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
      return fail(SKGEMM_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  cuuint32_t estr[5] = {1, 1, 1, 1, 1};
  CUresult r = fn(map, dtype, (cuuint32_t)rank, const_cast<void*>(base),
                  reinterpret_cast<const cuuint64_t*>(dims),
                  reinterpret_cast<const cuuint64_t*>(strides_bytes),
                  reinterpret_cast<const cuuint32_t*>(box), estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    char buf[128];
    snprintf(buf, sizeof(buf), "cuTensorMapEncodeTiled failed (CUresult %d, rank %d)", (int)r,
             rank);
    return fail(SKGEMM_ERR_INVALID_ARG, buf);
  }
  return SKGEMM_OK;
}

// ------------------------------------------------------- K == 0 epilogues
namespace {

__global__ void k0_kernel(int mode, int64_t M, int64_t N, double* D, int64_t ld, double gamma,
                          int beta_zero) {
  int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= M * N) return;
  int64_t m = idx / N, n = idx % N;
  if (mode == kOutRowMajor) {
    D[m * ld + n] = gamma;  // alpha * 0 + gamma
  } else if (mode == kOutSyrkUpper) {
    if (m <= n) {
      double* c = D + m + n * ld;
      *c = beta_zero ? 0.0 : gamma * (*c);
    }
  }
}

}  // namespace

int run_k0(int mode, int64_t M, int64_t N, double* D, int64_t ld, double gamma, bool beta_zero,
           cudaStream_t s) {
  if (M == 0 || N == 0) return SKGEMM_OK;
  int64_t n = M * N;
  k0_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(mode, M, N, D, ld, gamma,
                                                        beta_zero ? 1 : 0);
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

// Native FP64 entry shared by the C ABI functions below.
int run_native(const Fp64Problem& prob, cudaStream_t s) {
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (prob.M == 0 || prob.N == 0) return SKGEMM_OK;
  if (prob.K == 0)
    return run_k0(prob.out_kind, prob.M, prob.N, prob.D, prob.ldd, prob.gamma, prob.beta_zero,
                  s);
  return launch_fp64(dev, prob, s);
}

Fp64Problem gemm_packed_problem(int64_t M, int64_t N, int64_t K, const double* Ap,
                                const double* Bp, double* D, int64_t ldd, double alpha,
                                double gamma) {
  Fp64Problem p;
  p.a = {Ap, kOpPacked16, M, 0};
  p.b = {Bp, kOpPacked32, N, 0};
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
  return p;
}

Fp64Problem syrk_problem(int64_t K, int64_t M, const double* Ap, double* C, int64_t ldc,
                         double alpha, double beta) {
  Fp64Problem p;
  p.a = {Ap, kOpPacked16, M, 0};
  p.b = {Ap, kOpPacked16, M, 0};
  p.M = M;
  p.N = M;
  p.K = K;
  p.tile_order = kTilesUpper;
  p.out_kind = kOutSyrkUpper;
  p.D = C;
  p.ldd = ldc;
  p.alpha = alpha;
  p.gamma = beta;
  p.beta_zero = (beta == 0.0);
  return p;
}

Fp64Problem rot_problem(int64_t Nd, int64_t nb, const double* A, const double* Q, double* D,
                        bool a_band) {
  Fp64Problem p;
  p.a = {A, a_band ? kOpBandK : kOpPacked16, Nd, 0};
  p.b = {Q, kOpDense, nb, nb};
  p.M = Nd;
  p.N = nb;
  p.K = nb;
  p.tile_order = kTilesAll;
  p.out_kind = kOutBand16;
  p.D = D;
  p.ldd = 0;
  p.alpha = 1.0;
  p.gamma = 0.0;
  p.beta_zero = true;
  return p;
}

int check_dims(int64_t a, int64_t b, int64_t c) {
  if (a < 0 || b < 0 || c < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative dimension");
  return SKGEMM_OK;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// SKGEMM_PREC_AUTO on one call: the Ozaki split (INT8) when its cost-model
// time is below 0.8 of the native kernels' (the batched plans' rule), native
// otherwise. `t_ozaki` < 0 means the split does not take the shape.
int auto_precision(double t_ozaki, double t_native) {
  return (t_ozaki >= 0.0 && t_ozaki < 0.8 * t_native) ? SKGEMM_PREC_OZAKI_I8 : SKGEMM_PREC_NATIVE;
}

// Runs `call` with a copy of `opts` whose precision AUTO is resolved; the
// caller's options get the outputs (slices_used_out = 0: native ran).
template <typename Call>
int run_resolved(skgemm_options_t* opts, int precision, Call call) {
  skgemm_options_t o = *opts;
  o.precision = precision;
  const int st = call(&o);
  opts->err_bound_out = o.err_bound_out;
  opts->slices_used_out = precision == SKGEMM_PREC_NATIVE ? 0 : o.slices_used_out;
  return st;
}

namespace {

// Blocking host-pointer execution: copies `nin` inputs to device staging
// buffers, runs `body` with the device pointers, copies `out` back.
struct HostIO {
  const void* src;
  size_t bytes;
};

template <typename Body>
int run_host(int nin, const HostIO* in, void* out_host, size_t out_bytes, bool out_is_input,
             Body body) {
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  std::lock_guard<std::mutex> lk(dev->host_mu);
  if (!dev->host_stream) SKG_CUDA(cudaStreamCreateWithFlags(&dev->host_stream, cudaStreamNonBlocking));
  cudaStream_t s = dev->host_stream;
  void* dptr[4] = {nullptr, nullptr, nullptr, nullptr};
  for (int i = 0; i < nin; ++i) {
    if ((st = dev->stage[i].ensure(in[i].bytes ? in[i].bytes : 16)) != SKGEMM_OK) return st;
    dptr[i] = dev->stage[i].ptr;
    if (in[i].bytes) SKG_CUDA(cudaMemcpyAsync(dptr[i], in[i].src, in[i].bytes, cudaMemcpyHostToDevice, s));
  }
  if ((st = dev->stage[3].ensure(out_bytes ? out_bytes : 16)) != SKGEMM_OK) return st;
  dptr[3] = dev->stage[3].ptr;
  if (out_is_input && out_bytes)
    SKG_CUDA(cudaMemcpyAsync(dptr[3], out_host, out_bytes, cudaMemcpyHostToDevice, s));
  if ((st = body(dptr, s)) != SKGEMM_OK) {
    cudaStreamSynchronize(s);
    return st;
  }
  if (out_bytes) SKG_CUDA(cudaMemcpyAsync(out_host, dptr[3], out_bytes, cudaMemcpyDeviceToHost, s));
  StreamWorkspace* ws = nullptr;
  {
    std::lock_guard<std::mutex> lk2(dev->mu);
    auto it = dev->ws.find(s);
    if (it != dev->ws.end()) ws = it->second;
  }
  return consume_device_error(ws, s);
}

}  // namespace
}  // namespace skg

using namespace skg;

#define SKG_EXPORT extern "C" __attribute__((visibility("default")))

SKG_EXPORT const char* skgemm_version(void) { return "skgemm 0.1.0 (sm_100a)"; }

SKG_EXPORT const char* skgemm_last_error(void) { return g_last_error.c_str(); }

SKG_EXPORT int skgemm_stream_status(void* stream) {
  NvtxRange nvtx_(__func__);
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  StreamWorkspace* ws = nullptr;
  {
    std::lock_guard<std::mutex> lk(dev->mu);
    auto it = dev->ws.find(s);
    if (it != dev->ws.end()) ws = it->second;
  }
  int e = consume_device_error(ws, s);
  if (e != SKGEMM_OK) return e;
  if ((e = batch_consume_error(dev, s)) != SKGEMM_OK) return e;
  return ozaki_consume_error(dev, s);
}

SKG_EXPORT int skgemm_stream_release(void* stream) {
  NvtxRange nvtx_(__func__);
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  SKG_CUDA(cudaStreamSynchronize(s));
  {
    std::lock_guard<std::mutex> lk(dev->mu);
    auto it = dev->ws.find(s);
    if (it != dev->ws.end()) {
      StreamWorkspace* ws = it->second;
      if (ws->partials) cudaFree(ws->partials);
      if (ws->flags) cudaFree(ws->flags);
      if (ws->err) cudaFree(ws->err);
      delete ws;
      dev->ws.erase(it);
    }
  }
  return ozaki_release_stream(dev, s);
}

SKG_EXPORT int skgemm_debug_fill(void) { return debug_fill_enabled() ? 1 : 0; }

SKG_EXPORT int skgemm_kernel_timing(int enable) {
  std::lock_guard<std::mutex> lk(g_kt_mu);
  if (enable) {
    for (auto& r : g_kt_records) {
      g_kt_pool.push_back(r.start);
      g_kt_pool.push_back(r.stop);
    }
    g_kt_records.clear();
    for (auto& o : g_kt_open) g_kt_pool.push_back(o.second.second);
    g_kt_open.clear();
  }
  g_ktimer_on = enable != 0;
  return SKGEMM_OK;
}

SKG_EXPORT int skgemm_kernel_timing_report(char* buf, int64_t len) {
  std::lock_guard<std::mutex> lk(g_kt_mu);
  std::map<std::string, std::pair<int64_t, double>> sum;
  int st = SKGEMM_OK;
  for (auto& r : g_kt_records) {
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(r.stop);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, r.start, r.stop);
    if (e != cudaSuccess) {
      st = cuda_fail(e, "kernel timing events");
      break;
    }
    auto& v = sum[r.name];
    v.first += 1;
    v.second += ms;
  }
  for (auto& r : g_kt_records) {
    g_kt_pool.push_back(r.start);
    g_kt_pool.push_back(r.stop);
  }
  g_kt_records.clear();
  if (st) return st;
  std::string out;
  char line[256];
  for (auto& kv : sum) {
    snprintf(line, sizeof(line), "%s %lld %.6f\n", kv.first.c_str(), (long long)kv.second.first,
             kv.second.second);
    out += line;
  }
  if (!buf || len <= (int64_t)out.size())
    return fail(SKGEMM_ERR_INVALID_ARG, "kernel timing report: buffer too small");
  memcpy(buf, out.c_str(), out.size() + 1);
  return (int)sum.size();
}

SKG_EXPORT int skgemm_diag_expire_wait(double budget_ms, void* stream) {
  NvtxRange nvtx_(__func__);
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  return expire_wait(dev, budget_ms, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_diag_expire_fixup_wait(double budget_ms, void* stream) {
  NvtxRange nvtx_(__func__);
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  return expire_fixup_wait(dev, budget_ms, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_probe_fp64_peak(double* tflops_out) {
  NvtxRange nvtx_(__func__);
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  return probe_fp64_peak(dev, tflops_out);
}

SKG_EXPORT int skgemm_probe_i8_peak(double* tops_out) {
  NvtxRange nvtx_(__func__);
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  if (!tops_out) return fail(SKGEMM_ERR_INVALID_ARG, "null output");
  return probe_i8_peak(dev, tops_out);
}

SKG_EXPORT int skgemm_igemm_s8_dev(int64_t M, int64_t N, int64_t K, const int8_t* A,
                                   int64_t lda, const int8_t* B, int64_t ldb, int32_t* C,
                                   int64_t ldc, void* stream) {
  NvtxRange nvtx_(__func__);
  return igemm_s8(M, N, K, A, lda, B, ldb, C, ldc, reinterpret_cast<cudaStream_t>(stream));
}

// ------------------------------------------------------------------- GEMM
SKG_EXPORT int skgemm_dgemm_packed_dev(int64_t M, int64_t N, int64_t K, const double* Ap,
                                       const double* Bp, double* D, int64_t ldd, double alpha,
                                       double gamma, void* stream) {
  NvtxRange nvtx_(__func__);
  int st = check_dims(M, N, K);
  if (st) return st;
  if (ldd < N) return fail(SKGEMM_ERR_INVALID_ARG, "ldd < N");
  return run_native(gemm_packed_problem(M, N, K, Ap, Bp, D, ldd, alpha, gamma),
                    reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_dgemm_dev(int64_t M, int64_t N, int64_t K, const double* A, int64_t lda,
                                const double* B, int64_t ldb, double* D, int64_t ldd,
                                double alpha, double gamma, void* stream) {
  NvtxRange nvtx_(__func__);
  int st = check_dims(M, N, K);
  if (st) return st;
  if (lda < M || ldb < N || ldd < N) return fail(SKGEMM_ERR_INVALID_ARG, "leading dimension too small");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (M == 0 || N == 0) return SKGEMM_OK;
  Fp64Problem p = gemm_packed_problem(M, N, K, nullptr, nullptr, D, ldd, alpha, gamma);
  // Operands whose columns are 16-byte aligned are read in place through 2-D
  // TMA maps; others are first packed on the device (HBM-bound, O(MK + KN)).
  double* scratch[2] = {nullptr, nullptr};
  if (K > 0 && (lda % 2 == 0) && aligned16(A)) {
    p.a = {A, kOpDense, M, lda};
  } else if (K > 0) {
    SKG_CUDA(cudaMallocAsync(&scratch[0], (size_t)((M + 15) / 16 * 16) * K * 8, s));
    if ((st = launch_pack(M, K, A, 1, lda, 16, scratch[0], s))) return st;
    p.a = {scratch[0], kOpPacked16, M, 0};
  }
  if (K > 0 && (ldb % 2 == 0) && aligned16(B)) {
    p.b = {B, kOpDense, N, ldb};
  } else if (K > 0) {
    SKG_CUDA(cudaMallocAsync(&scratch[1], (size_t)((N + 31) / 32 * 32) * K * 8, s));
    if ((st = launch_pack(N, K, B, 1, ldb, 32, scratch[1], s))) return st;
    p.b = {scratch[1], kOpPacked32, N, 0};
  }
  st = run_native(p, s);
  for (double* x : scratch)
    if (x) cudaFreeAsync(x, s);
  return st;
}

SKG_EXPORT int skgemm_dgemm_packed_dev_opt(int64_t M, int64_t N, int64_t K, const double* Ap,
                                           const double* Bp, double* D, int64_t ldd,
                                           double alpha, double gamma, skgemm_options_t* opts,
                                           void* stream) {
  NvtxRange nvtx_(__func__);
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const int pr = auto_precision(
        ozaki_time_estimate(SKGEMM_OP_GEMM_PACKED, M, N, K, opts->slices),
        batch_native_estimate(gemm_packed_problem(M, N, K, Ap, Bp, D, ldd, alpha, gamma)));
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return skgemm_dgemm_packed_dev_opt(M, N, K, Ap, Bp, D, ldd, alpha, gamma, o, stream);
    });
  }
  if (!opts || opts->precision == SKGEMM_PREC_NATIVE) {
    if (opts) {
      opts->err_bound_out = 0.0;
      opts->slices_used_out = 0;
    }
    return skgemm_dgemm_packed_dev(M, N, K, Ap, Bp, D, ldd, alpha, gamma, stream);
  }
  int st = check_dims(M, N, K);
  if (st) return st;
  if (ldd < N) return fail(SKGEMM_ERR_INVALID_ARG, "ldd < N");
  return ozaki_gemm_packed(M, N, K, Ap, Bp, D, ldd, alpha, gamma, opts,
                           reinterpret_cast<cudaStream_t>(stream));
}

// ------------------------------------------- K-chunked blocking host calls
// Long reductions (K >= 2 * kHostChunkK) are uploaded in k-chunks: chunk c + 1
// goes up on the copy stream while chunk c is multiplied on the compute
// stream, so the products hide under the upload. A packed-T operand
// [ceil(R/T)][K][T] gives chunk [k0, k0 + kc) as one strided copy (ceil(R/T)
// rows of kc*T doubles) into a compact [ceil(R/T)][kc][T] buffer; the chunks
// sit one after another in the staging buffer, so no chunk overwrites another.
constexpr int64_t kHostChunkK = 8192;
constexpr int kHostChunks = 4;

int host_chunks(int64_t K) {
  return (int)std::min<int64_t>(kHostChunks, std::max<int64_t>(1, K / kHostChunkK));
}

cudaError_t upload_packed_chunk(double* dst, const double* src, int T, int64_t R, int64_t K,
                                int64_t k0, int64_t kc, cudaStream_t s) {
  const int64_t panels = (R + T - 1) / T;
  return cudaMemcpy2DAsync(dst, (size_t)kc * T * 8, src + k0 * T, (size_t)K * T * 8,
                           (size_t)kc * T * 8, (size_t)panels, cudaMemcpyHostToDevice, s);
}

struct HostPipe {
  DeviceState* dev = nullptr;
  cudaStream_t sc = nullptr, si = nullptr;
  std::vector<cudaEvent_t> ev;
  int init(DeviceState* d, int n) {
    dev = d;
    for (cudaStream_t* ps : {&dev->host_stream, &dev->host_h2d, &dev->host_d2h})
      if (!*ps) SKG_CUDA(cudaStreamCreateWithFlags(ps, cudaStreamNonBlocking));
    sc = dev->host_stream;
    si = dev->host_h2d;
    ev.assign(n, nullptr);
    for (auto& e : ev) SKG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return SKGEMM_OK;
  }
  // Waits for both streams, frees the events, reports device-side errors.
  int finish(int st) {
    cudaStreamSynchronize(si);
    cudaStreamSynchronize(sc);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    ev.clear();
    if (st) return st;
    StreamWorkspace* ws = nullptr;
    {
      std::lock_guard<std::mutex> lk2(dev->mu);
      auto it = dev->ws.find(sc);
      if (it != dev->ws.end()) ws = it->second;
    }
    return consume_device_error(ws, sc);
  }
};

SKG_EXPORT int skgemm_dgemm_packed(int64_t M, int64_t N, int64_t K, const double* Ap,
                                   const double* Bp, double* D, double alpha, double gamma) {
  NvtxRange nvtx_(__func__);
  int st = check_dims(M, N, K);
  if (st) return st;
  if (M == 0 || N == 0) return SKGEMM_OK;
  if (!Ap || !Bp || !D) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  const int C = host_chunks(K);
  if (C > 1) {
    // Chunk c: D_c = alpha A_c B_c into its own M x N buffer, then
    // D = sum_c D_c + gamma (the GEMM contract has no accumulate form).
    DeviceState* dev = current_device(&st);
    if (!dev) return st;
    std::lock_guard<std::mutex> lk(dev->host_mu);
    HostPipe hp;
    if ((st = hp.init(dev, C))) return hp.finish(st);
    const int64_t PA = (M + 15) / 16, PB = (N + 31) / 32;
    if ((st = dev->stage[0].ensure((size_t)PA * 16 * K * 8)) ||
        (st = dev->stage[1].ensure((size_t)PB * 32 * K * 8)) ||
        (st = dev->stage[3].ensure((size_t)C * M * N * 8)))
      return hp.finish(st);
    double* dA = (double*)dev->stage[0].ptr;
    double* dB = (double*)dev->stage[1].ptr;
    double* dD = (double*)dev->stage[3].ptr;
    for (int c = 0; c < C && st == SKGEMM_OK; ++c) {
      const int64_t k0 = K * c / C, kc = K * (c + 1) / C - k0;
      double* a = dA + PA * 16 * k0;
      double* b = dB + PB * 32 * k0;
      cudaError_t e = upload_packed_chunk(a, Ap, 16, M, K, k0, kc, hp.si);
      if (e == cudaSuccess) e = upload_packed_chunk(b, Bp, 32, N, K, k0, kc, hp.si);
      if (e == cudaSuccess) e = cudaEventRecord(hp.ev[c], hp.si);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.sc, hp.ev[c], 0);
      if (e != cudaSuccess) {
        st = cuda_fail(e, "GEMM chunk upload");
        break;
      }
      st = skgemm_dgemm_packed_dev(M, N, kc, a, b, dD + (size_t)c * M * N, N, alpha, 0.0, hp.sc);
    }
    if (!st) st = launch_sum_parts(dD, C, M * N, gamma, dD, hp.sc);
    if (!st) {
      const cudaError_t e = cudaMemcpyAsync(D, dD, (size_t)M * N * 8, cudaMemcpyDeviceToHost,
                                            hp.sc);
      if (e != cudaSuccess) st = cuda_fail(e, "GEMM download");
    }
    return hp.finish(st);
  }
  HostIO in[2] = {{Ap, (size_t)((M + 15) / 16) * 16 * K * 8},
                  {Bp, (size_t)((N + 31) / 32) * 32 * K * 8}};
  return run_host(2, in, D, (size_t)M * N * 8, false, [&](void** d, cudaStream_t s) {
    return skgemm_dgemm_packed_dev(M, N, K, (const double*)d[0], (const double*)d[1],
                                   (double*)d[3], N, alpha, gamma, s);
  });
}

SKG_EXPORT int skgemm_dgemm(int64_t M, int64_t N, int64_t K, const double* A, const double* B,
                            double* D, double alpha, double gamma) {
  NvtxRange nvtx_(__func__);
  int st = check_dims(M, N, K);
  if (st) return st;
  if (M == 0 || N == 0) return SKGEMM_OK;
  if (!A || !B || !D) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  HostIO in[2] = {{A, (size_t)M * K * 8}, {B, (size_t)K * N * 8}};
  return run_host(2, in, D, (size_t)M * N * 8, false, [&](void** d, cudaStream_t s) {
    return skgemm_dgemm_dev(M, N, K, (const double*)d[0], M, (const double*)d[1], N,
                            (double*)d[3], N, alpha, gamma, s);
  });
}

// ------------------------------------------------------------------- SYRK
SKG_EXPORT int skgemm_dsyrk_packed_dev(int64_t K, int64_t M, const double* Ap, double* C,
                                       int64_t ldc, double alpha, double beta, void* stream) {
  NvtxRange nvtx_(__func__);
  int st = check_dims(K, M, 0);
  if (st) return st;
  if (ldc < M) return fail(SKGEMM_ERR_INVALID_ARG, "ldc < M");
  return run_native(syrk_problem(K, M, Ap, C, ldc, alpha, beta),
                    reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_dsyrk_packed_dev_opt(int64_t K, int64_t M, const double* Ap, double* C,
                                           int64_t ldc, double alpha, double beta,
                                           skgemm_options_t* opts, void* stream) {
  NvtxRange nvtx_(__func__);
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const int pr = auto_precision(
        ozaki_time_estimate(SKGEMM_OP_SYRK_PACKED, M, M, K, opts->slices),
        batch_native_estimate(syrk_problem(K, M, Ap, C, ldc, alpha, beta)));
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return skgemm_dsyrk_packed_dev_opt(K, M, Ap, C, ldc, alpha, beta, o, stream);
    });
  }
  if (!opts || opts->precision == SKGEMM_PREC_NATIVE) {
    if (opts) {
      opts->err_bound_out = 0.0;
      opts->slices_used_out = 0;
    }
    return skgemm_dsyrk_packed_dev(K, M, Ap, C, ldc, alpha, beta, stream);
  }
  int st = check_dims(K, M, 0);
  if (st) return st;
  if (ldc < M) return fail(SKGEMM_ERR_INVALID_ARG, "ldc < M");
  return ozaki_syrk_packed(K, M, Ap, C, ldc, alpha, beta, opts,
                           reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_dsubspace_packed_dev(int64_t K, int64_t M, const double* Psi,
                                           const double* HPsi, double* S, int64_t lds, double* Hs,
                                           int64_t ldh, skgemm_options_t* opts, void* stream) {
  NvtxRange nvtx_(__func__);
  int st = check_dims(K, M, 0);
  if (st) return st;
  if (lds < M || ldh < M) return fail(SKGEMM_ERR_INVALID_ARG, "lds or ldh < M");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const double tn = batch_native_estimate(syrk_problem(K, M, Psi, S, lds, 1.0, 0.0)) +
                      batch_native_estimate(gemm_packed_problem(M, M, K, Psi, HPsi, Hs, ldh,
                                                                1.0, 0.0));
    const int pr = auto_precision(ozaki_pair_time_estimate(K, M, opts->slices), tn);
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return skgemm_dsubspace_packed_dev(K, M, Psi, HPsi, S, lds, Hs, ldh, o, stream);
    });
  }
  if (!opts || opts->precision == SKGEMM_PREC_NATIVE || K == 0) {
    // Native FP64 (an empty reduction needs no split either).
    if (opts) {
      opts->err_bound_out = 0.0;
      opts->slices_used_out = 0;
    }
    if ((st = run_native(syrk_problem(K, M, Psi, S, lds, 1.0, 0.0), s))) return st;
    return run_native(gemm_packed_problem(M, M, K, Psi, HPsi, Hs, ldh, 1.0, 0.0), s);
  }
  return ozaki_subspace(K, M, Psi, HPsi, S, lds, 1.0, 0.0, Hs, ldh, 1.0, 0.0, opts, s);
}

SKG_EXPORT int skgemm_dsyrk_packed(int64_t K, int64_t M, const double* Ap, double* C,
                                   double alpha, double beta) {
  NvtxRange nvtx_(__func__);
  int st = check_dims(K, M, 0);
  if (st) return st;
  if (M == 0) return SKGEMM_OK;
  if (!Ap || !C) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  const int nch = host_chunks(K);
  if (nch > 1) {
    // Chunk c accumulates into C through the SYRK contract: beta for the
    // first chunk, 1 for the others (alpha on every chunk).
    DeviceState* dev = current_device(&st);
    if (!dev) return st;
    std::lock_guard<std::mutex> lk(dev->host_mu);
    HostPipe hp;
    if ((st = hp.init(dev, nch))) return hp.finish(st);
    const int64_t PA = (M + 15) / 16;
    if ((st = dev->stage[0].ensure((size_t)PA * 16 * K * 8)) ||
        (st = dev->stage[3].ensure((size_t)M * M * 8)))
      return hp.finish(st);
    double* dA = (double*)dev->stage[0].ptr;
    double* dC = (double*)dev->stage[3].ptr;
    // C goes up whole: beta != 0 reads it, and its strict lower triangle
    // returns as the caller passed it.
    cudaError_t e = cudaMemcpyAsync(dC, C, (size_t)M * M * 8, cudaMemcpyHostToDevice, hp.si);
    if (e != cudaSuccess) return hp.finish(cuda_fail(e, "SYRK upload"));
    for (int c = 0; c < nch && st == SKGEMM_OK; ++c) {
      const int64_t k0 = K * c / nch, kc = K * (c + 1) / nch - k0;
      double* a = dA + PA * 16 * k0;
      e = upload_packed_chunk(a, Ap, 16, M, K, k0, kc, hp.si);
      if (e == cudaSuccess) e = cudaEventRecord(hp.ev[c], hp.si);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(hp.sc, hp.ev[c], 0);
      if (e != cudaSuccess) {
        st = cuda_fail(e, "SYRK chunk upload");
        break;
      }
      st = skgemm_dsyrk_packed_dev(kc, M, a, dC, M, alpha, c == 0 ? beta : 1.0, hp.sc);
    }
    if (!st) {
      e = cudaMemcpyAsync(C, dC, (size_t)M * M * 8, cudaMemcpyDeviceToHost, hp.sc);
      if (e != cudaSuccess) st = cuda_fail(e, "SYRK download");
    }
    return hp.finish(st);
  }
  HostIO in[1] = {{Ap, (size_t)((M + 15) / 16) * 16 * K * 8}};
  // C is copied in and out whole: the strict lower triangle is returned as the
  // caller passed it, and beta != 0 reads the upper triangle.
  return run_host(1, in, C, (size_t)M * M * 8, true, [&](void** d, cudaStream_t s) {
    return skgemm_dsyrk_packed_dev(K, M, (const double*)d[0], (double*)d[3], M, alpha, beta, s);
  });
}

// --------------------------------------------------------------- rotation
static int check_rot(int64_t Nd, int64_t nb) {
  if (Nd < 0 || nb < 0) return fail(SKGEMM_ERR_INVALID_ARG, "negative dimension");
  if (Nd % 16 || nb % 16)
    return fail(SKGEMM_ERR_INVALID_ARG, "rotation layouts need Nd and nb multiples of 16");
  return SKGEMM_OK;
}

SKG_EXPORT int skgemm_drot_dev(int64_t Nd, int64_t nb, const double* A, const double* Q,
                               double* D, void* stream) {
  NvtxRange nvtx_(__func__);
  int st = check_rot(Nd, nb);
  if (st) return st;
  return run_native(rot_problem(Nd, nb, A, Q, D), reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_drot_dev_opt(int64_t Nd, int64_t nb, const double* A, const double* Q,
                                   double* D, skgemm_options_t* opts, void* stream) {
  NvtxRange nvtx_(__func__);
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const int pr = auto_precision(ozaki_time_estimate(SKGEMM_OP_ROT, Nd, nb, nb, opts->slices),
                                  batch_native_estimate(rot_problem(Nd, nb, A, Q, D)));
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return skgemm_drot_dev_opt(Nd, nb, A, Q, D, o, stream);
    });
  }
  if (!opts || opts->precision == SKGEMM_PREC_NATIVE) {
    if (opts) {
      opts->err_bound_out = 0.0;
      opts->slices_used_out = 0;
    }
    return skgemm_drot_dev(Nd, nb, A, Q, D, stream);
  }
  int st = check_rot(Nd, nb);
  if (st) return st;
  return ozaki_rot(Nd, nb, A, Q, D, opts, reinterpret_cast<cudaStream_t>(stream));
}

// The rotation reading band-packed Psi ([nb/16][Nd][16], the layout of SYRK's
// and GEMM's A): the band -> grid transposition of the grid-packed entry's
// input (sme_pack<double>::band_to_grid_tile, include/sme_pack.hpp:232-249)
// folded into the operand loads (FP64: K-major TMA boxes; Ozaki: the
// residue conversion's reads). Results equal skgemm_drot_dev /
// skgemm_drot_dev_opt on the grid-packed copy, bit for bit.
SKG_EXPORT int skgemm_drot_band_dev(int64_t Nd, int64_t nb, const double* A_band,
                                    const double* Q, double* D, void* stream) {
  NvtxRange nvtx_(__func__);
  int st = check_rot(Nd, nb);
  if (st) return st;
  return run_native(rot_problem(Nd, nb, A_band, Q, D, true),
                    reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_drot_band_dev_opt(int64_t Nd, int64_t nb, const double* A_band,
                                        const double* Q, double* D, skgemm_options_t* opts,
                                        void* stream) {
  NvtxRange nvtx_(__func__);
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const int pr = auto_precision(ozaki_time_estimate(SKGEMM_OP_ROT, Nd, nb, nb, opts->slices),
                                  batch_native_estimate(rot_problem(Nd, nb, A_band, Q, D)));
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return skgemm_drot_band_dev_opt(Nd, nb, A_band, Q, D, o, stream);
    });
  }
  if (!opts || opts->precision == SKGEMM_PREC_NATIVE) {
    if (opts) {
      opts->err_bound_out = 0.0;
      opts->slices_used_out = 0;
    }
    return skgemm_drot_band_dev(Nd, nb, A_band, Q, D, stream);
  }
  int st = check_rot(Nd, nb);
  if (st) return st;
  return ozaki_rot(Nd, nb, A_band, Q, D, opts, reinterpret_cast<cudaStream_t>(stream), true);
}

// Blocking host-pointer rotation, pipelined over row chunks of Psi: chunk c's
// grid-packed rows go up on one copy stream, its rotation runs on the compute
// stream into a chunk-local band-packed buffer, and its nb/16 band segments
// come back (one strided copy) on a second copy stream, so the upload of
// chunk c + 1 and the download of chunk c - 1 overlap (PCIe is full duplex)
// and the compute hides under both.
// `opts` (optional) selects the precision of every chunk; AUTO is resolved
// once for the whole Nd, so all chunks take the same path. The Ozaki split
// scales each grid row by its own norm and each column of Q by its norm over
// the same nb, so a chunk of rows gets exactly the bits the whole call would.
static int host_rot(int64_t Nd, int64_t nb, const double* A, const double* Q, double* D,
                    skgemm_options_t* opts) {
  int st = check_rot(Nd, nb);
  if (st) return st;
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const int pr = auto_precision(ozaki_time_estimate(SKGEMM_OP_ROT, Nd, nb, nb, opts->slices),
                                  batch_native_estimate(rot_problem(Nd, nb, A, Q, D)));
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return host_rot(Nd, nb, A, Q, D, o);
    });
  }
  if (opts) {
    opts->err_bound_out = 0.0;
    opts->slices_used_out = 0;
  }
  if (Nd == 0 || nb == 0) return SKGEMM_OK;
  if (!A || !Q || !D) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  std::lock_guard<std::mutex> lk(dev->host_mu);
  for (cudaStream_t* ps : {&dev->host_stream, &dev->host_h2d, &dev->host_d2h})
    if (!*ps) SKG_CUDA(cudaStreamCreateWithFlags(ps, cudaStreamNonBlocking));
  cudaStream_t sc = dev->host_stream, si = dev->host_h2d, so = dev->host_d2h;
  const size_t bytes = (size_t)Nd * nb * 8;
  if ((st = dev->stage[0].ensure(bytes)) || (st = dev->stage[1].ensure((size_t)nb * nb * 8)) ||
      (st = dev->stage[3].ensure(bytes)))
    return st;
  double* dA = (double*)dev->stage[0].ptr;
  double* dQ = (double*)dev->stage[1].ptr;
  double* dD = (double*)dev->stage[3].ptr;
  const int64_t panels = Nd / 16;
  const int C = (int)std::min<int64_t>(8, panels);
  std::vector<cudaEvent_t> ev(2 * C, nullptr);
  for (auto& e : ev) SKG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  SKG_CUDA(cudaMemcpyAsync(dQ, Q, (size_t)nb * nb * 8, cudaMemcpyHostToDevice, si));
  for (int c = 0; c < C && st == SKGEMM_OK; ++c) {
    const int64_t p0 = panels * c / C, p1 = panels * (c + 1) / C;
    const int64_t g0 = p0 * 16, rows = (p1 - p0) * 16;
    const size_t off = (size_t)g0 * nb;  // doubles: grid-packed rows and the chunk's output block
    cudaError_t e = cudaMemcpyAsync(dA + off, A + off, (size_t)rows * nb * 8,
                                    cudaMemcpyHostToDevice, si);
    if (e == cudaSuccess) e = cudaEventRecord(ev[2 * c], si);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(sc, ev[2 * c], 0);
    if (e != cudaSuccess) {
      st = cuda_fail(e, "rotation upload");
      break;
    }
    if ((st = skgemm_drot_dev_opt(rows, nb, dA + off, dQ, dD + off, opts, sc)) != SKGEMM_OK)
      break;
    e = cudaEventRecord(ev[2 * c + 1], sc);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(so, ev[2 * c + 1], 0);
    // Band b of the chunk (rows x 16 doubles at dD + off + b rows 16) goes to
    // D + b Nd 16 + g0 16.
    if (e == cudaSuccess)
      e = cudaMemcpy2DAsync(D + g0 * 16, (size_t)Nd * 16 * 8, dD + off, (size_t)rows * 16 * 8,
                            (size_t)rows * 16 * 8, (size_t)(nb / 16), cudaMemcpyDeviceToHost, so);
    if (e != cudaSuccess) st = cuda_fail(e, "rotation download");
  }
  cudaStreamSynchronize(si);
  cudaStreamSynchronize(sc);
  cudaStreamSynchronize(so);
  for (auto& e : ev) cudaEventDestroy(e);
  if (st) return st;
  StreamWorkspace* ws = nullptr;
  {
    std::lock_guard<std::mutex> lk2(dev->mu);
    auto it = dev->ws.find(sc);
    if (it != dev->ws.end()) ws = it->second;
  }
  return consume_device_error(ws, sc);
}

SKG_EXPORT int skgemm_drot(int64_t Nd, int64_t nb, const double* A, const double* Q,
                           double* D) {
  NvtxRange nvtx_(__func__);
  return host_rot(Nd, nb, A, Q, D, nullptr);
}

SKG_EXPORT int skgemm_drot_opt(int64_t Nd, int64_t nb, const double* A, const double* Q,
                               double* D, skgemm_options_t* opts) {
  NvtxRange nvtx_(__func__);
  return host_rot(Nd, nb, A, Q, D, opts);
}

// Host-pointer GEMM and SYRK with a precision selector. Native runs the
// k-chunked pipelines of skgemm_dgemm_packed / skgemm_dsyrk_packed. The Ozaki
// split scales every row by its norm over the whole K, so its operands go up
// whole and one device call runs them: the result is the device entry's bit
// for bit (its products are a small fraction of the upload time).
SKG_EXPORT int skgemm_dgemm_packed_opt(int64_t M, int64_t N, int64_t K, const double* Ap,
                                       const double* Bp, double* D, double alpha, double gamma,
                                       skgemm_options_t* opts) {
  NvtxRange nvtx_(__func__);
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const int pr = auto_precision(
        ozaki_time_estimate(SKGEMM_OP_GEMM_PACKED, M, N, K, opts->slices),
        batch_native_estimate(gemm_packed_problem(M, N, K, Ap, Bp, D, N, alpha, gamma)));
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return skgemm_dgemm_packed_opt(M, N, K, Ap, Bp, D, alpha, gamma, o);
    });
  }
  if (!opts || opts->precision == SKGEMM_PREC_NATIVE) {
    if (opts) {
      opts->err_bound_out = 0.0;
      opts->slices_used_out = 0;
    }
    return skgemm_dgemm_packed(M, N, K, Ap, Bp, D, alpha, gamma);
  }
  int st = check_dims(M, N, K);
  if (st) return st;
  if (M == 0 || N == 0) return SKGEMM_OK;
  if (!Ap || !Bp || !D) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  HostIO in[2] = {{Ap, (size_t)((M + 15) / 16) * 16 * K * 8},
                  {Bp, (size_t)((N + 31) / 32) * 32 * K * 8}};
  return run_host(2, in, D, (size_t)M * N * 8, false, [&](void** d, cudaStream_t s) {
    return skgemm_dgemm_packed_dev_opt(M, N, K, (const double*)d[0], (const double*)d[1],
                                       (double*)d[3], N, alpha, gamma, opts, s);
  });
}

SKG_EXPORT int skgemm_dsyrk_packed_opt(int64_t K, int64_t M, const double* Ap, double* C,
                                       double alpha, double beta, skgemm_options_t* opts) {
  NvtxRange nvtx_(__func__);
  if (opts && opts->precision == SKGEMM_PREC_AUTO) {
    const int pr = auto_precision(
        ozaki_time_estimate(SKGEMM_OP_SYRK_PACKED, M, M, K, opts->slices),
        batch_native_estimate(syrk_problem(K, M, Ap, C, M, alpha, beta)));
    return run_resolved(opts, pr, [&](skgemm_options_t* o) {
      return skgemm_dsyrk_packed_opt(K, M, Ap, C, alpha, beta, o);
    });
  }
  if (!opts || opts->precision == SKGEMM_PREC_NATIVE) {
    if (opts) {
      opts->err_bound_out = 0.0;
      opts->slices_used_out = 0;
    }
    return skgemm_dsyrk_packed(K, M, Ap, C, alpha, beta);
  }
  int st = check_dims(K, M, 0);
  if (st) return st;
  if (M == 0) return SKGEMM_OK;
  if (!Ap || !C) return fail(SKGEMM_ERR_INVALID_ARG, "null pointer");
  HostIO in[1] = {{Ap, (size_t)((M + 15) / 16) * 16 * K * 8}};
  return run_host(1, in, C, (size_t)M * M * 8, true, [&](void** d, cudaStream_t s) {
    return skgemm_dsyrk_packed_dev_opt(K, M, (const double*)d[0], (double*)d[3], M, alpha, beta,
                                       opts, s);
  });
}

// ------------------------------------------------------ layout converters
SKG_EXPORT int skgemm_pack_dev(int64_t R, int64_t K, const double* X, int64_t sr, int64_t sk,
                               int T, double* Xp, void* stream) {
  NvtxRange nvtx_(__func__);
  return launch_pack(R, K, X, sr, sk, T, Xp, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_unpack_dev(int64_t R, int64_t K, const double* X_packed, int T, double* X,
                                 int64_t sr, int64_t sk, void* stream) {
  NvtxRange nvtx_(__func__);
  return launch_unpack(R, K, X_packed, T, X, sr, sk, reinterpret_cast<cudaStream_t>(stream));
}

// The reference's extern "C" converters (include/sme_pack.hpp:319-329): grid
// g, band b; column-major [Nd, nb] and row-major [nb, Nd] are the same bytes
// src[g + b*Nd], and the packed side is grid-packed [Nd/16][nb][16].
namespace {
int c16_check(int64_t Nd, int64_t nb) {
  if (Nd < 0 || nb < 0 || Nd % 16)
    return skg::fail(SKGEMM_ERR_INVALID_ARG, "grid packing needs Nd >= 0 a multiple of 16");
  return SKGEMM_OK;
}
}  // namespace

SKG_EXPORT int skgemm_pack_c16_dev(int64_t Nd, int64_t nb, const double* src, double* dst,
                                   void* stream) {
  NvtxRange nvtx_(__func__);
  if (int st = c16_check(Nd, nb)) return st;
  return launch_pack(Nd, nb, src, 1, Nd, 16, dst, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_pack_r16_dev(int64_t Nd, int64_t nb, const double* src, double* dst,
                                   void* stream) {
  NvtxRange nvtx_(__func__);
  return skgemm_pack_c16_dev(Nd, nb, src, dst, stream);
}

SKG_EXPORT int skgemm_unpack_c16_dev(int64_t Nd, int64_t nb, const double* src, double* dst,
                                     void* stream) {
  NvtxRange nvtx_(__func__);
  if (int st = c16_check(Nd, nb)) return st;
  return launch_unpack(Nd, nb, src, 16, dst, 1, Nd, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_unpack_r16_dev(int64_t Nd, int64_t nb, const double* src, double* dst,
                                     void* stream) {
  NvtxRange nvtx_(__func__);
  return skgemm_unpack_c16_dev(Nd, nb, src, dst, stream);
}

// The reference's extern "C" converters under their own names and signatures
// (include/sme_pack.hpp:316-352): host pointers, blocking, no status (the
// reference returns void; a refused call leaves dst as it was and records
// the reason for skgemm_last_error, which a successful call clears). As in
// the reference, only the first 16 * floor(Nd / 16) grid points are
// converted (its g_tiles = Nd / 16); the dense side keeps its column stride Nd.
namespace {
void linalg_convert(int Nd, int nb, const double* src, double* dst, bool pack) {
  g_last_error.clear();  // no status to return: an empty message means success
  if (Nd < 0 || nb < 0) {
    skg::fail(SKGEMM_ERR_INVALID_ARG, "linalg converters: Nd and nb must be >= 0");
    return;
  }
  const int64_t R = (int64_t)Nd / 16 * 16;
  if (R == 0 || nb == 0) return;
  if (!src || !dst) {
    skg::fail(SKGEMM_ERR_INVALID_ARG, "linalg converters: null pointer");
    return;
  }
  const size_t dense = (size_t)Nd * nb * 8, packed = (size_t)R * nb * 8;
  const HostIO in{src, pack ? dense : packed};
  // Unpacking a ragged Nd writes only the first R rows of each column: the
  // rest of dst must come back unchanged, so it goes up first.
  const bool keep = !pack && R != Nd;
  run_host(1, &in, dst, pack ? packed : dense, keep, [&](void** d, cudaStream_t s) {
    return pack ? launch_pack(R, nb, (const double*)d[0], 1, Nd, 16, (double*)d[3], s)
                : launch_unpack(R, nb, (const double*)d[0], 16, (double*)d[3], 1, Nd, s);
  });
}
}  // namespace

SKG_EXPORT void linalg_pack_c16_f64(const int Nd, const int nb, const double* src,
                                    double* dst) {
  NvtxRange nvtx_(__func__);
  linalg_convert(Nd, nb, src, dst, true);
}

// Row-major [nb, Nd] (src[b*Nd + g]) is the same bytes as column-major [Nd, nb].
SKG_EXPORT void linalg_pack_r16_f64(const int Nd, const int nb, const double* src,
                                    double* dst) {
  NvtxRange nvtx_(__func__);
  linalg_convert(Nd, nb, src, dst, true);
}

SKG_EXPORT void linalg_unpack_c16_f64(const int Nd, const int nb, const double* src,
                                      double* dst) {
  NvtxRange nvtx_(__func__);
  linalg_convert(Nd, nb, src, dst, false);
}

SKG_EXPORT void linalg_unpack_r16_f64(const int Nd, const int nb, const double* src,
                                      double* dst) {
  NvtxRange nvtx_(__func__);
  linalg_convert(Nd, nb, src, dst, false);
}

SKG_EXPORT int skgemm_stencil_ext_dev(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                                      const double* psi_ext16, const double* A_diag,
                                      const double* coef_x, const double* coef_y,
                                      const double* coef_z, double coef_0, double* out,
                                      int out_tile, void* stream) {
  NvtxRange nvtx_(__func__);
  int st;
  DeviceState* dev = current_device(&st);
  if (!dev) return st;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  return launch_stencil_ext(ni, nj, nk, nb, FDn, psi_ext16, A_diag, coef_x, coef_y, coef_z,
                            coef_0, out, out_tile, dev->num_sms, ws->err, s);
}

SKG_EXPORT int skgemm_halo_periodic_dev(int64_t ni, int64_t nj, int64_t nk, int64_t nb, int FDn,
                                        const double* psi_local16, double* psi_ext16,
                                        void* stream) {
  NvtxRange nvtx_(__func__);
  return launch_halo_periodic(ni, nj, nk, nb, FDn, psi_local16, psi_ext16,
                              reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_nloc_create(int64_t P, const uint32_t* nrow, const uint32_t* ncol,
                                  const int32_t* atom, const uint32_t* offsets,
                                  const uint32_t* index, const double* chi, const double* gamma,
                                  int64_t K, skgemm_nloc_t* out) {
  NvtxRange nvtx_(__func__);
  return nloc_create(P, nrow, ncol, atom, offsets, index, chi, gamma, K, out);
}

SKG_EXPORT int skgemm_nloc_apply_dev(skgemm_nloc_t h, int64_t nb, double dv,
                                     const double* psi16, double* out, int out_tile,
                                     void* stream) {
  NvtxRange nvtx_(__func__);
  return nloc_apply(h, nb, dv, psi16, out, out_tile, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT void skgemm_nloc_destroy(skgemm_nloc_t h) { nloc_destroy(h); }

SKG_EXPORT int skgemm_band_to_grid_dev(int64_t Nd, int64_t nb, const double* src, double* dst,
                                       void* stream) {
  NvtxRange nvtx_(__func__);
  return launch_band_to_grid(Nd, nb, src, dst, reinterpret_cast<cudaStream_t>(stream));
}

SKG_EXPORT int skgemm_grid_to_band_dev(int64_t Nd, int64_t nb, const double* src, double* dst,
                                       void* stream) {
  NvtxRange nvtx_(__func__);
  return launch_grid_to_band(Nd, nb, src, dst, reinterpret_cast<cudaStream_t>(stream));
}
