// FP64 tensor-core peak probe: register-resident DMMA m16n8k8 loop on every
// SM, timed with CUDA events. It plays the role of the reference's FMOPA peak
// microbenchmark (sme_peak_microbench.cpp:16-61) and supplies the FP64
// roofline denominator, which the driver-measured peaks do not include.
#include "skg_common.cuh"
#include "skg_runtime.h"

namespace skg {

namespace {

constexpr int kProbeAcc = 8;

__global__ void __launch_bounds__(256) dmma_peak_kernel(int iters, double* sink) {
  double acc[kProbeAcc][4];
#pragma unroll
  for (int j = 0; j < kProbeAcc; ++j)
#pragma unroll
    for (int r = 0; r < 4; ++r) acc[j][r] = 0.0;
  const double a0 = 1e-3 * threadIdx.x, a1 = a0 + 1e-4, a2 = a0 - 1e-4, a3 = a0 + 2e-4;
  const double b0 = 1e-3 * (32 - (int)(threadIdx.x & 31)), b1 = b0 + 1e-4;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int j = 0; j < kProbeAcc; ++j) dmma_16x8x8(acc[j], a0, a1, a2, a3, b0, b1);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < kProbeAcc; ++j) s += acc[j][0] + acc[j][1] + acc[j][2] + acc[j][3];
  if (s == 1.0e300) sink[0] = s;  // keeps the loop live; never true
}

// One thread waits on an mbarrier that nothing arrives on, with the same
// bounded wait the kernels use (a shorter budget): the wait gives up, the
// timeout lands in the stream's device error word, the kernel returns.
__global__ void expire_wait_kernel(uint32_t* err, uint64_t budget_ns) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_wait_ns(&bar, 0, err, budget_ns);  // phase 0 never completes
  }
}

// One thread runs the Stream-K fixup's flag wait on a flag that is never
// set to the awaited value (the stream's first partial-tile flag holds call
// epochs, which count up from 1 and never reach 0xffffffff): the wait gives
// up after its budget, records the fixup timeout, and the kernel returns.
__global__ void expire_fixup_wait_kernel(const uint32_t* flag, uint32_t* err,
                                         uint64_t budget_ns) {
  if (threadIdx.x == 0) fixup_flag_wait(flag, 0xffffffffu, err, budget_ns);
}

}  // namespace

int expire_fixup_wait(DeviceState* dev, double budget_ms, cudaStream_t s) {
  if (!(budget_ms > 0.0 && budget_ms <= 1000.0))
    return fail(SKGEMM_ERR_INVALID_ARG, "budget_ms must be in (0, 1000]");
  int st;
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  expire_fixup_wait_kernel<<<1, 32, 0, s>>>(ws->flags, ws->err, (uint64_t)(budget_ms * 1e6));
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int expire_wait(DeviceState* dev, double budget_ms, cudaStream_t s) {
  if (!(budget_ms > 0.0 && budget_ms <= 1000.0))
    return fail(SKGEMM_ERR_INVALID_ARG, "budget_ms must be in (0, 1000]");
  int st;
  StreamWorkspace* ws = stream_workspace(dev, s, 1, &st);
  if (!ws) return st;
  expire_wait_kernel<<<1, 32, 0, s>>>(ws->err, (uint64_t)(budget_ms * 1e6));
  SKG_CUDA(cudaGetLastError());
  return SKGEMM_OK;
}

int probe_fp64_peak(DeviceState* dev, double* tflops) {
  if (!tflops) return fail(SKGEMM_ERR_INVALID_ARG, "null output");
  double* sink = nullptr;
  SKG_CUDA(cudaMalloc(&sink, sizeof(double)));
  cudaEvent_t e0, e1;
  SKG_CUDA(cudaEventCreate(&e0));
  SKG_CUDA(cudaEventCreate(&e1));
  const int grid = dev->num_sms * 2, iters = 4096;
  dmma_peak_kernel<<<grid, 256>>>(iters / 8, sink);  // warm-up
  SKG_CUDA(cudaEventRecord(e0));
  const int reps = 3;
  for (int r = 0; r < reps; ++r) dmma_peak_kernel<<<grid, 256>>>(iters, sink);
  SKG_CUDA(cudaEventRecord(e1));
  SKG_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  SKG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  const double flops = 2.0 * 16 * 8 * 8 * (double)kProbeAcc * iters * (grid * 8.0) * reps;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return SKGEMM_OK;
}

}  // namespace skg
