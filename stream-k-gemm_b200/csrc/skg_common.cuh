// Shared device helpers for the sm_100a kernels: status codes, bounded waits,
// mbarrier / TMA wrappers (inline PTX) and the FP64 DMMA instruction.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "skgemm.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "skgemm kernels target sm_100a only"
#endif

namespace skg {

// --------------------------------------------------------------------------
// Device error word. Kernels never trap: a wait that runs past its budget ORs
// a code into this word and the kernel winds down; the host maps it to
// SKGEMM_ERR_DEVICE_TIMEOUT after the launch completes.
// --------------------------------------------------------------------------
enum DeviceError : uint32_t {
  kDevErrNone = 0,
  kDevErrMbarTimeout = 1u << 0,   // an mbarrier wait exceeded its iteration cap
  kDevErrFixupTimeout = 1u << 1,  // a Stream-K partial-tile flag never arrived
  kDevErrBadSchedule = 1u << 2,   // schedule arithmetic produced an impossible segment
};

// Budgets of the spin loops. An mbarrier wait normally completes within
// microseconds; the budgets only bound pathological cases. The mbarrier budget
// exceeds the fixup budget because a producer may legitimately wait while its
// consumers sit in a fixup wait. Iteration caps back up the timers.
constexpr uint64_t kFixupBudgetNs = 4ull * 1000ull * 1000ull * 1000ull;  // 4 s
constexpr uint32_t kFixupSpinCap = 1u << 26;
constexpr uint64_t kMbarBudgetNs = 8ull * 1000ull * 1000ull * 1000ull;   // 8 s
constexpr uint32_t kMbarSpinCap = 1u << 30;

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// --------------------------------------------------------------------------
// mbarrier
// --------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile(
      "{\n\t.reg .b64 st;\n\t"
      "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
      "r"(bytes)
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: returns false (and records the error) when `budget_ns` of
// device time or kMbarSpinCap polls run out.
__device__ __forceinline__ bool mbar_wait_ns(uint64_t* bar, uint32_t parity, uint32_t* err,
                                             uint64_t budget_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t it = 1; it < kMbarSpinCap; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 255u) == 0 && globaltimer_ns() - t0 > budget_ns) break;
  }
  if (err) atomicOr(err, kDevErrMbarTimeout);
  return false;
}
// The kernels' wait: the 8 s budget.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t* err) {
  return mbar_wait_ns(bar, parity, err, kMbarBudgetNs);
}

// --------------------------------------------------------------------------
// TMA (cp.async.bulk.tensor), no multicast.
// --------------------------------------------------------------------------
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int32_t c0, int32_t c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int32_t c0, int32_t c1, int32_t c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
// TMA store shared -> global (tile mode, bulk-group completion). The box
// must lie at non-negative coordinates; parts outside the tensor are not
// written.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int32_t c0,
                                             int32_t c1, int32_t c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
__device__ __forceinline__ void bulk_commit_group() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
// The source shared memory of every committed bulk store may be reused.
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// Every committed bulk store has completed.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void tma_load_1d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int32_t c0) {
  asm volatile(
      "cp.async.bulk.tensor.1d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0)
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int32_t c0, int32_t c1, int32_t c2, int32_t c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cta.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2),
      "r"(c3)
      : "memory");
}

// --------------------------------------------------------------------------
// FP64 tensor-core MMA (DMMA), m16n8k8, row.col, D = A*B + D.
// Fragment ownership (lane = 4*g + t):
//   A: a0=(g,t) a1=(g+8,t) a2=(g,t+4) a3=(g+8,t+4)      [row, k]
//   B: b0=(k=t, n=g) b1=(k=t+4, n=g)
//   C: c0=(g,2t) c1=(g,2t+1) c2=(g+8,2t) c3=(g+8,2t+1)  [row, col]
// --------------------------------------------------------------------------
__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], double a0, double a1, double a2,
                                            double a3, double b0, double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

__device__ __forceinline__ double2 lds128(uint32_t addr) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr));
  return v;
}

// 8-byte asynchronous global -> shared copy; src_bytes = 0 writes zeros.
__device__ __forceinline__ void cp_async8(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
// 16-byte asynchronous global -> shared copy (L2 only); src_bytes = 0 writes
// zeros. Both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Release / acquire flag accesses at GPU scope for the Stream-K fixup.
__device__ __forceinline__ void st_release_gpu(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The Stream-K fixup's wait for a later CTA's partial tile: spin (acquire)
// until *flag == want, bounded by budget_ns of %globaltimer and
// kFixupSpinCap polls. On expiry the timeout is ORed into *err and false is
// returned; the caller skips that partial and finishes normally.
__device__ __forceinline__ bool fixup_flag_wait(const uint32_t* flag, uint32_t want,
                                                uint32_t* err, uint64_t budget_ns) {
  const uint64_t t0 = globaltimer_ns();
  uint32_t spins = 0;
  while (ld_acquire_gpu(flag) != want) {
    __nanosleep(128);
    if (++spins > kFixupSpinCap || globaltimer_ns() - t0 > budget_ns) {
      atomicOr(err, kDevErrFixupTimeout);
      return false;
    }
  }
  return true;
}

}  // namespace skg
