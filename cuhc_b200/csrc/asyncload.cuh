// Bulk asynchronous copies global -> shared (the untiled TMA engine,
// cp.async.bulk) completed on a shared-memory mbarrier, and bounded waits.
//
// Rules kept by every caller: source and destination 16-byte aligned, sizes a
// multiple of 16 bytes, sources entirely inside their allocation (per-tile
// arrays are padded to whole tiles), and never a load from another GPU's
// memory. Waits spin at most kSpinLimit times; a wait that runs out returns
// false and the kernel records kErrorTimeout and leaves.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace cuhc {

__device__ __forceinline__ uint32_t smemAddress(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbarrierInit(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddress(bar)), "r"(count)
               : "memory");
}

// Makes the barrier initialisation visible to the async proxy.
__device__ __forceinline__ void fenceBarrierInit() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier shared-memory accesses (generic proxy) before
// later async-proxy writes to the same buffer.
__device__ __forceinline__ void fenceProxyAsync() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbarrierArriveExpectTx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddress(bar)),
               "r"(bytes)
               : "memory");
}

// Plain arrival of `count` on the barrier, releasing this thread's earlier
// shared-memory writes to the threads that wait on the phase.
__device__ __forceinline__ void mbarrierArrive(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddress(bar)),
               "r"(count)
               : "memory");
}

// Named barrier `id` over `threads` threads (a multiple of 32) that also ORs a
// predicate across them: every participant gets the same answer.
__device__ __forceinline__ bool namedBarrierOr(int id, int threads, bool predicate) {
  uint32_t out;
  asm volatile("{\n\t.reg .pred p, q;\n\t"
               "setp.ne.u32 p, %1, 0;\n\t"
               "bar.red.or.pred q, %2, %3, p;\n\t"
               "selp.u32 %0, 1, 0, q;\n\t}"
               : "=r"(out)
               : "r"((uint32_t)predicate), "r"(id), "r"(threads)
               : "memory");
  return out != 0;
}

__device__ __forceinline__ void bulkCopyToShared(void *dst, const void *src, uint32_t bytes,
                                                 uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smemAddress(dst)),
      "l"(src), "r"(bytes), "r"(smemAddress(bar))
      : "memory");
}

__device__ __forceinline__ bool mbarrierTryWait(uint64_t *bar, uint32_t phase) {
  uint32_t done;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(done)
               : "r"(smemAddress(bar)), "r"(phase)
               : "memory");
  return done != 0;
}

__device__ __forceinline__ uint64_t globalTimerNs() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// A wait on a copy or an MMA that has not completed after this long never
// will: the kernel records kErrorTimeout and leaves.
constexpr uint64_t kWaitLimitNs = 1000000000ull;

// try_wait that lets the hardware suspend the thread (issuing nothing) until
// the phase completes or about `hintNs` nanoseconds pass.
__device__ __forceinline__ bool mbarrierTryWaitSuspend(uint64_t *bar, uint32_t phase,
                                                       uint32_t hintNs) {
  uint32_t done;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(done)
               : "r"(smemAddress(bar)), "r"(phase), "r"(hintNs)
               : "memory");
  return done != 0;
}

// Waits for the barrier's phase `phase` to complete, suspended in between
// (a waiting warp takes no issue slots from the warps doing the work); false
// if a second of wall-clock time (or the iteration limit) ran out first.
// limitNs shortens the limit (the bounded-wait self-test only).
__device__ __forceinline__ bool mbarrierWait(uint64_t *bar, uint32_t phase,
                                             uint64_t limitNs = kWaitLimitNs) {
  if (mbarrierTryWait(bar, phase))
    return true;
  const uint64_t start = globalTimerNs();
  for (long long spins = 0; spins < kSpinLimit; ++spins) {
    if (mbarrierTryWaitSuspend(bar, phase, 100000u))
      return true;
    if (globalTimerNs() - start > limitNs)
      return false;
  }
  return false;
}

} // namespace cuhc
