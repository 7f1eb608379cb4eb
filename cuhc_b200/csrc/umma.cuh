// Fifth-generation tensor core (tcgen05) helpers: tensor-memory allocation,
// shared-memory operand descriptors, the TF32 MMA with an FP32 accumulator in
// tensor memory, commit to an mbarrier, and tensor-memory loads.
//
// Operands live in shared memory in the K-major, non-swizzled canonical
// layout: "core matrices" of 8 rows x 16 bytes (8 rows x 4 TF32 values),
// stored contiguously (128 B each). Element (row r, k) of a rows x K operand
// sits at
//     (r / 8) * SBO + (k / 4) * LBO + (r % 8) * 16 + (k % 4) * 4   bytes,
// with LBO = 128 (core matrices adjacent along K) and SBO = K * 32 (one
// 8-row group of all K). One MMA consumes K = 8 (two core matrices along K);
// step s starts at byte 256 * s. Descriptor bit layout: start address >> 4
// in [0,14), LBO >> 4 in [16,30), SBO >> 4 in [32,46), version 1 in
// [46,48), layout type (0 = no swizzle) in [61,64). Instruction descriptor:
// D format F32 (1) in [4,6), A / B format TF32 (2) in [7,10) / [10,13),
// K-major A and B, N >> 3 in [17,23), M >> 4 in [24,29).
#pragma once

#include <cstdint>

#include "asyncload.cuh"

namespace cuhc {

__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint64_t umma_smem_desc(const void *base, uint32_t lbo, uint32_t sbo) {
  const uint32_t addr = smemAddress(base);
  uint64_t desc = 0;
  desc |= (uint64_t)((addr >> 4) & 0x3fffu);
  desc |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
  desc |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
  desc |= (uint64_t)1 << 46; // descriptor version for sm_100
  return desc;                // layout type 0: no swizzle
}

// Byte offset of element (row, k) in the canonical K-major layout.
__device__ __forceinline__ uint32_t umma_offset(int row, int k, uint32_t sbo) {
  return (uint32_t)(row >> 3) * sbo + (uint32_t)(k >> 2) * 128u + (uint32_t)(row & 7) * 16u +
         (uint32_t)(k & 3) * 4u;
}

// TF32 (round to nearest, ties away) of an FP32 value, as an FP32 bit
// pattern with the 13 low mantissa bits zero.
__device__ __forceinline__ float toTf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Whole warp: allocates `cols` tensor-memory columns; the address lands in
// *dst (shared memory). cols is a power of two >= 32.
__device__ __forceinline__ void tmemAlloc(uint32_t *dst, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smemAddress(dst)),
               "r"(cols)
               : "memory");
}

__device__ __forceinline__ void tmemRelinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmemDealloc(uint32_t taddr, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
               : "memory");
}

__device__ __forceinline__ void tcgenFenceBefore() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tcgenFenceAfter() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// One thread: D (tensor memory) = A * B^T (+ D when accumulate).
__device__ __forceinline__ void mmaTf32(uint32_t tmemD, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, bool accumulate) {
  const uint32_t zero = 0, acc = accumulate ? 1u : 0u;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
               :
               : "r"(tmemD), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc), "r"(zero),
                 "r"(zero), "r"(zero), "r"(zero)
               : "memory");
}

// One thread: the mbarrier gets one arrival when this thread's earlier MMAs
// have completed.
__device__ __forceinline__ void mmaCommit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smemAddress(bar))
               : "memory");
}

// Whole warp: 32 consecutive FP32 columns of this thread's lane.
__device__ __forceinline__ void tmemLoad32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
               "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
               "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
               "[%32];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                 "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                 "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                 "=r"(r[30]), "=r"(r[31])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i)
    v[i] = __uint_as_float(r[i]);
}

// Whole warp: starts loading 32 consecutive FP32 columns of this thread's
// lane; the registers are valid only after tmemWaitLoads.
__device__ __forceinline__ void tmemLoad32Async(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
               "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
               "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
               "[%32];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                 "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                 "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                 "=r"(r[30]), "=r"(r[31])
               : "r"(taddr));
}

// Whole warp: waits for this thread's outstanding tensor-memory loads. The
// registers pass through the statement so that no use moves above the wait.
__device__ __forceinline__ void tmemWaitLoads(uint32_t (&r)[32]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                 "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                 "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                 "+r"(r[30]), "+r"(r[31])
               :
               : "memory");
}

// Orders later uses of r after the preceding (volatile) wait; emits nothing.
__device__ __forceinline__ void tmemHold(uint32_t (&r)[32]) {
  asm volatile(""
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]),
                 "+r"(r[6]), "+r"(r[7]), "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]),
                 "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]), "+r"(r[16]), "+r"(r[17]),
                 "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                 "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]),
                 "+r"(r[30]), "+r"(r[31]));
}

} // namespace cuhc
