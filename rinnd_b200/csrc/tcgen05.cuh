// tcgen05.cuh -- inline-PTX wrappers for the 5th-generation tensor cores (sm_100a):
// tensor-memory allocation, tcgen05.mma (kind::f16, BF16 in / FP32 accumulate,
// one CTA), completion via tcgen05.commit on an mbarrier, and tcgen05.ld of the
// accumulator.
//
// Operand layout used here: K-major without swizzle.  A "core matrix" is 8 rows
// x 16 bytes (8 BF16 along K) stored contiguously (128 bytes); core matrices
// adjacent along K are LBO bytes apart and 8-row groups SBO bytes apart.  With
// the K-chunks of a row group stored back to back, element (r, k) of a tile
// with K columns sits at (r/8)*SBO + (k/8)*128 + (r%8)*16 + (k%8)*2, where
// LBO = 128 and SBO = (K/8)*128; one MMA consumes K = 16 (two core matrices),
// so K-step s starts 256*s bytes further.
// Accumulator layout (cta_group::1): M = 128 -> row i in TMEM lane i; M = 64 ->
// rows 16q..16q+15 in lanes 32q..32q+15 (q = 0..3); column n = TMEM column n.
// (Both checked on a B200 against a CPU product for M = 64 with N = 16..64 and
// K = 80..256, and for M = 128.)
#pragma once
#include <stdint.h>

namespace rinnd {
namespace umma {

// Shared-memory matrix descriptor (K-major, no swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, absolute LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Whole warp: allocate `ncols` (power of two >= 32) TMEM columns; the address
// is written to shared memory at `slot`.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

// Whole warp (the allocating one).
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A * B^T, one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
      : "memory");
}

// Arrive on `bar` (one arrival) when all earlier tcgen05.mma of this thread completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(bar))
               : "memory");
}

// Whole warp: 16 consecutive 32-bit columns of the warp's 32 TMEM lanes.
__device__ __forceinline__ void ld_32x32b_x16(uint32_t taddr, uint32_t* r) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace umma
}  // namespace rinnd
