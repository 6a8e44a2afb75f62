// join_common.cuh -- pieces shared by the pipelined local-join kernels
// (join_tma.cu: FP32 SIMT tiles; join_tc.cu: BF16 tensor-core Gram tiles with
// FP32 recheck): the per-vertex descriptor format, bounded mbarrier waits,
// packed FP32x2 arithmetic and the exact FP32 pair distance both kernels use.
#pragma once
#include "async_copy.cuh"
#include "dist.cuh"
#include "heap.cuh"

namespace rinnd {
namespace joinc {

constexpr uint32_t WAIT_POLLS = 1u << 21;
constexpr int NDESC = 4;   // descriptor ring depth
constexpr int NQMAX = 16;  // max item quads per vertex (na <= 64)

// Per-vertex descriptor (ints): [0] na, [1] nb, [2] nq, [3] items,
// [4..20) quad item prefix, [20..) ids (2*maxc, new first), thresholds (2*maxc;
// filled in the stage by the producer), norms (2*maxc; dot-form metrics).
struct Desc {
  static constexpr int HDR = 4 + NQMAX;
  __host__ __device__ static int ids(int) { return HDR; }
  __host__ __device__ static int thr(int maxc) { return HDR + 2 * maxc; }
  __host__ __device__ static int nrm(int maxc) { return HDR + 4 * maxc; }
  __host__ __device__ static int stride(int maxc) { return (HDR + 6 * maxc + 15) / 16 * 16; }
};

// Bounded wait that also gives up when another warp has aborted.
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  for (uint32_t i = 0; i < WAIT_POLLS; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 63) == 63 && *abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Packed FP32x2 arithmetic (each half rounded as the scalar instruction).
__device__ __forceinline__ unsigned long long f2_sub(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long f2_add(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ float f2_sum(unsigned long long a) {
  return __uint_as_float((uint32_t)a) + __uint_as_float((uint32_t)(a >> 32));
}

// Exact FP32 join distance between two staged rows (Dp floats, 16-byte
// aligned): packed accumulators over dimension pairs (4q, 4q+1) and
// (4q+2, 4q+3), summed at the end -- the FP32 join's per-item arithmetic, so
// both join kernels push identical distances.  Dot-form kinds return the raw
// dot product (finalized by the caller with the norms).
__device__ __forceinline__ float join_dist_fp32(int kind, const float* a, const float* b, int Dp) {
  const ulonglong2* pa = reinterpret_cast<const ulonglong2*>(a);
  const ulonglong2* pb = reinterpret_cast<const ulonglong2*>(b);
  unsigned long long acc = 0ull;
  if (kind == DK_SQEUCLIDEAN) {
#pragma unroll 4
    for (int q = 0; q < Dp / 4; ++q) {
      const ulonglong2 x = pa[q], y = pb[q];
      const unsigned long long d01 = f2_sub(x.x, y.x), d23 = f2_sub(x.y, y.y);
      acc = f2_fma(d01, d01, acc);
      acc = f2_fma(d23, d23, acc);
    }
  } else if (kind == DK_MANHATTAN) {
    const unsigned long long absmask = 0x7FFFFFFF7FFFFFFFull;
#pragma unroll 4
    for (int q = 0; q < Dp / 4; ++q) {
      const ulonglong2 x = pa[q], y = pb[q];
      acc = f2_add(acc, f2_sub(x.x, y.x) & absmask);
      acc = f2_add(acc, f2_sub(x.y, y.y) & absmask);
    }
  } else {
#pragma unroll 4
    for (int q = 0; q < Dp / 4; ++q) {
      const ulonglong2 x = pa[q], y = pb[q];
      acc = f2_fma(x.x, y.x, acc);
      acc = f2_fma(x.y, y.y, acc);
    }
  }
  return f2_sum(acc);
}

}  // namespace joinc
}  // namespace rinnd
