// common.cuh -- shared device utilities for the B200 NN-Descent engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <float.h>

#include <atomic>
#include <stdexcept>
#include <string>

namespace rinnd {

// Distance kinds (include/rinnd.h RINND_DIST_*).
enum DistKind : int {
  DK_SQEUCLIDEAN = 0,
  DK_MANHATTAN = 1,
  DK_COSINE = 2,
  DK_ALT_COSINE = 3,
  DK_ALT_DOT = 4,
  DK_DIRECT_COSINE = 5,
  DK_INNER_PRODUCT = 6,
  DK_ALT_INNER_PRODUCT = 7,
  // the reference's other metrics (core/distance/{minkowski,angular,binary,hellinger}.rs),
  // evaluated per pair by the generic kernels
  DK_CHEBYSHEV = 8,
  DK_CANBERRA = 9,
  DK_BRAYCURTIS = 10,
  DK_CORRELATION = 11,
  DK_TRUE_ANGULAR = 12,
  DK_TSSS = 13,
  DK_HAMMING = 14,
  DK_JACCARD = 15,
  DK_DICE = 16,
  DK_MATCHING = 17,
  DK_KULSINSKI = 18,
  DK_ROGERSTANIMOTO = 19,
  DK_RUSSELLRAO = 20,
  DK_SOKALMICHENER = 21,
  DK_SOKALSNEATH = 22,
  DK_YULE = 23,
  DK_HELLINGER = 24,
  DK_JENSEN_SHANNON = 25,
  DK_SYMMETRIC_KL = 26,
  DK_COUNT = 27
};
constexpr int DK_FIRST_GENERIC = DK_CHEBYSHEV;

enum CorrKind : int { CK_NONE = 0, CK_SQRT = 1, CK_ALT_COSINE = 2, CK_ALT_IP = 3 };

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define RINND_CUDA(call)                                                                   \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      throw ::rinnd::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + \
                               __FILE__ + ":" + std::to_string(__LINE__) + ")");           \
  } while (0)

// Every kernel launch of this library is followed by RINND_LAUNCH_CHECK, which
// also counts it (rinnd_kernel_launches).
std::atomic<unsigned long long>& launch_counter();
#define RINND_LAUNCH_CHECK()               \
  do {                                     \
    ++::rinnd::launch_counter();           \
    RINND_CUDA(cudaGetLastError());        \
  } while (0)

// ---------------------------------------------------------------------------
// Order-preserving float <-> u32 map.  -0.0 is folded onto +0.0 so that the
// map agrees with IEEE comparison (the reference compares with `>=` on f32).
// NaN maps above +inf and is therefore never accepted by a push.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint32_t fkey(float f) {
  f = f + 0.0f;  // -0 -> +0
#ifdef __CUDA_ARCH__
  uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
#endif
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float fkey_inv(uint32_t k) {
  uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

constexpr uint32_t KEY_INF = 0xFF800000u;  // fkey(+inf)
constexpr uint32_t LO_EMPTY = 0xFFFFFFFFu;
constexpr uint64_t SLOT_EMPTY = ((uint64_t)KEY_INF << 32) | LO_EMPTY;  // (+inf, id -1)
constexpr uint64_t CAND_EMPTY = ~0ull;                                 // (prio max, id -1)

// Neighbor slot: hi = fkey(distance), lo = id | (is_new << 31); empty lo = 0xFFFFFFFF.
__host__ __device__ __forceinline__ uint64_t slot_pack(float d, int32_t id, int is_new) {
  return ((uint64_t)fkey(d) << 32) | (uint32_t)id | ((uint32_t)(is_new != 0) << 31);
}
__host__ __device__ __forceinline__ int32_t slot_id(uint64_t s) {
  uint32_t lo = (uint32_t)s;
  return lo == LO_EMPTY ? -1 : (int32_t)(lo & 0x7FFFFFFFu);
}
__host__ __device__ __forceinline__ int slot_new(uint64_t s) {
  uint32_t lo = (uint32_t)s;
  return lo == LO_EMPTY ? 0 : (int)(lo >> 31);
}
__host__ __device__ __forceinline__ float slot_dist(uint64_t s) { return fkey_inv((uint32_t)(s >> 32)); }

// ---------------------------------------------------------------------------
// Counter-based randomness (SplitMix64 finalizer).  Streams are keyed by
// (seed, purpose, coordinates) so every kernel is deterministic for a seed and
// independent of scheduling order.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t hash3(uint64_t seed, uint64_t a, uint64_t b) {
  return mix64(mix64(seed ^ mix64(a)) ^ b);
}

__host__ __device__ __forceinline__ int round_up(int x, int m) { return (x + m - 1) / m * m; }

}  // namespace rinnd
