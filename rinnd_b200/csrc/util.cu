// util.cu -- row layout, pair distances, permutations, corrections.
#include "dist.cuh"
#include "engine.h"

namespace rinnd {
namespace {

__global__ void k_distance_pairs(int kind, const float* A, const float* B, long long n, int D, int Dp,
                                 float* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = exact_distance(kind, A + (size_t)i * Dp, B + (size_t)i * Dp, D);
}

__global__ void k_pad_rows(const float* src, long long n, int D, int Dp, float* dst) {
  long long total = n * Dp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e / Dp;
    int c = (int)(e % Dp);
    dst[e] = c < D ? src[r * D + c] : 0.f;
  }
}

__global__ void k_gather_rows(const float4* src, const int32_t* order, long long n, int q4,
                              float4* dst) {
  long long total = n * q4;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    long long r = e / q4;
    int c = (int)(e % q4);
    dst[e] = src[(size_t)order[r] * q4 + c];
  }
}

// crates/rinnd/src/lib.rs normalize_rows_inplace: sequential f32 sum of squares,
// rows with norm_sq <= 1e-12 untouched, x *= 1/sqrt(norm_sq).
__global__ void k_normalize_rows(float* X, long long n, int D, int Dp) {
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    float* x = X + (size_t)r * Dp;
    float s = 0.f;
    for (int i = 0; i < D; ++i) s = __fadd_rn(s, __fmul_rn(x[i], x[i]));
    if (s <= 1e-12f) continue;
    float inv = __frcp_rn(__fsqrt_rn(s));
    for (int i = 0; i < D; ++i) x[i] = __fmul_rn(x[i], inv);
  }
}

__global__ void k_invert(const int32_t* order, int N, int32_t* inv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) inv[order[i]] = i;
}

__global__ void k_correct(float* d, long long n, int corr) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    d[i] = apply_correction(corr, d[i]);
}

}  // namespace

void distance_pairs(int kind, const float* A, const float* B, int64_t n, int D, int Dp, float* out,
                    cudaStream_t st) {
  k_distance_pairs<<<grid_for(n, 128, 148 * 64), 128, 0, st>>>(kind, A, B, n, D, Dp, out);
  RINND_LAUNCH_CHECK();
}

void pad_rows(const float* src, int64_t n, int D, int Dp, float* dst, cudaStream_t st) {
  if (D == Dp) {
    RINND_CUDA(cudaMemcpyAsync(dst, src, sizeof(float) * (size_t)n * D, cudaMemcpyDeviceToDevice, st));
    return;
  }
  k_pad_rows<<<grid_for(n * Dp, 256, 148 * 64), 256, 0, st>>>(src, n, D, Dp, dst);
  RINND_LAUNCH_CHECK();
}

void gather_rows(const float* src, const int32_t* order, int64_t n, int Dp, float* dst,
                 cudaStream_t st) {
  int q4 = Dp / 4;
  k_gather_rows<<<grid_for(n * q4, 256, 148 * 64), 256, 0, st>>>(
      reinterpret_cast<const float4*>(src), order, n, q4, reinterpret_cast<float4*>(dst));
  RINND_LAUNCH_CHECK();
}

void normalize_rows(float* X, int64_t n, int D, int Dp, cudaStream_t st) {
  k_normalize_rows<<<grid_for(n, 128, 148 * 64), 128, 0, st>>>(X, n, D, Dp);
  RINND_LAUNCH_CHECK();
}

void invert_permutation(const int32_t* order, int N, int32_t* inverse, cudaStream_t st) {
  k_invert<<<grid_for(N, 256), 256, 0, st>>>(order, N, inverse);
  RINND_LAUNCH_CHECK();
}

void apply_correction_dev(float* d, int64_t n, int corr, cudaStream_t st) {
  if (corr == CK_NONE || n == 0) return;
  k_correct<<<grid_for(n, 256, 148 * 64), 256, 0, st>>>(d, n, corr);
  RINND_LAUNCH_CHECK();
}

}  // namespace rinnd
