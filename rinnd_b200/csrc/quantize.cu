// quantize.cu -- int8 scalar quantization of index rows and queries.
//
// Restates QuantizedI8Index::new (crates/rinnd/src/lib.rs:159-223) and
// quantize_query (lib.rs:325-358) bit for bit:
//   multiplier = 127 / max|x| of the row (per-vector encodings) or of all rows
//                (sq8u global symmetric), 0 when the max is 0;
//   code       = clamp(round_half_away(x * multiplier), -127, 127);
//   scale      = 1 / sqrt(sum code^2)  (int8 per-vector cosine, 0 if the sum is 0),
//                1 / multiplier        (sq8p per-vector symmetric, 0 if 0),
//                1 / global multiplier (sq8u).
// Each product, quotient and square root is a single IEEE round-to-nearest
// operation as in the reference; maxima and integer sums are order-free, so
// the codes and scales are identical to the reference's.  A NaN product
// becomes code 0 (the reference's saturating float-to-int cast).
#include <cstring>

#include "engine.h"

namespace rinnd {
namespace {

__global__ void k_absmax(const float* __restrict__ X, long long total, unsigned int* out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(X[i]));
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  // non-negative floats order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// One warp per row; rows of `Dp` floats (first D used), codes of Dq bytes
// (zero beyond D).
__global__ void k_quantize(const float* __restrict__ X, long long n, int D, int Dp, int Dq, int encoding,
                           float gmult, float gscale, int8_t* __restrict__ codes, float* __restrict__ scale) {
  const long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const float* row = X + r * Dp;
  float mult = gmult;
  if (encoding != Q8_GLOBAL_SYMMETRIC) {
    float mx = 0.f;
    for (int j = lane; j < D; j += 32) mx = fmaxf(mx, fabsf(row[j]));
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mult = mx > 0.f ? __fdiv_rn(127.0f, mx) : 0.f;
  }
  int nsq = 0;
  int8_t* out = codes + r * Dq;
  for (int j = lane; j < Dq; j += 32) {
    int c = 0;
    if (j < D) {
      const float v = roundf(__fmul_rn(row[j], mult));
      if (v == v) c = (int)fminf(fmaxf(v, -127.0f), 127.0f);
    }
    out[j] = (int8_t)c;
    nsq += c * c;
  }
  for (int o = 16; o; o >>= 1) nsq += __shfl_xor_sync(0xffffffffu, nsq, o);
  if (lane == 0) {
    float s;
    if (encoding == Q8_PER_VECTOR_COSINE) s = nsq > 0 ? __frcp_rn(__fsqrt_rn((float)nsq)) : 0.f;
    else if (encoding == Q8_PER_VECTOR_SYMMETRIC) s = mult > 0.f ? __frcp_rn(mult) : 0.f;
    else s = gscale;
    scale[r] = s;
  }
}

}  // namespace

float quant_global_multiplier(const float* X, long long total, cudaStream_t st) {
  DVec<unsigned int> m(1, st);
  m.fill_bytes(0);
  k_absmax<<<grid_for(total, 256, 148 * 8), 256, 0, st>>>(X, total, m.p);
  RINND_LAUNCH_CHECK();
  unsigned int h = 0;
  m.to_host(&h, 1);
  RINND_CUDA(cudaStreamSynchronize(st));
  float gmax;
  std::memcpy(&gmax, &h, sizeof(gmax));
  return gmax > 0.f ? 127.0f / gmax : 0.f;  // lib.rs:170-174
}

void quantize_rows(const float* X, long long n, int D, int Dp, int Dq, int encoding, float gmult, int8_t* codes,
                   float* scale, cudaStream_t st) {
  if (n <= 0) return;
  const float gscale = gmult > 0.f ? 1.0f / gmult : 0.f;  // lib.rs:175-179
  k_quantize<<<grid_for(n * 32, 256), 256, 0, st>>>(X, n, D, Dp, Dq, encoding, gmult, gscale, codes, scale);
  RINND_LAUNCH_CHECK();
}

}  // namespace rinnd
