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
// Per-dimension symmetric codes (encoding 3), the operand format of the
// reference's quantized_i8_per_dimension_dot (core/distance/quantized.rs:42-56),
// which has no production encoder there: scale_j = max_i |x_ij| / 127 over the
// index rows (0 for a zero column), code = clamp(round_half_away(x / scale_j),
// -127, 127), 0 where scale_j = 0; queries use the index's scales.
// Each product, quotient and square root is a single IEEE round-to-nearest
// operation as in the reference; maxima and integer sums are order-free, so
// the codes and scales are identical to the reference's.  A NaN product
// becomes code 0 (the reference's saturating float-to-int cast).
#include <algorithm>
#include <cstring>
#include <stdexcept>

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

// Column maxima of |x| over rows [blockIdx.y-th chunk): one thread per column.
__global__ void k_colmax(const float* __restrict__ X, long long n, int D, int Dp, long long rows_per_block,
                         unsigned int* colmax) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D) return;
  const long long r0 = blockIdx.y * rows_per_block, r1 = min(n, r0 + rows_per_block);
  float m = 0.f;
  for (long long r = r0; r < r1; ++r) m = fmaxf(m, fabsf(X[r * Dp + j]));
  atomicMax(colmax + j, __float_as_uint(m));  // non-negative floats order like their bits
}

__global__ void k_dim_scales(const unsigned int* colmax, int D, int Dq, float* dim_scales) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= Dq) return;
  const float m = j < D ? __uint_as_float(colmax[j]) : 0.f;
  dim_scales[j] = m > 0.f ? __fdiv_rn(m, 127.0f) : 0.f;
}

// Per-dimension codes: one thread per element.
__global__ void k_quantize_dims(const float* __restrict__ X, long long n, int D, int Dp, int Dq,
                                const float* __restrict__ dim_scales, int8_t* __restrict__ codes) {
  const long long total = n * Dq;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / Dq;
    const int j = (int)(e - r * Dq);
    int c = 0;
    if (j < D) {
      const float sc = dim_scales[j];
      if (sc > 0.f) {
        const float v = roundf(__fdiv_rn(X[r * Dp + j], sc));
        if (v == v) c = (int)fminf(fmaxf(v, -127.0f), 127.0f);
      }
    }
    codes[e] = (int8_t)c;
  }
}

// QuantizedFlatTree::quantize_hyperplanes (flat_tree.rs:47-64), one warp per
// node: scale = max|h| / 127 (0 for a zero hyperplane, leaves included), code =
// clamp(round_half_away(h / scale), -127, 127); codes of Dq bytes, zero beyond D.
__global__ void k_quantize_tree(const float* __restrict__ H, long long n_nodes, int D, int Dp, int Dq,
                                int8_t* __restrict__ codes, float* __restrict__ scales) {
  const long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n_nodes) return;
  const float* h = H + r * Dp;
  float mx = 0.f;
  for (int j = lane; j < D; j += 32) mx = fmaxf(mx, fabsf(h[j]));
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  const float sc = mx > 0.f ? __fdiv_rn(mx, 127.0f) : 0.f;
  for (int j = lane; j < Dq; j += 32) {
    int c = 0;
    if (j < D && sc > 0.f) {
      const float v = roundf(__fdiv_rn(h[j], sc));
      if (v == v) c = (int)fminf(fmaxf(v, -127.0f), 127.0f);
    }
    codes[r * Dq + j] = (int8_t)c;
  }
  if (lane == 0) scales[r] = sc;
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

void quantize_tree_hyperplanes(const float* H, long long n_nodes, int D, int Dp, int Dq, int8_t* codes, float* scales,
                               cudaStream_t st) {
  if (n_nodes <= 0) return;
  k_quantize_tree<<<grid_for(n_nodes * 32, 256), 256, 0, st>>>(H, n_nodes, D, Dp, Dq, codes, scales);
  RINND_LAUNCH_CHECK();
}

void quant_dim_scales(const float* X, long long n, int D, int Dp, int Dq, float* dim_scales, cudaStream_t st) {
  DVec<unsigned int> colmax((size_t)std::max(D, 1), st);
  colmax.fill_bytes(0);
  if (n > 0) {
    const long long rpb = std::max<long long>(64, (n + 2047) / 2048);
    const dim3 grid((unsigned)((D + 127) / 128), (unsigned)((n + rpb - 1) / rpb));
    k_colmax<<<grid, 128, 0, st>>>(X, n, D, Dp, rpb, colmax.p);
    RINND_LAUNCH_CHECK();
  }
  k_dim_scales<<<(Dq + 127) / 128, 128, 0, st>>>(colmax.p, D, Dq, dim_scales);
  RINND_LAUNCH_CHECK();
}

void quantize_rows(const float* X, long long n, int D, int Dp, int Dq, int encoding, float gmult,
                   const float* dim_scales, int8_t* codes, float* scale, cudaStream_t st) {
  if (n <= 0) return;
  if (encoding == Q8_PER_DIMENSION) {
    if (!dim_scales) throw std::invalid_argument("per-dimension codes need the per-dimension scales");
    k_quantize_dims<<<grid_for(n * Dq, 256, 148 * 32), 256, 0, st>>>(X, n, D, Dp, Dq, dim_scales, codes);
    RINND_LAUNCH_CHECK();
    return;
  }
  const float gscale = gmult > 0.f ? 1.0f / gmult : 0.f;  // lib.rs:175-179
  k_quantize<<<grid_for(n * 32, 256), 256, 0, st>>>(X, n, D, Dp, Dq, encoding, gmult, gscale, codes, scale);
  RINND_LAUNCH_CHECK();
}

}  // namespace rinnd
