// dist.cuh -- per-pair distance functions.
//
// The `exact_*` functions reproduce the reference's AVX2+FMA code path
// bit-for-bit: eight (or 4x8) FMA lanes over chunks of 8 (or 32) elements, the
// same horizontal-sum tree, and a separately rounded multiply-add remainder
// (__fmul_rn/__fadd_rn prevent contraction).  They are used wherever an
// individual distance decides a comparison the reference makes: the pair
// distance kernel, RNG-style diversification, tree margins and graph search.
//
// References (core/ = crates/rinnd-core/src/):
//   sqeuclidean core/distance/euclidean.rs:66-110
//   manhattan   core/distance/minkowski.rs:57-83
//   cosine      core/distance/cosine.rs:41-80
//   alt cosine  core/distance/alternatives.rs:207-226
//   alt dot / direct normalized cosine  alternatives.rs:38-150 (normalized_dot_avx2)
//   inner product  core/distance/inner_product.rs:61-101
//   alt inner product  alternatives.rs:163-187
#pragma once
#include "common.cuh"

namespace rinnd {

// euclidean.rs:95-110 hsum256_ps_avx
__device__ __forceinline__ float hsum_a(const float* s) {
  float a0 = __fadd_rn(s[4], s[0]), a1 = __fadd_rn(s[5], s[1]);
  float a2 = __fadd_rn(s[6], s[2]), a3 = __fadd_rn(s[7], s[3]);
  return __fadd_rn(__fadd_rn(a0, a1), __fadd_rn(a2, a3));
}
// alternatives.rs:92-103 horizontal_sum_avx
__device__ __forceinline__ float hsum_b(const float* s) {
  float a0 = __fadd_rn(s[0], s[4]), a1 = __fadd_rn(s[1], s[5]);
  float a2 = __fadd_rn(s[2], s[6]), a3 = __fadd_rn(s[3], s[7]);
  return __fadd_rn(__fadd_rn(a0, a2), __fadd_rn(a1, a3));
}

// Packed FP32x2 arithmetic: each 32-bit half is computed and rounded exactly
// as the scalar instruction (sub.rn / add.rn / fma.rn), so a pair of
// independent accumulator chains advances in one instruction with the same
// results.  Element 2t of a chunk is the low half of 64-bit word t.
__device__ __forceinline__ unsigned long long pk_sub(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long pk_add(unsigned long long a, unsigned long long b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ unsigned long long pk_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
// A chunk of 8 as four packed pairs: rows are 16-byte aligned (the row stride
// is a multiple of 4 floats), so a chunk is two 16-byte loads.
__device__ __forceinline__ void load8p(const float* p, unsigned long long* v) {
  const ulonglong2 x = *reinterpret_cast<const ulonglong2*>(p);
  const ulonglong2 y = *reinterpret_cast<const ulonglong2*>(p + 4);
  v[0] = x.x; v[1] = x.y; v[2] = y.x; v[3] = y.y;
}
// Packed accumulators back to the eight chains s[0..7].
__device__ __forceinline__ void unpack8(const unsigned long long* p, float* s) {
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    s[2 * t] = __uint_as_float((uint32_t)p[t]);
    s[2 * t + 1] = __uint_as_float((uint32_t)(p[t] >> 32));
  }
}


__device__ __forceinline__ float exact_sqeuclid(const float* a, const float* b, int n) {
  unsigned long long p[4] = {0ull, 0ull, 0ull, 0ull};  // chains (0,1) (2,3) (4,5) (6,7)
  int chunks = n >> 3;
  for (int c = 0; c < chunks; ++c) {
    unsigned long long x[4], y[4];
    load8p(a + 8 * c, x);
    load8p(b + 8 * c, y);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const unsigned long long d = pk_sub(x[t], y[t]);
      p[t] = pk_fma(d, d, p[t]);
    }
  }
  float s[8];
  unpack8(p, s);
  float r = hsum_a(s);
  for (int i = chunks * 8; i < n; ++i) {
    float d = __fsub_rn(a[i], b[i]);
    r = __fadd_rn(r, __fmul_rn(d, d));
  }
  return r;
}

__device__ __forceinline__ float exact_manhattan(const float* a, const float* b, int n) {
  unsigned long long p[4] = {0ull, 0ull, 0ull, 0ull};
  int chunks = n >> 3;
  for (int c = 0; c < chunks; ++c) {
    unsigned long long x[4], y[4];
    load8p(a + 8 * c, x);
    load8p(b + 8 * c, y);
#pragma unroll
    for (int t = 0; t < 4; ++t) p[t] = pk_add(p[t], pk_sub(x[t], y[t]) & 0x7FFFFFFF7FFFFFFFull);
  }
  float s[8];
  unpack8(p, s);
  float r = hsum_a(s);
  for (int i = chunks * 8; i < n; ++i) r = __fadd_rn(r, fabsf(__fsub_rn(a[i], b[i])));
  return r;
}

__device__ __forceinline__ float exact_dot_a(const float* a, const float* b, int n) {
  unsigned long long p[4] = {0ull, 0ull, 0ull, 0ull};
  int chunks = n >> 3;
  for (int c = 0; c < chunks; ++c) {
    unsigned long long x[4], y[4];
    load8p(a + 8 * c, x);
    load8p(b + 8 * c, y);
#pragma unroll
    for (int t = 0; t < 4; ++t) p[t] = pk_fma(x[t], y[t], p[t]);
  }
  float s[8];
  unpack8(p, s);
  float r = hsum_a(s);
  for (int i = chunks * 8; i < n; ++i) r = __fadd_rn(r, __fmul_rn(a[i], b[i]));
  return r;
}

__device__ __forceinline__ float exact_dot_b(const float* a, const float* b, int n) {
  // four sets of eight chains, advanced in packed pairs
  unsigned long long q[4][4] = {{0ull, 0ull, 0ull, 0ull}, {0ull, 0ull, 0ull, 0ull},
                                {0ull, 0ull, 0ull, 0ull}, {0ull, 0ull, 0ull, 0ull}};
  int chunks = n >> 5;
  for (int c = 0; c < chunks; ++c) {
    const float* pa = a + 32 * c;
    const float* pb = b + 32 * c;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      unsigned long long x[4], y[4];
      load8p(pa + 8 * g, x);
      load8p(pb + 8 * g, y);
#pragma unroll
      for (int t = 0; t < 4; ++t) q[g][t] = pk_fma(x[t], y[t], q[g][t]);
    }
  }
  float t0[8], t1[8], t2[8], t3[8];
  unpack8(q[0], t0);
  unpack8(q[1], t1);
  unpack8(q[2], t2);
  unpack8(q[3], t3);
  float s[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) s[l] = __fadd_rn(__fadd_rn(t0[l], t1[l]), __fadd_rn(t2[l], t3[l]));
  float r = hsum_b(s);
  for (int i = chunks * 32; i < n; ++i) r = __fadd_rn(r, __fmul_rn(a[i], b[i]));
  return r;
}

__device__ __forceinline__ float exact_dot_c(const float* a, const float* b, int n) {
  float dot = 0.f;
  int chunks = n >> 2;
  for (int c = 0; c < chunks; ++c) {
    float4 x = *reinterpret_cast<const float4*>(a + 4 * c);
    float4 y = *reinterpret_cast<const float4*>(b + 4 * c);
    float p = __fmul_rn(x.x, y.x);
    p = __fadd_rn(p, __fmul_rn(x.y, y.y));
    p = __fadd_rn(p, __fmul_rn(x.z, y.z));
    p = __fadd_rn(p, __fmul_rn(x.w, y.w));
    dot = __fadd_rn(dot, p);
  }
  for (int i = chunks * 4; i < n; ++i) dot = __fadd_rn(dot, __fmul_rn(a[i], b[i]));
  return dot;
}

__device__ __forceinline__ float exact_cosine(const float* a, const float* b, int n) {
  unsigned long long pd[4] = {0ull, 0ull, 0ull, 0ull}, pa[4] = {0ull, 0ull, 0ull, 0ull};
  unsigned long long pb[4] = {0ull, 0ull, 0ull, 0ull};
  int chunks = n >> 3;
  for (int c = 0; c < chunks; ++c) {
    unsigned long long x[4], y[4];
    load8p(a + 8 * c, x);
    load8p(b + 8 * c, y);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      pd[t] = pk_fma(x[t], y[t], pd[t]);
      pa[t] = pk_fma(x[t], x[t], pa[t]);
      pb[t] = pk_fma(y[t], y[t], pb[t]);
    }
  }
  float sd[8], sa[8], sb[8];
  unpack8(pd, sd);
  unpack8(pa, sa);
  unpack8(pb, sb);
  float dot = hsum_a(sd), na = hsum_a(sa), nb = hsum_a(sb);
  for (int i = chunks * 8; i < n; ++i) {
    dot = __fadd_rn(dot, __fmul_rn(a[i], b[i]));
    na = __fadd_rn(na, __fmul_rn(a[i], a[i]));
    nb = __fadd_rn(nb, __fmul_rn(b[i], b[i]));
  }
  float denom = __fsqrt_rn(__fmul_rn(na, nb));
  if (denom < 1e-12f) return 1.0f;
  float sim = fminf(fmaxf(__fdiv_rn(dot, denom), -1.0f), 1.0f);
  return __fsub_rn(1.0f, sim);
}

__device__ __forceinline__ float exact_alt_cosine(const float* a, const float* b, int n) {
  float dot = 0.f, na = 0.f, nb = 0.f;
  for (int i = 0; i < n; ++i) {
    dot = __fadd_rn(dot, __fmul_rn(a[i], b[i]));
    na = __fadd_rn(na, __fmul_rn(a[i], a[i]));
    nb = __fadd_rn(nb, __fmul_rn(b[i], b[i]));
  }
  if (na == 0.f && nb == 0.f) return 0.f;
  if (na == 0.f || nb == 0.f) return FLT_MAX;
  if (dot <= 0.f) return FLT_MAX;
  return log2f(__fdiv_rn(__fsqrt_rn(__fmul_rn(na, nb)), dot));
}

// ---- the reference's other metrics: scalar loops in the reference's order, every
// operation separately rounded (Rust does not fuse a multiply and an add) ----
// core/distance/binary.rs: counts of (a != 0, b != 0) combinations as f32 sums.
struct BinCounts {
  float tt, tf, ft, ne;
};
__device__ __forceinline__ BinCounts binary_counts(const float* a, const float* b, int n) {
  BinCounts c{0.f, 0.f, 0.f, 0.f};
  for (int i = 0; i < n; ++i) {
    const bool x = a[i] != 0.f, y = b[i] != 0.f;
    if (x && y) c.tt = __fadd_rn(c.tt, 1.0f);
    if (x && !y) c.tf = __fadd_rn(c.tf, 1.0f);
    if (!x && y) c.ft = __fadd_rn(c.ft, 1.0f);
    if (x != y) c.ne = __fadd_rn(c.ne, 1.0f);
  }
  return c;
}

static __device__ __noinline__ float generic_distance(int kind, const float* a, const float* b, int n) {
  const float nf = (float)n;
  switch (kind) {
    case DK_CHEBYSHEV: {  // minkowski.rs:106-121
      float r = 0.f;
      for (int i = 0; i < n; ++i) {
        const float d = fabsf(__fsub_rn(a[i], b[i]));
        if (d > r) r = d;
      }
      return r;
    }
    case DK_CANBERRA: {  // minkowski.rs:165-181
      float s = 0.f;
      for (int i = 0; i < n; ++i) {
        const float den = __fadd_rn(fabsf(a[i]), fabsf(b[i]));
        if (den > 0.f) s = __fadd_rn(s, __fdiv_rn(fabsf(__fsub_rn(a[i], b[i])), den));
      }
      return s;
    }
    case DK_BRAYCURTIS: {  // minkowski.rs:191-212
      float num = 0.f, den = 0.f;
      for (int i = 0; i < n; ++i) {
        num = __fadd_rn(num, fabsf(__fsub_rn(a[i], b[i])));
        den = __fadd_rn(den, fabsf(__fadd_rn(a[i], b[i])));
      }
      return den > 0.f ? __fdiv_rn(num, den) : 0.f;
    }
    case DK_CORRELATION: {  // angular.rs:13-52
      if (n == 0) return 0.f;
      float ma = 0.f, mb = 0.f;
      for (int i = 0; i < n; ++i) {
        ma = __fadd_rn(ma, a[i]);
        mb = __fadd_rn(mb, b[i]);
      }
      ma = __fdiv_rn(ma, nf);
      mb = __fdiv_rn(mb, nf);
      float dot = 0.f, na = 0.f, nb = 0.f;
      for (int i = 0; i < n; ++i) {
        const float sa = __fsub_rn(a[i], ma), sb = __fsub_rn(b[i], mb);
        dot = __fadd_rn(dot, __fmul_rn(sa, sb));
        na = __fadd_rn(na, __fmul_rn(sa, sa));
        nb = __fadd_rn(nb, __fmul_rn(sb, sb));
      }
      if (na == 0.f && nb == 0.f) return 0.f;
      if (dot == 0.f) return 1.0f;
      return __fsub_rn(1.0f, __fdiv_rn(dot, __fsqrt_rn(__fmul_rn(na, nb))));
    }
    case DK_TRUE_ANGULAR:  // angular.rs:62-90
    case DK_TSSS: {        // angular.rs:99-133
      float de = 0.f, dot = 0.f, na = 0.f, nb = 0.f;
      for (int i = 0; i < n; ++i) {
        const float d = __fsub_rn(a[i], b[i]);
        de = __fadd_rn(de, __fmul_rn(d, d));
        dot = __fadd_rn(dot, __fmul_rn(a[i], b[i]));
        na = __fadd_rn(na, __fmul_rn(a[i], a[i]));
        nb = __fadd_rn(nb, __fmul_rn(b[i], b[i]));
      }
      if (kind == DK_TRUE_ANGULAR) {
        if (na == 0.f && nb == 0.f) return 0.f;
        if (na == 0.f || nb == 0.f || dot <= 0.f) return FLT_MAX;
        const float sim = fminf(fmaxf(__fdiv_rn(dot, __fsqrt_rn(__fmul_rn(na, nb))), -1.0f), 1.0f);
        return __fsub_rn(1.0f, __fdiv_rn(acosf(sim), 3.14159265358979f));
      }
      na = __fsqrt_rn(na);
      nb = __fsqrt_rn(nb);
      const float mag = fabsf(__fsub_rn(na, nb));
      const float den = __fmul_rn(na, nb);
      if (den < 1e-12f) return 0.f;
      const float cs = fminf(fmaxf(__fdiv_rn(dot, den), -1.0f), 1.0f);
      // + 10 degrees in radians: 10 * (pi / 180) in f32 arithmetic (f32::to_radians)
      const float theta = __fadd_rn(acosf(cs), __fmul_rn(10.0f, __fdiv_rn(3.14159265358979f, 180.0f)));
      const float t = __fadd_rn(__fsqrt_rn(de), mag);
      const float sector = __fmul_rn(__fmul_rn(t, t), theta);
      const float triangle = __fdiv_rn(__fmul_rn(den, sinf(theta)), 2.0f);
      return __fmul_rn(triangle, sector);
    }
    case DK_HAMMING: {  // binary.rs:13-32
      if (n == 0) return 0.f;
      unsigned cnt = 0;
      for (int i = 0; i < n; ++i) cnt += a[i] != b[i];
      return __fdiv_rn((float)cnt, nf);
    }
    case DK_MATCHING: {  // binary.rs:113-132
      if (n == 0) return 0.f;
      unsigned cnt = 0;
      for (int i = 0; i < n; ++i) cnt += (a[i] != 0.f) != (b[i] != 0.f);
      return __fdiv_rn((float)cnt, nf);
    }
    case DK_RUSSELLRAO: {  // binary.rs:239-258
      if (n == 0) return 0.f;
      const BinCounts c = binary_counts(a, b, n);
      return __fdiv_rn(__fsub_rn(nf, c.tt), nf);
    }
    case DK_JACCARD:
    case DK_DICE:
    case DK_KULSINSKI:
    case DK_ROGERSTANIMOTO:
    case DK_SOKALMICHENER:
    case DK_SOKALSNEATH:
    case DK_YULE: {
      const BinCounts c = binary_counts(a, b, n);
      switch (kind) {
        case DK_JACCARD: {  // binary.rs:42-68 (non-zero in either = tt + ne, exact integer counts)
          const float nnz = __fadd_rn(c.tt, c.ne);
          return nnz == 0.f ? 0.f : __fdiv_rn(__fsub_rn(nnz, c.tt), nnz);
        }
        case DK_DICE:  // binary.rs:142-167
          return c.ne == 0.f ? 0.f : __fdiv_rn(c.ne, __fadd_rn(__fmul_rn(2.0f, c.tt), c.ne));
        case DK_KULSINSKI:  // binary.rs:177-203
          return c.ne == 0.f ? 0.f : __fdiv_rn(__fadd_rn(__fsub_rn(c.ne, c.tt), nf), __fadd_rn(c.ne, nf));
        case DK_SOKALSNEATH:  // binary.rs:286-311
          return c.ne == 0.f ? 0.f : __fdiv_rn(c.ne, __fadd_rn(__fmul_rn(0.5f, c.tt), c.ne));
        case DK_YULE: {  // binary.rs:321-353
          const float ff = __fsub_rn(__fsub_rn(__fsub_rn(nf, c.tt), c.tf), c.ft);
          if (c.tf == 0.f || c.ft == 0.f) return 0.f;
          return __fdiv_rn(__fmul_rn(__fmul_rn(2.0f, c.tf), c.ft),
                           __fadd_rn(__fmul_rn(c.tt, ff), __fmul_rn(c.tf, c.ft)));
        }
        default:  // rogerstanimoto, binary.rs:213-229; sokalmichener is the same, :268-276
          return __fdiv_rn(__fmul_rn(2.0f, c.ne), __fadd_rn(nf, c.ne));
      }
    }
    case DK_HELLINGER: {  // hellinger.rs:16-44
      float bc = 0.f, la = 0.f, lb = 0.f;
      for (int i = 0; i < n; ++i) {
        bc = __fadd_rn(bc, __fsqrt_rn(__fmul_rn(a[i], b[i])));
        la = __fadd_rn(la, a[i]);
        lb = __fadd_rn(lb, b[i]);
      }
      if (la == 0.f && lb == 0.f) return 0.f;
      if (la == 0.f || lb == 0.f) return 1.0f;
      const float v = __fsub_rn(1.0f, __fdiv_rn(bc, __fsqrt_rn(__fmul_rn(la, lb))));
      return __fsqrt_rn(fmaxf(v, 0.f));
    }
    case DK_JENSEN_SHANNON:  // hellinger.rs:98-128
    case DK_SYMMETRIC_KL: {  // hellinger.rs:137-166
      float la = 0.f, lb = 0.f;
      for (int i = 0; i < n; ++i) {
        la = __fadd_rn(la, a[i]);
        lb = __fadd_rn(lb, b[i]);
      }
      const float et = __fmul_rn(FLT_EPSILON, nf);
      la = __fadd_rn(la, et);
      lb = __fadd_rn(lb, et);
      float r = 0.f;
      for (int i = 0; i < n; ++i) {
        const float px = __fdiv_rn(__fadd_rn(a[i], FLT_EPSILON), la);
        const float py = __fdiv_rn(__fadd_rn(b[i], FLT_EPSILON), lb);
        if (kind == DK_JENSEN_SHANNON) {
          const float m = __fmul_rn(0.5f, __fadd_rn(px, py));
          const float t = __fadd_rn(__fmul_rn(px, logf(__fdiv_rn(px, m))), __fmul_rn(py, logf(__fdiv_rn(py, m))));
          r = __fadd_rn(r, __fmul_rn(0.5f, t));
        } else {
          r = __fadd_rn(r, __fadd_rn(__fmul_rn(px, logf(__fdiv_rn(px, py))), __fmul_rn(py, logf(__fdiv_rn(py, px)))));
        }
      }
      return r;
    }
  }
  return __int_as_float(0x7fc00000);
}

// Dispatch.  `n` is the true dimension; rows may be padded beyond it.
__device__ __forceinline__ float exact_distance(int kind, const float* a, const float* b, int n) {
  if (kind >= DK_FIRST_GENERIC) return generic_distance(kind, a, b, n);
  switch (kind) {
    case DK_SQEUCLIDEAN: return exact_sqeuclid(a, b, n);
    case DK_MANHATTAN: return exact_manhattan(a, b, n);
    case DK_COSINE: return exact_cosine(a, b, n);
    case DK_ALT_COSINE: return exact_alt_cosine(a, b, n);
    case DK_ALT_DOT: {
      float dot = exact_dot_b(a, b, n);
      return dot <= 0.f ? FLT_MAX : -log2f(dot);
    }
    case DK_DIRECT_COSINE: {
      float dot = exact_dot_b(a, b, n);
      return __fsub_rn(1.0f, fminf(fmaxf(dot, -1.0f), 1.0f));
    }
    case DK_INNER_PRODUCT: return -exact_dot_a(a, b, n);
    case DK_ALT_INNER_PRODUCT: {
      float dot = exact_dot_c(a, b, n);
      return dot <= 0.f ? FLT_MAX : __fdiv_rn(1.0f, dot);
    }
  }
  return __int_as_float(0x7fc00000);
}

// Metrics evaluated from (dot, |a|^2, |b|^2) in the tiled join kernels.
__host__ __device__ __forceinline__ bool kind_is_dot(int kind) {
  return kind != DK_SQEUCLIDEAN && kind != DK_MANHATTAN && kind < DK_FIRST_GENERIC;
}
// Metrics the tiled joins do not evaluate (the generic per-pair kernels do).
__host__ __device__ __forceinline__ bool kind_is_generic(int kind) { return kind >= DK_FIRST_GENERIC; }
__device__ __forceinline__ float finalize_dot(int kind, float dot, float na, float nb) {
  switch (kind) {
    case DK_COSINE: {
      float denom = sqrtf(na * nb);
      if (denom < 1e-12f) return 1.0f;
      return 1.0f - fminf(fmaxf(dot / denom, -1.0f), 1.0f);
    }
    case DK_ALT_COSINE:
      if (na == 0.f && nb == 0.f) return 0.f;
      if (na == 0.f || nb == 0.f || dot <= 0.f) return FLT_MAX;
      return log2f(sqrtf(na * nb) / dot);
    case DK_ALT_DOT: return dot <= 0.f ? FLT_MAX : -log2f(dot);
    case DK_DIRECT_COSINE: return 1.0f - fminf(fmaxf(dot, -1.0f), 1.0f);
    case DK_INNER_PRODUCT: return -dot;
    case DK_ALT_INNER_PRODUCT: return dot <= 0.f ? FLT_MAX : 1.0f / dot;
  }
  return dot;
}

// alternatives.rs:273-287, index.rs:587
__host__ __device__ __forceinline__ float apply_correction(int corr, float d) {
  switch (corr) {
    case CK_SQRT: return sqrtf(d);
    case CK_ALT_COSINE: return 1.0f - exp2f(-d);
    case CK_ALT_IP: return d >= FLT_MAX ? 0.0f : -1.0f / d;
  }
  return d;
}

}  // namespace rinnd
