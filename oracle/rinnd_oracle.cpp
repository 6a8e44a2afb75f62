// rinnd_oracle.cpp -- TEST INFRASTRUCTURE ONLY (parity checker + timed CPU baseline).
//
// A C++17 restatement of lmcinnes/rinnd's CPU hot path: distances with the
// reference's AVX2 accumulation orders, the 3-component NeighborHeap, random
// candidate sampling, RP-forest construction, the NN-Descent driver, search-
// graph diversification/pruning, and greedy graph search (FP32 and int8).
// Parallel sections use OpenMP with the same owner-block partitioning as the
// reference's Rayon code, so results are deterministic for a given thread count.
//
// The reference is Rust and cannot be compiled in this environment (no cargo or
// rustc, no crates registry).  Its RNG comes from the third-party crates
// rand 0.8.5 / rand_core 0.6.4 / rand_xoshiro 0.6.0 (Cargo.lock); FastRng below
// restates their published algorithms (Xoshiro256++ seeded by SplitMix64,
// rand's f32/bool/range sampling).  No reference test pins an RNG stream, so the
// stream-level equality is unverified; the known-answer tests in
// tests/golden/reference_kats.json pin everything else this file computes.
//
// Paths in citations are relative to the reference root; "core/" means
// crates/rinnd-core/src/.  Build: oracle/Makefile (-O3 -mavx2 -mfma
// -ffp-contract=off -fopenmp): no mul+add is fused unless the reference fuses it.

#include "rinnd_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <utility>
#include <vector>
#include <chrono>
#include <cstdio>

#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__AVX2__) && defined(__FMA__)
#include <immintrin.h>
#define ORC_AVX2 1
#endif

namespace {

// ---------------------------------------------------------------------------
// RNG -- core/rng.rs:15-86 (FastRng = rand_xoshiro::Xoshiro256PlusPlus)
// ---------------------------------------------------------------------------
struct FastRng {
  uint64_t s[4];
  explicit FastRng(uint64_t seed) {
    // Xoshiro256PlusPlus::seed_from_u64: SplitMix64 fills the 4 state words.
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) {
      x += 0x9e3779b97f4a7c15ULL;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      s[i] = z ^ (z >> 31);
    }
  }
  static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
  // rng.rs:30-32 next_u64
  uint64_t next_u64() {
    uint64_t result = rotl(s[0] + s[3], 23) + s[0];
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
  }
  uint32_t next_u32() { return (uint32_t)(next_u64() >> 32); }
  // rng.rs:42-44: rand's Standard f32 = (u32 >> 8) * 2^-24
  float next_float() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
  // rng.rs:54-56: rand's Standard bool = sign bit of a u32
  bool next_bool() { return (int32_t)next_u32() < 0; }
  // rng.rs:48-50: gen_range(0..n), widening-multiply rejection sampling
  uint64_t next_index(uint64_t n) {
    uint64_t range = n;  // high - low + 1 with high = n - 1
    if (range == 0) return next_u64();
    int lz = __builtin_clzll(range);
    uint64_t zone = (range << lz) - 1;
    for (;;) {
      uint64_t v = next_u64();
      unsigned __int128 m = (unsigned __int128)v * (unsigned __int128)range;
      uint64_t hi = (uint64_t)(m >> 64), lo = (uint64_t)m;
      if (lo <= zone) return hi;
    }
  }
};

// ---------------------------------------------------------------------------
// Distances.  Each follows the reference's AVX2+FMA code path exactly (the
// path taken on x86 hosts with AVX2/FMA), including horizontal-sum order and
// the scalar remainder loop (separately rounded mul and add).
// ---------------------------------------------------------------------------

// core/distance/euclidean.rs:95-110 hsum256_ps_avx: ((s0+s4)+(s1+s5))+((s2+s6)+(s3+s7))
static inline float hsum_a(const float* s) {
  float a0 = s[4] + s[0], a1 = s[5] + s[1], a2 = s[6] + s[2], a3 = s[7] + s[3];
  return (a0 + a1) + (a2 + a3);
}
// core/distance/alternatives.rs:92-103 horizontal_sum_avx: ((s0+s4)+(s2+s6))+((s1+s5)+(s3+s7))
static inline float hsum_b(const float* s) {
  float a0 = s[0] + s[4], a1 = s[1] + s[5], a2 = s[2] + s[6], a3 = s[3] + s[7];
  return (a0 + a2) + (a1 + a3);
}

#ifdef ORC_AVX2
static inline void store8(__m256 v, float* out) { _mm256_storeu_ps(out, v); }
#endif

// core/distance/euclidean.rs:66-93 l2_sqr_avx2
static float sqeuclid(const float* a, const float* b, int n) {
  int chunks = n / 8;
  float s[8];
#ifdef ORC_AVX2
  __m256 sum = _mm256_setzero_ps();
  for (int i = 0; i < chunks; ++i) {
    __m256 d = _mm256_sub_ps(_mm256_loadu_ps(a + 8 * i), _mm256_loadu_ps(b + 8 * i));
    sum = _mm256_fmadd_ps(d, d, sum);
  }
  store8(sum, s);
#else
  for (int l = 0; l < 8; ++l) s[l] = 0.f;
  for (int i = 0; i < chunks; ++i)
    for (int l = 0; l < 8; ++l) {
      float d = a[8 * i + l] - b[8 * i + l];
      s[l] = std::fmaf(d, d, s[l]);
    }
#endif
  float r = hsum_a(s);
  for (int i = chunks * 8; i < n; ++i) {
    float d = a[i] - b[i];
    r += d * d;
  }
  return r;
}

// core/distance/minkowski.rs:57-83 manhattan_avx2 (abs via sign mask, plain add)
static float manhattan(const float* a, const float* b, int n) {
  int chunks = n / 8;
  float s[8];
#ifdef ORC_AVX2
  __m256 mask = _mm256_castsi256_ps(_mm256_set1_epi32(0x7FFFFFFF));
  __m256 sum = _mm256_setzero_ps();
  for (int i = 0; i < chunks; ++i) {
    __m256 d = _mm256_sub_ps(_mm256_loadu_ps(a + 8 * i), _mm256_loadu_ps(b + 8 * i));
    sum = _mm256_add_ps(sum, _mm256_and_ps(d, mask));
  }
  store8(sum, s);
#else
  for (int l = 0; l < 8; ++l) s[l] = 0.f;
  for (int i = 0; i < chunks; ++i)
    for (int l = 0; l < 8; ++l) s[l] = s[l] + std::fabs(a[8 * i + l] - b[8 * i + l]);
#endif
  float r = hsum_a(s);
  for (int i = chunks * 8; i < n; ++i) r += std::fabs(a[i] - b[i]);
  return r;
}

// core/distance/inner_product.rs:61-81 dot_avx2 (also tree/builder.rs:27-60)
static float dot_a(const float* a, const float* b, int n) {
  int chunks = n / 8;
  float s[8];
#ifdef ORC_AVX2
  __m256 sum = _mm256_setzero_ps();
  for (int i = 0; i < chunks; ++i)
    sum = _mm256_fmadd_ps(_mm256_loadu_ps(a + 8 * i), _mm256_loadu_ps(b + 8 * i), sum);
  store8(sum, s);
#else
  for (int l = 0; l < 8; ++l) s[l] = 0.f;
  for (int i = 0; i < chunks; ++i)
    for (int l = 0; l < 8; ++l) s[l] = std::fmaf(a[8 * i + l], b[8 * i + l], s[l]);
#endif
  float r = hsum_a(s);
  for (int i = chunks * 8; i < n; ++i) r += a[i] * b[i];
  return r;
}

// core/distance/alternatives.rs:53-90 normalized_dot_avx2 (4 x 8-lane accumulators)
static float dot_b(const float* a, const float* b, int n) {
  int chunks = n / 32;
  float s[8];
#ifdef ORC_AVX2
  __m256 s0 = _mm256_setzero_ps(), s1 = s0, s2 = s0, s3 = s0;
  for (int c = 0; c < chunks; ++c) {
    const float* pa = a + 32 * c;
    const float* pb = b + 32 * c;
    s0 = _mm256_fmadd_ps(_mm256_loadu_ps(pa), _mm256_loadu_ps(pb), s0);
    s1 = _mm256_fmadd_ps(_mm256_loadu_ps(pa + 8), _mm256_loadu_ps(pb + 8), s1);
    s2 = _mm256_fmadd_ps(_mm256_loadu_ps(pa + 16), _mm256_loadu_ps(pb + 16), s2);
    s3 = _mm256_fmadd_ps(_mm256_loadu_ps(pa + 24), _mm256_loadu_ps(pb + 24), s3);
  }
  store8(_mm256_add_ps(_mm256_add_ps(s0, s1), _mm256_add_ps(s2, s3)), s);
#else
  float t[4][8] = {};
  for (int c = 0; c < chunks; ++c)
    for (int q = 0; q < 4; ++q)
      for (int l = 0; l < 8; ++l)
        t[q][l] = std::fmaf(a[32 * c + 8 * q + l], b[32 * c + 8 * q + l], t[q][l]);
  for (int l = 0; l < 8; ++l) s[l] = (t[0][l] + t[1][l]) + (t[2][l] + t[3][l]);
#endif
  float r = hsum_b(s);
  for (int i = chunks * 32; i < n; ++i) r += a[i] * b[i];
  return r;
}

// core/distance/inner_product.rs:22-44 / alternatives.rs:170-183: 4-wide scalar chunks
static float dot_c(const float* a, const float* b, int n) {
  float dot = 0.f;
  int chunks = n / 4;
  for (int i = 0; i < chunks; ++i) {
    int j = 4 * i;
    float p = a[j] * b[j];
    p = p + a[j + 1] * b[j + 1];
    p = p + a[j + 2] * b[j + 2];
    p = p + a[j + 3] * b[j + 3];
    dot += p;
  }
  for (int i = chunks * 4; i < n; ++i) dot += a[i] * b[i];
  return dot;
}

// core/distance/cosine.rs:41-80 cosine_avx2
static float cosine(const float* a, const float* b, int n) {
  int chunks = n / 8;
  float sd[8], sa[8], sb[8];
#ifdef ORC_AVX2
  __m256 vd = _mm256_setzero_ps(), va = vd, vb = vd;
  for (int i = 0; i < chunks; ++i) {
    __m256 x = _mm256_loadu_ps(a + 8 * i), y = _mm256_loadu_ps(b + 8 * i);
    vd = _mm256_fmadd_ps(x, y, vd);
    va = _mm256_fmadd_ps(x, x, va);
    vb = _mm256_fmadd_ps(y, y, vb);
  }
  store8(vd, sd); store8(va, sa); store8(vb, sb);
#else
  for (int l = 0; l < 8; ++l) sd[l] = sa[l] = sb[l] = 0.f;
  for (int i = 0; i < chunks; ++i)
    for (int l = 0; l < 8; ++l) {
      float x = a[8 * i + l], y = b[8 * i + l];
      sd[l] = std::fmaf(x, y, sd[l]);
      sa[l] = std::fmaf(x, x, sa[l]);
      sb[l] = std::fmaf(y, y, sb[l]);
    }
#endif
  float dot = hsum_a(sd), na = hsum_a(sa), nb = hsum_a(sb);
  for (int i = chunks * 8; i < n; ++i) {
    dot += a[i] * b[i];
    na += a[i] * a[i];
    nb += b[i] * b[i];
  }
  float denom = std::sqrt(na * nb);
  if (denom < 1e-12f) return 1.0f;
  float sim = std::min(std::max(dot / denom, -1.0f), 1.0f);
  return 1.0f - sim;
}

// core/distance/alternatives.rs:207-226 AlternativeCosine (sequential scalar loop)
static float alt_cosine(const float* a, const float* b, int n) {
  float dot = 0.f, na = 0.f, nb = 0.f;
  for (int i = 0; i < n; ++i) {
    dot += a[i] * b[i];
    na += a[i] * a[i];
    nb += b[i] * b[i];
  }
  if (na == 0.f && nb == 0.f) return 0.f;
  if (na == 0.f || nb == 0.f) return FLT_MAX;
  if (dot <= 0.f) return FLT_MAX;
  return std::log2(std::sqrt(na * nb) / dot);
}

// The reference's other metrics (core/distance/{minkowski,angular,binary,
// hellinger}.rs), plain sequential loops as written there.
enum {
  ORC_CHEBYSHEV = 8, ORC_CANBERRA, ORC_BRAYCURTIS, ORC_CORRELATION, ORC_TRUE_ANGULAR, ORC_TSSS, ORC_HAMMING,
  ORC_JACCARD, ORC_DICE, ORC_MATCHING, ORC_KULSINSKI, ORC_ROGERSTANIMOTO, ORC_RUSSELLRAO, ORC_SOKALMICHENER,
  ORC_SOKALSNEATH, ORC_YULE, ORC_HELLINGER, ORC_JENSEN_SHANNON, ORC_SYMMETRIC_KL
};
static float other_metric(int kind, const float* a, const float* b, int n) {
  const float nf = (float)n;
  switch (kind) {
    case ORC_CHEBYSHEV: {  // minkowski.rs:106-121
      float r = 0.f;
      for (int i = 0; i < n; ++i) {
        float d = std::fabs(a[i] - b[i]);
        if (d > r) r = d;
      }
      return r;
    }
    case ORC_CANBERRA: {  // minkowski.rs:165-181
      float s = 0.f;
      for (int i = 0; i < n; ++i) {
        float den = std::fabs(a[i]) + std::fabs(b[i]);
        if (den > 0.f) s += std::fabs(a[i] - b[i]) / den;
      }
      return s;
    }
    case ORC_BRAYCURTIS: {  // minkowski.rs:191-212
      float num = 0.f, den = 0.f;
      for (int i = 0; i < n; ++i) {
        num += std::fabs(a[i] - b[i]);
        den += std::fabs(a[i] + b[i]);
      }
      return den > 0.f ? num / den : 0.f;
    }
    case ORC_CORRELATION: {  // angular.rs:13-52
      if (n == 0) return 0.f;
      float ma = 0.f, mb = 0.f;
      for (int i = 0; i < n; ++i) {
        ma += a[i];
        mb += b[i];
      }
      ma /= nf;
      mb /= nf;
      float dot = 0.f, na = 0.f, nb = 0.f;
      for (int i = 0; i < n; ++i) {
        float sa = a[i] - ma, sb = b[i] - mb;
        dot += sa * sb;
        na += sa * sa;
        nb += sb * sb;
      }
      if (na == 0.f && nb == 0.f) return 0.f;
      if (dot == 0.f) return 1.f;
      return 1.f - dot / std::sqrt(na * nb);
    }
    case ORC_TRUE_ANGULAR:  // angular.rs:62-90
    case ORC_TSSS: {        // angular.rs:99-133
      float de = 0.f, dot = 0.f, na = 0.f, nb = 0.f;
      for (int i = 0; i < n; ++i) {
        float d = a[i] - b[i];
        de += d * d;
        dot += a[i] * b[i];
        na += a[i] * a[i];
        nb += b[i] * b[i];
      }
      const float pi = 3.14159265358979f;
      if (kind == ORC_TRUE_ANGULAR) {
        if (na == 0.f && nb == 0.f) return 0.f;
        if (na == 0.f || nb == 0.f || dot <= 0.f) return FLT_MAX;
        float sim = std::min(std::max(dot / std::sqrt(na * nb), -1.f), 1.f);
        return 1.f - std::acos(sim) / pi;
      }
      na = std::sqrt(na);
      nb = std::sqrt(nb);
      float mag = std::fabs(na - nb);
      float den = na * nb;
      if (den < 1e-12f) return 0.f;
      float cs = std::min(std::max(dot / den, -1.f), 1.f);
      float theta = std::acos(cs) + 10.0f * (pi / 180.0f);  // f32::to_radians
      float t = std::sqrt(de) + mag;
      float sector = t * t * theta;
      float triangle = den * std::sin(theta) / 2.0f;
      return triangle * sector;
    }
    case ORC_HAMMING:
    case ORC_MATCHING: {  // binary.rs:13-32, :113-132
      if (n == 0) return 0.f;
      uint32_t cnt = 0;
      for (int i = 0; i < n; ++i)
        cnt += kind == ORC_HAMMING ? (a[i] != b[i]) : ((a[i] != 0.f) != (b[i] != 0.f));
      return (float)cnt / nf;
    }
    case ORC_HELLINGER: {  // hellinger.rs:16-44
      float bc = 0.f, la = 0.f, lb = 0.f;
      for (int i = 0; i < n; ++i) {
        bc += std::sqrt(a[i] * b[i]);
        la += a[i];
        lb += b[i];
      }
      if (la == 0.f && lb == 0.f) return 0.f;
      if (la == 0.f || lb == 0.f) return 1.f;
      float v = 1.f - bc / std::sqrt(la * lb);
      return std::sqrt(std::max(v, 0.f));
    }
    case ORC_JENSEN_SHANNON:  // hellinger.rs:98-128
    case ORC_SYMMETRIC_KL: {  // hellinger.rs:137-166
      float la = 0.f, lb = 0.f;
      for (int i = 0; i < n; ++i) {
        la += a[i];
        lb += b[i];
      }
      float et = FLT_EPSILON * nf;
      la += et;
      lb += et;
      float r = 0.f;
      for (int i = 0; i < n; ++i) {
        float px = (a[i] + FLT_EPSILON) / la, py = (b[i] + FLT_EPSILON) / lb;
        if (kind == ORC_JENSEN_SHANNON) {
          float m = 0.5f * (px + py);
          r += 0.5f * (px * std::log(px / m) + py * std::log(py / m));
        } else {
          r += px * std::log(px / py) + py * std::log(py / px);
        }
      }
      return r;
    }
  }
  // binary.rs: indicator counts (exact integers in f32)
  float tt = 0.f, tf = 0.f, ft = 0.f, ne = 0.f, nz = 0.f;
  for (int i = 0; i < n; ++i) {
    bool x = a[i] != 0.f, y = b[i] != 0.f;
    if (x || y) nz += 1.f;
    if (x && y) tt += 1.f;
    if (x && !y) tf += 1.f;
    if (!x && y) ft += 1.f;
    if (x != y) ne += 1.f;
  }
  switch (kind) {
    case ORC_JACCARD: return nz == 0.f ? 0.f : (nz - tt) / nz;                // binary.rs:42-68
    case ORC_DICE: return ne == 0.f ? 0.f : ne / (2.f * tt + ne);             // :142-167
    case ORC_KULSINSKI: return ne == 0.f ? 0.f : (ne - tt + nf) / (ne + nf);  // :177-203
    case ORC_ROGERSTANIMOTO:                                                  // :213-229
    case ORC_SOKALMICHENER: return (2.f * ne) / (nf + ne);                    // :268-276
    case ORC_RUSSELLRAO: return n == 0 ? 0.f : (nf - tt) / nf;                // :239-258
    case ORC_SOKALSNEATH: return ne == 0.f ? 0.f : ne / (0.5f * tt + ne);     // :286-311
    case ORC_YULE: {                                                          // :321-353
      float ff = nf - tt - tf - ft;
      if (tf == 0.f || ft == 0.f) return 0.f;
      return (2.f * tf * ft) / (tt * ff + tf * ft);
    }
  }
  return NAN;
}

static float distance_impl(int kind, const float* a, const float* b, int n) {
  if (kind >= ORC_CHEBYSHEV) return other_metric(kind, a, b, n);
  switch (kind) {
    case ORC_SQEUCLIDEAN: return sqeuclid(a, b, n);
    case ORC_MANHATTAN: return manhattan(a, b, n);
    case ORC_COSINE: return cosine(a, b, n);
    case ORC_ALT_COSINE: return alt_cosine(a, b, n);
    case ORC_ALT_DOT: {  // alternatives.rs:38-44
      float dot = dot_b(a, b, n);
      return dot <= 0.f ? FLT_MAX : -std::log2(dot);
    }
    case ORC_DIRECT_COSINE: {  // alternatives.rs:131-150
      float dot = dot_b(a, b, n);
      return 1.0f - std::min(std::max(dot, -1.0f), 1.0f);
    }
    case ORC_INNER_PRODUCT: return -dot_a(a, b, n);  // inner_product.rs:96-101
    case ORC_ALT_INNER_PRODUCT: {                    // alternatives.rs:163-187
      float dot = dot_c(a, b, n);
      return dot <= 0.f ? FLT_MAX : 1.0f / dot;
    }
  }
  return NAN;
}

// alternatives.rs:273-287 and index.rs:587
static float correct(int corr, float d) {
  switch (corr) {
    case ORC_CORR_SQRT: return std::sqrt(d);
    case ORC_CORR_ALT_COSINE: return 1.0f - std::pow(2.0f, -d);
    case ORC_CORR_ALT_IP: return d >= FLT_MAX ? 0.0f : -1.0f / d;
  }
  return d;
}

// core/distance/quantized.rs:26-40 quantized_i8_dot (exact integer dot)
static int32_t i8_dot(const int8_t* x, const int8_t* y, int n) {
  int32_t r = 0;
  for (int i = 0; i < n; ++i) r += (int32_t)x[i] * (int32_t)y[i];
  return r;
}

// ---------------------------------------------------------------------------
// NeighborHeap -- core/heap/neighbor_heap.rs:18-320
// ---------------------------------------------------------------------------
struct NeighborHeap {
  std::vector<int32_t> indices;
  std::vector<float> distances;
  std::vector<uint8_t> flags;
  size_t n_points, k;
  NeighborHeap(size_t n, size_t k_)  // neighbor_heap.rs:35-44
      : indices(n * k_, -1), distances(n * k_, INFINITY), flags(n * k_, 0), n_points(n), k(k_) {}
  float max_distance(size_t p) const { return distances[p * k]; }  // :54-56
  // neighbor_heap.rs:207-243 sift_down (shift technique)
  void sift_down(size_t off, size_t start) {
    size_t end = k;
    float vd = distances[off + start];
    int32_t vi = indices[off + start];
    uint8_t vf = flags[off + start];
    size_t pos = start, child = 2 * pos + 1;
    while (child < end) {
      size_t right = child + 1;
      if (right < end && distances[off + child] < distances[off + right]) child = right;
      if (vd >= distances[off + child]) break;
      distances[off + pos] = distances[off + child];
      indices[off + pos] = indices[off + child];
      flags[off + pos] = flags[off + child];
      pos = child;
      child = 2 * pos + 1;
    }
    distances[off + pos] = vd;
    indices[off + pos] = vi;
    flags[off + pos] = vf;
  }
  bool simple_push(size_t p, int32_t nb, float d) {  // :100-115
    size_t off = p * k;
    if (d >= distances[off]) return false;
    distances[off] = d; indices[off] = nb; flags[off] = 0;
    sift_down(off, 0);
    return true;
  }
  bool checked_push(size_t p, int32_t nb, float d) {  // :121-143
    size_t off = p * k;
    if (d >= distances[off]) return false;
    for (size_t i = 0; i < k; ++i)
      if (indices[off + i] == nb) return false;
    distances[off] = d; indices[off] = nb; flags[off] = 0;
    sift_down(off, 0);
    return true;
  }
  bool checked_flagged_push(size_t p, int32_t nb, float d, bool is_new) {  // :149-177
    size_t off = p * k;
    if (d >= distances[off]) return false;
    for (size_t i = 0; i < k; ++i)
      if (indices[off + i] == nb) return false;
    distances[off] = d; indices[off] = nb; flags[off] = is_new ? 1 : 0;
    sift_down(off, 0);
    return true;
  }
  void unchecked_flagged_push(size_t p, int32_t nb, float d, bool is_new) {  // :183-198
    size_t off = p * k;
    distances[off] = d; indices[off] = nb; flags[off] = is_new ? 1 : 0;
    sift_down(off, 0);
  }
  // :293-320 sort_all / sort_row: stable sort by distance (partial_cmp)
  void sort_all() {
    std::vector<std::pair<float, std::pair<int32_t, uint8_t>>> tmp(k);
    for (size_t p = 0; p < n_points; ++p) {
      size_t off = p * k;
      for (size_t i = 0; i < k; ++i) tmp[i] = {distances[off + i], {indices[off + i], flags[off + i]}};
      std::stable_sort(tmp.begin(), tmp.end(),
                       [](const auto& a, const auto& b) { return a.first < b.first; });
      for (size_t i = 0; i < k; ++i) {
        distances[off + i] = tmp[i].first;
        indices[off + i] = tmp[i].second.first;
        flags[off + i] = tmp[i].second.second;
      }
    }
  }
};

// core/nndescent/candidates.rs:433-484 checked_heap_push_flat
static inline void checked_heap_push_flat(float* pri, int32_t* idx, size_t n, float priority,
                                          int32_t index) {
  if (priority >= pri[0]) return;
  for (size_t i = 0; i < n; ++i)
    if (idx[i] == index) return;
  pri[0] = priority;
  idx[0] = index;
  size_t pos = 0;
  for (;;) {
    size_t left = 2 * pos + 1, right = 2 * pos + 2, largest = pos;
    if (left < n && pri[left] > pri[largest]) largest = left;
    if (right < n && pri[right] > pri[largest]) largest = right;
    if (largest != pos) {
      pri[pos] = pri[largest];
      idx[pos] = idx[largest];
      pri[largest] = priority;
      idx[largest] = index;
      pos = largest;
    } else {
      break;
    }
  }
}

// ---------------------------------------------------------------------------
// Rust std BinaryHeap restatement (push/pop/into_vec order), used for the
// search heaps so tie order of BoundedHeap::into_sorted matches
// (core/heap/candidate_heap.rs:78-163; ordered-float 4.6 total order on (d, idx)).
// ---------------------------------------------------------------------------
struct Item {
  float d;
  int32_t i;
};
static inline int ord_cmp_f(float a, float b) {  // OrderedFloat: NaN greatest, -0 == 0
  bool na = std::isnan(a), nb = std::isnan(b);
  if (na || nb) return na == nb ? 0 : (na ? 1 : -1);
  return a < b ? -1 : (a > b ? 1 : 0);
}
static inline int item_cmp(const Item& a, const Item& b) {
  int c = ord_cmp_f(a.d, b.d);
  if (c) return c;
  return a.i < b.i ? -1 : (a.i > b.i ? 1 : 0);
}
template <bool MaxHeap>
struct RustBinaryHeap {
  std::vector<Item> data;
  static bool le(const Item& a, const Item& b) {  // a <= b in heap order
    int c = item_cmp(a, b);
    return MaxHeap ? c <= 0 : c >= 0;  // Reverse<> for the min-heap
  }
  size_t sift_up(size_t start, size_t pos) {
    Item elem = data[pos];
    while (pos > start) {
      size_t parent = (pos - 1) / 2;
      if (le(elem, data[parent])) break;
      data[pos] = data[parent];
      pos = parent;
    }
    data[pos] = elem;
    return pos;
  }
  void sift_down_to_bottom(size_t pos) {
    size_t end = data.size(), start = pos;
    Item elem = data[pos];
    size_t child = 2 * pos + 1;
    while (end >= 2 && child <= end - 2) {
      child += le(data[child], data[child + 1]) ? 1 : 0;
      data[pos] = data[child];
      pos = child;
      child = 2 * pos + 1;
    }
    if (child == end - 1) {
      data[pos] = data[child];
      pos = child;
    }
    data[pos] = elem;
    sift_up(start, pos);
  }
  void push(Item it) {
    data.push_back(it);
    sift_up(0, data.size() - 1);
  }
  bool pop(Item* out) {
    if (data.empty()) return false;
    Item item = data.back();
    data.pop_back();
    if (!data.empty()) {
      std::swap(item, data[0]);
      sift_down_to_bottom(0);
    }
    *out = item;
    return true;
  }
  const Item& peek() const { return data[0]; }
  size_t size() const { return data.size(); }
  void clear() { data.clear(); }
};

// core/heap/candidate_heap.rs:78-163 BoundedHeap
struct BoundedHeap {
  RustBinaryHeap<true> heap;
  size_t k;
  explicit BoundedHeap(size_t k_) : k(k_) {}
  bool push(float d, int32_t idx) {  // :97-113
    if (heap.size() < k) {
      heap.push({d, idx});
      return true;
    }
    if (heap.size() > 0 && d < heap.peek().d) {
      Item tmp;
      heap.pop(&tmp);
      heap.push({d, idx});
      return true;
    }
    return false;
  }
  float max_distance() const { return heap.size() ? heap.peek().d : INFINITY; }
  bool is_full() const { return heap.size() >= k; }
  // :140-148 into_sorted: stable sort by OrderedFloat distance only
  void into_sorted(std::vector<int32_t>& ids, std::vector<float>& ds) const {
    std::vector<Item> v = heap.data;
    std::stable_sort(v.begin(), v.end(),
                     [](const Item& a, const Item& b) { return ord_cmp_f(a.d, b.d) < 0; });
    ids.clear();
    ds.clear();
    for (auto& it : v) {
      ids.push_back(it.i);
      ds.push_back(it.d);
    }
  }
};

// core/visited.rs:8-63 (epoch-stamped); the epoch value itself is not observable.
struct VisitedSet {
  std::vector<uint16_t> epochs;
  uint16_t epoch = 1;
  explicit VisitedSet(size_t n) : epochs(n, 0) {}
  bool check_and_mark(int32_t idx) {
    bool was = epochs[idx] == epoch;
    epochs[idx] = epoch;
    return was;
  }
  void clear() {
    epoch = (uint16_t)(epoch + 1);
    if (epoch == 0) {
      std::fill(epochs.begin(), epochs.end(), 0);
      epoch = 1;
    }
  }
};

// ---------------------------------------------------------------------------
// FlatTree -- core/tree/flat_tree.rs:14-356 and builder -- core/tree/builder.rs:62-348
// ---------------------------------------------------------------------------
struct FlatTree {
  std::vector<float> hyperplanes;
  std::vector<float> offsets;
  std::vector<int32_t> children;  // 2 per node
  std::vector<int32_t> indices;
  size_t dim = 0, n_nodes = 0;

  // flat_tree.rs:239-311 search_leaves
  int search_leaves(const float* point, FastRng& rng, size_t budget,
                    std::vector<std::pair<size_t, size_t>>& leaves) const {
    return search_leaves_with(
        [&](size_t node) { return dot_a(point, &hyperplanes[node * dim], (int)dim) + offsets[node]; }, rng, budget,
        leaves);
  }
  // search_leaves with the node margin given by `margin` (FP32 hyperplanes
  // above; the int8 routing tree's reconstructed margin, flat_tree.rs:96-183)
  template <class M>
  int search_leaves_with(M&& margin_of, FastRng& rng, size_t budget,
                         std::vector<std::pair<size_t, size_t>>& leaves) const {
    leaves.clear();
    if (n_nodes == 0 || budget == 0) return 0;
    int evals = 0;
    if (budget == 1) {
      size_t node = 0;
      while (children[2 * node] > 0) {
        float margin = margin_of(node);
        ++evals;
        size_t side = std::fabs(margin) < 1e-8f ? (size_t)rng.next_bool() : (size_t)(margin > 0.f);
        node = (size_t)children[2 * node + side];
      }
      leaves.push_back({(size_t)(-children[2 * node]), (size_t)(-children[2 * node + 1])});
      return evals;
    }
    std::vector<std::pair<float, size_t>> frontier;
    frontier.push_back({0.f, 0});
    while (leaves.size() < budget && !frontier.empty()) {
      size_t best = 0;  // Iterator::min_by: first minimum under f32::total_cmp
      for (size_t i = 1; i < frontier.size(); ++i) {
        float a = frontier[i].first, b = frontier[best].first;
        int32_t ia, ib;
        std::memcpy(&ia, &a, 4);
        std::memcpy(&ib, &b, 4);
        ia ^= (int32_t)(((uint32_t)(ia >> 31)) >> 1);
        ib ^= (int32_t)(((uint32_t)(ib >> 31)) >> 1);
        if (ia < ib) best = i;
      }
      auto pr = frontier[best];
      frontier.erase(frontier.begin() + (long)best);
      size_t node = pr.second;
      if (children[2 * node] <= 0) {
        leaves.push_back({(size_t)(-children[2 * node]), (size_t)(-children[2 * node + 1])});
        continue;
      }
      float margin = margin_of(node);
      ++evals;
      size_t side = std::fabs(margin) < 1e-8f ? (size_t)rng.next_bool() : (size_t)(margin > 0.f);
      frontier.push_back({pr.first, (size_t)children[2 * node + side]});
      frontier.push_back({std::max(pr.first, std::fabs(margin)), (size_t)children[2 * node + 1 - side]});
    }
    return evals;
  }
  // flat_tree.rs:339-356 get_all_leaves (DFS)
  void collect_leaves(size_t node, std::vector<std::pair<size_t, size_t>>& out) const {
    if (children[2 * node] <= 0) {
      out.push_back({(size_t)(-children[2 * node]), (size_t)(-children[2 * node + 1])});
    } else {
      collect_leaves((size_t)children[2 * node], out);
      collect_leaves((size_t)children[2 * node + 1], out);
    }
  }
};

struct TreeBuilder {  // builder.rs:138-348
  const float* data;
  size_t dim, leaf_size, max_depth;
  bool angular;
  FlatTree out;

  int32_t build_recursive(int32_t* idx, size_t n, size_t depth, FastRng& rng) {  // :172-226
    int32_t node_id = (int32_t)(out.children.size() / 2);
    auto make_leaf = [&]() {
      int32_t start = (int32_t)out.indices.size();
      out.indices.insert(out.indices.end(), idx, idx + n);
      int32_t end = (int32_t)out.indices.size();
      out.hyperplanes.resize(out.hyperplanes.size() + dim, 0.f);
      out.offsets.push_back(0.f);
      out.children.push_back(-start);
      out.children.push_back(-end);
      return node_id;
    };
    if (n <= leaf_size || depth >= max_depth) return make_leaf();
    std::vector<float> hp(dim);
    float offset = make_split(idx, n, rng, hp);
    size_t split = partition_inplace(idx, n, hp.data(), offset, rng);
    if (split == 0 || split == n) return make_leaf();
    out.hyperplanes.insert(out.hyperplanes.end(), hp.begin(), hp.end());
    out.offsets.push_back(offset);
    out.children.push_back(0);
    out.children.push_back(0);
    int32_t l = build_recursive(idx, split, depth + 1, rng);
    int32_t r = build_recursive(idx + split, n - split, depth + 1, rng);
    out.children[2 * node_id] = l;
    out.children[2 * node_id + 1] = r;
    return node_id;
  }
  float make_split(const int32_t* idx, size_t n, FastRng& rng, std::vector<float>& hp) {  // :228-247
    size_t i1 = rng.next_index(n);
    size_t i2 = rng.next_index(n);
    while (i2 == i1 && n > 1) i2 = rng.next_index(n);
    const float* p1 = data + (size_t)idx[i1] * dim;
    const float* p2 = data + (size_t)idx[i2] * dim;
    return split_hyperplane(p1, p2, dim, angular, hp.data());
  }
  // builder.rs:249-308: the hyperplane of two split points (euclidean
  // perpendicular bisector, or angular difference of the normalized points)
  static float split_hyperplane(const float* p1, const float* p2, size_t dim, bool angular, float* hp) {
    if (angular) {  // :281-308
      float n1 = 0.f, n2 = 0.f;
      for (size_t i = 0; i < dim; ++i) n1 += p1[i] * p1[i];
      for (size_t i = 0; i < dim; ++i) n2 += p2[i] * p2[i];
      n1 = std::sqrt(n1);
      n2 = std::sqrt(n2);
      if (n1 < 1e-8f || n2 < 1e-8f) {
        std::fill(hp, hp + dim, 0.f);
        return 0.f;
      }
      for (size_t i = 0; i < dim; ++i) hp[i] = p2[i] / n2 - p1[i] / n1;
      float nn = 0.f;
      for (size_t i = 0; i < dim; ++i) nn += hp[i] * hp[i];
      nn = std::sqrt(nn);
      if (nn > 1e-8f)
        for (size_t i = 0; i < dim; ++i) hp[i] /= nn;
      return 0.f;
    }
    // :249-279 euclidean perpendicular bisector
    float norm_sq = 0.f, dot_nm = 0.f;
    for (size_t i = 0; i < dim; ++i) {
      float h = p2[i] - p1[i];
      float m = (p1[i] + p2[i]) * 0.5f;
      hp[i] = h;
      norm_sq += h * h;
      dot_nm += h * m;
    }
    float norm = std::sqrt(norm_sq);
    if (norm > 1e-8f) {
      float inv = 1.0f / norm;
      for (size_t i = 0; i < dim; ++i) hp[i] *= inv;
      return -dot_nm * inv;
    }
    return 0.f;
  }
  size_t partition_inplace(int32_t* idx, size_t n, const float* hp, float offset,
                           FastRng& rng) {  // :312-348
    size_t left = 0, right = n;
    while (left < right) {
      const float* p = data + (size_t)idx[left] * dim;
      float margin = dot_a(p, hp, (int)dim) + offset;
      bool goes_left = std::fabs(margin) < 1e-8f ? !rng.next_bool() : margin < 0.f;
      if (goes_left) {
        ++left;
      } else {
        --right;
        std::swap(idx[left], idx[right]);
      }
    }
    return left;
  }
};

// flat_tree.rs:47-64 QuantizedFlatTree::quantize_hyperplanes: per node scale =
// max|h| / 127 (0 for zero hyperplanes, leaves included), code =
// (h / scale).round().clamp(-127, 127).
static void quantize_hyperplanes(const float* hp, size_t n_nodes, size_t dim, int8_t* codes, float* scales) {
  for (size_t v = 0; v < n_nodes; ++v) {
    const float* h = hp + v * dim;
    float mx = 0.f;
    for (size_t j = 0; j < dim; ++j) mx = std::max(mx, std::fabs(h[j]));
    const float sc = mx > 0.f ? mx / 127.0f : 0.f;
    scales[v] = sc;
    for (size_t j = 0; j < dim; ++j) {
      float c = sc > 0.f ? std::round(h[j] / sc) : 0.f;
      if (c != c) c = 0.f;
      codes[v * dim + j] = (int8_t)std::min(std::max(c, -127.0f), 127.0f);
    }
  }
}

// flat_tree.rs:96-103 QuantizedFlatTree::margin: ((dot as f32) * scale) * query_scale + offset.
static inline float quantized_margin(const int8_t* codes, const float* scales, const float* offsets, size_t dim,
                                     size_t node, const int8_t* q, float qscale) {
  return (float)i8_dot(codes + node * dim, q, (int)dim) * scales[node] * qscale + offsets[node];
}

// builder.rs:72-86 build_rp_tree
static FlatTree build_rp_tree(const float* data, size_t n, size_t dim, size_t leaf_size,
                              FastRng& rng, bool angular, size_t max_depth) {
  std::vector<int32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  TreeBuilder b{data, dim, leaf_size, max_depth, angular, FlatTree()};
  b.out.dim = dim;
  b.build_recursive(idx.data(), n, 0, rng);
  b.out.n_nodes = b.out.children.size() / 2;
  return std::move(b.out);
}

static int num_threads_of(int requested) {
#ifdef _OPENMP
  return requested > 0 ? requested : omp_get_max_threads();
#else
  (void)requested;
  return 1;
#endif
}

// builder.rs:89-118 build_rp_forest (seeds drawn from the master rng, trees in parallel)
static std::vector<FlatTree> build_rp_forest(const float* data, size_t n, size_t dim,
                                             size_t n_trees, size_t leaf_size, FastRng& rng,
                                             bool angular, size_t max_depth, int nt) {
  std::vector<uint64_t> seeds(n_trees);
  for (auto& s : seeds) s = rng.next_u64();
  std::vector<FlatTree> forest(n_trees);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
  for (long t = 0; t < (long)n_trees; ++t) {
    FastRng tr(seeds[(size_t)t]);
    forest[(size_t)t] = build_rp_tree(data, n, dim, leaf_size, tr, angular, max_depth);
  }
  return forest;
}

// builder.rs:123-135 rptree_leaf_array
static std::vector<std::vector<int32_t>> rptree_leaf_array(const std::vector<FlatTree>& forest) {
  std::vector<std::vector<int32_t>> res;
  for (auto& t : forest) {
    std::vector<std::pair<size_t, size_t>> leaves;
    t.collect_leaves(0, leaves);
    for (auto& l : leaves)
      res.emplace_back(t.indices.begin() + (long)l.first, t.indices.begin() + (long)l.second);
  }
  return res;
}

// ---------------------------------------------------------------------------
// NN-Descent -- core/nndescent/mod.rs
// ---------------------------------------------------------------------------
struct Cands {
  std::vector<int32_t> new_idx, old_idx;
  size_t mc;
};

// candidates.rs:354-417 mark_old_flags
static void mark_old_flags(NeighborHeap& g, const std::vector<int32_t>& new_idx, size_t mc,
                           int nt) {
  long n = (long)g.n_points;
  size_t k = g.k;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (long i = 0; i < n; ++i) {
    size_t ro = (size_t)i * k, no = (size_t)i * mc;
    for (size_t j = 0; j < k; ++j) {
      int32_t nb = g.indices[ro + j];
      if (nb < 0 || g.flags[ro + j] == 0) continue;
      for (size_t c = 0; c < mc; ++c)
        if (new_idx[no + c] == nb) {
          g.flags[ro + j] = 0;
          break;
        }
    }
  }
}

// candidates.rs:68-144 build_from_graph_sequential
static Cands build_candidates_sequential(NeighborHeap& g, size_t mc, FastRng& rng) {
  size_t n = g.n_points, k = g.k;
  Cands c{std::vector<int32_t>(n * mc, -1), std::vector<int32_t>(n * mc, -1), mc};
  std::vector<float> np(n * mc, INFINITY), op(n * mc, INFINITY);
  for (size_t i = 0; i < n; ++i) {
    for (size_t j = 0; j < k; ++j) {
      int32_t nb = g.indices[i * k + j];
      if (nb < 0) continue;
      bool is_new = g.flags[i * k + j] != 0;
      float pr = rng.next_float();
      size_t oi = i * mc;
      if (is_new) checked_heap_push_flat(&np[oi], &c.new_idx[oi], mc, pr, nb);
      else checked_heap_push_flat(&op[oi], &c.old_idx[oi], mc, pr, nb);
      float rpr = rng.next_float();
      size_t on = (size_t)nb * mc;
      if (is_new) checked_heap_push_flat(&np[on], &c.new_idx[on], mc, rpr, (int32_t)i);
      else checked_heap_push_flat(&op[on], &c.old_idx[on], mc, rpr, (int32_t)i);
    }
  }
  mark_old_flags(g, c.new_idx, mc, 1);
  return c;
}

struct RevEdge {
  size_t dest;
  int32_t cand;
  float pri;
  bool is_new;
};

// candidates.rs:153-351 build_from_graph_parallel
static Cands build_candidates_parallel(NeighborHeap& g, size_t mc, FastRng& rng, int nt) {
  size_t n = g.n_points, k = g.k;
  size_t T = (size_t)nt;
  size_t bs = (n + T - 1) / T;
  Cands c{std::vector<int32_t>(n * mc, -1), std::vector<int32_t>(n * mc, -1), mc};
  std::vector<float> np(n * mc, INFINITY), op(n * mc, INFINITY);
  std::vector<uint64_t> seeds(T);
  for (auto& s : seeds) s = rng.next_u64();
  std::vector<std::vector<std::vector<RevEdge>>> buckets(T, std::vector<std::vector<RevEdge>>(T));
#pragma omp parallel for schedule(static, 1) num_threads(nt)
  for (long tl = 0; tl < (long)T; ++tl) {
    size_t t = (size_t)tl;
    size_t b0 = t * bs, b1 = std::min((t + 1) * bs, n);
    if (b0 >= n) continue;
    FastRng lr(seeds[t]);
    for (size_t i = b0; i < b1; ++i) {
      for (size_t j = 0; j < k; ++j) {
        int32_t nb = g.indices[i * k + j];
        if (nb < 0) continue;
        bool is_new = g.flags[i * k + j] != 0;
        float pr = lr.next_float();
        size_t oi = i * mc;
        if (is_new) checked_heap_push_flat(&np[oi], &c.new_idx[oi], mc, pr, nb);
        else checked_heap_push_flat(&op[oi], &c.old_idx[oi], mc, pr, nb);
        size_t dest_block = (size_t)nb / bs;
        if (dest_block < T) {
          if (dest_block == t) {
            size_t on = (size_t)nb * mc;
            if (is_new) checked_heap_push_flat(&np[on], &c.new_idx[on], mc, pr, (int32_t)i);
            else checked_heap_push_flat(&op[on], &c.old_idx[on], mc, pr, (int32_t)i);
          } else {
            buckets[t][dest_block].push_back({(size_t)nb, (int32_t)i, pr, is_new});
          }
        }
      }
    }
  }
#pragma omp parallel for schedule(static, 1) num_threads(nt)
  for (long tl = 0; tl < (long)T; ++tl) {
    size_t t = (size_t)tl;
    if (t * bs >= n) continue;
    for (size_t src = 0; src < T; ++src) {
      if (src == t) continue;
      for (auto& e : buckets[src][t]) {
        size_t off = e.dest * mc;
        if (e.is_new) checked_heap_push_flat(&np[off], &c.new_idx[off], mc, e.pri, e.cand);
        else checked_heap_push_flat(&op[off], &c.old_idx[off], mc, e.pri, e.cand);
      }
    }
  }
  mark_old_flags(g, c.new_idx, mc, nt);
  return c;
}

// candidates.rs:51-65 dispatch
static Cands build_candidates(NeighborHeap& g, size_t mc, FastRng& rng, int nt) {
  if (g.n_points >= 256 && nt > 1) return build_candidates_parallel(g, mc, rng, nt);
  return build_candidates_sequential(g, mc, rng);
}

struct Upd {
  int32_t p, q;
  float d;
};

// nndescent/mod.rs:203-300 initialize_from_leaves
static void initialize_from_leaves(NeighborHeap& g, const std::vector<std::vector<int32_t>>& leaves,
                                   const float* data, size_t dim, int kind, int nt) {
  size_t n = g.n_points, T = (size_t)nt;
  size_t nl = leaves.size();
  size_t block = std::max(T * 64, (size_t)128);
  size_t vbs = (n + T - 1) / T;
  std::vector<std::vector<Upd>> ups(T);
  for (size_t b0 = 0; b0 < nl; b0 += block) {
    size_t b1 = std::min(b0 + block, nl);
    size_t blen = b1 - b0;
#pragma omp parallel for schedule(static, 1) num_threads(nt)
    for (long tl = 0; tl < (long)T; ++tl) {
      size_t t = (size_t)tl;
      auto& tu = ups[t];
      tu.clear();
      size_t per = (blen + T - 1) / T;
      size_t s = t * per, e = std::min(s + per, blen);
      for (size_t li = s; li < e; ++li) {
        const auto& leaf = leaves[b0 + li];
        for (size_t i = 0; i < leaf.size(); ++i) {
          int32_t p = leaf[i];
          if (p < 0) break;
          for (size_t j = i + 1; j < leaf.size(); ++j) {
            int32_t q = leaf[j];
            if (q < 0) break;
            float d = distance_impl(kind, data + (size_t)p * dim, data + (size_t)q * dim, (int)dim);
            float thr = std::max(g.max_distance((size_t)p), g.max_distance((size_t)q));
            if (d < thr) tu.push_back({p, q, d});
          }
        }
      }
    }
#pragma omp parallel for schedule(static, 1) num_threads(nt)
    for (long tl = 0; tl < (long)T; ++tl) {
      size_t t = (size_t)tl;
      size_t v0 = t * vbs, v1 = std::min(v0 + vbs, n);
      for (size_t src = 0; src < T; ++src)
        for (auto& u : ups[src]) {
          size_t p = (size_t)u.p, q = (size_t)u.q;
          if (p >= v0 && p < v1) g.checked_flagged_push(p, u.q, u.d, true);
          if (q >= v0 && q < v1) g.checked_flagged_push(q, u.p, u.d, true);
        }
    }
  }
}

// nndescent/mod.rs:321-491 update_iteration
static size_t update_iteration(NeighborHeap& g, const Cands& c, const float* data, size_t dim,
                               int kind, int nt) {
  size_t n = g.n_points, T = (size_t)nt, mc = c.mc;
  const size_t BLOCK = 16384;
  size_t vbs = (n + T - 1) / T;
  std::vector<std::vector<std::vector<Upd>>> buckets(T, std::vector<std::vector<Upd>>(T));
  size_t total = 0;
  size_t nblocks = (n + BLOCK - 1) / BLOCK;
  for (size_t bi = 0; bi < nblocks; ++bi) {
    size_t bstart = bi * BLOCK, bend = std::min((bi + 1) * BLOCK, n);
    size_t rpt = (bend - bstart + T - 1) / T;
    for (auto& tb : buckets)
      for (auto& b : tb) b.clear();
#pragma omp parallel for schedule(static, 1) num_threads(nt)
    for (long tl = 0; tl < (long)T; ++tl) {
      size_t t = (size_t)tl;
      auto& lb = buckets[t];
      size_t r0 = bstart + t * rpt, r1 = std::min(r0 + rpt, bend);
      for (size_t i = r0; i < r1; ++i) {
        const int32_t* nc = &c.new_idx[i * mc];
        const int32_t* oc = &c.old_idx[i * mc];
        for (size_t j = 0; j < mc; ++j) {
          int32_t p = nc[j];
          if (p < 0) continue;
          const float* dp = data + (size_t)p * dim;
          float tp = g.max_distance((size_t)p);
          auto emit = [&](int32_t q, float d) {
            size_t pb = (size_t)p / vbs, qb = (size_t)q / vbs;
            lb[std::min(pb, T - 1)].push_back({p, q, d});
            if (pb != qb) lb[std::min(qb, T - 1)].push_back({p, q, d});
          };
          for (size_t kk = j + 1; kk < mc; ++kk) {  // new x new
            int32_t q = nc[kk];
            if (q < 0) continue;
            float mt = std::max(tp, g.max_distance((size_t)q));
            float d = distance_impl(kind, dp, data + (size_t)q * dim, (int)dim);
            if (d <= mt) emit(q, d);
          }
          for (size_t kk = 0; kk < mc; ++kk) {  // new x old
            int32_t q = oc[kk];
            if (q < 0 || p == q) continue;
            float mt = std::max(tp, g.max_distance((size_t)q));
            float d = distance_impl(kind, dp, data + (size_t)q * dim, (int)dim);
            if (d <= mt) emit(q, d);
          }
        }
      }
    }
    size_t changes = 0;
#pragma omp parallel for schedule(static, 1) num_threads(nt) reduction(+ : changes)
    for (long tl = 0; tl < (long)T; ++tl) {
      size_t t = (size_t)tl;
      size_t v0 = t * vbs, v1 = std::min(v0 + vbs, n);
      for (size_t src = 0; src < T; ++src)
        for (auto& u : buckets[src][t]) {
          size_t p = (size_t)u.p, q = (size_t)u.q;
          if (p >= v0 && p < v1 && g.checked_flagged_push(p, u.q, u.d, true)) ++changes;
          if (q >= v0 && q < v1 && g.checked_flagged_push(q, u.p, u.d, true)) ++changes;
        }
    }
    total += changes;
  }
  return total;
}

// ---------------------------------------------------------------------------
// Search graph -- core/graph/search_graph.rs
// ---------------------------------------------------------------------------
struct CSR {
  std::vector<int32_t> indptr, indices;
  size_t n = 0;
};

// search_graph.rs:432-473 diversify_row.  A qualifying prune (:457-460) is
// taken always at probability >= 1 (no draw), else when an f32 draw is below
// the probability; the reference draws from rand::thread_rng() (OS-seeded, not
// reproducible), this restatement from a FastRng seeded per row.
static void diversify_row(const int32_t* ri, const float* rd, size_t len, const float* data,
                          size_t dim, int kind, size_t max_degree,
                          std::vector<std::pair<int32_t, float>>& out, float prob = 1.0f, uint64_t rseed = 0) {
  out.clear();
  FastRng rng(rseed);
  for (size_t pos = 0; pos < len; ++pos) {
    int32_t j = ri[pos];
    if (j < 0) break;
    float dij = rd[pos];
    bool keep = true;
    for (auto& cd : out) {
      float dcj = distance_impl(kind, data + (size_t)cd.first * dim, data + (size_t)j * dim, (int)dim);
      if (cd.second > FLT_MIN && dcj < dij) {
        if (prob >= 1.0f || rng.next_float() < prob) {
          keep = false;
          break;
        }
      }
    }
    if (keep) {
      out.push_back({j, dij});
      if (out.size() >= max_degree) break;
    }
  }
}

// search_graph.rs:478-523 diversify_sorted_csr (prune probability as diversify_row)
static void diversify_sorted(const int32_t* ri, const float* rd, const std::vector<size_t>& order,
                             const float* data, size_t dim, int kind, size_t max_degree,
                             std::vector<std::pair<int32_t, float>>& out, float prob = 1.0f, uint64_t rseed = 0) {
  out.clear();
  FastRng rng(rseed);
  for (size_t pos : order) {
    int32_t j = ri[pos];
    if (j < 0) continue;
    float dij = rd[pos];
    bool keep = true;
    for (auto& cd : out) {
      float dcj = distance_impl(kind, data + (size_t)cd.first * dim, data + (size_t)j * dim, (int)dim);
      if (cd.second > FLT_MIN && dcj < dij) {
        if (prob >= 1.0f || rng.next_float() < prob) {
          keep = false;
          break;
        }
      }
    }
    if (keep) {
      out.push_back({j, dij});
      if (out.size() >= max_degree) break;
    }
  }
}

static inline int total_cmp_f(float a, float b) {  // f32::total_cmp
  int32_t ia, ib;
  std::memcpy(&ia, &a, 4);
  std::memcpy(&ib, &b, 4);
  ia ^= (int32_t)(((uint32_t)(ia >> 31)) >> 1);
  ib ^= (int32_t)(((uint32_t)(ib >> 31)) >> 1);
  return ia < ib ? -1 : (ia > ib ? 1 : 0);
}

// search_graph.rs:368-426 weighted_union_pruned
static CSR weighted_union_pruned(const std::vector<std::vector<std::pair<int32_t, float>>>& fwd,
                                 const std::vector<std::vector<std::pair<int32_t, float>>>& rev,
                                 size_t n, size_t max_degree) {
  CSR g;
  g.n = n;
  g.indptr.reserve(n + 1);
  g.indptr.push_back(0);
  std::vector<std::pair<int32_t, float>> row, dd;
  for (size_t v = 0; v < n; ++v) {
    row.clear();
    for (auto& e : fwd[v])
      if (e.first >= 0 && e.first != (int32_t)v && std::isfinite(e.second)) row.push_back(e);
    for (auto& e : rev[v])
      if (e.first >= 0 && e.first != (int32_t)v && std::isfinite(e.second)) row.push_back(e);
    std::sort(row.begin(), row.end(),
              [](const auto& a, const auto& b) { return a.first < b.first; });
    dd.clear();
    for (auto& e : row) {
      if (!dd.empty() && dd.back().first == e.first) {
        dd.back().second = std::max(dd.back().second, e.second);
        continue;
      }
      dd.push_back(e);
    }
    std::sort(dd.begin(), dd.end(), [](const auto& a, const auto& b) {
      int c = total_cmp_f(a.second, b.second);
      return c != 0 ? c < 0 : a.first < b.first;
    });
    if (dd.size() > max_degree) dd.resize(max_degree);
    std::sort(dd.begin(), dd.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    for (auto& e : dd) g.indices.push_back(e.first);
    g.indptr.push_back((int32_t)g.indices.size());
  }
  return g;
}

// search_graph.rs:263-360 from_dense_diversified
static CSR from_dense_diversified(const int32_t* ni, const float* nd, const float* data, size_t n,
                                  size_t k, size_t dim, int kind, float mult, int nt,
                                  float* min_distance, float prob = 1.0f, uint64_t seed = 0) {
  size_t max_degree = (size_t)std::round(mult * (float)k);  // f32::round, half away from zero
  std::vector<std::vector<std::pair<int32_t, float>>> fwd(n), rev(n);
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
  for (long i = 0; i < (long)n; ++i)
    diversify_row(ni + (size_t)i * k, nd + (size_t)i * k, k, data, dim, kind, max_degree, fwd[(size_t)i], prob,
                  seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(i + 1)));
  // forward CSR with data (:299-309) and transpose (:526-567)
  std::vector<int32_t> fptr(n + 1, 0), findx;
  std::vector<float> fdat;
  for (size_t i = 0; i < n; ++i) {
    for (auto& e : fwd[i]) {
      findx.push_back(e.first);
      fdat.push_back(e.second);
    }
    fptr[i + 1] = (int32_t)findx.size();
  }
  std::vector<int32_t> indeg(n, 0);
  for (int32_t x : findx)
    if (x >= 0) indeg[(size_t)x]++;
  std::vector<int32_t> tptr(n + 1, 0);
  for (size_t i = 0; i < n; ++i) tptr[i + 1] = tptr[i] + indeg[i];
  std::vector<int32_t> tidx((size_t)tptr[n]);
  std::vector<float> tdat((size_t)tptr[n]);
  std::vector<int32_t> cur(tptr.begin(), tptr.end() - 1);
  for (size_t v = 0; v < n; ++v)
    for (int32_t e = fptr[v]; e < fptr[v + 1]; ++e) {
      int32_t nb = findx[(size_t)e];
      if (nb >= 0) {
        size_t pos = (size_t)cur[(size_t)nb]++;
        tidx[pos] = (int32_t)v;
        tdat[pos] = fdat[(size_t)e];
      }
    }
  // reverse diversification (:316-346); rows sorted by distance.  Ties keep
  // source-id order (std::stable_sort): matches the reference's sort_unstable
  // whenever a row has no tied distances.
#pragma omp parallel for schedule(dynamic, 256) num_threads(nt)
  for (long il = 0; il < (long)n; ++il) {
    size_t i = (size_t)il;
    size_t s = (size_t)tptr[i], e = (size_t)tptr[i + 1];
    if (s == e) continue;
    std::vector<size_t> order(e - s);
    std::iota(order.begin(), order.end(), 0);
    const float* rd = &tdat[s];
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return rd[a] < rd[b]; });
    diversify_sorted(&tidx[s], rd, order, data, dim, kind, max_degree, rev[i], prob,
                     ~seed ^ (0x9E3779B97F4A7C15ull * (uint64_t)(i + 1)));
  }
  CSR g = weighted_union_pruned(fwd, rev, n, max_degree);
  float md = INFINITY;  // :353-357
  for (float d : fdat) {
    float v = d == 0.f ? FLT_EPSILON : d;
    if (std::isfinite(v)) md = std::min(md, v);
  }
  *min_distance = md;
  return g;
}

// search_graph.rs:199-229 reorder
static void csr_reorder(CSR& g, const std::vector<size_t>& order) {
  size_t n = g.n;
  std::vector<size_t> inv(n);
  for (size_t i = 0; i < n; ++i) inv[order[i]] = i;
  std::vector<int32_t> np, ni;
  np.reserve(n + 1);
  np.push_back(0);
  for (size_t v = 0; v < n; ++v) {
    size_t ov = order[v];
    for (int32_t e = g.indptr[ov]; e < g.indptr[ov + 1]; ++e) {
      int32_t nb = g.indices[(size_t)e];
      if (nb >= 0) ni.push_back((int32_t)inv[(size_t)nb]);
    }
    np.push_back((int32_t)ni.size());
  }
  g.indptr.swap(np);
  g.indices.swap(ni);
}

// ---------------------------------------------------------------------------
// Greedy search -- core/search/greedy.rs
// ---------------------------------------------------------------------------
struct Workspace {  // greedy.rs:32-68
  VisitedSet visited;
  BoundedHeap result;
  RustBinaryHeap<false> seeds;
  std::vector<std::pair<size_t, size_t>> leaves;
  Workspace(size_t n, size_t k) : visited(n), result(k) {}
  void reset(size_t k) {
    visited.clear();
    result.heap.clear();
    result.k = k;
    seeds.clear();
  }
};

template <class F>
static void fill_random(size_t n, size_t k, F&& dist_to, FastRng& rng, Workspace& ws) {  // :148-163
  size_t cnt = k > ws.seeds.size() ? k - ws.seeds.size() : 0;
  for (size_t r = 0; r < cnt; ++r) {
    int32_t idx = (int32_t)rng.next_index(n);
    if (!ws.visited.check_and_mark(idx)) {
      float d = dist_to(idx);
      ws.result.push(d, idx);
      ws.seeds.push({d, idx});
    }
  }
}

template <class F>
static void traverse(const CSR& g, float eps, float min_distance, F&& dist_to, Workspace& ws) {  // :165-201
  float mx = ws.result.max_distance();
  float bound = mx + eps * (mx - min_distance);
  Item it;
  while (ws.seeds.pop(&it)) {
    if (ws.result.is_full() && it.d >= bound) break;
    for (int32_t e = g.indptr[(size_t)it.i]; e < g.indptr[(size_t)it.i + 1]; ++e) {
      int32_t nb = g.indices[(size_t)e];
      if (nb < 0 || ws.visited.check_and_mark(nb)) continue;
      float d = dist_to(nb);
      if (d < bound) {
        bool ins = ws.result.push(d, nb);
        ws.seeds.push({d, nb});
        if (ins) {
          mx = ws.result.max_distance();
          bound = mx + eps * (mx - min_distance);
        }
      }
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Index -- core/index.rs:24-733 + Python dispatch crates/rinnd/src/lib.rs
// ---------------------------------------------------------------------------
struct orc_index {
  std::vector<float> data;  // reordered (internal order)
  size_t n = 0, dim = 0, k = 0;
  int kind = 0, corr = 0;
  std::vector<int32_t> nbr_idx;
  std::vector<float> nbr_dist;  // corrected
  CSR graph;                    // internal order
  std::vector<FlatTree> trees;  // internal ids
  size_t leaf_budget = 1;
  std::vector<size_t> vertex_order;
  float min_distance = 0.f;
  uint64_t seed = 42;
  int iters = 0;
  double t[5] = {0, 0, 0, 0, 0};
  int nt = 1;
};

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// index.rs:157-202 process_query_with_workspace + greedy.rs:203-241 search
static void process_query(const orc_index* ix, const float* q, size_t qid, size_t k, float eps,
                          Workspace& ws, int32_t* oi, float* od) {
  FastRng rng(ix->seed + (uint64_t)qid);
  ws.reset(k);
  const float* data = ix->data.data();
  size_t dim = ix->dim;
  int kind = ix->kind;
  auto dist_to = [&](int32_t i) { return distance_impl(kind, q, data + (size_t)i * dim, (int)dim); };
  for (auto& t : ix->trees) {  // initialize_fp32 :70-99
    t.search_leaves(q, rng, ix->leaf_budget, ws.leaves);
    for (auto& l : ws.leaves)
      for (size_t p = l.first; p < l.second; ++p) {
        int32_t idx = t.indices[p];
        if (idx >= 0 && !ws.visited.check_and_mark(idx)) {
          float d = dist_to(idx);
          ws.result.push(d, idx);
          ws.seeds.push({d, idx});
        }
      }
  }
  fill_random(ix->n, k, dist_to, rng, ws);
  traverse(ix->graph, eps, ix->min_distance, dist_to, ws);
  std::vector<int32_t> ids;
  std::vector<float> ds;
  ws.result.into_sorted(ids, ds);
  for (size_t j = 0; j < k; ++j) {
    if (j < ids.size()) {
      oi[j] = ids[j] >= 0 ? (int32_t)ix->vertex_order[(size_t)ids[j]] : ids[j];
      od[j] = correct(ix->corr, ds[j]);
    } else {
      oi[j] = -1;
      od[j] = INFINITY;
    }
  }
}

extern "C" {

int32_t orc_max_threads(void) { return num_threads_of(0); }

float orc_distance(int kind, const float* a, const float* b, int32_t dim) {
  return distance_impl(kind, a, b, dim);
}

void orc_distance_pairs(int kind, const float* a, const float* b, int64_t n_pairs, int32_t dim,
                        float* out) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < (long)n_pairs; ++i)
    out[i] = distance_impl(kind, a + (size_t)i * (size_t)dim, b + (size_t)i * (size_t)dim, dim);
}

float orc_correct(int correction, float d) { return correct(correction, d); }

int32_t orc_i8_dot(const int8_t* x, const int8_t* y, int32_t dim) { return i8_dot(x, y, dim); }

// quantized.rs:48-56 quantized_i8_per_dimension_dot (sequential f32 sum)
float orc_i8_per_dimension_dot(const int8_t* x, const int8_t* y, const float* scales, int32_t dim) {
  float s = 0.f;
  for (int i = 0; i < dim; ++i) s += (float)x[i] * (float)y[i] * scales[i] * scales[i];
  return s;
}

void orc_rng_u64(uint64_t seed, int32_t n, uint64_t* out) {
  FastRng r(seed);
  for (int i = 0; i < n; ++i) out[i] = r.next_u64();
}
void orc_rng_float(uint64_t seed, int32_t n, float* out) {
  FastRng r(seed);
  for (int i = 0; i < n; ++i) out[i] = r.next_float();
}
void orc_rng_index(uint64_t seed, uint64_t range, int32_t n, uint64_t* out) {
  FastRng r(seed);
  for (int i = 0; i < n; ++i) out[i] = r.next_index(range);
}

void orc_neighbor_heap_sequence(int32_t k, int32_t n_ops, const int32_t* op, const int32_t* ids,
                                const float* dists, const uint8_t* flags, int32_t* results,
                                int32_t* out_idx, float* out_dist, uint8_t* out_flags) {
  NeighborHeap h(1, (size_t)k);
  for (int i = 0; i < n_ops; ++i) {
    int r = 1;
    switch (op[i]) {
      case 0: r = h.simple_push(0, ids[i], dists[i]); break;
      case 1: r = h.checked_push(0, ids[i], dists[i]); break;
      case 2: r = h.checked_flagged_push(0, ids[i], dists[i], flags[i] != 0); break;
      default: h.unchecked_flagged_push(0, ids[i], dists[i], flags[i] != 0); break;
    }
    results[i] = r;
  }
  for (int j = 0; j < k; ++j) {
    out_idx[j] = h.indices[(size_t)j];
    out_dist[j] = h.distances[(size_t)j];
    out_flags[j] = h.flags[(size_t)j];
  }
}

void orc_neighbor_heap_apply(int32_t n, int32_t k, int64_t n_ops, const int32_t* rows,
                             const int32_t* ids, const float* dists, const uint8_t* flags,
                             int32_t* out_idx, float* out_dist, uint8_t* out_flags,
                             int64_t* n_accepted) {
  NeighborHeap h((size_t)n, (size_t)k);
  int64_t acc = 0;
  for (int64_t i = 0; i < n_ops; ++i)
    acc += h.checked_flagged_push((size_t)rows[i], ids[i], dists[i], flags[i] != 0);
  h.sort_all();
  std::memcpy(out_idx, h.indices.data(), sizeof(int32_t) * (size_t)n * (size_t)k);
  std::memcpy(out_dist, h.distances.data(), sizeof(float) * (size_t)n * (size_t)k);
  std::memcpy(out_flags, h.flags.data(), (size_t)n * (size_t)k);
  *n_accepted = acc;
}

void orc_candidate_heap_sequence(int32_t size, int32_t n_ops, const float* priorities,
                                 const int32_t* ids, float* out_pri, int32_t* out_idx) {
  for (int i = 0; i < size; ++i) {
    out_pri[i] = INFINITY;
    out_idx[i] = -1;
  }
  for (int i = 0; i < n_ops; ++i)
    checked_heap_push_flat(out_pri, out_idx, (size_t)size, priorities[i], ids[i]);
}

int32_t orc_bounded_heap_sequence(int32_t k, int32_t n_ops, const float* dists, const int32_t* ids,
                                  int32_t* accepted, int32_t* out_idx, float* out_dist) {
  BoundedHeap h((size_t)k);
  for (int i = 0; i < n_ops; ++i) accepted[i] = h.push(dists[i], ids[i]);
  std::vector<int32_t> oi;
  std::vector<float> od;
  h.into_sorted(oi, od);
  for (size_t i = 0; i < oi.size(); ++i) {
    out_idx[i] = oi[i];
    out_dist[i] = od[i];
  }
  return (int32_t)oi.size();
}

void orc_build_candidates(int32_t n, int32_t k, const int32_t* heap_idx, uint8_t* heap_flags,
                          int32_t max_candidates, uint64_t seed, int32_t n_threads,
                          int32_t* new_idx, int32_t* old_idx) {
  NeighborHeap h((size_t)n, (size_t)k);
  std::memcpy(h.indices.data(), heap_idx, sizeof(int32_t) * (size_t)n * (size_t)k);
  std::memcpy(h.flags.data(), heap_flags, (size_t)n * (size_t)k);
  FastRng rng(seed);
  int nt = num_threads_of(n_threads);
  Cands c = build_candidates(h, (size_t)max_candidates, rng, nt);
  std::memcpy(new_idx, c.new_idx.data(), sizeof(int32_t) * c.new_idx.size());
  std::memcpy(old_idx, c.old_idx.data(), sizeof(int32_t) * c.old_idx.size());
  std::memcpy(heap_flags, h.flags.data(), (size_t)n * (size_t)k);
}

int32_t orc_tree_search_leaves(int32_t n_nodes, int32_t dim, const float* hyperplanes,
                               const float* offsets, const int32_t* children, const float* point,
                               uint64_t seed, int32_t leaf_budget, int32_t* out_leaves,
                               int32_t* n_leaves) {
  FlatTree t;
  t.dim = (size_t)dim;
  t.n_nodes = (size_t)n_nodes;
  t.hyperplanes.assign(hyperplanes, hyperplanes + (size_t)n_nodes * (size_t)dim);
  t.offsets.assign(offsets, offsets + n_nodes);
  t.children.assign(children, children + 2 * (size_t)n_nodes);
  FastRng rng(seed);
  std::vector<std::pair<size_t, size_t>> leaves;
  int ev = t.search_leaves(point, rng, (size_t)leaf_budget, leaves);
  for (size_t i = 0; i < leaves.size(); ++i) {
    out_leaves[2 * i] = (int32_t)leaves[i].first;
    out_leaves[2 * i + 1] = (int32_t)leaves[i].second;
  }
  *n_leaves = (int32_t)leaves.size();
  return ev;
}

int32_t orc_tree_search_leaves_quantized(int32_t n_nodes, int32_t dim, const float* hyperplanes,
                                         const float* offsets, const int32_t* children, const int8_t* qcodes,
                                         float qscale, uint64_t seed, int32_t leaf_budget, int32_t* out_leaves,
                                         int32_t* n_leaves) {
  FlatTree t;
  t.dim = (size_t)dim;
  t.n_nodes = (size_t)n_nodes;
  t.offsets.assign(offsets, offsets + n_nodes);
  t.children.assign(children, children + 2 * (size_t)n_nodes);
  std::vector<int8_t> codes((size_t)n_nodes * (size_t)dim);
  std::vector<float> scales((size_t)n_nodes);
  quantize_hyperplanes(hyperplanes, (size_t)n_nodes, (size_t)dim, codes.data(), scales.data());
  FastRng rng(seed);
  std::vector<std::pair<size_t, size_t>> leaves;
  int ev = t.search_leaves_with(
      [&](size_t node) {
        return quantized_margin(codes.data(), scales.data(), t.offsets.data(), (size_t)dim, node, qcodes, qscale);
      },
      rng, (size_t)leaf_budget, leaves);
  for (size_t i = 0; i < leaves.size(); ++i) {
    out_leaves[2 * i] = (int32_t)leaves[i].first;
    out_leaves[2 * i + 1] = (int32_t)leaves[i].second;
  }
  *n_leaves = (int32_t)leaves.size();
  return ev;
}

void orc_quantize_tree_hyperplanes(int32_t n_nodes, int32_t dim, const float* hyperplanes, int8_t* codes,
                                   float* scales) {
  quantize_hyperplanes(hyperplanes, (size_t)n_nodes, (size_t)dim, codes, scales);
}

float orc_tree_hyperplane(const float* p1, const float* p2, int32_t dim, int32_t angular, float* hp) {
  return TreeBuilder::split_hyperplane(p1, p2, (size_t)dim, angular != 0, hp);
}

// flat_tree.rs:253-273 (leaf budget 1) for many points: the side of every node
// is margin > 0 (margin = dot_a + offset, builder.rs:331); a margin with
// |m| < 1e-8 is a random side in the reference, reported here as a tie
// (leaf_node = -1) instead of drawn.
void orc_tree_route_points(int32_t n_nodes, int32_t dim, const float* hyperplanes, const float* offsets,
                           const int32_t* children, const float* points, int64_t n, int32_t* leaf_node) {
  (void)n_nodes;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const float* x = points + (size_t)i * (size_t)dim;
    size_t node = 0;
    int32_t out = 0;
    while (children[2 * node] > 0) {
      const float margin = dot_a(x, hyperplanes + node * (size_t)dim, dim) + offsets[node];
      if (std::fabs(margin) < 1e-8f) {
        out = -1;
        break;
      }
      node = (size_t)children[2 * node + (margin > 0.f ? 1 : 0)];
    }
    leaf_node[i] = out < 0 ? -1 : (int32_t)node;
  }
}

int64_t orc_search_graph_from_knn(const int32_t* knn_idx, const float* knn_dist, const float* data,
                                  int32_t n, int32_t k, int32_t dim, int kind, float diversify_prob,
                                  float mult, int32_t* indptr, int32_t* indices, int64_t cap,
                                  float* min_distance) {
  CSR g = from_dense_diversified(knn_idx, knn_dist, data, (size_t)n, (size_t)k, (size_t)dim, kind,
                                 mult, num_threads_of(0), min_distance, diversify_prob, 42);
  std::memcpy(indptr, g.indptr.data(), sizeof(int32_t) * ((size_t)n + 1));
  int64_t nnz = (int64_t)g.indices.size();
  if (nnz <= cap) std::memcpy(indices, g.indices.data(), sizeof(int32_t) * (size_t)nnz);
  return nnz;
}

int64_t orc_weighted_union_pruned(int32_t n, const int32_t* fwd_ptr, const int32_t* fwd_idx,
                                  const float* fwd_dist, const int32_t* rev_ptr,
                                  const int32_t* rev_idx, const float* rev_dist,
                                  int32_t max_degree, int32_t* indptr, int32_t* indices) {
  std::vector<std::vector<std::pair<int32_t, float>>> f((size_t)n), r((size_t)n);
  for (int32_t v = 0; v < n; ++v) {
    for (int32_t e = fwd_ptr[v]; e < fwd_ptr[v + 1]; ++e) f[(size_t)v].push_back({fwd_idx[e], fwd_dist[e]});
    for (int32_t e = rev_ptr[v]; e < rev_ptr[v + 1]; ++e) r[(size_t)v].push_back({rev_idx[e], rev_dist[e]});
  }
  CSR g = weighted_union_pruned(f, r, (size_t)n, (size_t)max_degree);
  std::memcpy(indptr, g.indptr.data(), sizeof(int32_t) * ((size_t)n + 1));
  std::memcpy(indices, g.indices.data(), sizeof(int32_t) * g.indices.size());
  return (int64_t)g.indices.size();
}

void orc_params_default(orc_params* p) {  // index.rs:475-494
  p->n_neighbors = 30;
  p->n_trees = 8;
  p->n_search_trees = 1;
  p->search_tree_leaf_budget = 1;
  p->leaf_size = 0;
  p->max_candidates = 0;
  p->n_iters = 0;
  p->delta = 0.001f;
  p->random_seed = 42;
  p->diversify_prob = 1.0f;
  p->pruning_degree_multiplier = 1.5f;
  p->angular = 0;
  p->distance_kind = ORC_SQEUCLIDEAN;
  p->correction = ORC_CORR_SQRT;
  p->n_threads = 0;
  p->verbose = 0;
}

// index.rs:601-733 build_with_distance
orc_index* orc_build(const float* data, int64_t n_, int32_t dim_, const orc_params* p) {
  size_t n = (size_t)n_, dim = (size_t)dim_, k = (size_t)p->n_neighbors;
  int nt = num_threads_of(p->n_threads);
  orc_index* ix = new orc_index();
  ix->n = n;
  ix->dim = dim;
  ix->k = k;
  ix->kind = p->distance_kind;
  ix->corr = p->correction;
  ix->seed = p->random_seed;
  ix->nt = nt;
  ix->leaf_budget = (size_t)std::max(1, p->search_tree_leaf_budget);
  size_t leaf_size = p->leaf_size > 0 ? (size_t)p->leaf_size : std::max((size_t)60, std::min(5 * k, (size_t)256));
  size_t mc = p->max_candidates > 0 ? (size_t)p->max_candidates : std::min(k, (size_t)60);
  size_t n_iters = p->n_iters > 0 ? (size_t)p->n_iters
                                  : std::max((size_t)5, (size_t)std::ceil(std::log2((double)n)));
  FastRng rng(p->random_seed);
  // nndescent/mod.rs:79-197
  size_t emc = std::min(std::min(mc, (size_t)60), k);
  double t0 = now_s();
  std::vector<FlatTree> forest =
      build_rp_forest(data, n, dim, (size_t)p->n_trees, leaf_size, rng, p->angular != 0, 200, nt);
  double t1 = now_s();
  NeighborHeap g(n, k);
  auto leaves = rptree_leaf_array(forest);
  initialize_from_leaves(g, leaves, data, dim, ix->kind, nt);
  double t2 = now_s();
  size_t iters = 0;
  for (size_t it = 0; it < n_iters; ++it) {
    iters = it + 1;
    Cands c = build_candidates(g, emc, rng, nt);
    size_t changes = update_iteration(g, c, data, dim, ix->kind, nt);
    if (p->verbose) std::printf("Iteration %zu: %zu updates\n", it + 1, changes);
    size_t thr = (size_t)(p->delta * (float)k * (float)n);
    if (changes <= thr) break;
  }
  double t3 = now_s();
  ix->iters = (int)iters;
  g.sort_all();
  ix->graph = from_dense_diversified(g.indices.data(), g.distances.data(), data, n, k, dim, ix->kind,
                                     p->pruning_degree_multiplier, nt, &ix->min_distance, p->diversify_prob,
                                     p->random_seed);
  ix->nbr_idx = g.indices;
  ix->nbr_dist.resize(g.distances.size());
  for (size_t i = 0; i < g.distances.size(); ++i) ix->nbr_dist[i] = correct(ix->corr, g.distances[i]);
  size_t nst = std::min((size_t)std::max(0, p->n_search_trees), forest.size());
  ix->trees.assign(forest.begin(), forest.begin() + (long)nst);
  ix->vertex_order.resize(n);
  if (!ix->trees.empty())
    for (size_t i = 0; i < n; ++i) ix->vertex_order[i] = (size_t)ix->trees[0].indices[i];
  else
    std::iota(ix->vertex_order.begin(), ix->vertex_order.end(), (size_t)0);
  std::vector<size_t> old_to_new(n);
  for (size_t i = 0; i < n; ++i) old_to_new[ix->vertex_order[i]] = i;
  ix->data.resize(n * dim);
  for (size_t i = 0; i < n; ++i)
    std::memcpy(&ix->data[i * dim], data + ix->vertex_order[i] * dim, sizeof(float) * dim);
  ix->graph.n = n;
  csr_reorder(ix->graph, ix->vertex_order);
  for (auto& t : ix->trees)
    for (auto& v : t.indices) v = (int32_t)old_to_new[(size_t)v];
  double t4 = now_s();
  ix->t[0] = t1 - t0;
  ix->t[1] = t2 - t1;
  ix->t[2] = t3 - t2;
  ix->t[3] = t4 - t3;
  ix->t[4] = t4 - t0;
  return ix;
}

// A search-only index from another index's parts (test infrastructure: the GPU
// search and this search on one shared graph and tree set).  Rows, CSR and
// tree leaf orders are in the index's internal order; vertex_order maps
// internal ids to original ids (index.rs:679-715); the trees' nodes are
// concatenated (tree_nodes[t] nodes each) in FlatTree layout (flat_tree.rs:14-28).
orc_index* orc_index_from_parts(const float* data, int64_t n_, int32_t dim_, int32_t kind, int32_t corr,
                                const int32_t* indptr, const int32_t* indices, float min_distance, int32_t n_trees,
                                const int64_t* tree_nodes, const float* hyperplanes, const float* offsets,
                                const int32_t* children, const int32_t* tree_indices, int32_t leaf_budget,
                                const int32_t* vertex_order, uint64_t seed, int32_t n_threads) {
  const size_t n = (size_t)n_, dim = (size_t)dim_;
  orc_index* ix = new orc_index();
  ix->n = n;
  ix->dim = dim;
  ix->kind = kind;
  ix->corr = corr;
  ix->seed = seed;
  ix->nt = num_threads_of(n_threads);
  ix->leaf_budget = (size_t)std::max(1, leaf_budget);
  ix->min_distance = min_distance;
  ix->data.assign(data, data + n * dim);
  ix->graph.n = n;
  ix->graph.indptr.assign(indptr, indptr + n + 1);
  ix->graph.indices.assign(indices, indices + (size_t)indptr[n]);
  size_t node0 = 0;
  for (int32_t t = 0; t < n_trees; ++t) {
    FlatTree ft;
    ft.dim = dim;
    ft.n_nodes = (size_t)tree_nodes[t];
    ft.hyperplanes.assign(hyperplanes + node0 * dim, hyperplanes + (node0 + ft.n_nodes) * dim);
    ft.offsets.assign(offsets + node0, offsets + node0 + ft.n_nodes);
    ft.children.assign(children + 2 * node0, children + 2 * (node0 + ft.n_nodes));
    ft.indices.assign(tree_indices + (size_t)t * n, tree_indices + (size_t)(t + 1) * n);
    ix->trees.push_back(std::move(ft));
    node0 += (size_t)tree_nodes[t];
  }
  ix->vertex_order.resize(n);
  for (size_t i = 0; i < n; ++i) ix->vertex_order[i] = (size_t)vertex_order[i];
  return ix;
}

void orc_free(orc_index* idx) { delete idx; }
int32_t orc_index_k(const orc_index* idx) { return (int32_t)idx->k; }
int32_t orc_iterations(const orc_index* idx) { return idx->iters; }
void orc_timings(const orc_index* idx, double* out5) {
  for (int i = 0; i < 5; ++i) out5[i] = idx->t[i];
}

void orc_neighbor_graph(const orc_index* idx, int32_t* out_idx, float* out_dist) {
  std::memcpy(out_idx, idx->nbr_idx.data(), sizeof(int32_t) * idx->nbr_idx.size());
  std::memcpy(out_dist, idx->nbr_dist.data(), sizeof(float) * idx->nbr_dist.size());
}

int64_t orc_search_graph_nnz(const orc_index* idx) { return (int64_t)idx->graph.indices.size(); }

// index.rs:137-141 search_graph_original_order
void orc_search_graph(const orc_index* idx, int32_t* indptr, int32_t* indices, float* min_distance) {
  CSR g = idx->graph;
  std::vector<size_t> o2i(idx->n);
  for (size_t i = 0; i < idx->n; ++i) o2i[idx->vertex_order[i]] = i;
  csr_reorder(g, o2i);
  std::memcpy(indptr, g.indptr.data(), sizeof(int32_t) * (idx->n + 1));
  std::memcpy(indices, g.indices.data(), sizeof(int32_t) * g.indices.size());
  *min_distance = idx->min_distance;
}

void orc_vertex_order(const orc_index* idx, int32_t* out) {
  for (size_t i = 0; i < idx->n; ++i) out[i] = (int32_t)idx->vertex_order[i];
}

// index.rs:406-439 query (serial for <= 4 queries, parallel otherwise; same per-query seeds)
void orc_query(const orc_index* idx, const float* queries, int64_t nq, int32_t k, float epsilon,
               int32_t* out_idx, float* out_dist) {
#pragma omp parallel num_threads(idx->nt)
  {
    Workspace ws(idx->n, (size_t)k);
#pragma omp for schedule(dynamic, 16)
    for (long i = 0; i < (long)nq; ++i)
      process_query(idx, queries + (size_t)i * idx->dim, (size_t)i, (size_t)k, epsilon, ws,
                    out_idx + (size_t)i * (size_t)k, out_dist + (size_t)i * (size_t)k);
  }
}

void orc_query_one(const orc_index* idx, const float* query, int32_t k, float epsilon,
                   int32_t* out_idx, float* out_dist) {
  Workspace ws(idx->n, (size_t)k);
  process_query(idx, query, 0, (size_t)k, epsilon, ws, out_idx, out_dist);
}

// crates/rinnd/src/lib.rs:159-223 QuantizedI8Index::new (encode rows)
void orc_quantize_rows(const float* data, int64_t n, int32_t dim, int32_t encoding, int8_t* codes,
                       float* inv_norms, float* global_mult) {
  float gmax = 0.f;
  for (int64_t i = 0; i < n * dim; ++i) gmax = std::max(gmax, std::fabs(data[i]));
  float gm = gmax > 0.f ? 127.0f / gmax : 0.f;
  float gds = gm > 0.f ? 1.0f / gm : 0.f;
  for (int64_t r = 0; r < n; ++r) {
    const float* row = data + r * dim;
    float mult;
    if (encoding == 1) {
      mult = gm;
    } else {
      float mx = 0.f;
      for (int j = 0; j < dim; ++j) mx = std::max(mx, std::fabs(row[j]));
      mult = mx > 0.f ? 127.0f / mx : 0.f;
    }
    int8_t* c = codes + r * dim;
    for (int j = 0; j < dim; ++j) {
      float v = std::round(row[j] * mult);
      v = std::min(std::max(v, -127.0f), 127.0f);
      c[j] = (int8_t)v;
    }
    if (encoding == 0) {
      int32_t nsq = i8_dot(c, c, dim);
      inv_norms[r] = nsq > 0 ? 1.0f / std::sqrt((float)nsq) : 0.f;
    } else if (encoding == 2) {
      inv_norms[r] = mult > 0.f ? 1.0f / mult : 0.f;
    } else {
      inv_norms[r] = gds;
    }
  }
  *global_mult = gm;
}

// lib.rs:325-358 quantize_query: the row multiplier of the per-vector encodings or
// the index's global multiplier (sq8u); scale = 1/sqrt(sum code^2), 1/multiplier
// or the global dequantization scale.
void orc_quantize_queries(const float* queries, int64_t nq, int32_t dim, int32_t encoding, float global_mult,
                          int8_t* codes, float* scales) {
  const float gds = global_mult > 0.f ? 1.0f / global_mult : 0.f;
  for (int64_t r = 0; r < nq; ++r) {
    const float* q = queries + r * dim;
    float mult = global_mult;
    if (encoding != 1) {
      float mx = 0.f;
      for (int j = 0; j < dim; ++j) mx = std::max(mx, std::fabs(q[j]));
      mult = mx > 0.f ? 127.0f / mx : 0.f;
    }
    int8_t* c = codes + r * dim;
    for (int j = 0; j < dim; ++j) {
      float v = std::round(q[j] * mult);
      c[j] = (int8_t)std::min(std::max(v, -127.0f), 127.0f);
    }
    int32_t nsq = i8_dot(c, c, dim);
    scales[r] = encoding == 0 ? (nsq > 0 ? 1.0f / std::sqrt((float)nsq) : 0.f)
                              : (encoding == 1 ? gds : (mult > 0.f ? 1.0f / mult : 0.f));
  }
}

// Per-dimension symmetric int8 encoding, the operand format of
// quantized_i8_per_dimension_dot (core/distance/quantized.rs:42-56: one
// dequantization scale per dimension, shared by queries and rows).  The
// reference has no production encoder for it; this one follows its other
// symmetric encoders (lib.rs:185-199, flat_tree.rs:47-64): scale_j = max_i |x_ij| / 127
// over the index rows (0 when the column is zero), code = clamp(round(x / scale_j),
// -127, 127) with round half away from zero, 0 where scale_j = 0.
void orc_quantize_per_dimension(const float* data, int64_t n, int32_t dim, int8_t* codes, float* dim_scales) {
  for (int j = 0; j < dim; ++j) {
    float mx = 0.f;
    for (int64_t r = 0; r < n; ++r) mx = std::max(mx, std::fabs(data[r * dim + j]));
    dim_scales[j] = mx > 0.f ? mx / 127.0f : 0.f;
  }
  orc_quantize_queries_per_dimension(data, n, dim, dim_scales, codes);
}

void orc_quantize_queries_per_dimension(const float* queries, int64_t nq, int32_t dim, const float* dim_scales,
                                        int8_t* codes) {
  for (int64_t r = 0; r < nq; ++r)
    for (int j = 0; j < dim; ++j) {
      const float sc = dim_scales[j];
      float v = sc > 0.f ? std::round(queries[r * dim + j] / sc) : 0.f;
      if (v != v) v = 0.f;
      codes[r * dim + j] = (int8_t)std::min(std::max(v, -127.0f), 127.0f);
    }
}

// lib.rs:1131-1146 normalize_rows_inplace: sequential f32 sum of squares; rows
// with norm^2 <= 1e-12 are left unchanged; x *= 1/sqrt(norm^2).
void orc_normalize_rows(float* data, int64_t n, int32_t dim) {
  for (int64_t r = 0; r < n; ++r) {
    float* row = data + r * dim;
    float nsq = 0.f;
    for (int j = 0; j < dim; ++j) nsq += row[j] * row[j];
    if (nsq <= 1e-12f) continue;
    float inv = 1.0f / std::sqrt(nsq);
    for (int j = 0; j < dim; ++j) row[j] *= inv;
  }
}

// lib.rs:325-358 quantize_query + index.rs:283-334 + greedy.rs:365-413 + index.rs:103-126.
// The index must have been built with ORC_DIRECT_COSINE on normalized rows.  Search
// trees are the FP32 trees (tree_quantization="none").  Returns 0, or -1 when the
// width combination is invalid (index.rs:55-78).
int32_t orc_query_quantized(const orc_index* ix, const float* queries, int64_t nq, int32_t k,
                            float epsilon, int32_t encoding, int32_t candidate_width,
                            int32_t rerank_width, int32_t* out_idx, float* out_dist) {
  return orc_query_quantized_trees(ix, queries, nq, k, epsilon, encoding, candidate_width, rerank_width, 0, out_idx,
                                   out_dist);
}

// With quantize_trees != 0 the search trees route over int8 routing trees
// (QuantizedFlatTree, flat_tree.rs:35-183; lib.rs:231-240) with the query's
// int8 codes and tree_query_scale = max|q| / 127 (lib.rs:283-296, greedy.rs:109-146).
int32_t orc_query_quantized_trees(const orc_index* ix, const float* queries, int64_t nq, int32_t k,
                                  float epsilon, int32_t encoding, int32_t candidate_width,
                                  int32_t rerank_width, int32_t quantize_trees, int32_t* out_idx, float* out_dist) {
  size_t resolved = candidate_width == 0 ? (size_t)std::max(k, rerank_width) : (size_t)candidate_width;
  if (resolved < (size_t)k || (size_t)rerank_width > resolved ||
      !(candidate_width == 0 || rerank_width == 0 || rerank_width >= k))
    return -1;
  bool rerank = candidate_width == 0 ? rerank_width > k : rerank_width > 0;
  size_t dim = ix->dim, n = ix->n;
  std::vector<int8_t> codes(n * dim);
  std::vector<float> inv(n), dsc(dim);
  float gm = 0.f;
  const bool per_dim = encoding == 3;
  if (per_dim) orc_quantize_per_dimension(ix->data.data(), (int64_t)n, (int32_t)dim, codes.data(), dsc.data());
  else orc_quantize_rows(ix->data.data(), (int64_t)n, (int32_t)dim, encoding, codes.data(), inv.data(), &gm);
  float gds = gm > 0.f ? 1.0f / gm : 0.f;
  Workspace ws(n, resolved);
  std::vector<int8_t> qc(dim);
  std::vector<std::vector<int8_t>> tcodes(ix->trees.size());
  std::vector<std::vector<float>> tscales(ix->trees.size());
  if (quantize_trees)
    for (size_t t = 0; t < ix->trees.size(); ++t) {
      const FlatTree& tr = ix->trees[t];
      tcodes[t].resize(tr.n_nodes * dim);
      tscales[t].resize(tr.n_nodes);
      quantize_hyperplanes(tr.hyperplanes.data(), tr.n_nodes, dim, tcodes[t].data(), tscales[t].data());
    }
  for (int64_t qi = 0; qi < nq; ++qi) {
    const float* q = queries + qi * (int64_t)dim;
    float mult;
    if (encoding == 1) {
      mult = gm;
    } else {
      float mx = 0.f;
      for (size_t j = 0; j < dim; ++j) mx = std::max(mx, std::fabs(q[j]));
      mult = mx > 0.f ? 127.0f / mx : 0.f;
    }
    for (size_t j = 0; j < dim; ++j) {
      float v = std::round(q[j] * mult);
      qc[j] = (int8_t)std::min(std::max(v, -127.0f), 127.0f);
    }
    if (per_dim) orc_quantize_queries_per_dimension(q, 1, (int32_t)dim, dsc.data(), qc.data());
    int32_t nsq = i8_dot(qc.data(), qc.data(), (int)dim);
    float qinv = encoding == 0 ? (nsq > 0 ? 1.0f / std::sqrt((float)nsq) : 0.f)
                               : (encoding == 1 ? gds : (mult > 0.f ? 1.0f / mult : 0.f));
    FastRng rng(ix->seed);  // index.rs:298: quantized queries seed with rng_seed only
    ws.reset(resolved);
    auto dist_to = [&](int32_t i) {
      // per-dimension codes: the reconstructed inner product (quantized.rs:48-56)
      float sim = per_dim ? orc_i8_per_dimension_dot(qc.data(), &codes[(size_t)i * dim], dsc.data(), (int32_t)dim)
                          : (float)i8_dot(qc.data(), &codes[(size_t)i * dim], (int)dim) * qinv * inv[(size_t)i];
      return 1.0f - std::min(std::max(sim, -1.0f), 1.0f);
    };
    float tqs = 0.f;
    if (quantize_trees) {
      float mx = 0.f;
      for (size_t j = 0; j < dim; ++j) mx = std::max(mx, std::fabs(q[j]));
      tqs = mx > 0.f ? mx / 127.0f : 0.f;
    }
    for (size_t ti = 0; ti < ix->trees.size(); ++ti) {
      const FlatTree& t = ix->trees[ti];
      if (quantize_trees)
        t.search_leaves_with(
            [&](size_t node) {
              return quantized_margin(tcodes[ti].data(), tscales[ti].data(), t.offsets.data(), dim, node, qc.data(),
                                      tqs);
            },
            rng, ix->leaf_budget, ws.leaves);
      else
        t.search_leaves(q, rng, ix->leaf_budget, ws.leaves);
      for (auto& l : ws.leaves)
        for (size_t p = l.first; p < l.second; ++p) {
          int32_t idx = t.indices[p];
          if (idx >= 0 && !ws.visited.check_and_mark(idx)) {
            float d = dist_to(idx);
            ws.result.push(d, idx);
            ws.seeds.push({d, idx});
          }
        }
    }
    fill_random(n, resolved, dist_to, rng, ws);
    traverse(ix->graph, epsilon, ix->min_distance, dist_to, ws);
    std::vector<int32_t> ids;
    std::vector<float> ds;
    ws.result.into_sorted(ids, ds);
    if (rerank) {  // index.rs:103-126
      std::vector<std::pair<float, int32_t>> rr;
      for (int32_t id : ids) {
        if (id < 0) continue;
        if (rr.size() >= (size_t)rerank_width) break;
        rr.push_back({distance_impl(ix->kind, q, &ix->data[(size_t)id * dim], (int)dim), id});
      }
      std::sort(rr.begin(), rr.end(), [](const auto& a, const auto& b) {
        int c = total_cmp_f(a.first, b.first);
        return c != 0 ? c < 0 : a.second < b.second;
      });
      if (rr.size() > (size_t)k) rr.resize((size_t)k);
      ids.clear();
      ds.clear();
      for (auto& e : rr) {
        ids.push_back(e.second);
        ds.push_back(e.first);
      }
    }
    int32_t* oi = out_idx + qi * k;
    float* od = out_dist + qi * k;
    for (int32_t j = 0; j < k; ++j) {
      if ((size_t)j < ids.size()) {
        oi[j] = ids[(size_t)j] >= 0 ? (int32_t)ix->vertex_order[(size_t)ids[(size_t)j]] : ids[(size_t)j];
        od[j] = ds[(size_t)j];
      } else {
        oi[j] = -1;
        od[j] = INFINITY;
      }
    }
  }
  return 0;
}

// FP64 exact kNN: base metric in double precision (ranking-equivalent to the
// proxies for euclidean/cosine/inner-product).  Ties broken by id.
void orc_exact_knn_f64(int kind, const float* data, int64_t n, const float* queries, int64_t nq,
                       int32_t dim, int32_t k, int32_t exclude_self, int32_t* out_idx,
                       double* out_dist) {
  std::vector<double> nrm;
  bool angular = kind == ORC_COSINE || kind == ORC_ALT_COSINE || kind == ORC_ALT_DOT ||
                 kind == ORC_DIRECT_COSINE;
  if (angular) {
    nrm.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      double s = 0;
      for (int j = 0; j < dim; ++j) s += (double)data[i * dim + j] * data[i * dim + j];
      nrm[(size_t)i] = std::sqrt(s);
    }
  }
#pragma omp parallel
  {
    std::vector<std::pair<double, int32_t>> best;
#pragma omp for schedule(dynamic, 4)
    for (long qi = 0; qi < (long)nq; ++qi) {
      const float* q = queries + qi * dim;
      double qn = 0;
      if (angular) {
        for (int j = 0; j < dim; ++j) qn += (double)q[j] * q[j];
        qn = std::sqrt(qn);
      }
      best.clear();
      for (int64_t i = 0; i < n; ++i) {
        if (exclude_self && i == qi) continue;
        const float* x = data + i * dim;
        double d = 0;
        if (kind == ORC_SQEUCLIDEAN) {
          for (int j = 0; j < dim; ++j) {
            double t = (double)q[j] - x[j];
            d += t * t;
          }
        } else if (kind == ORC_MANHATTAN) {
          for (int j = 0; j < dim; ++j) d += std::fabs((double)q[j] - x[j]);
        } else {
          double dot = 0;
          for (int j = 0; j < dim; ++j) dot += (double)q[j] * x[j];
          if (angular) {
            double den = qn * nrm[(size_t)i];
            d = den > 0 ? 1.0 - dot / den : 1.0;
          } else {
            d = -dot;
          }
        }
        std::pair<double, int32_t> e{d, (int32_t)i};
        if ((int32_t)best.size() < k) {
          best.push_back(e);
          std::push_heap(best.begin(), best.end());
        } else if (e < best.front()) {
          std::pop_heap(best.begin(), best.end());
          best.back() = e;
          std::push_heap(best.begin(), best.end());
        }
      }
      std::sort(best.begin(), best.end());
      for (int32_t j = 0; j < k; ++j) {
        if ((size_t)j < best.size()) {
          out_idx[qi * k + j] = best[(size_t)j].second;
          out_dist[qi * k + j] = best[(size_t)j].first;
        } else {
          out_idx[qi * k + j] = -1;
          out_dist[qi * k + j] = INFINITY;
        }
      }
    }
  }
}

}  // extern "C"
