// brute.cu -- brute-force exact kNN: every query against every row.
//
// No counterpart in the reference, which has no exact pass; the exact
// neighbors are what its recall criteria are measured against.  For each
// query the k rows of smallest (distance, id), in that order.
//
// Tiles.  A CTA holds 64 queries (FP32; 32 in FP64) and walks its share of
// the rows in chunks of 64 (the rows of a large call are split over gridDim.y
// CTAs per query tile when there are few query tiles, and the splits merged
// after).  Query and row tiles are staged in shared memory 64 dimensions at a
// time, so any D fits; each thread accumulates a 4 x 4 (2 x 4) block of
// (query, row) pairs, its rows 16 apart so a warp's 16-byte reads of them
// spread over all banks.  Two arithmetics:
//   FP32: the FP32 join's per-pair arithmetic (join_dist_fp32: packed
//     accumulators over dimension pairs (4q, 4q+1) and (4q+2, 4q+3), summed at
//     the end; dot forms finalized with FP32 squared norms), so a distance
//     equals the one the build would compute for that pair;
//   FP64: every term in double and accumulated sequentially -- the checker
//     that the FP32 form's ids are compared with.
// Selection.  After each chunk, the pairs whose key beats the query's current
// k-th key are staged (at most 64 a query), sorted by a warp, and merged into
// the query's sorted list of k keys (merge path: each output position finds
// its split by binary search); the k-th key then filters the next chunks.
// Metrics: squared Euclidean and Manhattan (difference form), inner product,
// cosine and direct cosine (dot form).
//
// Tensor-core form (BF16 filter + FP32 recheck; D <= 128, k <= 32; squared
// Euclidean and the dot forms).  Rows and queries get a BF16 copy written in
// the tcgen05 operand layout (K-major core matrices, no swizzle), one 128-row
// tile after another, with per row |b|^2 and a bound e >= |b - x| of its
// rounding error.  A CTA holds 128 queries as the A operand and streams 128-row
// tiles as B, each arriving with one bulk copy on an mbarrier (two stages);
// one thread issues the M = 128, N = 128 MMAs (FP32 accumulate) into two
// tensor-memory accumulators; eight epilogue warps each read 64 columns of
// their lane quadrant (lane = query).  A pair survives when its lower bound --
// the local join's (join_tc.cu): squared Euclidean |b_i - b_j| from the Gram
// value with its FP32 error and the rows' rounding bounds, dot forms from an
// upper bound of the dot -- beats the k-th key of the query's list; survivors
// are recomputed with the FP32 form's arithmetic and inserted by (distance,
// id).  Each (query, epilogue half) keeps its own list and the two are merged
// at the end, so the results equal the FP32 form's exactly.
#include <cuda_bf16.h>

#include "dist.cuh"
#include "engine.h"
#include "join_common.cuh"
#include "tcgen05.cuh"

namespace rinnd {
namespace {

using namespace joinc;

constexpr int BF_RT = 64;   // rows per chunk
constexpr int BF_NT = 256;  // threads: thread t takes queries QT/16 (t / 16) + i and rows t % 16 + 16 j, j < 4
constexpr int BF_KC = 64;   // dimensions staged at a time
constexpr int BF_KS = BF_KC + 4;  // staged row stride (floats): conflict-free 16-byte reads
constexpr int BF_KMAX = 128;      // largest k
enum BfMode { BF_SQ = 0, BF_MAN = 1, BF_DOT = 2 };

template <typename T>
struct BfKey {
  T d;
  int32_t id;
};
template <typename T>
__device__ __forceinline__ bool key_less(const BfKey<T>& a, const BfKey<T>& b) {
  return a.d < b.d || (a.d == b.d && a.id < b.id);
}
template <typename T>
__device__ __forceinline__ BfKey<T> key_max() {
  return BfKey<T>{(T)INFINITY, 0x7FFFFFFF};
}

bool bf_dot_kind(int kind) { return kind == DK_INNER_PRODUCT || kind == DK_COSINE || kind == DK_DIRECT_COSINE; }

template <typename T>
__device__ __forceinline__ T bf_finalize(int kind, T dot, T na, T nb) {
  if (kind == DK_INNER_PRODUCT) return -dot;
  if (kind == DK_DIRECT_COSINE) return (T)1 - fmin(fmax(dot, (T)-1), (T)1);
  const T denom = sqrt(na * nb);  // cosine.rs:76-79
  if (denom < (T)1e-12) return (T)1;
  return (T)1 - fmin(fmax(dot / denom, (T)-1), (T)1);
}
template <>
__device__ __forceinline__ float bf_finalize<float>(int kind, float dot, float na, float nb) {
  return finalize_dot(kind, dot, na, nb);
}

// Squared norms of rows (the dot forms' normalization), one warp per row: the
// build's order (lane-strided fma, then a shuffle reduction), in T.
template <typename T>
__global__ void k_bf_norms(const float* __restrict__ X, long long n, int Dp, T* __restrict__ out) {
  const long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n) return;
  const float* x = X + (size_t)r * Dp;
  T s = (T)0;
  for (int t = lane; t < Dp; t += 32) s = fma((T)x[t], (T)x[t], s);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) out[r] = s;
}

struct BfArgs {
  const float* Q;       // nq x Dp
  const float* X;       // n x Dp
  const void* qn;       // squared norms (dot forms), T
  const void* xn;
  const int32_t* excl;  // per query: a row id to leave out, or null
  long long n;
  int nq, Dp, k, kind, splits;
  void* out_key;        // splits > 1: nq x splits x k partial lists (BfKey<T>)
  int32_t* out_idx;     // splits == 1: final results
  float* out_dist;
};

template <typename T, int MODE, int QT>
__global__ void __launch_bounds__(BF_NT) k_brute(BfArgs a) {
  constexpr int QPT = QT / 16;  // queries per thread
  extern __shared__ __align__(16) unsigned char smem[];
  float* sq = reinterpret_cast<float*>(smem);                  // QT x BF_KS
  float* sx = sq + QT * BF_KS;                                  // BF_RT x BF_KS
  BfKey<T>* cand = reinterpret_cast<BfKey<T>*>(sx + BF_RT * BF_KS);  // QT x BF_RT
  BfKey<T>* list = cand + QT * BF_RT;                           // QT x k
  int* ccount = reinterpret_cast<int*>(list + (size_t)QT * a.k);  // QT
  int* lcount = ccount + QT;                                    // QT
  BfKey<T>* thr = reinterpret_cast<BfKey<T>*>(lcount + QT + 2);     // QT (8-byte aligned)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q0 = blockIdx.x * QT;
  const long long per = (a.n + a.splits - 1) / a.splits;
  const long long r_lo = (long long)blockIdx.y * per, r_hi = min(a.n, r_lo + per);
  const int tq = QPT * (tid >> 4), tr = tid & 15;
  const T* qn = reinterpret_cast<const T*>(a.qn);
  const T* xn = reinterpret_cast<const T*>(a.xn);
  for (int t = tid; t < QT; t += BF_NT) {
    ccount[t] = 0;
    lcount[t] = 0;
    thr[t] = key_max<T>();
  }
  __syncthreads();
  int32_t my_excl[QPT];
#pragma unroll
  for (int i = 0; i < QPT; ++i) my_excl[i] = (a.excl && q0 + tq + i < a.nq) ? a.excl[q0 + tq + i] : -1;
  for (long long r0 = r_lo; r0 < r_hi; r0 += BF_RT) {
    // ---- distances of the QT x 64 tile, 64 dimensions at a time ----
    unsigned long long accf[QPT][4];
    T accd[QPT][4];
#pragma unroll
    for (int i = 0; i < QPT; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        accf[i][j] = 0ull;
        accd[i][j] = (T)0;
      }
    for (int k0 = 0; k0 < a.Dp; k0 += BF_KC) {
      const int kc = min(BF_KC, a.Dp - k0);  // a multiple of 4
      __syncthreads();
      for (int e = tid; e < QT * (BF_KC / 4); e += BF_NT) {
        const int qi = e / (BF_KC / 4), c = 4 * (e % (BF_KC / 4));
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < kc && q0 + qi < a.nq) v = *reinterpret_cast<const float4*>(a.Q + (size_t)(q0 + qi) * a.Dp + k0 + c);
        *reinterpret_cast<float4*>(sq + qi * BF_KS + c) = v;
      }
      for (int e = tid; e < BF_RT * (BF_KC / 4); e += BF_NT) {
        const int ri = e / (BF_KC / 4), c = 4 * (e % (BF_KC / 4));
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c < kc && r0 + ri < r_hi) v = *reinterpret_cast<const float4*>(a.X + (size_t)(r0 + ri) * a.Dp + k0 + c);
        *reinterpret_cast<float4*>(sx + ri * BF_KS + c) = v;
      }
      __syncthreads();
      for (int c = 0; c < kc; c += 4) {
        if constexpr (sizeof(T) == 4) {
          // join_dist_fp32's arithmetic on (x0, x1) and (x2, x3) as packed pairs
          ulonglong2 qv[QPT], xv[4];
#pragma unroll
          for (int i = 0; i < QPT; ++i) qv[i] = *reinterpret_cast<const ulonglong2*>(sq + (tq + i) * BF_KS + c);
#pragma unroll
          for (int j = 0; j < 4; ++j) xv[j] = *reinterpret_cast<const ulonglong2*>(sx + (tr + 16 * j) * BF_KS + c);
#pragma unroll
          for (int i = 0; i < QPT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              if (MODE == BF_SQ) {
                const unsigned long long d01 = f2_sub(xv[j].x, qv[i].x), d23 = f2_sub(xv[j].y, qv[i].y);
                accf[i][j] = f2_fma(d01, d01, accf[i][j]);
                accf[i][j] = f2_fma(d23, d23, accf[i][j]);
              } else if (MODE == BF_MAN) {
                const unsigned long long absmask = 0x7FFFFFFF7FFFFFFFull;
                accf[i][j] = f2_add(accf[i][j], f2_sub(xv[j].x, qv[i].x) & absmask);
                accf[i][j] = f2_add(accf[i][j], f2_sub(xv[j].y, qv[i].y) & absmask);
              } else {
                accf[i][j] = f2_fma(xv[j].x, qv[i].x, accf[i][j]);
                accf[i][j] = f2_fma(xv[j].y, qv[i].y, accf[i][j]);
              }
            }
        } else {
          float4 qv[QPT], xv[4];
#pragma unroll
          for (int i = 0; i < QPT; ++i) qv[i] = *reinterpret_cast<const float4*>(sq + (tq + i) * BF_KS + c);
#pragma unroll
          for (int j = 0; j < 4; ++j) xv[j] = *reinterpret_cast<const float4*>(sx + (tr + 16 * j) * BF_KS + c);
#pragma unroll
          for (int i = 0; i < QPT; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float xs[4] = {xv[j].x, xv[j].y, xv[j].z, xv[j].w};
              const float qs[4] = {qv[i].x, qv[i].y, qv[i].z, qv[i].w};
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const T dx = (T)xs[u] - (T)qs[u];
                if (MODE == BF_SQ) accd[i][j] = fma(dx, dx, accd[i][j]);
                else if (MODE == BF_MAN) accd[i][j] = accd[i][j] + fabs(dx);
                else accd[i][j] = fma((T)xs[u], (T)qs[u], accd[i][j]);
              }
            }
        }
      }
    }
    // ---- keys that beat the query's k-th key -> the query's staging list ----
#pragma unroll
    for (int i = 0; i < QPT; ++i) {
      const int qi = tq + i;
      if (q0 + qi >= a.nq) continue;
      const BfKey<T> t = thr[qi];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const long long r = r0 + tr + 16 * j;
        if (r >= r_hi || (int32_t)r == my_excl[i]) continue;
        T d;
        if constexpr (sizeof(T) == 4) d = f2_sum(accf[i][j]);
        else d = accd[i][j];
        if (MODE == BF_DOT) d = bf_finalize<T>(a.kind, d, xn[r], qn[q0 + qi]);
        if (d != d) d = (T)INFINITY;  // NaN ranks last
        const BfKey<T> key{d, (int32_t)r};
        if (key_less(key, t)) cand[qi * BF_RT + atomicAdd(&ccount[qi], 1)] = key;
      }
    }
    __syncthreads();
    // ---- merge: warp w takes queries w, w + 8, ... ----
    for (int qi = warp; qi < QT; qi += BF_NT / 32) {
      const int nc = ccount[qi];
      if (nc == 0) continue;
      BfKey<T>* c = cand + qi * BF_RT;
      for (int e = nc + lane; e < BF_RT; e += 32) c[e] = key_max<T>();
      __syncwarp();
      // bitonic sort of the 64 staged keys
      for (int size = 2; size <= BF_RT; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          for (int e = lane; e < BF_RT; e += 32) {
            const int p = e ^ stride;
            if (p > e) {
              const bool up = (e & size) == 0;
              const BfKey<T> x = c[e], y = c[p];
              if (key_less(y, x) == up) {
                c[e] = y;
                c[p] = x;
              }
            }
          }
          __syncwarp();
        }
      // merge path of (list[0, nl), c[0, nc)) -> the first min(nl + nc, k)
      BfKey<T>* L = list + (size_t)qi * a.k;
      const int nl = lcount[qi], nout = min(nl + nc, a.k);
      BfKey<T> outv[BF_KMAX / 32];
#pragma unroll
      for (int t = 0; t < BF_KMAX / 32; ++t) {
        const int p = lane + 32 * t;
        if (p >= nout) continue;
        int lo = max(0, p - nc), hi = min(p, nl);  // i = list elements before position p
        while (lo < hi) {
          const int i = (lo + hi) >> 1;
          // take more from the list while list[i] < c[p - 1 - i]
          if (key_less(L[i], c[p - 1 - i])) lo = i + 1; else hi = i;
        }
        const int i = lo, j = p - i;
        const bool from_list = j >= nc || (i < nl && key_less(L[i], c[j]));
        outv[t] = from_list ? L[i] : c[j];
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < BF_KMAX / 32; ++t) {
        const int p = lane + 32 * t;
        if (p < nout) L[p] = outv[t];
      }
      __syncwarp();
      if (lane == 0) {
        lcount[qi] = nout;
        ccount[qi] = 0;
        if (nout == a.k) thr[qi] = L[a.k - 1];
      }
    }
    __syncthreads();
  }
  // ---- results ----
  for (int qi = warp; qi < QT; qi += BF_NT / 32) {
    if (q0 + qi >= a.nq) continue;
    const BfKey<T>* L = list + (size_t)qi * a.k;
    const int nl = lcount[qi];
    for (int p = lane; p < a.k; p += 32) {
      const BfKey<T> key = p < nl ? L[p] : BfKey<T>{(T)INFINITY, -1};
      if (a.splits > 1) {
        reinterpret_cast<BfKey<T>*>(a.out_key)[((size_t)(q0 + qi) * a.splits + blockIdx.y) * a.k + p] = key;
      } else {
        a.out_idx[(size_t)(q0 + qi) * a.k + p] = key.id;
        a.out_dist[(size_t)(q0 + qi) * a.k + p] = (float)key.d;
      }
    }
  }
}

// The splits' sorted lists of one query -> its first k keys (warp per query;
// lane l holds the heads of splits l, l + 32, l + 64, l + 96): repeatedly the
// smallest head, by a reduction within the lane and then over the warp.
constexpr int BF_MAXSPLIT = 128;
template <typename T>
__global__ void k_brute_merge(const BfKey<T>* __restrict__ part, int nq, int splits, int k, int32_t* out_idx,
                              float* out_dist) {
  const int q = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (q >= nq) return;
  const BfKey<T>* P = part + (size_t)q * splits * k;
  int head[BF_MAXSPLIT / 32] = {0, 0, 0, 0};
  auto head_key = [&](int u) {
    const int sp = lane + 32 * u;
    BfKey<T> key{(T)INFINITY, 0x7FFFFFFF};
    if (sp < splits && head[u] < k) {
      key = P[(size_t)sp * k + head[u]];
      if (key.id < 0) key = BfKey<T>{(T)INFINITY, 0x7FFFFFFF};
    }
    return key;
  };
  for (int p = 0; p < k; ++p) {
    BfKey<T> best = head_key(0);
    int src = lane;  // split number of the best head
#pragma unroll
    for (int u = 1; u < BF_MAXSPLIT / 32; ++u) {
      const BfKey<T> h = head_key(u);
      if (key_less(h, best)) {
        best = h;
        src = lane + 32 * u;
      }
    }
    for (int o = 16; o; o >>= 1) {
      const T od = __shfl_xor_sync(0xffffffffu, best.d, o);
      const int32_t oi = __shfl_xor_sync(0xffffffffu, best.id, o);
      const int os = __shfl_xor_sync(0xffffffffu, src, o);
      const BfKey<T> other{od, oi};
      if (key_less(other, best) || (!key_less(best, other) && os < src)) {
        best = other;
        src = os;
      }
    }
#pragma unroll
    for (int u = 0; u < BF_MAXSPLIT / 32; ++u)
      if (src == lane + 32 * u) ++head[u];
    if (lane == 0) {
      const bool empty = best.id == 0x7FFFFFFF;
      out_idx[(size_t)q * k + p] = empty ? -1 : best.id;
      out_dist[(size_t)q * k + p] = empty ? __int_as_float(0x7f800000) : (float)best.d;
    }
  }
}

// Row splits per query tile: the fewest in [1, 128] (the merge kernel's limit,
// and at least `min_tiles` row tiles a split) whose CTAs fill 90 % of the
// resident slots over their waves -- a grid that barely exceeds the slots
// would double the time with its last wave -- else the count that fills them
// best.  Fewer splits keep the per-CTA start (the first tile's keys all enter
// the lists) and the merge small.
int choose_splits(long long qtiles, long long row_tiles, int slots, int min_tiles) {
  int best = 1;
  double best_eff = 0.0;
  for (int s = 1; s <= BF_MAXSPLIT; ++s) {
    if (s > 1 && (long long)s * min_tiles > row_tiles) break;
    const long long ctas = qtiles * s;
    const long long waves = (ctas + slots - 1) / slots;
    const double eff = (double)ctas / (double)(waves * slots);
    if (eff >= 0.9) return s;
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = s;
    }
  }
  return best;
}

int resident_slots(const void* kernel, int threads, size_t smem) {
  int dev = 0, per_sm = 0, sms = 0;
  RINND_CUDA(cudaGetDevice(&dev));
  RINND_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  RINND_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return std::max(1, per_sm) * std::max(1, sms);
}

template <typename T, int QT>
size_t bf_smem(int k) {
  return (size_t)(QT + BF_RT) * BF_KS * 4 + (size_t)QT * (BF_RT + k) * sizeof(BfKey<T>) + (size_t)(2 * QT + 2) * 4 +
         (size_t)QT * sizeof(BfKey<T>);
}

template <typename T, int MODE, int QT>
void brute_launch(BfArgs& a, int qtiles, DVec<BfKey<T>>& part, cudaStream_t st) {
  const size_t smem = bf_smem<T, QT>(a.k);
  const void* kern = reinterpret_cast<const void*>(k_brute<T, MODE, QT>);
  set_smem_limit_once(kern, 200 * 1024);
  a.splits = choose_splits(qtiles, (a.n + BF_RT - 1) / BF_RT, resident_slots(kern, BF_NT, smem), 4);
  if (a.splits > 1) {
    part.alloc((size_t)a.nq * a.splits * a.k, st);
    a.out_key = part.p;
  }
  k_brute<T, MODE, QT><<<dim3((unsigned)qtiles, (unsigned)a.splits), BF_NT, smem, st>>>(a);
  RINND_LAUNCH_CHECK();
}

// FP32: 64 queries a CTA (4 x 4 pairs a thread); FP64: 32 (2 x 4), its keys
// being twice as wide.
template <typename T>
void brute_run(const float* Q, int nq, const float* X, long long n, int Dp, int k, int kind, const int32_t* excl,
               int32_t* out_idx, float* out_dist, cudaStream_t st) {
  constexpr int QT = sizeof(T) == 4 ? 64 : 32;
  const int mode = kind == DK_SQEUCLIDEAN ? BF_SQ : (kind == DK_MANHATTAN ? BF_MAN : BF_DOT);
  DVec<T> qn, xn;
  if (mode == BF_DOT) {
    qn.alloc((size_t)nq, st);
    xn.alloc((size_t)n, st);
    k_bf_norms<T><<<(unsigned)(((long long)nq * 32 + 255) / 256), 256, 0, st>>>(Q, nq, Dp, qn.p);
    RINND_LAUNCH_CHECK();
    k_bf_norms<T><<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(X, n, Dp, xn.p);
    RINND_LAUNCH_CHECK();
  }
  const int qtiles = (nq + QT - 1) / QT;
  DVec<BfKey<T>> part;
  BfArgs a{Q, X, qn.p, xn.p, excl, n, nq, Dp, k, kind, 1, nullptr, out_idx, out_dist};
  if (mode == BF_SQ) brute_launch<T, BF_SQ, QT>(a, qtiles, part, st);
  else if (mode == BF_MAN) brute_launch<T, BF_MAN, QT>(a, qtiles, part, st);
  else brute_launch<T, BF_DOT, QT>(a, qtiles, part, st);
  if (a.splits > 1) {
    k_brute_merge<T><<<(unsigned)((nq * 32 + 255) / 256), 256, 0, st>>>(part.p, nq, a.splits, k, out_idx, out_dist);
    RINND_LAUNCH_CHECK();
  }
}

// ---------------------------------------------------------------------------
// Tensor-core form
// ---------------------------------------------------------------------------
constexpr int TC_M = 128;       // queries per CTA (tensor-memory lanes)
constexpr int TC_N = 128;       // rows per tile (accumulator columns)
constexpr int TC_KPMAX = 128;   // padded dimension limit
constexpr int TC_KMAX = 32;     // k limit
constexpr int TC_NEPI = 8;      // epilogue warps: lane quadrant warp % 4, column half (warp - 2) / 4
constexpr int TC_NT = 32 * (2 + TC_NEPI);

// BF16 copy of rows 0..n_pad-1 (rows >= n zero) in the tiled operand layout:
// tile t = rows 128 t.., at t * 128 Kp elements; element (r, k) of a tile at
// byte (r / 8) SBO + (k / 8) 128 + (r % 8) 16 + (k % 8) 2, SBO = (Kp / 8) 128.
// info[r] = (|b_r|^2, e_r >= |b_r - x_r|), one warp per row.
__global__ void k_bf16_tiled(const float* __restrict__ X, long long n, long long n_pad, int Dp, int Kp,
                             __nv_bfloat16* __restrict__ out, float2* __restrict__ info) {
  const long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= n_pad) return;
  const long long tile = r / TC_N;
  const int rr = (int)(r % TC_N);
  const size_t sbo = (size_t)(Kp / 8) * 128;
  unsigned char* base = reinterpret_cast<unsigned char*>(out) + (size_t)tile * TC_N * Kp * 2 + (size_t)(rr / 8) * sbo +
                        (size_t)(rr % 8) * 16;
  float bn = 0.f, ee = 0.f;
  for (int k = lane; k < Kp; k += 32) {
    const float x = (r < n && k < Dp) ? X[(size_t)r * Dp + k] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    const float bf = __bfloat162float(b);
    *reinterpret_cast<__nv_bfloat16*>(base + (size_t)(k / 8) * 128 + (k % 8) * 2) = b;
    bn = fmaf(bf, bf, bn);
    const float d = bf - x;  // exact: b is x rounded to 8 significant bits
    ee = fmaf(d, d, ee);
  }
  for (int o = 16; o; o >>= 1) {
    bn += __shfl_xor_sync(0xffffffffu, bn, o);
    ee += __shfl_xor_sync(0xffffffffu, ee, o);
  }
  // the FP32 sum of squares is within Kp 2^-24 of its value; 2^-10 covers it and the sqrt
  if (lane == 0) info[r] = make_float2(bn, sqrtf(ee) * 1.0009765625f + 1e-30f);
}

struct TcArgs {
  const __nv_bfloat16* Qb;  // tiled BF16 queries
  const float2* qinfo;
  const float* Q;           // FP32 queries, nq x Dp
  const float* qn;          // FP32 squared norms (dot forms)
  const __nv_bfloat16* Xb;  // tiled BF16 rows
  const float2* xinfo;
  const float* X;
  const float* xn;
  const int32_t* excl;
  long long n;
  int nq, Dp, Kp, k, kind, splits, ntiles;
  BfKey<float>* out_key;  // splits > 1: nq x splits x k
  int32_t* out_idx;
  float* out_dist;
  int* err;
};

__host__ __device__ inline size_t tc_smem(int Kp, int k) {
  return (size_t)3 * TC_N * Kp * 2 + (size_t)TC_M * 2 * k * sizeof(BfKey<float>) + 16 * 8 + 16 + TC_M * 2 * 4;
}

// Bounded wait whose outcome is the same in every lane of the warp.
__device__ __forceinline__ bool warp_wait_tc(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  return __all_sync(0xffffffffu, wait_or_abort(bar, parity, abort_flag));
}

template <bool SQ>
__global__ void __launch_bounds__(TC_NT) k_brute_tc(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  const uint32_t tile_bytes = (uint32_t)(TC_N * a.Kp * 2);
  unsigned char* A = smem;
  unsigned char* Bst = smem + tile_bytes;  // two stages
  BfKey<float>* lists = reinterpret_cast<BfKey<float>*>(smem + 3 * (size_t)tile_bytes);  // (query, half) x k
  uint64_t* bar = reinterpret_cast<uint64_t*>(lists + (size_t)TC_M * 2 * a.k);
  uint64_t* a_full = bar;
  uint64_t* tile_full = bar + 1;   // [2]
  uint64_t* tile_empty = bar + 3;  // [2]
  uint64_t* mma_done = bar + 5;    // [2]
  uint64_t* tmem_empty = bar + 7;  // [2]
  uint64_t* drain = bar + 9;
  int* ints = reinterpret_cast<int*>(bar + 16);
  volatile int* abort_flag = ints;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(ints + 1);
  int* lcnt = ints + 4;  // entries of each (query, half) list
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int per = (a.ntiles + a.splits - 1) / a.splits;
  const int t_lo = blockIdx.y * per;
  const int nt = max(0, min(a.ntiles, t_lo + per) - t_lo);
  if (tid == 0) {
    mbar_init(a_full, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tile_full[i], 1);
      mbar_init(&tile_empty[i], 1);
      mbar_init(&mma_done[i], 1);
      mbar_init(&tmem_empty[i], TC_NEPI);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) umma::tmem_alloc(tmem_slot, 2 * TC_N);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t taddr = *tmem_slot;

  if (warp == 0) {
    // ------------------------------ producer ------------------------------
    if (lane == 0) {
      bool ok = true;
      int issued = 0;
      mbar_arrive_expect_tx(a_full, tile_bytes);
      bulk_g2s(A, a.Qb + (size_t)blockIdx.x * TC_M * a.Kp, tile_bytes, a_full);
      for (int t = 0; t < nt; ++t) {
        const int s = t & 1;
        if (t >= 2 && !(ok = wait_or_abort(&tile_empty[s], (uint32_t)((t >> 1) - 1) & 1u, abort_flag))) break;
        mbar_arrive_expect_tx(&tile_full[s], tile_bytes);
        bulk_g2s(Bst + (size_t)s * tile_bytes, a.Xb + (size_t)(t_lo + t) * TC_N * a.Kp, tile_bytes, &tile_full[s]);
        issued = t + 1;
      }
      if (!ok) {
        *abort_flag = 1;
        atomicExch(a.err, 1);
      }
      // no copy may land after the CTA exits: wait (bounded) for the last ones issued
      mbar_wait_bounded(a_full, 0u, WAIT_POLLS);
      for (int t = max(0, issued - 2); t < issued; ++t)
        mbar_wait_bounded(&tile_full[t & 1], (uint32_t)(t >> 1) & 1u, WAIT_POLLS);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------ MMA issuer ------------------------------
    if (lane == 0) {
      bool ok = wait_or_abort(a_full, 0u, abort_flag);
      const uint32_t idesc = umma::idesc_bf16_f32(TC_M, TC_N);
      const uint32_t sbo = (uint32_t)(a.Kp / 8) * 128u;
      const uint32_t a0 = smem_addr(A), b0 = smem_addr(Bst);
      for (int t = 0; ok && t < nt; ++t) {
        const int s = t & 1;
        if (!(ok = wait_or_abort(&tile_full[s], (uint32_t)(t >> 1) & 1u, abort_flag))) break;
        if (t >= 2 && !(ok = wait_or_abort(&tmem_empty[s], (uint32_t)((t >> 1) - 1) & 1u, abort_flag))) break;
        umma::fence_after_sync();
        for (int kk = 0; kk < a.Kp / 16; ++kk) {
          const uint64_t ad = umma::smem_desc(a0 + 256u * kk, 128u, sbo);
          const uint64_t bd = umma::smem_desc(b0 + (uint32_t)s * tile_bytes + 256u * kk, 128u, sbo);
          umma::mma_bf16(taddr + (uint32_t)(TC_N * s), ad, bd, idesc, kk > 0);
        }
        umma::commit(&tile_empty[s]);  // the stage is free once these MMAs completed
        umma::commit(&mma_done[s]);
      }
      if (!ok) {
        *abort_flag = 1;
        atomicExch(a.err, 1);
      }
      // no MMA may run once the tensor memory is freed: a last commit tracks every MMA issued
      umma::commit(drain);
      mbar_wait_bounded(drain, 0u, WAIT_POLLS);
    }
    __syncwarp();
  } else {
    // ------------------------------ epilogue ------------------------------
    const int quad = warp & 3, half = (warp - 2) >> 2;
    const int qi = 32 * quad + lane;
    const int q = blockIdx.x * TC_M + qi;
    const bool qv = q < a.nq;
    BfKey<float>* L = lists + ((size_t)qi * 2 + half) * a.k;
    int cnt = 0;
    BfKey<float> thr = key_max<float>();
    const float2 qinf = qv ? a.qinfo[q] : make_float2(0.f, 0.f);
    const float bn_q = qinf.x, e_q = qinf.y;
    const float xn_q = (!SQ && qv) ? a.qn[q] : 0.f;
    const float bt = sqrtf(bn_q);
    const int32_t excl = (a.excl && qv) ? a.excl[q] : -1;
    const float* qrow = a.Q + (size_t)(qv ? q : 0) * a.Dp;
    const float gam = SQ ? (float)a.Kp * 1.9073486328125e-06f + 9.5367431640625e-07f   // Kp 2^-19 + 2^-20
                         : (float)a.Kp * 9.5367431640625e-07f + 9.5367431640625e-07f;  // Kp 2^-20 + 2^-20
    float sthr = INFINITY;  // squared Euclidean: sqrt(T (1 + 2^-11)) of the list's k-th distance T
    for (int t = 0; t < nt; ++t) {
      const int b = t & 1;
      if (!warp_wait_tc(&mma_done[b], (uint32_t)(t >> 1) & 1u, abort_flag)) {
        if (lane == 0) {
          *abort_flag = 1;
          atomicExch(a.err, 1);
        }
        break;
      }
      umma::fence_after_sync();
      uint32_t g[64];
      const uint32_t ta = taddr + ((uint32_t)(32 * quad) << 16) + (uint32_t)(TC_N * b + 64 * half);
#pragma unroll
      for (int c = 0; c < 4; ++c) umma::ld_32x32b_x16(ta + 16u * c, g + 16 * c);
      umma::wait_ld();
      umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tmem_empty[b]);  // this warp's reads of the accumulator are done
      const long long row0 = (long long)(t_lo + t) * TC_N + 64 * half;
      // the 64 columns' row terms, one column a lane per 32, passed by shuffles
      float2 xi_l[2];
      float xn_l[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long long row = row0 + 32 * h + lane;
        xi_l[h] = row < a.n ? __ldg(a.xinfo + row) : make_float2(0.f, 0.f);
        xn_l[h] = (!SQ && row < a.n) ? __ldg(a.xn + row) : 0.f;
      }
      // survivors of the filter against the list's k-th key at the tile's start
      unsigned long long keepm = 0ull;
#pragma unroll
      for (int j = 0; j < 64; ++j) {
        const long long row = row0 + j;
        const float G = __uint_as_float(g[j]);
        const float2 xi = make_float2(__shfl_sync(0xffffffffu, xi_l[j >> 5].x, j & 31),
                                      __shfl_sync(0xffffffffu, xi_l[j >> 5].y, j & 31));
        bool keep;
        if (SQ) {
          const float sum = bn_q + xi.x;
          const float x = sum - 2.0f * G - gam * sum;
          const float c = sthr + e_q + xi.y;
          keep = fmaxf(x, 0.f) < c * c;
        } else {
          const float bj = sqrtf(xi.x);
          const float ub = G + e_q * bj + xi.y * (bt + e_q) + gam * bt * bj;
          float lb = finalize_dot(a.kind, ub, __shfl_sync(0xffffffffu, xn_l[j >> 5], j & 31), xn_q);
          lb = lb - fabsf(lb) * 4.8828125e-4f - 1e-30f;
          keep = lb < thr.d;
        }
        keepm |= (unsigned long long)(keep && row < a.n) << j;
      }
      if (!qv) keepm = 0ull;
      while (keepm) {
        const int j = __ffsll((long long)keepm) - 1;
        keepm &= keepm - 1;
        const long long row = row0 + j;
        if ((int32_t)row == excl) continue;
        // exact FP32 recheck: the FP32 form's arithmetic (row first)
        float d = join_dist_fp32(a.kind, a.X + (size_t)row * a.Dp, qrow, a.Dp);
        if (!SQ) d = finalize_dot(a.kind, d, __ldg(a.xn + row), xn_q);
        if (d != d) d = INFINITY;
        const BfKey<float> key{d, (int32_t)row};
        if (!key_less(key, thr)) continue;
        int p = cnt < a.k ? cnt : a.k - 1;  // the slot the key may take
        while (p > 0 && key_less(key, L[p - 1])) {
          L[p] = L[p - 1];
          --p;
        }
        L[p] = key;
        if (cnt < a.k) ++cnt;
        if (cnt == a.k) {
          thr = L[a.k - 1];
          sthr = SQ ? sqrtf(thr.d * 1.00048828125f) : 0.f;
        }
      }
    }
    lcnt[qi * 2 + half] = cnt;  // the two halves' lists of a query are merged after the barrier
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 1) umma::tmem_dealloc(taddr, 2 * TC_N);
  if (warp >= 2 && ((warp - 2) >> 2) == 0) {
    const int qi = 32 * (warp & 3) + lane;
    const int q = blockIdx.x * TC_M + qi;
    if (q < a.nq) {
      const BfKey<float>* L0 = lists + (size_t)qi * 2 * a.k;
      const BfKey<float>* L1 = L0 + a.k;
      const int n0 = lcnt[qi * 2], n1 = lcnt[qi * 2 + 1];
      int i0 = 0, i1 = 0;
      for (int p = 0; p < a.k; ++p) {
        BfKey<float> key{INFINITY, -1};
        if (i0 < n0 && (i1 >= n1 || key_less(L0[i0], L1[i1]))) key = L0[i0++];
        else if (i1 < n1) key = L1[i1++];
        if (a.splits > 1) {
          a.out_key[((size_t)q * a.splits + blockIdx.y) * a.k + p] = key;
        } else {
          a.out_idx[(size_t)q * a.k + p] = key.id;
          a.out_dist[(size_t)q * a.k + p] = key.d;
        }
      }
    }
  }
}

bool tc_supported(int kind, int Dp, int k) {
  return (kind == DK_SQEUCLIDEAN || bf_dot_kind(kind)) && (Dp + 15) / 16 * 16 <= TC_KPMAX && k <= TC_KMAX;
}

void brute_tc_run(const float* Q, int nq, const float* X, long long n, int Dp, int k, int kind, const int32_t* excl,
                  int32_t* out_idx, float* out_dist, cudaStream_t st) {
  const int Kp = (Dp + 15) / 16 * 16;
  const long long ntiles = (n + TC_N - 1) / TC_N;
  const int qtiles = (nq + TC_M - 1) / TC_M;
  if (ntiles > 0x7FFFFFFF) throw std::invalid_argument("brute force: too many rows");
  DVec<__nv_bfloat16> Xb((size_t)ntiles * TC_N * Kp, st), Qb((size_t)qtiles * TC_M * Kp, st);
  DVec<float2> xinfo((size_t)ntiles * TC_N, st), qinfo((size_t)qtiles * TC_M, st);
  k_bf16_tiled<<<(unsigned)((ntiles * TC_N * 32 + 255) / 256), 256, 0, st>>>(X, n, ntiles * TC_N, Dp, Kp, Xb.p, xinfo.p);
  RINND_LAUNCH_CHECK();
  k_bf16_tiled<<<(unsigned)(((long long)qtiles * TC_M * 32 + 255) / 256), 256, 0, st>>>(Q, nq, (long long)qtiles * TC_M,
                                                                                       Dp, Kp, Qb.p, qinfo.p);
  RINND_LAUNCH_CHECK();
  DVec<float> qn, xn;
  const bool sq = kind == DK_SQEUCLIDEAN;
  if (!sq) {
    qn.alloc((size_t)nq, st);
    xn.alloc((size_t)n, st);
    k_bf_norms<float><<<(unsigned)(((long long)nq * 32 + 255) / 256), 256, 0, st>>>(Q, nq, Dp, qn.p);
    RINND_LAUNCH_CHECK();
    k_bf_norms<float><<<(unsigned)((n * 32 + 255) / 256), 256, 0, st>>>(X, n, Dp, xn.p);
    RINND_LAUNCH_CHECK();
  }
  // at least 116 KB: at most two CTAs (2 x 256 tensor-memory columns) share an SM
  const size_t smem = std::max<size_t>(tc_smem(Kp, k), 116 * 1024);
  const void* kern = sq ? reinterpret_cast<const void*>(k_brute_tc<true>) : reinterpret_cast<const void*>(k_brute_tc<false>);
  set_smem_limit_once(kern, 227 * 1024);
  const int splits = choose_splits(qtiles, ntiles, resident_slots(kern, TC_NT, smem), 8);
  DVec<BfKey<float>> part;
  if (splits > 1) part.alloc((size_t)nq * splits * k, st);
  DVec<int> err(1, st);
  err.fill_bytes(0);
  TcArgs a{Qb.p, qinfo.p, Q, qn.p, Xb.p, xinfo.p, X, xn.p, excl, n, nq, Dp, Kp, k, kind, splits, (int)ntiles,
           part.p, out_idx, out_dist, err.p};
  const dim3 grid((unsigned)qtiles, (unsigned)splits);
  if (sq) k_brute_tc<true><<<grid, TC_NT, smem, st>>>(a);
  else k_brute_tc<false><<<grid, TC_NT, smem, st>>>(a);
  RINND_LAUNCH_CHECK();
  if (splits > 1) {
    k_brute_merge<float><<<(unsigned)(((long long)nq * 32 + 255) / 256), 256, 0, st>>>(part.p, nq, splits, k, out_idx,
                                                                                       out_dist);
    RINND_LAUNCH_CHECK();
  }
  int h_err = 0;
  RINND_CUDA(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  if (h_err) throw std::runtime_error("brute force: a tensor-core pipeline wait timed out");
}

}  // namespace

bool brute_supported(int kind) {
  return kind == DK_SQEUCLIDEAN || kind == DK_MANHATTAN || bf_dot_kind(kind);
}

void brute_force_knn(const float* Q, int nq, const float* X, long long n, int Dp, int k, int kind, int precision,
                     const int32_t* excl, int32_t* out_idx, float* out_dist, cudaStream_t st) {
  if (nq <= 0) return;
  if (k < 1 || k > BF_KMAX) throw std::invalid_argument("brute force: k must be in [1, 128]");
  if (!brute_supported(kind)) throw std::invalid_argument("brute force: unsupported distance kind");
  if (Dp % 4 != 0) throw std::invalid_argument("brute force: row stride must be a multiple of 4");
  if (precision == 2) {
    brute_run<double>(Q, nq, X, n, Dp, k, kind, excl, out_idx, out_dist, st);
  } else if (precision == 0) {
    brute_run<float>(Q, nq, X, n, Dp, k, kind, excl, out_idx, out_dist, st);
  } else if (precision == 1) {
    if (!tc_supported(kind, Dp, k))
      throw std::invalid_argument(
          "brute force: the BF16 tensor-core form takes D <= 128, k <= 32 and squared Euclidean or a dot form");
    brute_tc_run(Q, nq, X, n, Dp, k, kind, excl, out_idx, out_dist, st);
  } else {
    throw std::invalid_argument("brute force: precision must be 0 (FP32), 1 (BF16 tensor cores) or 2 (FP64)");
  }
}

}  // namespace rinnd
