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
#include "dist.cuh"
#include "engine.h"
#include "join_common.cuh"

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

// The splits' sorted lists of one query -> its first k keys (warp per query):
// repeatedly the smallest head, found by a warp reduction over the splits.
template <typename T>
__global__ void k_brute_merge(const BfKey<T>* __restrict__ part, int nq, int splits, int k, int32_t* out_idx,
                              float* out_dist) {
  const int q = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (q >= nq) return;
  const BfKey<T>* P = part + (size_t)q * splits * k;
  int head = 0;  // this lane's position in split `lane` (splits <= 32)
  for (int p = 0; p < k; ++p) {
    BfKey<T> mine = (lane < splits && head < k) ? P[(size_t)lane * k + head] : BfKey<T>{(T)INFINITY, -1};
    if (mine.id < 0) mine = BfKey<T>{(T)INFINITY, 0x7FFFFFFF};
    BfKey<T> best = mine;
    int src = lane;
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
    if (lane == src) ++head;
    if (lane == 0) {
      const bool empty = best.id == 0x7FFFFFFF;
      out_idx[(size_t)q * k + p] = empty ? -1 : best.id;
      out_dist[(size_t)q * k + p] = empty ? __int_as_float(0x7f800000) : (float)best.d;
    }
  }
}

template <typename T, int QT>
size_t bf_smem(int k) {
  return (size_t)(QT + BF_RT) * BF_KS * 4 + (size_t)QT * (BF_RT + k) * sizeof(BfKey<T>) + (size_t)(2 * QT + 2) * 4 +
         (size_t)QT * sizeof(BfKey<T>);
}

template <typename T, int MODE, int QT>
void brute_launch(const BfArgs& a, int qtiles, cudaStream_t st) {
  const size_t smem = bf_smem<T, QT>(a.k);
  set_smem_limit_once(reinterpret_cast<const void*>(k_brute<T, MODE, QT>), 200 * 1024);
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
  // enough CTAs for a few waves, rows split over the CTAs of one query tile
  int splits = 1;
  while (splits < 32 && (long long)qtiles * splits < 148 * 4 && (long long)splits * 4 * BF_RT < n) splits *= 2;
  DVec<BfKey<T>> part;
  if (splits > 1) part.alloc((size_t)nq * splits * k, st);
  BfArgs a{Q, X, qn.p, xn.p, excl, n, nq, Dp, k, kind, splits, part.p, out_idx, out_dist};
  if (mode == BF_SQ) brute_launch<T, BF_SQ, QT>(a, qtiles, st);
  else if (mode == BF_MAN) brute_launch<T, BF_MAN, QT>(a, qtiles, st);
  else brute_launch<T, BF_DOT, QT>(a, qtiles, st);
  if (splits > 1) {
    k_brute_merge<T><<<(unsigned)((nq * 32 + 255) / 256), 256, 0, st>>>(part.p, nq, splits, k, out_idx, out_dist);
    RINND_LAUNCH_CHECK();
  }
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
  if (precision == 2) brute_run<double>(Q, nq, X, n, Dp, k, kind, excl, out_idx, out_dist, st);
  else if (precision == 0) brute_run<float>(Q, nq, X, n, Dp, k, kind, excl, out_idx, out_dist, st);
  else throw std::invalid_argument("brute force: precision must be 0 (FP32) or 2 (FP64)");
}

}  // namespace rinnd
