// graph.cu -- diversified, pruned CSR search graph.
//
// Restates SearchGraph::from_dense_diversified (core/graph/search_graph.rs:263-360):
//   1. forward diversify every sorted kNN row (diversify_row :432-473): keep j
//      unless a retained c has d_ic > f32::MIN_POSITIVE and d(c, j) < d_ij;
//   2. transpose the forward rows with their distances (transpose_csr :526-567)
//      and order each reverse row by (distance, source id);
//   3. diversify the reverse rows (diversify_sorted_csr :478-523);
//   4. union forward and reverse rows (weighted_union_pruned :368-426): drop
//      -1, self loops and non-finite distances, merge duplicate ids with the
//      max distance, keep the max_degree nearest by (distance, id), emit by id;
//   5. min_distance = min forward distance (0 -> f32::EPSILON), :353-357.
// With diversify_prob = 1 (the default) no randomness is involved and the
// output equals the reference's for the same input graph: the d(c, j)
// comparisons use the reference's exact accumulation order (dist.cuh), and the
// reverse-row order (distance, then source id) equals the reference's whenever
// a reverse row has no tied distances.
#include <cub/cub.cuh>

#include "dist.cuh"
#include "engine.h"

namespace rinnd {
namespace {

constexpr int WARPS = 4;

// Prune probability (diversify_prob): the reference draws rand::thread_rng()'s
// f32 for every pruning decision that qualifies and prunes when the draw is below
// the probability (search_graph.rs:457-460, :506-509), an OS-seeded stream.  Here the draw of
// the decision (row, candidate j, retained c) is a keyed hash, 24-bit uniform
// like rand's f32: the outcome is reproducible, and since each decision has its
// own draw, "some retained c prunes j" does not depend on the order the retained
// entries are tested in.  prob >= 1 prunes every qualifying decision (no draw).
struct PruneDraw {
  float prob;
  uint64_t seed;
};
__device__ __forceinline__ bool prune_draw(const PruneDraw& pd, int row, int32_t j, int32_t c) {
  if (pd.prob >= 1.0f) return true;
  const uint64_t h = hash3(pd.seed ^ 0xD17E55ull, ((uint64_t)(uint32_t)row << 32) | (uint32_t)j, (uint32_t)c);
  return (float)(h >> 40) * 5.9604644775390625e-08f < pd.prob;  // (h >> 40) / 2^24
}

// exact_distance with the metric fixed at compile time (KIND >= 0) or chosen
// at run time (KIND < 0): the fixed form carries only its metric's code, so the
// kernels hold fewer registers and keep more warps resident.
template <int KIND>
__device__ __forceinline__ float pair_distance(int kind, const float* a, const float* b, int n) {
  if constexpr (KIND == DK_SQEUCLIDEAN) return exact_sqeuclid(a, b, n);
  else return exact_distance(kind, a, b, n);
}

// Squared Euclidean distances of the row pairs (a0, b0), (a0, b1), (a1, b0),
// (a1, b1), each with exact_sqeuclid's arithmetic (the same chains, packed
// pairs, horizontal sum and remainder); the four pairs share their chunk loads.
__device__ __forceinline__ void exact_sqeuclid_2x2(const float* a0, const float* a1, const float* b0,
                                                   const float* b1, int n, float* out) {
  unsigned long long p[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int t = 0; t < 4; ++t) p[u][t] = 0ull;
  const int chunks = n >> 3;
  for (int c = 0; c < chunks; ++c) {
    unsigned long long x0[4], x1[4], y0[4], y1[4];
    load8p(a0 + 8 * c, x0);
    load8p(a1 + 8 * c, x1);
    load8p(b0 + 8 * c, y0);
    load8p(b1 + 8 * c, y1);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      unsigned long long d = pk_sub(x0[t], y0[t]);
      p[0][t] = pk_fma(d, d, p[0][t]);
      d = pk_sub(x0[t], y1[t]);
      p[1][t] = pk_fma(d, d, p[1][t]);
      d = pk_sub(x1[t], y0[t]);
      p[2][t] = pk_fma(d, d, p[2][t]);
      d = pk_sub(x1[t], y1[t]);
      p[3][t] = pk_fma(d, d, p[3][t]);
    }
  }
  const float* A[4] = {a0, a0, a1, a1};
  const float* B[4] = {b0, b1, b0, b1};
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    float s[8];
    unpack8(p[u], s);
    float r = hsum_a(s);
    for (int i = chunks * 8; i < n; ++i) {
      const float d = __fsub_rn(A[u][i], B[u][i]);
      r = __fadd_rn(r, __fmul_rn(d, d));
    }
    out[u] = r;
  }
}

// Warp-cooperative RNG-style prune step: does any retained c (in smem) prune j?
template <int KIND>
__device__ __forceinline__ bool pruned_by_retained(const int32_t* ret_id, const float* ret_d, int nret,
                                                   int32_t j, float dij, const float* X, int D,
                                                   int Dp, int kind, const PruneDraw& pd, int row) {
  const int lane = threadIdx.x & 31;
  for (int r0 = 0; r0 < nret; r0 += 32) {
    int r = r0 + lane;
    bool pr = false;
    if (r < nret) {
      float dic = ret_d[r];
      if (dic > FLT_MIN) {
        float dcj = pair_distance<KIND>(kind, X + (size_t)ret_id[r] * Dp, X + (size_t)j * Dp, D);
        pr = dcj < dij && prune_draw(pd, row, j, ret_id[r]);
      }
    }
    if (__any_sync(0xffffffffu, pr)) return true;
  }
  return false;
}

template <int MAXR, int KIND>
__global__ void k_diversify_fwd(const int32_t* knn_idx, const float* knn_dist, int N, int k,
                                const float* X, int D, int Dp, int kind, int max_degree,
                                int32_t* fwd_idx, float* fwd_dist, int32_t* fwd_cnt,
                                uint32_t* min_key, PruneDraw pd) {
  __shared__ int32_t s_id[WARPS][MAXR];
  __shared__ float s_d[WARPS][MAXR];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * WARPS + w;
  if (row >= N) return;
  int nret = 0;
  uint32_t local_min = KEY_INF;
  for (int pos = 0; pos < k; ++pos) {
    int32_t j = knn_idx[(size_t)row * k + pos];
    if (j < 0) break;
    float dij = knn_dist[(size_t)row * k + pos];
    bool pruned = pruned_by_retained<KIND>(s_id[w], s_d[w], nret, j, dij, X, D, Dp, kind, pd, row);
    if (!pruned) {
      if (lane == 0) {
        s_id[w][nret] = j;
        s_d[w][nret] = dij;
      }
      __syncwarp();
      ++nret;
      float v = dij == 0.f ? FLT_EPSILON : dij;
      if (isfinite(v)) local_min = min(local_min, fkey(v));
      if (nret >= max_degree) break;
    }
  }
  for (int r = lane; r < nret; r += 32) {
    fwd_idx[(size_t)row * k + r] = s_id[w][r];
    fwd_dist[(size_t)row * k + r] = s_d[w][r];
  }
  if (lane == 0) {
    fwd_cnt[row] = nret;
    if (local_min != KEY_INF) atomicMin(min_key, local_min);
  }
}

// Forward diversify with a row's candidates staged in shared memory (<= 32
// candidates, Dp <= 256): the warp first evaluates d(a, b) for every candidate pair a < b
// from shared memory, in parallel and in the reference's exact order (the same
// exact_distance call as the sequential form, argument order (earlier, later)),
// then runs the sequential keep/prune pass (diversify_row / diversify_sorted_csr)
// on that table.  Same output as the sequential kernels; the pairs of pruned
// candidates are evaluated too, trading a little arithmetic for the latency of
// evaluating one candidate at a time against rows in global memory.
constexpr int SK = 32;
struct StagedSmem {
  // rows padded to Dp + 4 floats: lanes reading the same offset of different rows hit different banks
  __host__ __device__ static size_t per_warp(int Dp) {
    return (size_t)SK * (Dp + 4) * 4 + (size_t)SK * SK * 4 + SK * 12;
  }
};

struct StagedWarp {
  float* rows;   // SK x (Dp + 4)
  float* M;      // SK x SK, M[a * SK + b] = d(a, b), a < b
  int32_t* ret;  // retained candidate positions
  float* dpos;   // d(row, candidate)
  int32_t* cid;  // candidate ids
};

__device__ __forceinline__ StagedWarp staged_warp(unsigned char* smem, int w, int Dp) {
  unsigned char* base = smem + (size_t)w * StagedSmem::per_warp(Dp);
  StagedWarp sw;
  sw.rows = reinterpret_cast<float*>(base);
  sw.M = sw.rows + (size_t)SK * (Dp + 4);
  sw.ret = reinterpret_cast<int32_t*>(sw.M + SK * SK);
  sw.dpos = reinterpret_cast<float*>(sw.ret + SK);
  sw.cid = reinterpret_cast<int32_t*>(sw.dpos + SK);
  return sw;
}

// The n candidates (cid/dpos filled, synchronized) -> sw.ret[0, nret); returns nret.
template <int KIND>
__device__ __forceinline__ int staged_prune(const StagedWarp& sw, int n, const float* X, int D, int Dp, int kind,
                                            int max_degree, const PruneDraw& pd, int row) {
  const int lane = threadIdx.x & 31, rs = Dp + 4, q4 = Dp / 4;
  // every 16-byte piece of every candidate row in flight at once (cp.async, L2 only)
  for (int e = lane; e < n * q4; e += 32) {
    const int r = e / q4, t = e - r * q4;
    const float* src = X + (size_t)sw.cid[r] * Dp + 4 * t;
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(sw.rows + (size_t)r * rs + 4 * t);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncwarp();
  if constexpr (KIND == DK_SQEUCLIDEAN) {
    // 2 x 2 blocks of pairs: rows (2p, 2p + 1) x (2q, 2q + 1), p <= q, block e
    // = (p, q) with q = floor((sqrt(1 + 8e) - 1) / 2); rows past n repeat row
    // n - 1 and pairs with a >= b or b >= n are not stored
    const int h = (n + 1) >> 1;
    for (int e = lane; e < h * (h + 1) / 2; e += 32) {
      int q = (int)((sqrtf((float)(8 * e + 1)) - 1.0f) * 0.5f);
      if (q * (q + 1) / 2 > e) --q;
      else if ((q + 1) * (q + 2) / 2 <= e) ++q;
      const int p = e - q * (q + 1) / 2;
      const int a0 = 2 * p, a1 = min(2 * p + 1, n - 1), b0 = 2 * q, b1 = min(2 * q + 1, n - 1);
      float d4[4];
      exact_sqeuclid_2x2(sw.rows + (size_t)a0 * rs, sw.rows + (size_t)a1 * rs, sw.rows + (size_t)b0 * rs,
                         sw.rows + (size_t)b1 * rs, D, d4);
      const int as[4] = {2 * p, 2 * p, 2 * p + 1, 2 * p + 1};
      const int bs[4] = {2 * q, 2 * q + 1, 2 * q, 2 * q + 1};
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (as[u] < bs[u] && bs[u] < n) sw.M[as[u] * SK + bs[u]] = d4[u];
    }
  } else {
    // pairs a < b < n in the order (b, then a): pair e is (e - b(b-1)/2, b) with
    // b = floor((1 + sqrt(1 + 8e)) / 2), so no lane idles on a >= b
    for (int e = lane; e < n * (n - 1) / 2; e += 32) {
      int b = (int)((1.0f + sqrtf((float)(8 * e + 1))) * 0.5f);
      if (b * (b - 1) / 2 > e) --b;
      else if ((b + 1) * b / 2 <= e) ++b;
      const int a = e - b * (b - 1) / 2;
      sw.M[a * SK + b] = exact_distance(kind, sw.rows + (size_t)a * rs, sw.rows + (size_t)b * rs, D);
    }
  }
  __syncwarp();
  int nret = 0;
  for (int pos = 0; pos < n; ++pos) {
    const float dij = sw.dpos[pos];
    bool pr = false;
    if (lane < nret) {
      const int c = sw.ret[lane];
      pr = sw.dpos[c] > FLT_MIN && sw.M[c * SK + pos] < dij && prune_draw(pd, row, sw.cid[pos], sw.cid[c]);
    }
    if (!__any_sync(0xffffffffu, pr)) {
      if (lane == 0) sw.ret[nret] = pos;
      __syncwarp();
      ++nret;
      if (nret >= max_degree) break;
    }
  }
  __syncwarp();
  return nret;
}

template <int KIND>
__global__ void __launch_bounds__(32 * WARPS)
    k_diversify_fwd_staged(const int32_t* knn_idx, const float* knn_dist, int N, int k, const float* X, int D,
                           int Dp, int kind, int max_degree, int32_t* fwd_idx, float* fwd_dist, int32_t* fwd_cnt,
                           uint32_t* min_key, PruneDraw pd) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * WARPS + w;
  if (row >= N) return;
  const StagedWarp sw = staged_warp(smem, w, Dp);
  int32_t my_id = -1;
  float my_d = 0.f;
  if (lane < k) {
    my_id = knn_idx[(size_t)row * k + lane];
    my_d = knn_dist[(size_t)row * k + lane];
  }
  // candidates end at the first -1
  const unsigned valid = __ballot_sync(0xffffffffu, lane < k && my_id >= 0);
  const int n = (~valid) ? __ffs(~valid) - 1 : 32;
  sw.dpos[lane] = my_d;
  sw.cid[lane] = my_id;
  __syncwarp();
  const int nret = staged_prune<KIND>(sw, n, X, D, Dp, kind, max_degree, pd, row);
  uint32_t local_min = KEY_INF;
  for (int r = lane; r < nret; r += 32) {
    const int pos = sw.ret[r];
    const float dij = sw.dpos[pos];
    fwd_idx[(size_t)row * k + r] = sw.cid[pos];
    fwd_dist[(size_t)row * k + r] = dij;
    const float v = dij == 0.f ? FLT_EPSILON : dij;
    if (isfinite(v)) local_min = min(local_min, fkey(v));
  }
  for (int o = 16; o; o >>= 1) local_min = min(local_min, __shfl_xor_sync(0xffffffffu, local_min, o));
  if (lane == 0) {
    fwd_cnt[row] = nret;
    if (local_min != KEY_INF) atomicMin(min_key, local_min);
  }
}

__global__ void k_indegree(const int32_t* fwd_idx, const int32_t* fwd_cnt, int N, int k,
                           int32_t* indeg) {
  long long total = (long long)N * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e / k), r = (int)(e % k);
    if (r < fwd_cnt[i]) atomicAdd(&indeg[fwd_idx[e]], 1);
  }
}

__global__ void k_transpose(const int32_t* fwd_idx, const float* fwd_dist, const int32_t* fwd_cnt,
                            int N, int k, int32_t* cursor, uint64_t* rev_key) {
  long long total = (long long)N * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int i = (int)(e / k), r = (int)(e % k);
    if (r >= fwd_cnt[i]) continue;
    int32_t j = fwd_idx[e];
    int pos = atomicAdd(&cursor[j], 1);
    rev_key[pos] = ((uint64_t)fkey(fwd_dist[e]) << 32) | (uint32_t)i;
  }
}

template <int MAXR, int KIND>
__global__ void k_diversify_rev(const int32_t* rev_ptr, const uint64_t* rev_key, int N,
                                const float* X, int D, int Dp, int kind, int max_degree,
                                int32_t* rret_idx, float* rret_dist, int32_t* rret_cnt, PruneDraw pd) {
  __shared__ int32_t s_id[WARPS][MAXR];
  __shared__ float s_d[WARPS][MAXR];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * WARPS + w;
  if (row >= N) return;
  int nret = 0;
  const int e_end = rev_ptr[row + 1];
  for (int e = rev_ptr[row]; e < e_end; ++e) {
    uint64_t key = rev_key[e];
    int32_t j = (int32_t)(uint32_t)key;
    float dij = fkey_inv((uint32_t)(key >> 32));
    // warm L1 with the next candidate's row while this one is checked (the
    // candidate's row is the chain's global load; retained rows mostly hit L1)
    if (e + 1 < e_end && lane * 128 < Dp * 4) {
      const char* nxt = reinterpret_cast<const char*>(X + (size_t)(int32_t)(uint32_t)rev_key[e + 1] * Dp) + lane * 128;
      asm volatile("prefetch.global.L1 [%0];" ::"l"(nxt));
    }
    bool pruned = pruned_by_retained<KIND>(s_id[w], s_d[w], nret, j, dij, X, D, Dp, kind, pd, row);
    if (!pruned) {
      if (lane == 0) {
        s_id[w][nret] = j;
        s_d[w][nret] = dij;
      }
      __syncwarp();
      ++nret;
      if (nret >= max_degree) break;
    }
  }
  for (int r = lane; r < nret; r += 32) {
    rret_idx[(size_t)row * max_degree + r] = s_id[w][r];
    rret_dist[(size_t)row * max_degree + r] = s_d[w][r];
  }
  if (lane == 0) rret_cnt[row] = nret;
}

// Bitonic sort of b[0, n), n a power of two; entries from n on are ~0 (no
// smaller than any sorted key), so the whole array ends sorted.
__device__ __forceinline__ void warp_bitonic_n(uint64_t* b, int n) {
  const int lane = threadIdx.x & 31;
  for (int size = 2; size <= n; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int j = lane; j < n; j += 32) {
        int partner = j ^ stride;
        if (partner > j) {
          bool up = (j & size) == 0;
          uint64_t x = b[j], y = b[partner];
          if ((x > y) == up) {
            b[j] = y;
            b[partner] = x;
          }
        }
      }
      __syncwarp();
    }
}

// search_graph.rs:368-426 weighted_union_pruned, one warp per vertex.
template <int P>
__global__ void k_union(const int32_t* fwd_idx, const float* fwd_dist, const int32_t* fwd_cnt, int k,
                        const int32_t* rret_idx, const float* rret_dist, const int32_t* rret_cnt,
                        int N, int max_degree, int32_t* out_idx, int32_t* out_cnt) {
  __shared__ uint64_t buf[WARPS][P];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int v = blockIdx.x * WARPS + w;
  if (v >= N) return;
  uint64_t* b = buf[w];
  const int nf = fwd_cnt[v], nr = rret_cnt[v];
  int span = 32;  // sorts cover the live entries only (nf + nr <= P)
  while (span < nf + nr) span <<= 1;
  // (id, distance) keys; dropped entries become ~0.
  for (int e = lane; e < P; e += 32) {
    uint64_t key = ~0ull;
    int32_t id = -1;
    float d = 0.f;
    if (e < nf) {
      id = fwd_idx[(size_t)v * k + e];
      d = fwd_dist[(size_t)v * k + e];
    } else if (e < nf + nr) {
      id = rret_idx[(size_t)v * max_degree + (e - nf)];
      d = rret_dist[(size_t)v * max_degree + (e - nf)];
    }
    if (id >= 0 && id != v && isfinite(d)) key = ((uint64_t)(uint32_t)id << 32) | fkey(d);
    b[e] = key;
  }
  __syncwarp();
  warp_bitonic_n(b, span);
  // keep the last (max distance) entry of each id run; re-key by (distance, id)
  uint64_t nk[P / 32];
#pragma unroll
  for (int t = 0; t < P / 32; ++t) {
    int e = t * 32 + lane;
    uint64_t key = b[e];
    uint64_t out = ~0ull;
    if (key != ~0ull) {
      uint64_t nxt = e + 1 < P ? b[e + 1] : ~0ull;
      bool last = nxt == ~0ull || (nxt >> 32) != (key >> 32);
      if (last) out = ((key & 0xFFFFFFFFull) << 32) | (key >> 32);
    }
    nk[t] = out;
  }
  __syncwarp();
#pragma unroll
  for (int t = 0; t < P / 32; ++t) b[t * 32 + lane] = nk[t];
  __syncwarp();
  warp_bitonic_n(b, span);
  // first max_degree valid entries, re-keyed by id
#pragma unroll
  for (int t = 0; t < P / 32; ++t) {
    int e = t * 32 + lane;
    uint64_t key = b[e];
    nk[t] = (e < max_degree && key != ~0ull) ? (key & 0xFFFFFFFFull) : ~0ull;
  }
  __syncwarp();
#pragma unroll
  for (int t = 0; t < P / 32; ++t) b[t * 32 + lane] = nk[t];
  __syncwarp();
  warp_bitonic_n(b, span);
  int cnt = 0;
#pragma unroll
  for (int t = 0; t < P / 32; ++t) {
    int e = t * 32 + lane;
    uint64_t key = b[e];
    bool valid = key != ~0ull;
    cnt += __popc(__ballot_sync(0xffffffffu, valid));
    if (valid) out_idx[(size_t)v * max_degree + e] = (int32_t)key;
  }
  if (lane == 0) out_cnt[v] = cnt;
}

__global__ void k_compact(const int32_t* rows, int width, const int32_t* cnt, const int32_t* ptr,
                          int N, int32_t* out) {
  long long total = (long long)N * width;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int v = (int)(e / width), r = (int)(e % width);
    if (r < cnt[v]) out[ptr[v] + r] = rows[e];
  }
}

__global__ void k_reorder_count(const int32_t* in_ptr, const int32_t* order, int N, int32_t* cnt) {
  int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v < N) cnt[v] = in_ptr[order[v] + 1] - in_ptr[order[v]];
}
__global__ void k_reorder_fill(const int32_t* in_ptr, const int32_t* in_idx, const int32_t* order,
                               const int32_t* inverse, const int32_t* out_ptr, int N,
                               int32_t* out_idx) {
  int w = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (w >= N) return;
  int ov = order[w];
  int s = in_ptr[ov], e = in_ptr[ov + 1], o = out_ptr[w];
  for (int t = s + lane; t < e; t += 32) out_idx[o + (t - s)] = inverse[in_idx[t]];
}

template <class T>
void exclusive_scan(const T* in, T* out, long long n, TempStorage& tmp, cudaStream_t st) {
  size_t bytes = 0;
  RINND_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st));
  void* p = tmp.ensure(bytes, st);
  RINND_CUDA(cub::DeviceScan::ExclusiveSum(p, bytes, in, out, n, st));
}

}  // namespace

void build_search_graph(const int32_t* knn_idx, const float* knn_dist, const float* X, int N,
                        int k, int D, int Dp, int kind, float mult, cudaStream_t st,
                        TempStorage& tmp, Csr& out, float* min_distance_host, float prune_prob,
                        uint64_t seed) {
  const int max_degree = (int)roundf(mult * (float)k);  // f32::round (:276)
  const PruneDraw pd_fwd{prune_prob, seed}, pd_rev{prune_prob, seed ^ 0x5EEDull};
  if (k > 128 || max_degree < 1 || max_degree > 384)
    throw std::invalid_argument("search graph supports n_neighbors <= 128 and 1 <= round(mult * k) <= 384");
  const int blocks = (N + WARPS - 1) / WARPS;
  DVec<int32_t> fwd_idx((size_t)N * k, st), fwd_cnt((size_t)N, st);
  DVec<float> fwd_dist((size_t)N * k, st);
  DVec<uint32_t> min_key(1, st);
  RINND_CUDA(cudaMemcpyAsync(min_key.p, &KEY_INF, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  const size_t staged_bytes = StagedSmem::per_warp(Dp) * WARPS;
  const bool sq = kind == DK_SQEUCLIDEAN;
  if (k <= SK && Dp <= 256) {
    auto kern = sq ? k_diversify_fwd_staged<DK_SQEUCLIDEAN> : k_diversify_fwd_staged<-1>;
    set_smem_limit_once(reinterpret_cast<const void*>(kern), 227 * 1024);
    kern<<<blocks, 32 * WARPS, staged_bytes, st>>>(knn_idx, knn_dist, N, k, X, D, Dp, kind, max_degree, fwd_idx.p,
                                                   fwd_dist.p, fwd_cnt.p, min_key.p, pd_fwd);
  } else {
    auto kern = k <= 32 ? (sq ? k_diversify_fwd<32, DK_SQEUCLIDEAN> : k_diversify_fwd<32, -1>)
                        : (sq ? k_diversify_fwd<128, DK_SQEUCLIDEAN> : k_diversify_fwd<128, -1>);
    kern<<<blocks, 32 * WARPS, 0, st>>>(knn_idx, knn_dist, N, k, X, D, Dp, kind, max_degree, fwd_idx.p,
                                        fwd_dist.p, fwd_cnt.p, min_key.p, pd_fwd);
  }
  RINND_LAUNCH_CHECK();
  // transpose
  DVec<int32_t> indeg((size_t)N + 1, st), rev_ptr((size_t)N + 1, st), cursor((size_t)N + 1, st);
  indeg.fill_bytes(0);
  k_indegree<<<grid_for((long long)N * k, 256, 148 * 64), 256, 0, st>>>(fwd_idx.p, fwd_cnt.p, N, k, indeg.p);
  RINND_LAUNCH_CHECK();
  exclusive_scan(indeg.p, rev_ptr.p, (long long)N + 1, tmp, st);
  int32_t n_rev = 0;
  RINND_CUDA(cudaMemcpyAsync(&n_rev, rev_ptr.p + N, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaMemcpyAsync(cursor.p, rev_ptr.p, sizeof(int32_t) * ((size_t)N + 1),
                             cudaMemcpyDeviceToDevice, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  DVec<uint64_t> rev_key((size_t)std::max(n_rev, 1), st), rev_sorted((size_t)std::max(n_rev, 1), st);
  k_transpose<<<grid_for((long long)N * k, 256, 148 * 64), 256, 0, st>>>(fwd_idx.p, fwd_dist.p, fwd_cnt.p,
                                                                        N, k, cursor.p, rev_key.p);
  RINND_LAUNCH_CHECK();
  if (n_rev > 0) {
    size_t bytes = 0;
    RINND_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, bytes, rev_key.p, rev_sorted.p, n_rev, N,
                                                  rev_ptr.p, rev_ptr.p + 1, st));
    void* p = tmp.ensure(bytes, st);
    RINND_CUDA(cub::DeviceSegmentedSort::SortKeys(p, bytes, rev_key.p, rev_sorted.p, n_rev, N,
                                                  rev_ptr.p, rev_ptr.p + 1, st));
  }
  DVec<int32_t> rret_idx((size_t)N * max_degree, st), rret_cnt((size_t)N, st);
  DVec<float> rret_dist((size_t)N * max_degree, st);
  // (reverse rows stay sequential: they are short, and the early exits of the
  // sequential form beat the staged pair table there)
  {
    auto kern = max_degree <= 32 ? (sq ? k_diversify_rev<32, DK_SQEUCLIDEAN> : k_diversify_rev<32, -1>)
                : max_degree <= 64 ? (sq ? k_diversify_rev<64, DK_SQEUCLIDEAN> : k_diversify_rev<64, -1>)
                                   : (sq ? k_diversify_rev<384, DK_SQEUCLIDEAN> : k_diversify_rev<384, -1>);
    kern<<<blocks, 32 * WARPS, 0, st>>>(rev_ptr.p, rev_sorted.p, N, X, D, Dp, kind, max_degree, rret_idx.p,
                                        rret_dist.p, rret_cnt.p, pd_rev);
  }
  RINND_LAUNCH_CHECK();
  // union + prune
  DVec<int32_t> rows((size_t)N * max_degree, st), cnt((size_t)N + 1, st);
  RINND_CUDA(cudaMemsetAsync(cnt.p + N, 0, sizeof(int32_t), st));
  int need = k + max_degree;
  if (need <= 64)
    k_union<64><<<blocks, 32 * WARPS, 0, st>>>(fwd_idx.p, fwd_dist.p, fwd_cnt.p, k, rret_idx.p,
                                              rret_dist.p, rret_cnt.p, N, max_degree, rows.p, cnt.p);
  else if (need <= 128)
    k_union<128><<<blocks, 32 * WARPS, 0, st>>>(fwd_idx.p, fwd_dist.p, fwd_cnt.p, k, rret_idx.p,
                                               rret_dist.p, rret_cnt.p, N, max_degree, rows.p, cnt.p);
  else if (need <= 256)
    k_union<256><<<blocks, 32 * WARPS, 0, st>>>(fwd_idx.p, fwd_dist.p, fwd_cnt.p, k, rret_idx.p,
                                               rret_dist.p, rret_cnt.p, N, max_degree, rows.p, cnt.p);
  else
    k_union<512><<<blocks, 32 * WARPS, 0, st>>>(fwd_idx.p, fwd_dist.p, fwd_cnt.p, k, rret_idx.p,
                                               rret_dist.p, rret_cnt.p, N, max_degree, rows.p, cnt.p);
  RINND_LAUNCH_CHECK();
  out.N = N;
  out.indptr.alloc((size_t)N + 1, st);
  exclusive_scan(cnt.p, out.indptr.p, (long long)N + 1, tmp, st);
  int32_t nnz = 0;
  uint32_t mk = KEY_INF;
  RINND_CUDA(cudaMemcpyAsync(&nnz, out.indptr.p + N, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaMemcpyAsync(&mk, min_key.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  out.nnz = nnz;
  out.indices.alloc((size_t)std::max(nnz, 1), st);
  k_compact<<<grid_for((long long)N * max_degree, 256, 148 * 64), 256, 0, st>>>(rows.p, max_degree, cnt.p,
                                                                               out.indptr.p, N, out.indices.p);
  RINND_LAUNCH_CHECK();
  *min_distance_host = fkey_inv(mk);
}

void reorder_csr(const Csr& in, const int32_t* order, const int32_t* inverse, cudaStream_t st,
                 TempStorage& tmp, Csr& out) {
  const int N = in.N;
  out.N = N;
  out.nnz = in.nnz;
  DVec<int32_t> cnt((size_t)N + 1, st);
  RINND_CUDA(cudaMemsetAsync(cnt.p + N, 0, sizeof(int32_t), st));
  k_reorder_count<<<grid_for(N, 256), 256, 0, st>>>(in.indptr.p, order, N, cnt.p);
  RINND_LAUNCH_CHECK();
  out.indptr.alloc((size_t)N + 1, st);
  exclusive_scan(cnt.p, out.indptr.p, (long long)N + 1, tmp, st);
  out.indices.alloc((size_t)std::max<int64_t>(in.nnz, 1), st);
  k_reorder_fill<<<grid_for((long long)N * 32, 256), 256, 0, st>>>(in.indptr.p, in.indices.p, order,
                                                                   inverse, out.indptr.p, N, out.indices.p);
  RINND_LAUNCH_CHECK();
}

}  // namespace rinnd
