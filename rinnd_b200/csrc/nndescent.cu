// nndescent.cu -- NN-Descent on device-resident neighbor rows.
//
// Restates nn_descent (core/nndescent/mod.rs:79-197):
//   * leaf initialization (mod.rs:203-300): all pairs inside every RP leaf,
//     pushed both ways when d < the endpoint's threshold;
//   * candidate sampling (core/nndescent/candidates.rs:51-417): every heap edge
//     i->j is offered to i's and j's new/old candidate lists with one random
//     priority (the parallel reference reuses it for the reverse edge, :260);
//     lists keep the c lowest priorities without duplicates; neighbors that
//     made it into i's new list are then flagged old (mark_old_flags :354-417);
//   * local join (mod.rs:321-491): per vertex, new x new (q after p) and
//     new x old (q != p) candidate pairs; a pair is pushed into each endpoint's
//     row whose threshold it beats (the reference's `d <= max(thr_p, thr_q)`
//     followed by the per-row `d < root` check in checked_flagged_push).
// Rows are updated concurrently with the lock-free protocol in heap.cuh; the
// final row content equals the reference's sequential application (the k
// smallest distinct ids offered); the per-iteration change count is the number
// of successful pushes, as in the reference (mod.rs:473-481).
//
// The join is a tiled FP32 SIMT kernel: a CTA gathers the vertex's candidate
// rows chunk by chunk (32 dims) into shared memory in dimension-major layout and
// every thread accumulates a 4x4 block of pair distances in registers.
#include <cub/cub.cuh>

#include <cstring>

#include <vector>

#include "dist.cuh"
#include "engine.h"
#include "../../include/rinnd.h"
#include "heap.cuh"

namespace rinnd {
namespace {


__global__ void k_fill_u64(uint64_t* p, size_t n, uint64_t v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}
__global__ void k_fill_u32(uint32_t* p, size_t n, uint32_t v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void k_norms(const float* X, int N, int D, int Dp, float* norms) {
  int warp = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (warp >= N) return;
  const float* r = X + (size_t)warp * Dp;
  float s = 0.f;
  for (int i = lane; i < D; i += 32) s = fmaf(r[i], r[i], s);
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) norms[warp] = s;
}

// ---------------------------------------------------------------------------
// Pair join.  A job is a set A (na <= MAXA ids) against a set B (nb <= MAXB
// ids); the pairs are the rectangle A x B minus, where A is a prefix of B, the
// diagonal and lower triangle of A x A, and in a vertex job the new x old pairs
// with equal ids.  Rows are staged in shared memory JDC dimensions at a time,
// row-major with a 4-float pad (conflict-free 16-byte loads); each thread owns
// up to PPT pairs and accumulates their distances in registers.  Pairs that
// beat an endpoint's threshold are appended to a global update buffer (one
// atomic per warp); k_apply_updates performs the lock-free pushes in a
// separate, fully parallel launch.  Updates beyond the buffer capacity are
// pushed directly by the join thread.
// ---------------------------------------------------------------------------
constexpr int JDC = 64;        // dimensions per staged chunk
constexpr int JROW = JDC + 4;  // staged row stride in floats

enum JoinMode : int { MODE_JOIN = 0, MODE_TRI = 1, MODE_RECT = 2 };

template <int MAXA, int MAXB, int AROWS = MAXA>
struct __align__(16) PairSmem {
  int32_t aid[MAXA];
  int32_t bid[MAXB];
  uint32_t athr[MAXA];
  uint32_t bthr[MAXB];
  float an[MAXA];
  float bn[MAXB];
  float rows[(MAXB + AROWS) * JROW];  // B rows, then A rows (RECT only; AROWS = 0 when A prefixes B)
  unsigned int pairs;
  int na, nb;
};

struct UpdateBuf {
  uint32_t* row;
  uint64_t* key;
  unsigned long long* count;  // total appended (may exceed cap)
  unsigned long long cap;
  ItemCount ic;               // per-index accounting of direct pushes (grouped builds)
};

__device__ __forceinline__ void stage_rows(const float* __restrict__ X, int Dp, int c0, const int32_t* ids,
                                           int n, float* dst) {
  constexpr int Q = JDC / 4;
  for (int e = threadIdx.x; e < n * Q; e += blockDim.x) {
    int r = e / Q, q = e % Q;
    int d = c0 + 4 * q;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (d < Dp) v = __ldg(reinterpret_cast<const float4*>(X + (size_t)ids[r] * Dp + d));
    *reinterpret_cast<float4*>(dst + r * JROW + 4 * q) = v;
  }
}

template <int MAXA, int MAXB, int AROWS>
__device__ __forceinline__ void load_meta(PairSmem<MAXA, MAXB, AROWS>& sm, int na, int nb, bool a_prefix,
                                          const uint32_t* thr, const float* norms) {
  for (int t = threadIdx.x; t < nb; t += blockDim.x) {
    sm.bthr[t] = __ldcg(thr + sm.bid[t]);
    if (norms) sm.bn[t] = norms[sm.bid[t]];
  }
  if (!a_prefix)
    for (int t = threadIdx.x; t < na; t += blockDim.x) {
      sm.athr[t] = __ldcg(thr + sm.aid[t]);
      if (norms) sm.an[t] = norms[sm.aid[t]];
    }
}

template <int MAXA, int MAXB, int AROWS, int NT>
__device__ __forceinline__ void join_pairs(PairSmem<MAXA, MAXB, AROWS>& sm, int na, int nb, int mode,
                                           const float* __restrict__ X, int Dp, int kind, uint64_t* slots,
                                           uint32_t* thr, int k, int kp, UpdateBuf ub,
                                           unsigned long long* counters, bool direct = false) {
  constexpr int PPT = (MAXA * MAXB + NT - 1) / NT;
  const bool a_prefix = mode != MODE_RECT;
  const float* rowsB = sm.rows;
  const float* rowsA = a_prefix ? sm.rows : sm.rows + MAXB * JROW;
  const int npairs = na * nb;
  const int tid = threadIdx.x;
  // validity mask of this thread's pairs
  unsigned valid_mask = 0;
#pragma unroll
  for (int s = 0; s < PPT; ++s) {
    int t = tid + s * NT;
    if (t < npairs) {
      int i = t / nb, j = t % nb;
      bool v;
      if (mode == MODE_RECT) v = true;
      else if (j < na) v = j > i;                               // A x A: q after p (mod.rs:396)
      else v = (mode == MODE_JOIN) && (sm.bid[j] != sm.bid[i]);  // new x old: q != p (mod.rs:424)
      if (v) valid_mask |= 1u << s;
    }
  }
  float acc[PPT];
#pragma unroll
  for (int s = 0; s < PPT; ++s) acc[s] = 0.f;
  for (int c0 = 0; c0 < Dp; c0 += JDC) {
    __syncthreads();
    stage_rows(X, Dp, c0, sm.bid, nb, sm.rows);
    if (AROWS > 0 && !a_prefix) stage_rows(X, Dp, c0, sm.aid, na, sm.rows + MAXB * JROW);
    __syncthreads();
#pragma unroll
    for (int s = 0; s < PPT; ++s) {
      if (valid_mask & (1u << s)) {
        int t = tid + s * NT;
        const float4* a = reinterpret_cast<const float4*>(rowsA + (t / nb) * JROW);
        const float4* b = reinterpret_cast<const float4*>(rowsB + (t % nb) * JROW);
        float x = acc[s];
        if (kind == DK_SQEUCLIDEAN) {
#pragma unroll
          for (int q = 0; q < JDC / 4; ++q) {
            float4 u = a[q], w = b[q];
            float d0 = u.x - w.x, d1 = u.y - w.y, d2 = u.z - w.z, d3 = u.w - w.w;
            x = fmaf(d0, d0, x); x = fmaf(d1, d1, x); x = fmaf(d2, d2, x); x = fmaf(d3, d3, x);
          }
        } else if (kind == DK_MANHATTAN) {
#pragma unroll
          for (int q = 0; q < JDC / 4; ++q) {
            float4 u = a[q], w = b[q];
            x += fabsf(u.x - w.x) + fabsf(u.y - w.y) + fabsf(u.z - w.z) + fabsf(u.w - w.w);
          }
        } else {
#pragma unroll
          for (int q = 0; q < JDC / 4; ++q) {
            float4 u = a[q], w = b[q];
            x = fmaf(u.x, w.x, x); x = fmaf(u.y, w.y, x); x = fmaf(u.z, w.z, x); x = fmaf(u.w, w.w, x);
          }
        }
        acc[s] = x;
      }
    }
  }
  // ---- filter, then emit updates (warp-aggregated append) ----
  const bool is_dot = kind_is_dot(kind);
  uint32_t kd[PPT];
  unsigned emit_p = 0, emit_q = 0;
  int n_emit = 0;
#pragma unroll
  for (int s = 0; s < PPT; ++s) {
    kd[s] = 0;
    if (valid_mask & (1u << s)) {
      int t = tid + s * NT;
      int i = t / nb, j = t % nb;
      float d = acc[s];
      if (is_dot) d = finalize_dot(kind, d, a_prefix ? sm.bn[i] : sm.an[i], sm.bn[j]);
      kd[s] = fkey(d);
      uint32_t tp = a_prefix ? sm.bthr[i] : sm.athr[i];
      if (kd[s] < tp) { emit_p |= 1u << s; ++n_emit; }
      if (kd[s] < sm.bthr[j]) { emit_q |= 1u << s; ++n_emit; }
    }
  }
  if (direct) {
    // MODE_TRI job over rows nothing else writes, all empty (first tree's leaf
    // of at most k + 1 points): every passing (row, id) has its own slot --
    // row of point i holds point j at slot j - 1 (j > i), row of j holds i at
    // slot i -- the keys the updates would carry, in place of the updates.
#pragma unroll
    for (int s = 0; s < PPT; ++s) {
      if ((emit_p | emit_q) & (1u << s)) {
        const int t = tid + s * NT;
        const int i = t / nb, j = t % nb;
        const int32_t p = sm.bid[i], q = sm.bid[j];
        if (emit_p & (1u << s)) slots[(size_t)p * kp + (j - 1)] = ((uint64_t)kd[s] << 32) | (uint32_t)q | 0x80000000u;
        if (emit_q & (1u << s)) slots[(size_t)q * kp + i] = ((uint64_t)kd[s] << 32) | (uint32_t)p | 0x80000000u;
      }
    }
    const unsigned int my_pairs = __popc(valid_mask);
    if (my_pairs) atomicAdd(&sm.pairs, my_pairs);
    return;
  }
  const int lane = tid & 31;
  int incl = n_emit;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  int warp_total = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long base = 0;
  if (lane == 0 && warp_total) base = atomicAdd(ub.count, (unsigned long long)warp_total);
  base = __shfl_sync(0xffffffffu, base, 0) + (unsigned long long)(incl - n_emit);
  unsigned int my_pairs = __popc(valid_mask);
#pragma unroll
  for (int s = 0; s < PPT; ++s) {
    if ((emit_p | emit_q) & (1u << s)) {
      int t = tid + s * NT;
      int i = t / nb, j = t % nb;
      int32_t p = a_prefix ? sm.bid[i] : sm.aid[i], q = sm.bid[j];
      for (int side = 0; side < 2; ++side) {
        if (!((side == 0 ? emit_p : emit_q) & (1u << s))) continue;
        uint32_t row = side == 0 ? (uint32_t)p : (uint32_t)q;
        uint64_t key = ((uint64_t)kd[s] << 32) | (uint32_t)(side == 0 ? q : p) | 0x80000000u;
        if (base < ub.cap) {
          ub.row[base] = row;
          ub.key[base] = key;
        } else if (row_push(slots + (size_t)row * kp, k, thr + row, key, &counters[1])) {
          atomicAdd(&counters[0], 1ull);
          ub.ic.add(row);
        }
        ++base;
      }
    }
  }
  if (my_pairs) atomicAdd(&sm.pairs, my_pairs);
}

// One CTA per vertex (grid-stride over [v0, v1)): A = new candidates, B = new ++ old.
template <int MAXC, int NT>
__global__ void __launch_bounds__(NT)
    k_local_join(const uint64_t* cand_new, const uint64_t* cand_old, int v0, int v1, int c, int cp,
                 const float* __restrict__ X, int Dp, int kind, const float* norms, uint64_t* slots,
                 uint32_t* thr, int k, int kp, UpdateBuf ub, unsigned long long* counters) {
  __shared__ PairSmem<MAXC, 2 * MAXC, 0> sm;
  for (int v = v0 + blockIdx.x; v < v1; v += gridDim.x) {
    __syncthreads();
    if (threadIdx.x == 0) sm.pairs = 0;
    if (threadIdx.x < 32) {  // compact valid ids, new first then old
      int lane = threadIdx.x;
      int base = 0;
      for (int t0 = 0; t0 < c; t0 += 32) {
        int t = t0 + lane;
        int32_t id = t < c ? slot_id(cand_new[(size_t)v * cp + t]) : -1;
        unsigned m = __ballot_sync(0xffffffffu, id >= 0);
        if (id >= 0) sm.bid[base + __popc(m & ((1u << lane) - 1))] = id;
        base += __popc(m);
      }
      int na = base;
      for (int t0 = 0; t0 < c; t0 += 32) {
        int t = t0 + lane;
        int32_t id = t < c ? slot_id(cand_old[(size_t)v * cp + t]) : -1;
        unsigned m = __ballot_sync(0xffffffffu, id >= 0);
        if (id >= 0) sm.bid[base + __popc(m & ((1u << lane) - 1))] = id;
        base += __popc(m);
      }
      if (lane == 0) {
        sm.na = na;
        sm.nb = base;
      }
    }
    __syncthreads();
    const int na = sm.na, nb = sm.nb;
    if (na == 0) continue;  // uniform across the CTA
    load_meta(sm, na, nb, true, thr, kind_is_dot(kind) ? norms : nullptr);
    join_pairs<MAXC, 2 * MAXC, 0, NT>(sm, na, nb, MODE_JOIN, X, Dp, kind, slots, thr, k, kp, ub, counters);
    __syncthreads();
    if (threadIdx.x == 0) {
      atomicAdd(&counters[2], (unsigned long long)sm.pairs);
      atomicAdd(&counters[3], (unsigned long long)nb);
    }
  }
}

// ---------------------------------------------------------------------------
// Generic metrics (the reference's other metrics, core/distance/{minkowski,
// angular,binary,hellinger}.rs): the same pairs and pushes as the tiled joins,
// each pair's distance evaluated by one thread with exact_distance from the rows
// in global memory (the tiles' dot / difference forms do not apply to them).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void emit_generic(UpdateBuf ub, uint32_t row, uint64_t key, uint64_t* slots, uint32_t* thr,
                                             int k, int kp, unsigned long long* counters) {
  const unsigned long long at = atomicAdd(ub.count, 1ull);
  if (at < ub.cap) {
    ub.row[at] = row;
    ub.key[at] = key;
  } else if (row_push(slots + (size_t)row * kp, k, thr + row, key, &counters[1])) {
    atomicAdd(&counters[0], 1ull);
    ub.ic.add(row);
  }
}

// Pair (p, q) of ids with thresholds tp, tq: pushed into each row it beats.
__device__ __forceinline__ void generic_pair(int kind, const float* X, int D, int Dp, int32_t p, int32_t q, uint32_t tp,
                                             uint32_t tq, UpdateBuf ub, uint64_t* slots, uint32_t* thr, int k, int kp,
                                             unsigned long long* counters) {
  const float d = exact_distance(kind, X + (size_t)p * Dp, X + (size_t)q * Dp, D);
  const uint32_t kd = fkey(d);
  if (kd < tp) emit_generic(ub, (uint32_t)p, ((uint64_t)kd << 32) | (uint32_t)q | 0x80000000u, slots, thr, k, kp, counters);
  if (kd < tq) emit_generic(ub, (uint32_t)q, ((uint64_t)kd << 32) | (uint32_t)p | 0x80000000u, slots, thr, k, kp, counters);
}

// One CTA per vertex (grid-stride over [v0, v1)): new x new (q after p) and new x old (q != p).
template <int MAXC>
__global__ void k_local_join_generic(const uint64_t* cand_new, const uint64_t* cand_old, int v0, int v1, int c, int cp,
                                     const float* __restrict__ X, int D, int Dp, int kind, uint64_t* slots, uint32_t* thr,
                                     int k, int kp, UpdateBuf ub, unsigned long long* counters) {
  __shared__ int32_t ids[2 * MAXC];
  __shared__ uint32_t th[2 * MAXC];
  __shared__ int s_na, s_nb;
  for (int v = v0 + blockIdx.x; v < v1; v += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < 32) {  // compact valid ids, new first then old
      const int lane = threadIdx.x;
      int base = 0;
      for (int list = 0; list < 2; ++list) {
        const uint64_t* L = (list ? cand_old : cand_new) + (size_t)v * cp;
        for (int t0 = 0; t0 < c; t0 += 32) {
          const int t = t0 + lane;
          const int32_t id = t < c ? slot_id(L[t]) : -1;
          const unsigned m = __ballot_sync(0xffffffffu, id >= 0);
          if (id >= 0) ids[base + __popc(m & ((1u << lane) - 1))] = id;
          base += __popc(m);
        }
        if (list == 0 && lane == 0) s_na = base;
      }
      if (lane == 0) s_nb = base;
    }
    __syncthreads();
    const int na = s_na, nb = s_nb;
    if (na == 0) continue;  // uniform across the CTA
    for (int t = threadIdx.x; t < nb; t += blockDim.x) th[t] = __ldcg(thr + ids[t]);
    __syncthreads();
    unsigned int pairs = 0;
    for (int e = threadIdx.x; e < na * nb; e += blockDim.x) {
      const int i = e / nb, j = e - i * nb;
      const bool valid = j < na ? j > i : ids[j] != ids[i];  // mod.rs:396, :424
      if (!valid) continue;
      ++pairs;
      generic_pair(kind, X, D, Dp, ids[i], ids[j], th[i], th[j], ub, slots, thr, k, kp, counters);
    }
    for (int o = 16; o; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(&counters[2], (unsigned long long)pairs);
    if (threadIdx.x == 0) atomicAdd(&counters[3], (unsigned long long)nb);
  }
}

// Leaf jobs (leaf, block a, block b) of BS points: the pairs of initialize_from_leaves
// (mod.rs:203-300), evaluated per thread.
__global__ void k_leaf_join_generic(const int4* jobs, long long j0, long long j1, const int4* leaves, const int32_t* perm,
                                    int N, int BS, const float* __restrict__ X, int D, int Dp, int kind, uint64_t* slots,
                                    uint32_t* thr, int k, int kp, UpdateBuf ub, unsigned long long* counters) {
  for (long long jb = j0 + blockIdx.x; jb < j1; jb += gridDim.x) {
    const int4 job = jobs[jb];
    const int4 leaf = leaves[job.x];
    const int32_t* P = perm + (size_t)leaf.x * N + leaf.y;
    const int L = leaf.z - leaf.y;
    const int a0 = job.y * BS, b0 = job.z * BS;
    const int na = min(BS, L - a0), nb = min(BS, L - b0);
    const bool tri = job.y == job.z;
    unsigned int pairs = 0;
    for (int e = threadIdx.x; e < na * nb; e += blockDim.x) {
      const int i = e / nb, j = e - i * nb;
      if (tri && j <= i) continue;
      ++pairs;
      const int32_t p = P[a0 + i], q = P[b0 + j];
      generic_pair(kind, X, D, Dp, p, q, __ldcg(thr + p), __ldcg(thr + q), ub, slots, thr, k, kp, counters);
    }
    for (int o = 16; o; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    if ((threadIdx.x & 31) == 0 && pairs) atomicAdd(&counters[2], (unsigned long long)pairs);
  }
}

// Lock-free pushes of buffered updates (heap.cuh protocol).
// Entry handled in place e of n: consecutive entries of the leaf initialization
// come from one leaf block and target the same few rows (all racing for an
// empty row's max slot in the first trees), so they are spread over the launch
// (e * P mod n, a bijection when the prime P does not divide n).
__device__ __forceinline__ unsigned long long spread_entry(unsigned long long e, unsigned long long n) {
  constexpr unsigned long long P = 1000003ull;
  return n % P ? (e * P) % n : e;
}

__global__ void k_apply_updates(const uint32_t* urow, const uint64_t* ukey, const unsigned long long* count,
                                unsigned long long cap, uint64_t* slots, uint32_t* thr, int k, int kp,
                                unsigned long long* counters, bool spread, ItemCount ic) {
  const unsigned long long n = min(*count, cap);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    atomicAdd(&counters[5], n);
    atomicAdd(&counters[6], *count);  // appended, including overflow pushed directly
  }
  unsigned int mine = 0;
  ItemTally tally;
  for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < n;
       e += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long x = spread ? spread_entry(e, n) : e;
    uint32_t r = urow[x];
    if (row_push_fast(slots + (size_t)r * kp, k, thr + r, ukey[x], &counters[1])) {
      ++mine;
      tally.add(ic, r);
    }
  }
  tally.flush(ic);
  for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&counters[0], (unsigned long long)mine);
}

// k_apply_updates for the region form: region r of the buffer holds rcnt[r]
// updates from entry r * rsize; `sub` blocks share a region.  Updates under
// their row's bound are queued per warp and pushed 32 at a time (WarpQueue;
// 1.77 -> 1.60 ms per launch at 400k x 128, k = 30; the same queue in the
// reverse candidate offers was slower at 1M).  Launched with 256 threads.
__global__ void k_apply_regions(const uint32_t* urow, const uint64_t* ukey, const uint32_t* rcnt, int nreg,
                                unsigned int rsize, int sub, const unsigned long long* count, uint64_t* slots,
                                uint32_t* thr, int k, int kp, unsigned long long* counters, ItemCount ic) {
  const int r = blockIdx.x / sub, part = blockIdx.x - r * sub;
  if (r >= nreg) return;
  const unsigned int cnt = rcnt[r];
  if (threadIdx.x == 0) {
    if (part == 0) atomicAdd(&counters[5], (unsigned long long)cnt);
    if (blockIdx.x == 0) atomicAdd(&counters[6], *count);  // appended, including overflow pushed directly
  }
  const size_t base = (size_t)r * rsize;
  unsigned int mine = 0;
  ItemTally tally;
  __shared__ uint32_t q_row[8][64];
  __shared__ uint64_t q_key[8][64];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpQueue q{q_row[w], q_key[w], 0};
  uint32_t row;
  uint64_t key;
  auto push = [&]() {
    if (row_push_fast(slots + (size_t)row * kp, k, thr + row, key, &counters[1])) {
      ++mine;
      tally.add(ic, row);
    }
  };
  // (in order: the join's updates rarely share rows within a warp, and reads
  // in order are cheaper than spread ones)
  for (unsigned int e0 = part * blockDim.x + w * 32; e0 < cnt; e0 += sub * blockDim.x) {
    const unsigned int e = e0 + lane;
    bool pass = false;
    uint32_t rr = 0;
    uint64_t kk = 0;
    if (e < cnt) {
      rr = urow[base + e];
      kk = ukey[base + e];
      pass = (uint32_t)(kk >> 32) < __ldcg(thr + rr);
    }
    if (q.append(pass, rr, kk, row, key)) push();
  }
  if (q.drain(row, key)) push();
  tally.flush(ic);
  for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(&counters[0], (unsigned long long)mine);
}

// Leaf jobs: blocks of BS points of one leaf, (a, b) with a <= b.
__global__ void k_leaf_job_count(const int4* leaves, long long nl, int BS, int32_t* cnt) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nl;
       i += (long long)gridDim.x * blockDim.x) {
    int L = leaves[i].z - leaves[i].y;
    int nb = (L + BS - 1) / BS;
    cnt[i] = L >= 2 ? nb * (nb + 1) / 2 : 0;
  }
}
__global__ void k_leaf_job_emit(const int4* leaves, long long nl, int BS, const int32_t* off,
                                int4* jobs) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nl;
       i += (long long)gridDim.x * blockDim.x) {
    int L = leaves[i].z - leaves[i].y;
    if (L < 2) continue;
    int nb = (L + BS - 1) / BS;
    int o = off[i];
    for (int a = 0; a < nb; ++a)
      for (int b = a; b < nb; ++b) jobs[o++] = make_int4((int)i, a, b, 0);
  }
}

// nndescent/mod.rs:203-300 initialize_from_leaves, one CTA per (leaf, block pair).
// Pass 1 (first, on empty rows) takes only the first tree's leaves of at most
// min(BS, k + 1) points: each is one job, its rows belong to no other leaf of
// that tree, and all its passing pairs fit the rows, so it writes its slots
// directly.  Pass 0 takes every other job and appends updates.
template <int BS, int NT>
__global__ void __launch_bounds__(NT)
    k_leaf_join(const int4* jobs, long long j0, long long j1, const int4* leaves, const int32_t* perm, int N,
                const float* __restrict__ X, int Dp, int kind, const float* norms, uint64_t* slots,
                uint32_t* thr, int k, int kp, UpdateBuf ub, unsigned long long* counters, int pass) {
  __shared__ PairSmem<BS, BS, BS> sm;
  for (long long jb = j0 + blockIdx.x; jb < j1; jb += gridDim.x) {
    int4 job = jobs[jb];
    int4 leaf = leaves[job.x];
    const int32_t* P = perm + (size_t)leaf.x * N + leaf.y;
    int L = leaf.z - leaf.y;
    const bool direct = leaf.x == 0 && L <= BS && L <= k + 1;
    if (direct != (pass == 1)) continue;  // uniform over the CTA
    int a0 = job.y * BS, b0 = job.z * BS;
    int na = min(BS, L - a0), nb = min(BS, L - b0);
    int mode = job.y == job.z ? MODE_TRI : MODE_RECT;
    __syncthreads();
    if (threadIdx.x == 0) sm.pairs = 0;
    for (int t = threadIdx.x; t < nb; t += blockDim.x) sm.bid[t] = P[b0 + t];
    for (int t = threadIdx.x; t < na; t += blockDim.x) sm.aid[t] = P[a0 + t];
    __syncthreads();
    load_meta(sm, na, nb, mode != MODE_RECT, thr, kind_is_dot(kind) ? norms : nullptr);
    join_pairs<BS, BS, BS, NT>(sm, na, nb, mode, X, Dp, kind, slots, thr, k, kp, ub, counters, direct);
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&counters[2], (unsigned long long)sm.pairs);
  }
}

// candidates.rs:153-351: each heap edge i->j is offered to i's list (forward)
// and to j's list (reverse) with one random priority; a list keeps the c
// lowest priorities with distinct ids.  Forward offers to list i all come from
// row i, so one warp per row selects them without atomics (k_cand_forward) and
// records the list's priority bound; reverse offers then go through the
// lock-free push with that bound as a pre-filter (k_cand_reverse).
// The priority of edge (row, id) is a hash of (seed, iteration, {row, id}): a
// uniform draw per pair, used for both endpoints' lists like the reference's
// one draw pushed to both sides (candidates.rs:171-223).  It does not depend on
// where the entry sits in its row (slot order follows the order of concurrent
// pushes) nor on which endpoint's row holds the edge, so a candidate offered
// twice carries one key and the lists are a function of the rows' contents:
// runs (and join precisions) from equal rows sample alike.
// salt = cand_salt(seed, iter), computed once per iteration on the host.
__host__ __device__ __forceinline__ uint64_t cand_salt(uint64_t seed, int iter) {
  return seed ^ mix64(0xC0DE0000ull + (uint64_t)iter);
}
__device__ __forceinline__ uint32_t cand_priority(uint64_t salt, int row, int32_t id) {
  const uint32_t lo = (uint32_t)min(row, (int)id), hi = (uint32_t)max(row, (int)id);
  const uint64_t edge = ((uint64_t)lo << 32) | hi;
  return (uint32_t)(mix64(salt ^ edge) >> 33);
}

template <int P>
__global__ void k_cand_forward(const uint64_t* slots, int N, int k, int kp, int c, int cp, uint64_t* cnew,
                               uint64_t* cold, uint32_t* thr_new, uint32_t* thr_old, uint64_t salt,
                               GroupRows grp) {
  __shared__ uint64_t buf[4][P];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * 4 + w;
  if (row >= N) return;
  if (grp.frozen(row)) {  // a finished index of a grouped build: empty lists that accept no offer
    for (int t = lane; t < c; t += 32) {
      cnew[(size_t)row * cp + t] = CAND_EMPTY;
      cold[(size_t)row * cp + t] = CAND_EMPTY;
    }
    if (lane == 0) {
      thr_new[row] = 0u;
      thr_old[row] = 0u;
    }
    return;
  }
  uint64_t* b = buf[w];
  for (int flag = 1; flag >= 0; --flag) {
    int n = 0;
    for (int j0 = 0; j0 < P; j0 += 32) {
      int j = j0 + lane;
      uint64_t key = ~0ull;
      if (j < k) {
        uint64_t sl = slots[(size_t)row * kp + j];
        int32_t id = slot_id(sl);
        if (id >= 0 && slot_new(sl) == flag)
          key = ((uint64_t)cand_priority(salt, row, id) << 32) | (uint32_t)id;
      }
      n += __popc(__ballot_sync(0xffffffffu, key != ~0ull));
      b[j] = key;
    }
    __syncwarp();
    if (n > c) {  // keep the c lowest priorities (bitonic sort of P keys)
      for (int size = 2; size <= P; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
          for (int j = lane; j < P; j += 32) {
            int partner = j ^ stride;
            if (partner > j) {
              bool up = (j & size) == 0;
              uint64_t x = b[j], y = b[partner];
              if ((x > y) == up) { b[j] = y; b[partner] = x; }
            }
          }
          __syncwarp();
        }
    } else {  // compact in slot order
      uint64_t keep[P / 32];
#pragma unroll
      for (int t = 0; t < P / 32; ++t) keep[t] = b[t * 32 + lane];
      __syncwarp();
      int base = 0;
#pragma unroll
      for (int t = 0; t < P / 32; ++t) {
        unsigned m = __ballot_sync(0xffffffffu, keep[t] != ~0ull);
        if (keep[t] != ~0ull) b[base + __popc(m & ((1u << lane) - 1))] = keep[t];
        base += __popc(m);
      }
      __syncwarp();
    }
    uint64_t* list = (flag ? cnew : cold) + (size_t)row * cp;
    const int kept = min(n, c);
    for (int t = lane; t < c; t += 32) list[t] = t < kept ? b[t] : CAND_EMPTY;
    uint32_t bound = 0xFFFFFFFFu;  // accepts any priority until the list is full
    if (kept == c) {
      uint32_t mx = 0;
      for (int t = lane; t < kept; t += 32) mx = max(mx, (uint32_t)(b[t] >> 32));
      for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      bound = mx;
    }
    if (lane == 0) (flag ? thr_new : thr_old)[row] = bound;
    __syncwarp();
  }
}

// One warp per row (lane = slot): each of the row's entries is offered to its
// neighbor's list.
__global__ void k_cand_reverse(const uint64_t* slots, int N, int k, int kp, int c, int cp, uint64_t* cnew,
                               uint64_t* cold, uint32_t* thr_new, uint32_t* thr_old, uint64_t salt,
                               unsigned long long* contention, GroupRows grp) {
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < N; r += nwarps) {
    const int32_t i = (int32_t)r;
    if (grp.frozen(i)) continue;  // (a frozen row's neighbors are frozen rows too)
    for (int j = lane; j < k; j += 32) {
      const uint64_t sl = slots[(size_t)i * kp + j];
      const int32_t id = slot_id(sl);
      if (id < 0) continue;
      const bool nw = slot_new(sl);
      const uint64_t key = ((uint64_t)cand_priority(salt, i, id) << 32) | (uint32_t)i;
      row_push_fast((nw ? cnew : cold) + (size_t)id * cp, c, (nw ? thr_new : thr_old) + id, key, contention);
    }
  }
}

// candidates.rs:354-417 mark_old_flags, one warp per row.
// The new list is read once per warp (list entry t in lane t % 32) and each
// slot's id is tested against it by shuffles.
__global__ void k_mark_old(uint64_t* slots, int N, int k, int kp, const uint64_t* cnew, int c, int cp) {
  int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  int lane = threadIdx.x & 31;
  if (row >= N) return;
  const uint64_t* nl = cnew + (size_t)row * cp;
  const int32_t l0 = lane < c ? slot_id(nl[lane]) : -1;
  const int32_t l1 = lane + 32 < c ? slot_id(nl[lane + 32]) : -1;  // c <= 64
  for (int j0 = 0; j0 < k; j0 += 32) {
    int j = j0 + lane;
    uint64_t s = j < k ? slots[(size_t)row * kp + j] : SLOT_EMPTY;
    int32_t id = slot_id(s);
    const bool want = id >= 0 && slot_new(s);
    bool hit = false;
    if (__any_sync(0xffffffffu, want)) {
      for (int t = 0; t < 32 && t < c; ++t) hit |= __shfl_sync(0xffffffffu, l0, t) == id;
      for (int t = 0; t + 32 < c; ++t) hit |= __shfl_sync(0xffffffffu, l1, t) == id;
    }
    if (want && hit) slots[(size_t)row * kp + j] = s & ~(1ull << 31);
  }
}

// neighbor_heap.rs:293-320 sort_all: rows ascending by distance (ties by id),
// one warp per row, bitonic sort of P = next_pow2(k) keys in shared memory.
// Sort key = (fkey(d) << 32) | (id << 1) | flag; empty = ~0.
template <int P>
__global__ void k_finalize(const uint64_t* slots, int N, int k, int kp, int32_t* out_idx, float* out_dist,
                           uint8_t* out_flags) {
  __shared__ uint64_t buf[4][P];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int row = blockIdx.x * 4 + w;
  if (row >= N) return;
  uint64_t* b = buf[w];
  for (int j = lane; j < P; j += 32) {
    uint64_t key = ~0ull;
    if (j < k) {
      uint64_t s = slots[(size_t)row * kp + j];
      uint32_t lo = (uint32_t)s;
      if (lo != LO_EMPTY) key = (s & 0xFFFFFFFF00000000ull) | (((lo & 0x7FFFFFFFu) << 1) | (lo >> 31));
    }
    b[j] = key;
  }
  __syncwarp();
  for (int size = 2; size <= P; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int j = lane; j < P; j += 32) {
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
  for (int j = lane; j < k; j += 32) {
    uint64_t key = b[j];
    bool empty = key == ~0ull;
    uint32_t lo = (uint32_t)key;
    out_idx[(size_t)row * k + j] = empty ? -1 : (int32_t)(lo >> 1);
    out_dist[(size_t)row * k + j] = empty ? __int_as_float(0x7f800000) : fkey_inv((uint32_t)(key >> 32));
    if (out_flags) out_flags[(size_t)row * k + j] = empty ? 0 : (uint8_t)(lo & 1u);
  }
}

template <class T>
void exclusive_scan(const T* in, T* out, long long n, TempStorage& tmp, cudaStream_t st) {
  size_t bytes = 0;
  RINND_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st));
  void* p = tmp.ensure(bytes, st);
  RINND_CUDA(cub::DeviceScan::ExclusiveSum(p, bytes, in, out, n, st));
}

}  // namespace

void knn_init(KnnState& s, int N, int k, int c, cudaStream_t st) {
  s.N = N;
  s.k = k;
  s.c = c;
  s.kp = row_stride(k);
  s.cp = row_stride(c);
  s.slots.alloc((size_t)N * s.kp, st);
  s.thr.alloc((size_t)N, st);
  s.cand_new.alloc((size_t)N * s.cp, st);
  s.cand_old.alloc((size_t)N * s.cp, st);
  s.counters.alloc(8, st);
  s.counters.fill_bytes(0);
  k_fill_u64<<<grid_for((long long)N * s.kp, 256, 148 * 32), 256, 0, st>>>(s.slots.p, s.slots.n, SLOT_EMPTY);
  k_fill_u32<<<grid_for(N, 256, 148 * 32), 256, 0, st>>>(s.thr.p, s.thr.n, KEY_INF);
  RINND_LAUNCH_CHECK();
}

void compute_norms(const float* X, int N, int D, int Dp, float* norms, cudaStream_t st) {
  k_norms<<<grid_for((long long)N * 32, 256), 256, 0, st>>>(X, N, D, Dp, norms);
  RINND_LAUNCH_CHECK();
}

void ensure_update_buffer(KnnState& s, cudaStream_t st) {
  if (s.ucap) return;
  // Sized for one whole join iteration: at most ~70 buffered updates per vertex were
  // seen on 1M-point mixtures (k = 30); overflow falls back to direct pushes.
  s.ucap = std::max<unsigned long long>(1ull << 22, 96ull * (unsigned long long)s.N);
  s.urow.alloc(s.ucap, st);
  s.ukey.alloc(s.ucap, st);
}

namespace {
// `spread`: apply in the spread order (leaf-initialization updates).
void apply_pending(KnnState& s, cudaStream_t st, bool spread = false) {
  if (s.nreg > 0) {
    const int sub = std::max(1, (148 * 16) / s.nreg);
    k_apply_regions<<<s.nreg * sub, 256, 0, st>>>(s.urow.p, s.ukey.p, s.rcnt.p, s.nreg, s.rsize, sub,
                                                  s.counters.p + 4, s.slots.p, s.thr.p, s.k, s.kp, s.counters.p,
                                                  s.item_count());
    RINND_LAUNCH_CHECK();
    s.nreg = 0;
    return;
  }
  k_apply_updates<<<148 * 16, 256, 0, st>>>(s.urow.p, s.ukey.p, s.counters.p + 4, s.ucap, s.slots.p, s.thr.p,
                                            s.k, s.kp, s.counters.p, spread, s.item_count());
  RINND_LAUNCH_CHECK();
}
UpdateBuf update_buf(KnnState& s) { return UpdateBuf{s.urow.p, s.ukey.p, s.counters.p + 4, s.ucap, s.item_count()}; }
}  // namespace

void leaf_init(KnnState& s, const Forest& f, const float* X, int D, int Dp, int kind,
               cudaStream_t st) {
  if (f.n_leaves == 0) return;
  ensure_update_buffer(s, st);
  const int BS = f.max_leaf <= 32 ? 32 : 64;
  TempStorage tmp;
  DVec<int32_t> cnt((size_t)f.n_leaves + 1, st), off((size_t)f.n_leaves + 1, st);
  RINND_CUDA(cudaMemsetAsync(cnt.p + f.n_leaves, 0, sizeof(int32_t), st));
  k_leaf_job_count<<<grid_for(f.n_leaves, 256, 148 * 32), 256, 0, st>>>(f.leaves.p, f.n_leaves, BS, cnt.p);
  RINND_LAUNCH_CHECK();
  exclusive_scan(cnt.p, off.p, f.n_leaves + 1, tmp, st);
  int32_t njobs = 0;
  RINND_CUDA(cudaMemcpyAsync(&njobs, off.p + f.n_leaves, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  if (njobs == 0) return;
  s.seeded = true;
  DVec<int4> jobs((size_t)njobs, st);
  k_leaf_job_emit<<<grid_for(f.n_leaves, 256, 148 * 32), 256, 0, st>>>(f.leaves.p, f.n_leaves, BS, off.p, jobs.p);
  RINND_LAUNCH_CHECK();
  const float* norms = s.norms.p;
  const bool generic = kind_is_generic(kind);
  auto launch = [&](long long j0, long long j1, int pass) {
    const int grid = (int)std::min<long long>(j1 - j0, 148LL * 16);
    if (generic) {  // every job through the update buffer (no direct first pass)
      if (pass == 0) {
        k_leaf_join_generic<<<grid, 128, 0, st>>>(jobs.p, j0, j1, f.leaves.p, f.perm.p, f.N, BS, X, D, Dp, kind,
                                                  s.slots.p, s.thr.p, s.k, s.kp, update_buf(s), s.counters.p);
        RINND_LAUNCH_CHECK();
      }
      return;
    }
    if (BS == 32)
      k_leaf_join<32, 128><<<grid, 128, 0, st>>>(jobs.p, j0, j1, f.leaves.p, f.perm.p, f.N, X, Dp, kind, norms,
                                                 s.slots.p, s.thr.p, s.k, s.kp, update_buf(s), s.counters.p, pass);
    else
      k_leaf_join<64, 256><<<grid, 256, 0, st>>>(jobs.p, j0, j1, f.leaves.p, f.perm.p, f.N, X, Dp, kind, norms,
                                                 s.slots.p, s.thr.p, s.k, s.kp, update_buf(s), s.counters.p, pass);
    RINND_LAUNCH_CHECK();
  };
  // the first tree's small leaves write their (still empty) rows directly
  launch(0, njobs, 1);
  // Worst case 2 * BS^2 updates per job: batches never overflow the buffer.
  const long long per_batch = std::max<long long>(1, (long long)(s.ucap / (2ull * BS * BS)));
  for (long long j0 = 0; j0 < njobs; j0 += per_batch) {
    long long j1 = std::min<long long>(njobs, j0 + per_batch);
    RINND_CUDA(cudaMemsetAsync(s.counters.p + 4, 0, sizeof(unsigned long long), st));
    launch(j0, j1, 0);
    apply_pending(s, st, true);
  }
}

void candidates_reserve(KnnState& s, cudaStream_t st) {
  if (s.cthr.n < 2 * (size_t)s.N) s.cthr.alloc(2 * (size_t)s.N, st);
}

void build_candidates(KnnState& s, uint64_t seed, int iter, cudaStream_t st) {
  candidates_reserve(s, st);
  uint32_t* thr_new = s.cthr.p;
  uint32_t* thr_old = s.cthr.p + s.N;
  const uint64_t salt = cand_salt(seed, iter);
  const int grid = (s.N + 3) / 4;
  if (s.k <= 32)
    k_cand_forward<32><<<grid, 128, 0, st>>>(s.slots.p, s.N, s.k, s.kp, s.c, s.cp, s.cand_new.p, s.cand_old.p,
                                             thr_new, thr_old, salt, s.group_rows());
  else if (s.k <= 64)
    k_cand_forward<64><<<grid, 128, 0, st>>>(s.slots.p, s.N, s.k, s.kp, s.c, s.cp, s.cand_new.p, s.cand_old.p,
                                             thr_new, thr_old, salt, s.group_rows());
  else
    k_cand_forward<128><<<grid, 128, 0, st>>>(s.slots.p, s.N, s.k, s.kp, s.c, s.cp, s.cand_new.p, s.cand_old.p,
                                              thr_new, thr_old, salt, s.group_rows());
  RINND_LAUNCH_CHECK();
  k_cand_reverse<<<grid_for((long long)s.N * 32, 256, 148 * 64), 256, 0, st>>>(
      s.slots.p, s.N, s.k, s.kp, s.c, s.cp, s.cand_new.p, s.cand_old.p, thr_new, thr_old, salt, &s.counters.p[1],
      s.group_rows());
  RINND_LAUNCH_CHECK();
  k_mark_old<<<grid_for((long long)s.N * 32, 256), 256, 0, st>>>(s.slots.p, s.N, s.k, s.kp, s.cand_new.p,
                                                                 s.c, s.cp);
  RINND_LAUNCH_CHECK();
}

JoinPlan join_plan(KnnState& s, const float* X, int D, int Dp, int kind, cudaStream_t st) {
  ensure_update_buffer(s, st);
  JoinPlan p;
  p.generic = kind_is_generic(kind);
  p.use_tc = !p.generic && s.precision == 1 && join_tc_supported(kind, s.c, Dp);
  p.use_tma = !p.generic && (p.use_tc || (s.use_tma && join_tma_supported(s.c, Dp)));
  if (s.err.n == 0) {
    s.err.alloc(1, st);
    s.err.fill_bytes(0);
  }
  // one region of the update buffer per join CTA: enough counts for any grid
  if (s.rcnt.n < (size_t)JOIN_MAX_GRID) s.rcnt.alloc((size_t)JOIN_MAX_GRID, st);
  // The chunked kernel batches for its worst case, 4 c^2 updates per vertex (2 directions x
  // c new x 2c candidates).  The pipelined kernel batches for the expected count: the
  // previous iteration's appended updates per vertex (an estimate before the first), with
  // the buffer filled to 80%; rows tightened by one batch's pushes filter the next.
  p.per_batch =
      std::max<long long>(1, (long long)(s.ucap / (4ull * (unsigned long long)s.c * (unsigned long long)s.c)));
  if (p.use_tma) {
    // First join: rows seeded from the tree leaves already filter most pairs
    // (~0.09 c^2 updates per vertex measured on 1M-point mixtures, k = 30);
    // unseeded rows (no trees) pass nearly every pair.
    const double first = (s.seeded ? 0.25 : 1.2) * (double)s.c * (double)s.c;
    const double upv = s.upv_prev >= 0 ? 1.1 * s.upv_prev : first;
    const double nbatch = std::max(1.0, std::ceil(upv * (double)s.N / (0.8 * (double)s.ucap)));
    p.per_batch = std::max<long long>(1, (long long)std::ceil((double)s.N / nbatch));
    join_describe_reserve(s);
  }
  if (p.use_tc) {
    join_tc_prepare(s, X, D, Dp, st);
    join_tc_reserve(kind);
  } else if (p.use_tma) {
    join_tma_reserve(s, Dp);
  }
  return p;
}

void join_enqueue(KnnState& s, const JoinPlan& p, const float* X, int D, int Dp, int kind, cudaStream_t st,
                  std::vector<cudaEvent_t>* kev) {
  RINND_CUDA(cudaMemsetAsync(s.counters.p, 0, sizeof(unsigned long long), st));
  RINND_CUDA(cudaMemsetAsync(s.counters.p + 2, 0, 2 * sizeof(unsigned long long), st));
  RINND_CUDA(cudaMemsetAsync(s.counters.p + 5, 0, 2 * sizeof(unsigned long long), st));
  if (p.use_tma) join_describe(s, kind, st);
  for (long long v0 = 0; v0 < s.N; v0 += p.per_batch) {
    int v1 = (int)std::min<long long>(s.N, v0 + p.per_batch);
    RINND_CUDA(cudaMemsetAsync(s.counters.p + 4, 0, sizeof(unsigned long long), st));
    int grid = (int)std::min<long long>(v1 - v0, 148LL * 16);
    if (kev) {
      for (int e = 0; e < 2; ++e) {
        kev->emplace_back();
        RINND_CUDA(cudaEventCreate(&kev->back()));
      }
      RINND_CUDA(cudaEventRecord((*kev)[kev->size() - 2], st));
    }
    if (p.use_tc) {
      join_tc_batch(s, X, D, Dp, kind, (int)v0, v1, s.err.p, st);
    } else if (p.use_tma) {
      join_tma_batch(s, X, Dp, kind, (int)v0, v1, s.err.p, st);
    } else if (p.generic) {
      if (s.c <= 32)
        k_local_join_generic<32><<<grid, 128, 0, st>>>(s.cand_new.p, s.cand_old.p, (int)v0, v1, s.c, s.cp, X, D, Dp,
                                                        kind, s.slots.p, s.thr.p, s.k, s.kp, update_buf(s),
                                                        s.counters.p);
      else
        k_local_join_generic<64><<<grid, 128, 0, st>>>(s.cand_new.p, s.cand_old.p, (int)v0, v1, s.c, s.cp, X, D, Dp,
                                                        kind, s.slots.p, s.thr.p, s.k, s.kp, update_buf(s),
                                                        s.counters.p);
      RINND_LAUNCH_CHECK();
    } else if (s.c <= 32) {
      k_local_join<32, 128><<<grid, 128, 0, st>>>(s.cand_new.p, s.cand_old.p, (int)v0, v1, s.c, s.cp, X, Dp, kind,
                                                  s.norms.p, s.slots.p, s.thr.p, s.k, s.kp, update_buf(s),
                                                  s.counters.p);
      RINND_LAUNCH_CHECK();
    } else {
      k_local_join<64, 256><<<grid, 256, 0, st>>>(s.cand_new.p, s.cand_old.p, (int)v0, v1, s.c, s.cp, X, Dp, kind,
                                                  s.norms.p, s.slots.p, s.thr.p, s.k, s.kp, update_buf(s),
                                                  s.counters.p);
      RINND_LAUNCH_CHECK();
    }
    if (kev) RINND_CUDA(cudaEventRecord(kev->back(), st));
    apply_pending(s, st);
  }
}

JoinStats join_collect(KnnState& s, const JoinPlan& p, const unsigned long long* h, int herr) {
  if (herr) throw CudaError("local join: a shared-memory pipeline stage did not complete within its wait limit");
  JoinStats js;
  js.form = p.use_tc ? RINND_JOIN_TENSOR_BF16 : p.use_tma ? RINND_JOIN_PIPELINED_FP32 : RINND_JOIN_CHUNKED_FP32;
  js.changes = h[0];
  js.pairs = h[2];
  js.rows = h[3];
  js.updates = h[5];
  js.appended = h[6];
  s.upv_prev = (double)h[6] / (double)s.N;
  return js;
}

JoinStats local_join(KnnState& s, const float* X, int D, int Dp, int kind, cudaStream_t st) {
  const JoinPlan p = join_plan(s, X, D, Dp, kind, st);
  cudaEvent_t e0, e1;
  RINND_CUDA(cudaEventCreate(&e0));
  RINND_CUDA(cudaEventCreate(&e1));
  std::vector<cudaEvent_t> kev;  // start/stop of every join kernel launch
  RINND_CUDA(cudaEventRecord(e0, st));
  join_enqueue(s, p, X, D, Dp, kind, st, &kev);
  RINND_CUDA(cudaEventRecord(e1, st));
  unsigned long long h[7];
  int herr = 0;
  RINND_CUDA(cudaMemcpyAsync(h, s.counters.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaMemcpyAsync(&herr, s.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  JoinStats js = join_collect(s, p, h, herr);
  RINND_CUDA(cudaEventElapsedTime(&js.total_ms, e0, e1));
  for (size_t e = 0; e < kev.size(); e += 2) {
    float ms = 0.f;
    RINND_CUDA(cudaEventElapsedTime(&ms, kev[e], kev[e + 1]));
    js.kernel_ms += ms;
  }
  js.launches = (int)(kev.size() / 2);
  for (cudaEvent_t ev : kev) cudaEventDestroy(ev);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return js;
}

JoinTile choose_join_tile(KnnState& s, const float* X, int D, int Dp, int kind, uint64_t seed, int mode,
                          cudaStream_t st, bool* tuned) {
  if (tuned) *tuned = false;
  if (mode == RINND_TUNE_FIXED) {
    s.tile = JoinTile();
    return s.tile;
  }
  const JoinPlan p = join_plan(s, X, D, Dp, kind, st);
  if (!p.use_tma || p.use_tc) return s.tile;
  if (mode != RINND_TUNE_RETUNE && join_tile_lookup(s, Dp, kind)) return s.tile;
  // the first iteration's candidate lists, sampled; the heaps (with their
  // flags) are put back so the iteration itself starts from the same state
  const size_t nslots = (size_t)s.N * s.kp;
  DVec<uint64_t> slots0(nslots, st);
  DVec<uint32_t> thr0((size_t)s.N, st);
  RINND_CUDA(cudaMemcpyAsync(slots0.p, s.slots.p, sizeof(uint64_t) * nslots, cudaMemcpyDeviceToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(thr0.p, s.thr.p, sizeof(uint32_t) * s.N, cudaMemcpyDeviceToDevice, st));
  build_candidates(s, seed, 0, st);
  join_tune(s, X, Dp, kind, std::min<long long>(p.per_batch, 131072), st);
  RINND_CUDA(cudaMemcpyAsync(s.slots.p, slots0.p, sizeof(uint64_t) * nslots, cudaMemcpyDeviceToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(s.thr.p, thr0.p, sizeof(uint32_t) * s.N, cudaMemcpyDeviceToDevice, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  if (tuned) *tuned = true;
  return s.tile;
}

IterationGraph::~IterationGraph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (host) cudaFreeHost(host);
}

JoinStats iteration_graph(KnnState& s, IterationGraph& g, uint64_t seed, int iter, const float* X, int D, int Dp,
                          int kind, cudaStream_t st, unsigned long long* item_changes_host, int n_items) {
  // host-side preparation (allocations, BF16 copy, kernel attributes) happens
  // outside the capture; the graph holds only stream work
  const JoinPlan p = join_plan(s, X, D, Dp, kind, st);
  candidates_reserve(s, st);
  const size_t host_words = 8 + (size_t)std::max(n_items, 0);
  if (g.host_words < host_words) {
    if (g.host) cudaFreeHost(g.host);
    g.host = nullptr;
    RINND_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&g.host), host_words * sizeof(unsigned long long),
                             cudaHostAllocDefault));
    g.host_words = host_words;
  }
  cudaGraph_t graph = nullptr;
  RINND_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    if (n_items > 0 && s.item_changes.p)
      RINND_CUDA(cudaMemsetAsync(s.item_changes.p, 0, sizeof(unsigned long long) * n_items, st));
    build_candidates(s, seed, iter, st);
    join_enqueue(s, p, X, D, Dp, kind, st, nullptr);
    RINND_CUDA(cudaMemcpyAsync(g.host, s.counters.p, 7 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    RINND_CUDA(cudaMemcpyAsync(g.host + 7, s.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (n_items > 0 && s.item_changes.p)
      RINND_CUDA(cudaMemcpyAsync(g.host + 8, s.item_changes.p, sizeof(unsigned long long) * n_items,
                                 cudaMemcpyDeviceToHost, st));
  } catch (...) {
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  RINND_CUDA(cudaStreamEndCapture(st, &graph));
  bool updated = false;
  if (g.exec) {
    cudaGraphExecUpdateResultInfo info;
    updated = cudaGraphExecUpdate(g.exec, graph, &info) == cudaSuccess;
    if (!updated) {
      cudaGetLastError();
      cudaGraphExecDestroy(g.exec);
      g.exec = nullptr;
    }
  }
  if (!g.exec) {
    const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(graph);
      RINND_CUDA(e);
    }
  }
  g.updates += updated ? 1 : 0;
  g.launches += 1;
  cudaEvent_t e0, e1;
  RINND_CUDA(cudaEventCreate(&e0));
  RINND_CUDA(cudaEventCreate(&e1));
  RINND_CUDA(cudaEventRecord(e0, st));
  const cudaError_t le = cudaGraphLaunch(g.exec, st);
  RINND_CUDA(cudaEventRecord(e1, st));
  cudaGraphDestroy(graph);
  RINND_CUDA(le);
  RINND_CUDA(cudaStreamSynchronize(st));
  unsigned long long h[7];
  for (int i = 0; i < 7; ++i) h[i] = g.host[i];
  int herr = 0;
  std::memcpy(&herr, g.host + 7, sizeof(int));
  if (item_changes_host)
    for (int i = 0; i < n_items; ++i) item_changes_host[i] = g.host[8 + i];
  JoinStats js = join_collect(s, p, h, herr);
  RINND_CUDA(cudaEventElapsedTime(&js.total_ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return js;
}

void finalize_knn(const KnnState& s, int32_t* out_idx, float* out_dist, cudaStream_t st) {
  finalize_rows(s.slots.p, s.N, s.k, s.kp, out_idx, out_dist, nullptr, st);
}

void finalize_rows(const uint64_t* slots, int N, int k, int kp, int32_t* out_idx, float* out_dist,
                   uint8_t* out_flags, cudaStream_t st) {
  int grid = (N + 3) / 4;
  if (k <= 32) k_finalize<32><<<grid, 128, 0, st>>>(slots, N, k, kp, out_idx, out_dist, out_flags);
  else if (k <= 64) k_finalize<64><<<grid, 128, 0, st>>>(slots, N, k, kp, out_idx, out_dist, out_flags);
  else if (k <= 128) k_finalize<128><<<grid, 128, 0, st>>>(slots, N, k, kp, out_idx, out_dist, out_flags);
  else if (k <= 512) k_finalize<512><<<grid, 128, 0, st>>>(slots, N, k, kp, out_idx, out_dist, out_flags);
  else throw std::invalid_argument("n_neighbors must be <= 512");
  RINND_LAUNCH_CHECK();
}

// Applies (row, id, dist, flag) pushes concurrently to rows initialised empty.
__global__ void k_push_batch(uint64_t* slots, uint32_t* thr, int k, int kp, long long n_ops,
                             const int32_t* rows, const int32_t* ids, const float* dists,
                             const uint8_t* flags, unsigned long long* counters) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_ops;
       i += (long long)gridDim.x * blockDim.x) {
    int32_t r = rows[i];
    uint64_t key = slot_pack(dists[i], ids[i], flags[i]);
    if (row_push(slots + (size_t)r * kp, k, thr + r, key, &counters[1])) atomicAdd(&counters[0], 1ull);
  }
}

unsigned long long heap_push_batch(KnnState& s, long long n_ops, const int32_t* rows,
                                   const int32_t* ids, const float* dists, const uint8_t* flags,
                                   cudaStream_t st) {
  s.counters.fill_bytes(0);
  k_push_batch<<<grid_for(n_ops, 256, 148 * 32), 256, 0, st>>>(s.slots.p, s.thr.p, s.k, s.kp, n_ops, rows, ids,
                                                              dists, flags, s.counters.p);
  RINND_LAUNCH_CHECK();
  unsigned long long h[4];
  RINND_CUDA(cudaMemcpyAsync(h, s.counters.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  return h[0];
}

}  // namespace rinnd
