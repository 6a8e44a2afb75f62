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

#include "dist.cuh"
#include "engine.h"
#include "heap.cuh"

namespace rinnd {
namespace {

enum JoinMode : int { MODE_JOIN = 0, MODE_TRI = 1, MODE_RECT = 2 };

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
// Tile join: A ids (na <= MA) x B ids (nb <= MB), dimensions chunked by DC.
// ---------------------------------------------------------------------------
template <int MA, int MB, int DC>
struct __align__(16) JoinSmem {
  int32_t aid[MA];
  int32_t bid[MB];
  uint32_t athr[MA];
  uint32_t bthr[MB];
  float an[MA];
  float bn[MB];
  float a[DC * MA];  // dimension-major, used only when A is not a prefix of B
  float b[DC * MB];
  unsigned int pushes;
  unsigned int pairs;
};

template <int DC>
__device__ __forceinline__ void gather_chunk(const float* __restrict__ X, int Dp, int c0,
                                             const int32_t* ids, int n, int M, float* dst) {
  constexpr int Q = DC / 4;
  for (int e = threadIdx.x; e < M * Q; e += blockDim.x) {
    int r = e % M, q = e / M;
    int d = c0 + 4 * q;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (r < n && d < Dp) v = __ldg(reinterpret_cast<const float4*>(X + (size_t)ids[r] * Dp + d));
    dst[(4 * q + 0) * M + r] = v.x;
    dst[(4 * q + 1) * M + r] = v.y;
    dst[(4 * q + 2) * M + r] = v.z;
    dst[(4 * q + 3) * M + r] = v.w;
  }
}

// Loads ids' thresholds / norms into shared memory (threads < n).
template <int MA, int MB, int DC>
__device__ __forceinline__ void load_meta(JoinSmem<MA, MB, DC>& sm, int na, int nb, bool a_prefix,
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

template <int MA, int MB, int DC>
__device__ __forceinline__ void join_tile(JoinSmem<MA, MB, DC>& sm, int na, int nb, int mode,
                                          const float* __restrict__ X, int Dp, int kind,
                                          uint64_t* slots, uint32_t* thr, int k,
                                          unsigned long long* contention) {
  constexpr int TX = MB / 4;  // threads along B
  const int tx = threadIdx.x % TX, ty = threadIdx.x / TX;
  const int i0 = ty * 4, j0 = tx * 4;
  const bool a_prefix = (mode != MODE_RECT);
  const float* sa = a_prefix ? sm.b : sm.a;
  const int astride = a_prefix ? MB : MA;
  bool active = i0 < na && j0 < nb;
  if (active && mode != MODE_RECT) {
    // skip 4x4 blocks that lie entirely on/below the diagonal of the A x A part
    bool any_tri = (j0 + 3 > i0) && (j0 < na);
    bool any_rect = (mode == MODE_JOIN) && (j0 + 3 >= na);
    active = any_tri || any_rect;
  }
  const bool is_dot = kind_is_dot(kind);
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;

  for (int c0 = 0; c0 < Dp; c0 += DC) {
    __syncthreads();
    gather_chunk<DC>(X, Dp, c0, sm.bid, nb, MB, sm.b);
    if (!a_prefix) gather_chunk<DC>(X, Dp, c0, sm.aid, na, MA, sm.a);
    __syncthreads();
    if (active) {
      if (kind == DK_SQEUCLIDEAN) {
#pragma unroll 8
        for (int d = 0; d < DC; ++d) {
          float4 av = *reinterpret_cast<const float4*>(sa + d * astride + i0);
          float4 bv = *reinterpret_cast<const float4*>(sm.b + d * MB + j0);
          float a4[4] = {av.x, av.y, av.z, av.w};
          float b4[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              float t = a4[i] - b4[j];
              acc[i][j] = fmaf(t, t, acc[i][j]);
            }
        }
      } else if (kind == DK_MANHATTAN) {
#pragma unroll 8
        for (int d = 0; d < DC; ++d) {
          float4 av = *reinterpret_cast<const float4*>(sa + d * astride + i0);
          float4 bv = *reinterpret_cast<const float4*>(sm.b + d * MB + j0);
          float a4[4] = {av.x, av.y, av.z, av.w};
          float b4[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] += fabsf(a4[i] - b4[j]);
        }
      } else {
#pragma unroll 8
        for (int d = 0; d < DC; ++d) {
          float4 av = *reinterpret_cast<const float4*>(sa + d * astride + i0);
          float4 bv = *reinterpret_cast<const float4*>(sm.b + d * MB + j0);
          float a4[4] = {av.x, av.y, av.z, av.w};
          float b4[4] = {bv.x, bv.y, bv.z, bv.w};
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a4[i], b4[j], acc[i][j]);
        }
      }
    }
  }
  unsigned int my_pairs = 0, my_push = 0;
  if (active) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int ia = i0 + i;
      if (ia >= na) break;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int jb = j0 + j;
        if (jb >= nb) break;
        int32_t p = a_prefix ? sm.bid[ia] : sm.aid[ia], q = sm.bid[jb];
        bool valid;
        if (mode == MODE_RECT) valid = true;
        else if (jb < na) valid = jb > ia;            // new x new, q after p (mod.rs:396)
        else valid = (mode == MODE_JOIN) && (q != p);  // new x old, q != p (mod.rs:424)
        if (!valid) continue;
        ++my_pairs;
        float d = acc[i][j];
        if (is_dot) d = finalize_dot(kind, d, a_prefix ? sm.bn[ia] : sm.an[ia], sm.bn[jb]);
        uint32_t kd = fkey(d);
        uint32_t tp = a_prefix ? sm.bthr[ia] : sm.athr[ia];
        if (kd < tp)
          my_push += row_push(slots + (size_t)p * k, k, thr + p,
                              ((uint64_t)kd << 32) | (uint32_t)q | 0x80000000u, contention);
        if (kd < sm.bthr[jb])
          my_push += row_push(slots + (size_t)q * k, k, thr + q,
                              ((uint64_t)kd << 32) | (uint32_t)p | 0x80000000u, contention);
      }
    }
  }
  if (my_pairs) atomicAdd(&sm.pairs, my_pairs);
  if (my_push) atomicAdd(&sm.pushes, my_push);
}

// One CTA per vertex (grid-stride): A = new candidates, B = new ++ old.
template <int MA, int MB, int DC>
__global__ void __launch_bounds__((MA / 4) * (MB / 4))
    k_local_join(const uint64_t* cand_new, const uint64_t* cand_old, int N, int c,
                 const float* __restrict__ X, int Dp, int kind, const float* norms,
                 uint64_t* slots, uint32_t* thr, int k, unsigned long long* counters) {
  __shared__ JoinSmem<MA, MB, DC> sm;
  __shared__ int s_cnt[2];
  for (int v = blockIdx.x; v < N; v += gridDim.x) {
    __syncthreads();
    if (threadIdx.x == 0) {
      s_cnt[0] = 0;
      s_cnt[1] = 0;
      sm.pushes = 0;
      sm.pairs = 0;
    }
    __syncthreads();
    // compact valid ids, keeping list order: new first, then old
    if (threadIdx.x < 32) {
      int lane = threadIdx.x;
      int base = 0;
      for (int t0 = 0; t0 < c; t0 += 32) {
        int t = t0 + lane;
        int32_t id = t < c ? slot_id(cand_new[(size_t)v * c + t]) : -1;
        unsigned m = __ballot_sync(0xffffffffu, id >= 0);
        if (id >= 0) sm.bid[base + __popc(m & ((1u << lane) - 1))] = id;
        base += __popc(m);
      }
      int na = base;
      for (int t0 = 0; t0 < c; t0 += 32) {
        int t = t0 + lane;
        int32_t id = t < c ? slot_id(cand_old[(size_t)v * c + t]) : -1;
        unsigned m = __ballot_sync(0xffffffffu, id >= 0);
        if (id >= 0) sm.bid[base + __popc(m & ((1u << lane) - 1))] = id;
        base += __popc(m);
      }
      if (lane == 0) {
        s_cnt[0] = na;
        s_cnt[1] = base;
      }
    }
    __syncthreads();
    int na = s_cnt[0], nb = s_cnt[1];
    if (na == 0) continue;  // no new candidates: nothing to join (uniform across CTA)
    load_meta<MA, MB, DC>(sm, na, nb, true, thr, kind_is_dot(kind) ? norms : nullptr);
    join_tile<MA, MB, DC>(sm, na, nb, MODE_JOIN, X, Dp, kind, slots, thr, k, &counters[1]);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (sm.pushes) atomicAdd(&counters[0], (unsigned long long)sm.pushes);
      if (sm.pairs) atomicAdd(&counters[2], (unsigned long long)sm.pairs);
    }
  }
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
template <int BS, int DC>
__global__ void __launch_bounds__((BS / 4) * (BS / 4))
    k_leaf_join(const int4* jobs, long long njobs, const int4* leaves, const int32_t* perm, int N,
                const float* __restrict__ X, int Dp, int kind, const float* norms,
                uint64_t* slots, uint32_t* thr, int k, unsigned long long* counters) {
  __shared__ JoinSmem<BS, BS, DC> sm;
  for (long long jb = blockIdx.x; jb < njobs; jb += gridDim.x) {
    int4 job = jobs[jb];
    int4 leaf = leaves[job.x];
    const int32_t* P = perm + (size_t)leaf.x * N + leaf.y;
    int L = leaf.z - leaf.y;
    int a0 = job.y * BS, b0 = job.z * BS;
    int na = min(BS, L - a0), nb = min(BS, L - b0);
    int mode = job.y == job.z ? MODE_TRI : MODE_RECT;
    __syncthreads();
    if (threadIdx.x == 0) {
      sm.pushes = 0;
      sm.pairs = 0;
    }
    for (int t = threadIdx.x; t < nb; t += blockDim.x) sm.bid[t] = P[b0 + t];
    for (int t = threadIdx.x; t < na; t += blockDim.x) sm.aid[t] = P[a0 + t];
    __syncthreads();
    load_meta<BS, BS, DC>(sm, na, nb, mode != MODE_RECT, thr, kind_is_dot(kind) ? norms : nullptr);
    join_tile<BS, BS, DC>(sm, na, nb, mode, X, Dp, kind, slots, thr, k, &counters[1]);
    __syncthreads();
    if (threadIdx.x == 0) {
      if (sm.pushes) atomicAdd(&counters[0], (unsigned long long)sm.pushes);
      if (sm.pairs) atomicAdd(&counters[2], (unsigned long long)sm.pairs);
    }
  }
}

// candidates.rs:153-351: each heap edge offered forward and reverse with one priority.
__global__ void k_candidates(const uint64_t* slots, int N, int k, int c, uint64_t* cnew,
                             uint64_t* cold, uint64_t seed, int iter,
                             unsigned long long* contention) {
  long long total = (long long)N * k;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    uint64_t s = slots[e];
    int32_t id = slot_id(s);
    if (id < 0) continue;
    int32_t i = (int32_t)(e / k);
    uint64_t* lists = slot_new(s) ? cnew : cold;
    uint32_t prio = (uint32_t)(hash3(seed, 0xC0DE0000ull + (uint64_t)iter, (uint64_t)e) >> 33);
    uint64_t hi = (uint64_t)prio << 32;
    row_push(lists + (size_t)i * c, c, nullptr, hi | (uint32_t)id, contention);
    row_push(lists + (size_t)id * c, c, nullptr, hi | (uint32_t)i, contention);
  }
}

// candidates.rs:354-417 mark_old_flags, one warp per row.
__global__ void k_mark_old(uint64_t* slots, int N, int k, const uint64_t* cnew, int c) {
  int row = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  int lane = threadIdx.x & 31;
  if (row >= N) return;
  const uint64_t* nl = cnew + (size_t)row * c;
  for (int j0 = 0; j0 < k; j0 += 32) {
    int j = j0 + lane;
    uint64_t s = j < k ? slots[(size_t)row * k + j] : SLOT_EMPTY;
    int32_t id = slot_id(s);
    bool hit = false;
    if (id >= 0 && slot_new(s))
      for (int t = 0; t < c; ++t)
        if (slot_id(nl[t]) == id) { hit = true; break; }
    if (hit) slots[(size_t)row * k + j] = s & ~(1ull << 31);
  }
}

// neighbor_heap.rs:293-320 sort_all: rows ascending by distance (ties by id),
// one warp per row, bitonic sort of P = next_pow2(k) keys in shared memory.
// Sort key = (fkey(d) << 32) | (id << 1) | flag; empty = ~0.
template <int P>
__global__ void k_finalize(const uint64_t* slots, int N, int k, int32_t* out_idx, float* out_dist,
                           uint8_t* out_flags) {
  __shared__ uint64_t buf[4][P];
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int row = blockIdx.x * 4 + w;
  if (row >= N) return;
  uint64_t* b = buf[w];
  for (int j = lane; j < P; j += 32) {
    uint64_t key = ~0ull;
    if (j < k) {
      uint64_t s = slots[(size_t)row * k + j];
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
  s.slots.alloc((size_t)N * k, st);
  s.thr.alloc((size_t)N, st);
  s.cand_new.alloc((size_t)N * c, st);
  s.cand_old.alloc((size_t)N * c, st);
  s.counters.alloc(4, st);
  s.counters.fill_bytes(0);
  k_fill_u64<<<grid_for((long long)N * k, 256, 148 * 32), 256, 0, st>>>(s.slots.p, s.slots.n, SLOT_EMPTY);
  k_fill_u32<<<grid_for(N, 256, 148 * 32), 256, 0, st>>>(s.thr.p, s.thr.n, KEY_INF);
  RINND_LAUNCH_CHECK();
}

void compute_norms(const float* X, int N, int D, int Dp, float* norms, cudaStream_t st) {
  k_norms<<<grid_for((long long)N * 32, 256), 256, 0, st>>>(X, N, D, Dp, norms);
  RINND_LAUNCH_CHECK();
}

void leaf_init(KnnState& s, const Forest& f, const float* X, int D, int Dp, int kind,
               cudaStream_t st) {
  (void)D;
  if (f.n_leaves == 0) return;
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
  DVec<int4> jobs((size_t)njobs, st);
  k_leaf_job_emit<<<grid_for(f.n_leaves, 256, 148 * 32), 256, 0, st>>>(f.leaves.p, f.n_leaves, BS, off.p, jobs.p);
  RINND_LAUNCH_CHECK();
  const float* norms = s.norms.p;
  int grid = (int)std::min<long long>(njobs, 148LL * 16);
  if (BS == 32)
    k_leaf_join<32, 32><<<grid, 64, 0, st>>>(jobs.p, njobs, f.leaves.p, f.perm.p, f.N, X, Dp, kind,
                                             norms, s.slots.p, s.thr.p, s.k, s.counters.p);
  else
    k_leaf_join<64, 32><<<grid, 256, 0, st>>>(jobs.p, njobs, f.leaves.p, f.perm.p, f.N, X, Dp, kind,
                                              norms, s.slots.p, s.thr.p, s.k, s.counters.p);
  RINND_LAUNCH_CHECK();
}

void build_candidates(KnnState& s, uint64_t seed, int iter, cudaStream_t st) {
  s.cand_new.fill_bytes(0xFF);
  s.cand_old.fill_bytes(0xFF);
  long long total = (long long)s.N * s.k;
  k_candidates<<<grid_for(total, 256, 148 * 64), 256, 0, st>>>(s.slots.p, s.N, s.k, s.c, s.cand_new.p,
                                                              s.cand_old.p, seed, iter, &s.counters.p[1]);
  RINND_LAUNCH_CHECK();
  k_mark_old<<<grid_for((long long)s.N * 32, 256), 256, 0, st>>>(s.slots.p, s.N, s.k, s.cand_new.p, s.c);
  RINND_LAUNCH_CHECK();
}

unsigned long long local_join(KnnState& s, const float* X, int D, int Dp, int kind,
                              cudaStream_t st, unsigned long long* pairs_out) {
  (void)D;
  RINND_CUDA(cudaMemsetAsync(s.counters.p, 0, sizeof(unsigned long long), st));
  RINND_CUDA(cudaMemsetAsync(s.counters.p + 2, 0, sizeof(unsigned long long), st));
  int grid = std::min(s.N, 148 * 16);
  if (s.c <= 32)
    k_local_join<32, 64, 32><<<grid, 128, 0, st>>>(s.cand_new.p, s.cand_old.p, s.N, s.c, X, Dp, kind,
                                                   s.norms.p, s.slots.p, s.thr.p, s.k, s.counters.p);
  else
    k_local_join<64, 128, 32><<<grid, 512, 0, st>>>(s.cand_new.p, s.cand_old.p, s.N, s.c, X, Dp, kind,
                                                    s.norms.p, s.slots.p, s.thr.p, s.k, s.counters.p);
  RINND_LAUNCH_CHECK();
  unsigned long long h[4];
  RINND_CUDA(cudaMemcpyAsync(h, s.counters.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  if (pairs_out) *pairs_out = h[2];
  return h[0];
}

void finalize_knn(const KnnState& s, int32_t* out_idx, float* out_dist, cudaStream_t st) {
  finalize_rows(s.slots.p, s.N, s.k, out_idx, out_dist, nullptr, st);
}

void finalize_rows(const uint64_t* slots, int N, int k, int32_t* out_idx, float* out_dist,
                   uint8_t* out_flags, cudaStream_t st) {
  int grid = (N + 3) / 4;
  if (k <= 32) k_finalize<32><<<grid, 128, 0, st>>>(slots, N, k, out_idx, out_dist, out_flags);
  else if (k <= 64) k_finalize<64><<<grid, 128, 0, st>>>(slots, N, k, out_idx, out_dist, out_flags);
  else if (k <= 128) k_finalize<128><<<grid, 128, 0, st>>>(slots, N, k, out_idx, out_dist, out_flags);
  else if (k <= 512) k_finalize<512><<<grid, 128, 0, st>>>(slots, N, k, out_idx, out_dist, out_flags);
  else throw std::invalid_argument("n_neighbors must be <= 512");
  RINND_LAUNCH_CHECK();
}

// Applies (row, id, dist, flag) pushes concurrently to rows initialised empty.
__global__ void k_push_batch(uint64_t* slots, uint32_t* thr, int k, long long n_ops,
                             const int32_t* rows, const int32_t* ids, const float* dists,
                             const uint8_t* flags, unsigned long long* counters) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_ops;
       i += (long long)gridDim.x * blockDim.x) {
    int32_t r = rows[i];
    uint64_t key = slot_pack(dists[i], ids[i], flags[i]);
    if (row_push(slots + (size_t)r * k, k, thr + r, key, &counters[1])) atomicAdd(&counters[0], 1ull);
  }
}

unsigned long long heap_push_batch(KnnState& s, long long n_ops, const int32_t* rows,
                                   const int32_t* ids, const float* dists, const uint8_t* flags,
                                   cudaStream_t st) {
  s.counters.fill_bytes(0);
  k_push_batch<<<grid_for(n_ops, 256, 148 * 32), 256, 0, st>>>(s.slots.p, s.thr.p, s.k, n_ops, rows, ids,
                                                              dists, flags, s.counters.p);
  RINND_LAUNCH_CHECK();
  unsigned long long h[4];
  RINND_CUDA(cudaMemcpyAsync(h, s.counters.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  return h[0];
}

}  // namespace rinnd
