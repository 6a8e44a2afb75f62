// search.cu -- warp-per-query greedy graph search.
//
// Restates the reference query path (core/search/greedy.rs:70-241, 365-413;
// core/index.rs:157-202, 283-334) with one warp per query:
//   * tree seeding: each retained RP tree's search_leaves (flat_tree.rs:239-311):
//     hard descent with a leaf budget of 1, else the spill search over a
//     priority frontier; margin = dot(q, hyperplane) + offset in the reference
//     dot order (or the int8 routing tree's reconstructed margin for quantized
//     queries, flat_tree.rs:96-183), |m| < 1e-8 -> random side; every unvisited
//     leaf point is pushed to results and seeds;
//   * fill_random up to k seeds (greedy.rs:148-163);
//   * traverse (greedy.rs:165-201): pop the nearest seed; stop when the result
//     list is full and the seed is >= bound, bound = max + eps * (max - min_distance)
//     evaluated with separately rounded ops; expand CSR neighbors not yet
//     visited, push those with d < bound (results bounded to k, seeds
//     unbounded), recomputing the bound after every result insertion.
// Distances use the reference's exact accumulation order (dist.cuh), or the
// exact int8 dot with the reference's scaling (quantized.rs:26-40, greedy.rs:384-390)
// followed by an optional exact FP32 rerank of the leading results (index.rs:103-126).
//
// Per-warp state: the query, the result list (sorted by (distance, id)) and
// the front of the seed queue (a sorted array merged warp-parallel with each
// batch of accepted neighbors) in shared memory; the rest of the seed queue
// (an unsorted back store) and a second visited table in global memory,
// behind a first table in shared memory.  Seeds the traversal can no longer
// pop (distance >= bound with a full result list) are dropped.  The state is
// still bounded, while the reference's seed heap and visited set are not:
// dropping seeds from a full back store changes nothing unless the unbounded
// search would pop one of them (it ranks before a seed that is popped while
// still within the bound, or the seeds run out while it is); such a query, or
// one with an id neither table can place within 32 probes, is recorded and
// re-run from scratch, first with larger bounded state and, if that overflows
// too, with state sized to the index (a visited bitset of N bits and a back
// store of N seeds), so every query's result is the one of the unbounded
// search.
// Neighbor and tie order follow (distance, id); the reference's BinaryHeap
// orders exact distance ties by its internal layout.
#include <map>
#include <mutex>
#include <tuple>

#include "dist.cuh"
#include "engine.h"

namespace rinnd {
namespace {

constexpr int WPB = 4;  // warps per block
constexpr int HASH_PROBES = 32;

struct WarpLayout {
  int dp, kmax, s, h, f;  // f: spill-frontier entries (0 with a leaf budget of 1)
  __host__ __device__ size_t q_off() const { return 0; }
  __host__ __device__ size_t res_off() const { return (size_t)dp * 4; }
  __host__ __device__ size_t seed_off() const { return res_off() + (size_t)kmax * 8; }
  __host__ __device__ size_t batch_off() const { return seed_off() + (size_t)2 * s * 8; }
  // batch, keys leaving the front, keys staged for the front by a refill
  __host__ __device__ size_t vis_off() const { return batch_off() + 96 * 8; }
  __host__ __device__ size_t fr_off() const { return vis_off() + (size_t)h * 4; }
  // a warp's region is a multiple of 16 bytes (the tables are cleared with 16-byte stores)
  __host__ __device__ size_t bytes() const { return (fr_off() + (size_t)f * 8 + 15) & ~(size_t)15; }
};

__host__ __device__ __forceinline__ int seed_capacity(int width) {
  return width <= 32 ? 256 : (width <= 128 ? 512 : 1024);
}

__device__ __forceinline__ uint64_t rkey(float d, int32_t id) {
  return ((uint64_t)fkey(d) << 32) | (uint32_t)id;
}

// The query's random stream: the reference's FastRng (core/rng.rs), i.e.
// Xoshiro256++ (rand_xoshiro 0.6.0) seeded through SplitMix64 by
// seed_from_u64, with rand 0.8.5's samplers: a bool is the sign bit of a
// u32 draw (next_u32 = high word of next_u64), and gen_range(0..n) is the
// widening-multiply draw with rejection of the low word above the zone
// (range << lz) - 1.  Seeded with seed + query id (index.rs:165).  Every lane
// of the warp advances the same state, so draws are warp-uniform.
struct QRng {
  uint64_t s0, s1, s2, s3;
  __device__ explicit QRng(uint64_t seed) {
    uint64_t x = seed;
    uint64_t st[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      x += 0x9e3779b97f4a7c15ull;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
      st[i] = z ^ (z >> 31);
    }
    s0 = st[0];
    s1 = st[1];
    s2 = st[2];
    s3 = st[3];
  }
  __device__ static uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
  __device__ uint64_t next() {
    const uint64_t r = rotl(s0 + s3, 23) + s0;
    const uint64_t t = s1 << 17;
    s2 ^= s0;
    s3 ^= s1;
    s1 ^= s2;
    s0 ^= s3;
    s2 ^= t;
    s3 = rotl(s3, 45);
    return r;
  }
  __device__ bool next_bool() { return (int32_t)(uint32_t)(next() >> 32) < 0; }
  __device__ uint32_t next_index(uint32_t n) {
    const uint64_t range = n;
    const uint64_t zone = (range << __clzll((long long)range)) - 1;
    uint64_t hi = 0;
    for (int attempt = 0; attempt < 64; ++attempt) {  // a draw is rejected with probability < 1/2
      const uint64_t v = next();
      hi = __umul64hi(v, range);
      if (v * range <= zone) break;
    }
    return (uint32_t)hi;
  }
};

// Visited set (VisitedSet::check_and_mark).  Exact form: a bitset of N bits
// (bits != null).  Bounded form: an open-addressing table of h ids (shared
// memory, or global memory for widths above 32) backed by a second global table
// of h2 ids that a query clears when it first needs it.  The first table takes
// new ids until it holds 2/3 h (so that a lookup's probe run stays short);
// after that an id absent from it goes to the second.  An id that finds no
// free slot within HASH_PROBES probes of either table is counted, treated as
// visited and marks the search as lost (it is re-run with a larger state).
struct Visited {
  int32_t* tab;
  int h, n1;      // n1: ids the first table holds (warp-uniform)
  int32_t* tab2;  // second level (null: none)
  int h2;
  uint32_t* bits;
  bool lost;       // warp-uniform
  bool tab2_live;  // warp-uniform: tab2 cleared for this query
};

__device__ __forceinline__ uint32_t vis_slot(int32_t id, int h) {
  return __umulhi((uint32_t)id * 2654435761u, (uint32_t)h);
}

// insert: 0 id inserted, 1 id present, 2 no free slot within HASH_PROBES probes.
// lookup (!insert, no lane inserts meanwhile): 1 present, 2 absent.
__device__ __forceinline__ int table_mark(int32_t* tab, int h, int32_t id, bool insert) {
  uint32_t pos = vis_slot(id, h);
  for (int p = 0; p < HASH_PROBES; ++p) {
    const int32_t old = insert ? atomicCAS(&tab[pos], -1, id) : tab[pos];
    if (old == -1) return insert ? 0 : 2;
    if (old == id) return 1;
    pos = pos + 1 == (uint32_t)h ? 0u : pos + 1;
  }
  return 2;
}

// Whole warp: marks id on the lanes with `have` and returns, on those lanes,
// whether it was already visited.  An id is held by one table only: the first
// table never frees a slot, so an id it did not take (no free slot within
// HASH_PROBES probes, or the table closed) is never found there later either.
__device__ __forceinline__ bool visited_mark(Visited& v, int32_t id, bool have, unsigned long long* overflow) {
  if (v.bits) {
    if (!have) return false;
    const uint32_t m = 1u << (id & 31);
    return (atomicOr(&v.bits[id >> 5], m) & m) != 0u;
  }
  const bool open1 = v.n1 < v.h - v.h / 3;
  int r = have ? table_mark(v.tab, v.h, id, open1) : 1;
  if (open1) v.n1 += __popc(__ballot_sync(0xffffffffu, r == 0));
  if (__any_sync(0xffffffffu, r == 2)) {
    if (v.tab2) {
      if (!v.tab2_live) {
        const int lane = threadIdx.x & 31;
        int4* t4 = reinterpret_cast<int4*>(v.tab2);
        for (int t = lane; t < v.h2 / 4; t += 32) t4[t] = make_int4(-1, -1, -1, -1);
        __syncwarp();
        v.tab2_live = true;
      }
      if (r == 2) r = table_mark(v.tab2, v.h2, id, true);
    }
    if (r == 2) atomicAdd(overflow, 1ull);
    if (__any_sync(0xffffffffu, r == 2)) v.lost = true;
  }
  return have && r != 0;
}

// First-level visited-table entries for result width w: shared memory up to
// w = 32 (3072 entries keep three 4-warp blocks on an SM), beyond that a
// per-warp region of global memory (a search of width w evaluates on the order
// of 100 w nodes).
__host__ __device__ __forceinline__ int visited_capacity(int width) {
  if (width <= 32) return 3072;
  int h = 8192;
  while (h < 128 * width) h <<= 1;
  return h;
}

template <bool QUANT>
__device__ __forceinline__ float dist_to(const SearchIndex& ix, const float* q, const int8_t* q8,
                                         float qinv, int32_t id) {
  if (QUANT && ix.dim_scales) {
    // per-dimension codes: quantized_i8_per_dimension_dot (quantized.rs:48-56),
    // ((a * b) * s_j) * s_j summed sequentially over the dimensions
    const int4* b = reinterpret_cast<const int4*>(ix.codes + (size_t)id * ix.Dq);
    float acc = 0.f;
    for (int t = 0; t < ix.Dq / 16; ++t) {
      const int4 y = __ldg(b + t);
      const int8_t* yb = reinterpret_cast<const int8_t*>(&y);
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int j = 16 * t + u;
        if (j < ix.D) {
          const float s = __ldg(ix.dim_scales + j);
          acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(__fmul_rn((float)q8[j], (float)yb[u]), s), s));
        }
      }
    }
    return __fsub_rn(1.0f, fminf(fmaxf(acc, -1.0f), 1.0f));
  }
  if (QUANT) {
    const int4* a = reinterpret_cast<const int4*>(q8);
    const int4* b = reinterpret_cast<const int4*>(ix.codes + (size_t)id * ix.Dq);
    int acc = 0;  // exact: |sum| <= 127^2 D
    for (int t = 0; t < ix.Dq / 16; ++t) {
      const int4 x = a[t], y = __ldg(b + t);
      acc = __dp4a(x.x, y.x, acc);
      acc = __dp4a(x.y, y.y, acc);
      acc = __dp4a(x.z, y.z, acc);
      acc = __dp4a(x.w, y.w, acc);
    }
    float sim = __fmul_rn(__fmul_rn((float)acc, qinv), ix.inv_norms[id]);
    return __fsub_rn(1.0f, fminf(fmaxf(sim, -1.0f), 1.0f));
  }
  return exact_distance(ix.kind, q, ix.X + (size_t)id * ix.Dp, ix.D);
}

// Warp-parallel insertion into the sorted result list (BoundedHeap::push,
// candidate_heap.rs:97-113).  Returns true if inserted.  Uniform across the warp.
__device__ __forceinline__ bool result_push(uint64_t* res, int& rc, int k, float d, int32_t id) {
  const int lane = threadIdx.x & 31;
  uint64_t key = rkey(d, id);
  if (rc >= k) {
    float mx = fkey_inv((uint32_t)(res[rc - 1] >> 32));
    if (!(d < mx)) return false;
  }
  // duplicate guard (only reachable after a visited-table overflow)
  bool dup = false;
  for (int e = lane; e < rc; e += 32) dup |= ((uint32_t)res[e] == (uint32_t)id);
  if (__any_sync(0xffffffffu, dup)) return false;
  int pos = 0;
  for (int e0 = 0; e0 < rc; e0 += 32) {
    int e = e0 + lane;
    pos += __popc(__ballot_sync(0xffffffffu, e < rc && res[e] < key));
  }
  int last = rc < k ? rc : k - 1;  // entries [pos, last) shift right by one
  uint64_t tmp[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    int e = pos + lane + 32 * t;
    tmp[t] = e < last ? res[e] : 0;
  }
  __syncwarp();
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    int e = pos + lane + 32 * t;
    if (e < last) res[e + 1] = tmp[t];
  }
  __syncwarp();
  if (lane == 0) res[pos] = key;
  __syncwarp();
  if (rc < k) ++rc;
  return true;
}

__device__ __forceinline__ float result_max(const uint64_t* res, int rc) {
  return rc > 0 ? fkey_inv((uint32_t)(res[rc - 1] >> 32)) : __int_as_float(0x7f800000);
}

// Sort 32 keys held one per lane (ascending), bitonic via shuffles.
__device__ __forceinline__ uint64_t warp_sort32(uint64_t v) {
  const int lane = threadIdx.x & 31;
  for (int size = 2; size <= 32; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      uint64_t o = __shfl_xor_sync(0xffffffffu, v, stride);
      bool up = (lane & size) == 0;
      bool lower = (lane & stride) == 0;
      uint64_t mn = v < o ? v : o, mx = v < o ? o : v;
      v = (lower == up) ? mn : mx;
    }
  return v;
}

// Seed queue: the reference's unbounded min-heap of seeds (greedy.rs:165-201)
// as a sorted front in shared memory and an unsorted back store in global
// memory, with every front key < fence <= every back key.  The front's first
// key is the queue's minimum while the front is non-empty; an empty front is
// refilled with the smallest back keys.  Keys the traversal can no longer pop
// are dropped: with a full result list the traversal stops at the first seed
// whose distance is >= bound, and the bound never grows once the list is full
// (for a finite epsilon >= 0), so a key with distance >= bound is never popped
// ("prunable": key >= cut, cut = fkey(bound) << 32; keys of NaN distance are
// kept).  A full back store drops keys; min_drop keeps the smallest, which the
// traversal compares with the seeds it pops and its final bound.
struct SeedQueue {
  uint64_t* front;  // two arrays of S entries `stride` apart; live: [head, tail) of array cur
  int stride, S, cur, head, tail;
  uint64_t* back;  // B entries of this warp's global memory; live: [0, nback)
  int B, nback;
  uint64_t fence, min_drop;
  bool spilled;
};

__device__ __forceinline__ bool key_prunable(uint64_t key, uint64_t cut) {
  return key >= cut && (uint32_t)(key >> 32) <= KEY_INF;
}

__device__ __forceinline__ uint64_t warp_min64(uint64_t v) {
  for (int o = 16; o; o >>= 1) {
    const uint64_t x = __shfl_xor_sync(0xffffffffu, v, o);
    v = x < v ? x : v;
  }
  return v;
}

// Appends the keys of the lanes with `take` to the back store at w (capacity
// cap), in lane order; keys beyond cap are dropped into min_drop.
__device__ __forceinline__ void back_append(SeedQueue& s, uint64_t key, bool take, int& w, int cap) {
  const int lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(0xffffffffu, take);
  if (!m) return;
  const int pos = w + __popc(m & ((1u << lane) - 1u));
  const bool drop = take && pos >= cap;
  if (take && !drop) s.back[pos] = key;
  if (__any_sync(0xffffffffu, drop)) {
    const uint64_t d = warp_min64(drop ? key : ~0ull);
    s.min_drop = d < s.min_drop ? d : s.min_drop;
  }
  w = min(cap, w + __popc(m));
  s.spilled = true;
}

// Merges the sorted batch (one key per lane, ascending; the first nb lanes
// valid, all below the fence) into the front.  Entries merged beyond S leave
// the front: they are returned on lanes [0, E) in order (E is returned) and
// the fence becomes the smallest of them if that is lower.  Then prunable keys
// are cut off the front's end.
__device__ __forceinline__ int front_merge(SeedQueue& s, uint64_t* bbuf, uint64_t bkey, int nb, uint64_t cut,
                                           uint64_t& evicted) {
  const int lane = threadIdx.x & 31;
  uint64_t* ebuf = bbuf + 32;
  bbuf[lane] = bkey;
  __syncwarp();
  const uint64_t* A = s.front + (size_t)s.cur * s.stride;
  uint64_t* C = s.front + (size_t)(s.cur ^ 1) * s.stride;
  const int na = s.tail - s.head, S = s.S;
  for (int i = lane; i < na; i += 32) {  // out = i + #(b < a)
    const uint64_t a = A[s.head + i];
    int lo = 0, hi = nb;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (bbuf[mid] < a) lo = mid + 1; else hi = mid;
    }
    const int o = i + lo;
    if (o < S) C[o] = a; else ebuf[o - S] = a;
  }
  if (lane < nb) {  // out = j + #(a <= b)
    int lo = 0, hi = na;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (A[s.head + mid] <= bkey) lo = mid + 1; else hi = mid;
    }
    const int o = lane + lo;
    if (o < S) C[o] = bkey; else ebuf[o - S] = bkey;
  }
  __syncwarp();
  const int total = na + nb;
  const int E = total > S ? total - S : 0;  // <= nb <= 32, as na <= S
  evicted = lane < E ? ebuf[lane] : ~0ull;
  if (E > 0 && ebuf[0] < s.fence) s.fence = ebuf[0];
  __syncwarp();
  s.cur ^= 1;
  s.head = 0;
  s.tail = min(total, S);
  if (s.tail > 0 && key_prunable(C[s.tail - 1], cut)) {  // no NaN key at the end: cut the prunable run
    int lo = 0, hi = s.tail - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (C[mid] < cut) lo = mid + 1; else hi = mid;
    }
    s.tail = lo;
  }
  return E;
}

// Pushes a sorted batch (ascending, one key per lane, the first nb valid):
// keys below the fence merge into the front, the others and the front's
// overflow go to the back store, prunable ones nowhere.
__device__ __forceinline__ void seeds_push(SeedQueue& s, uint64_t* bbuf, uint64_t sorted, int nb, uint64_t cut) {
  const int lane = threadIdx.x & 31;
  if (nb == 0) return;
  const int nf = __popc(__ballot_sync(0xffffffffu, lane < nb && sorted < s.fence));
  back_append(s, sorted, lane >= nf && lane < nb && !key_prunable(sorted, cut), s.nback, s.B);
  if (nf == 0) return;
  uint64_t ev;
  const int E = front_merge(s, bbuf, sorted, nf, cut, ev);
  if (E > 0) back_append(s, ev, lane < E && !key_prunable(ev, cut), s.nback, s.B);
}

// Refills the empty front by merging the whole back store through it, 32
// keys at a time; what leaves the front is written back in place (never past
// the keys read so far), so the back store ends with the rest and the fence
// with the smallest of them.  Used when no threshold is found.
__device__ void seeds_refill_merge(SeedQueue& s, uint64_t* bbuf, uint64_t cut) {
  const int lane = threadIdx.x & 31;
  const int n = s.nback;
  s.head = s.tail = 0;
  s.fence = ~0ull;
  int w = 0;
  for (int c0 = 0; c0 < n; c0 += 32) {
    uint64_t key = c0 + lane < n ? s.back[c0 + lane] : ~0ull;
    if (key_prunable(key, cut)) key = ~0ull;
    const int nb = __popc(__ballot_sync(0xffffffffu, key != ~0ull));
    if (nb == 0) continue;
    const uint64_t sorted = warp_sort32(key);
    uint64_t ev;
    const int E = front_merge(s, bbuf, sorted, nb, cut, ev);
    if (E > 0) back_append(s, ev, lane < E && !key_prunable(ev, cut), w, n);
  }
  __syncwarp();
  s.nback = w;
  if (w == 0) s.fence = ~0ull;
}

constexpr int BACK_UNROLL = 8;  // 32-key chunks of the back store loaded at once

// Number of back keys below hi that are not prunable (whole warp).
__device__ __forceinline__ int back_count(const SeedQueue& s, uint64_t hi, uint64_t cut) {
  const int lane = threadIdx.x & 31;
  int c = 0;
  for (int c0 = 0; c0 < s.nback; c0 += 32 * BACK_UNROLL) {
    uint64_t key[BACK_UNROLL];
#pragma unroll
    for (int u = 0; u < BACK_UNROLL; ++u) {
      const int p = c0 + 32 * u + lane;
      key[u] = p < s.nback ? s.back[p] : ~0ull;
    }
#pragma unroll
    for (int u = 0; u < BACK_UNROLL; ++u) c += __popc(__ballot_sync(0xffffffffu, key[u] < hi && !key_prunable(key[u], cut)));
  }
  return c;
}

// Refills the empty front with the back keys below a threshold hi chosen so
// that at most S of them (about S / 2) qualify: hi follows a sorted sample of
// up to 32 qualifying keys (each lane takes the first one on its stride of
// the back store), and is narrowed with a new sample while more than S keys
// lie below it.  One pass then moves the keys below hi into the front, in
// sorted batches of 32 staged in shared memory, and compacts the others in
// place; hi becomes the fence.  Prunable keys are dropped.  Without a
// threshold after four samples the whole back store is merged through.
__device__ void seeds_refill(SeedQueue& s, uint64_t* bbuf, uint64_t cut) {
  const int lane = threadIdx.x & 31;
  const int n = s.nback;
  if (n == 0) return;
  uint64_t hi = ~0ull;
  int c = n;  // an upper bound of the keys below hi
  for (int round = 0; c > s.S; ++round) {
    if (round == 4) {
      seeds_refill_merge(s, bbuf, cut);
      return;
    }
    uint64_t smp = ~0ull;
    for (int p = lane; p < n; p += 32) {
      const uint64_t key = s.back[p];
      if (key < hi && !key_prunable(key, cut)) {
        smp = key;
        break;
      }
    }
    const int ns = __popc(__ballot_sync(0xffffffffu, smp != ~0ull));
    if (ns == 0) {  // every key prunable (c counted none) or none below hi
      c = 0;
      break;
    }
    const uint64_t sorted = warp_sort32(smp);
    // about (r + 1) / ns of the c keys lie at or below the sample's r-th key
    const int r = max(0, min(ns - 1, (int)(((long long)(s.S / 2) * ns) / c) - 1));
    const uint64_t t = __shfl_sync(0xffffffffu, sorted, r);
    hi = t + 1;  // t is a key (distinct, never ~0)
    c = back_count(s, hi, cut);
  }
  uint64_t* stage = bbuf + 64;
  int staged = 0, w = 0;
  s.head = s.tail = 0;
  s.fence = ~0ull;
  auto flush = [&]() {
    const uint64_t key = lane < staged ? stage[lane] : ~0ull;
    __syncwarp();
    uint64_t ev;
    front_merge(s, bbuf, warp_sort32(key), staged, cut, ev);  // at most S keys in all: nothing leaves
    staged = 0;
  };
  for (int c0 = 0; c0 < n; c0 += 32 * BACK_UNROLL) {
    uint64_t keys[BACK_UNROLL];
#pragma unroll
    for (int u = 0; u < BACK_UNROLL; ++u) {
      const int p = c0 + 32 * u + lane;
      keys[u] = p < n ? s.back[p] : ~0ull;
    }
    __syncwarp();  // every chunk read before the in-place writes (w stays at or below c0 + 32 u)
#pragma unroll
    for (int u = 0; u < BACK_UNROLL; ++u) {
      const uint64_t key = keys[u];
      const bool live = key != ~0ull && !key_prunable(key, cut);
      const bool sel = live && key < hi;
      back_append(s, key, live && !sel, w, n);
      const unsigned sm = __ballot_sync(0xffffffffu, sel);
      if (staged + __popc(sm) > 32) flush();
      if (sel) stage[staged + __popc(sm & ((1u << lane) - 1u))] = key;
      staged += __popc(sm);
      __syncwarp();
    }
  }
  if (staged > 0) flush();
  __syncwarp();
  s.nback = w;
  s.fence = w > 0 ? hi : ~0ull;
}

// tree_query_scale of a quantized query (lib.rs:283-296): max|q| / 127 of the
// FP32 query, 0 for a zero query.  Whole warp.
__device__ __forceinline__ float tree_query_scale(const float* qf, int D) {
  const int lane = threadIdx.x & 31;
  float mx = 0.f;
  for (int t = lane; t < D; t += 32) mx = fmaxf(mx, fabsf(qf[t]));
  for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  return mx > 0.f ? __fdiv_rn(mx, 127.0f) : 0.f;
}

// Margin of a query at an internal node: the FP32 hyperplane's dot in the
// reference order plus the offset (builder.rs:331), or with int8 routing trees
// (qtrees) the reconstructed margin dot(codes) * scale * tree_query_scale +
// offset (flat_tree.rs:96-103).  Every lane computes the same value.
__device__ __forceinline__ float tree_margin(const SearchIndex& ix, bool qtrees, const float* qf, const int8_t* q8,
                                             float tqs, int node) {
  if (qtrees) {
    const int4* a = reinterpret_cast<const int4*>(q8);
    const int4* b = reinterpret_cast<const int4*>(ix.tree_codes + (size_t)node * ix.Dq);
    int acc = 0;
    for (int t = 0; t < ix.Dq / 16; ++t) {
      const int4 x = a[t], y = __ldg(b + t);
      acc = __dp4a(x.x, y.x, acc);
      acc = __dp4a(x.y, y.y, acc);
      acc = __dp4a(x.z, y.z, acc);
      acc = __dp4a(x.w, y.w, acc);
    }
    return __fadd_rn(__fmul_rn(__fmul_rn((float)acc, ix.tree_scales[node]), tqs), ix.offsets[node]);
  }
  return __fadd_rn(exact_dot_a(qf, ix.hyperplanes + (size_t)node * ix.Dp, ix.D), ix.offsets[node]);
}

// FlatTree::search_leaves (flat_tree.rs:239-311), whole warp: calls
// on_leaf(start, end) for each leaf found, in order.  budget 1: hard descent
// (margin > 0 -> right, |m| < 1e-8 -> random side).  Otherwise the spill
// search over a frontier of (priority, node) kept in insertion order in `fr`
// (fcap entries): take the first entry of least priority (min_by over
// total_cmp; priorities are non-negative so their bits order them), emit a
// leaf, or split an internal node into the near child (same priority) and the
// far child (priority max(p, |margin|)), until `budget` leaves.  A frontier
// that would exceed fcap (not reachable with fcap = budget * depth + 2) ends
// the search early and is counted in *overflow.
template <class LeafF>
__device__ void tree_search_leaves(const SearchIndex& ix, int root, int budget, uint64_t* fr, int fcap, QRng& rng,
                                   bool qtrees, const float* qf, const int8_t* q8, float tqs,
                                   unsigned long long* overflow, LeafF&& on_leaf) {
  const int lane = threadIdx.x & 31;
  auto side_of = [&](float margin) -> int {
    if (fabsf(margin) < 1e-8f) return rng.next_bool() ? 1 : 0;
    return margin > 0.f ? 1 : 0;
  };
  if (budget <= 1 || fcap < 3) {
    int node = root;
    while (ix.children[2 * (size_t)node] > 0)
      node = ix.children[2 * (size_t)node + side_of(tree_margin(ix, qtrees, qf, q8, tqs, node))];
    on_leaf(-ix.children[2 * (size_t)node], -ix.children[2 * (size_t)node + 1]);
    return;
  }
  int nfr = 1, nleaves = 0;
  if (lane == 0) fr[0] = (uint64_t)(uint32_t)root;
  __syncwarp();
  while (nleaves < budget && nfr > 0) {
    uint64_t best = ~0ull;
    for (int e = lane; e < nfr; e += 32) {
      const uint64_t key = (fr[e] & 0xFFFFFFFF00000000ull) | (uint32_t)e;
      best = key < best ? key : best;
    }
    for (int o = 16; o; o >>= 1) {
      const uint64_t other = __shfl_xor_sync(0xffffffffu, best, o);
      best = other < best ? other : best;
    }
    const int pos = (int)(uint32_t)best;
    const uint64_t entry = fr[pos];
    __syncwarp();
    for (int c0 = pos; c0 < nfr - 1; c0 += 32) {  // Vec::remove: shift the tail left
      const int e = c0 + lane;
      const uint64_t v = e + 1 < nfr ? fr[e + 1] : 0ull;
      __syncwarp();
      if (e + 1 < nfr) fr[e] = v;
      __syncwarp();
    }
    --nfr;
    const int node = (int)(uint32_t)entry;
    const float prio = __uint_as_float((uint32_t)(entry >> 32));
    if (ix.children[2 * (size_t)node] <= 0) {
      on_leaf(-ix.children[2 * (size_t)node], -ix.children[2 * (size_t)node + 1]);
      ++nleaves;
      continue;
    }
    const float margin = tree_margin(ix, qtrees, qf, q8, tqs, node);
    const int side = side_of(margin);
    const float far = fmaxf(prio, fabsf(margin));
    if (nfr + 2 > fcap) {
      if (lane == 0) atomicAdd(overflow, 1ull);
      break;
    }
    if (lane == 0) {
      fr[nfr] = ((uint64_t)__float_as_uint(prio) << 32) | (uint32_t)ix.children[2 * (size_t)node + side];
      fr[nfr + 1] = ((uint64_t)__float_as_uint(far) << 32) | (uint32_t)ix.children[2 * (size_t)node + 1 - side];
    }
    __syncwarp();
    nfr += 2;
  }
}

// k: result-list width; k_out: entries written to oi/od; rerank (QUANT only):
// number of leading results re-ordered by exact FP32 distance before output;
// rng_seed: the query's random stream.
// W: this warp's global-memory state for the pass: the first-level visited
// table when the layout has none in shared memory (vis1), the second-level
// table (vis2, or null), the seed back store (back), and in the exact pass a
// visited bitset of N bits (bits; the tables are then unused) with a back store
// of N entries, neither of which can overflow.  Returns true when a bounded
// state could have changed the result (the query is then re-run).
struct WarpScratch {
  int32_t* vis1;
  int vis1_cap;
  int32_t* vis2;
  int vis2_cap;
  uint64_t* back;
  int back_cap;
  uint32_t* bits;
};
template <bool QUANT>
__device__ bool search_one(const SearchIndex& ix, const float* Qrow, const int8_t* Q8row,
                           float qinv, uint64_t rng_seed, int k, int k_out, int rerank, float eps,
                           const WarpLayout& L, unsigned char* wsm, const WarpScratch& W, int32_t* oi,
                           float* od, unsigned long long* stats) {
  const int lane = threadIdx.x & 31;
  float* q = reinterpret_cast<float*>(wsm + L.q_off());
  uint64_t* res = reinterpret_cast<uint64_t*>(wsm + L.res_off());
  uint64_t* seeds = reinterpret_cast<uint64_t*>(wsm + L.seed_off());
  int32_t* vis = W.vis1 ? W.vis1 : reinterpret_cast<int32_t*>(wsm + L.vis_off());
  uint64_t* bbuf = reinterpret_cast<uint64_t*>(wsm + L.batch_off());
  int8_t* q8 = reinterpret_cast<int8_t*>(q);  // QUANT: codes stored in the query slot
  if (QUANT) {
    for (int t = lane; t < ix.Dq / 16; t += 32)
      reinterpret_cast<int4*>(q8)[t] = reinterpret_cast<const int4*>(Q8row)[t];
  } else {
    for (int t = lane; t < ix.Dp; t += 32) q[t] = t < ix.D ? Qrow[t] : 0.f;
  }
  const int vcap = W.vis1 ? W.vis1_cap : L.h;
  Visited V{vis, vcap, 0, W.vis2, W.vis2_cap, W.bits, false, false};
  if (W.bits) {
    uint4* b4 = reinterpret_cast<uint4*>(W.bits);  // words padded to a multiple of 4
    for (long long t = lane; t < ((long long)ix.N + 127) / 128; t += 32) b4[t] = make_uint4(0u, 0u, 0u, 0u);
  } else {
    int4* v4 = reinterpret_cast<int4*>(vis);  // capacities are multiples of 4
    for (int t = lane; t < vcap / 4; t += 32) v4[t] = make_int4(-1, -1, -1, -1);
  }
  __syncwarp();
  QRng rng(rng_seed);
  SeedQueue sq{seeds, L.s, L.s, 0, 0, 0, W.back, W.back_cap, 0, ~0ull, ~0ull, false};
  // Dropped seeds change the result only if the unbounded search would pop
  // one: when a popped seed ranks after the smallest dropped one while that
  // one is still within the bound, or the seeds run out while it is.
  bool lost = false;  // the bounded state may have changed the result (warp-uniform)
  int rc = 0;
  unsigned long long evals = 0, expansions = 0;
  unsigned long long* overflow = &stats[2];
  const float min_d = ix.min_distance;
  auto bound_of = [&](float mx) { return __fadd_rn(mx, __fmul_rn(eps, __fsub_rn(mx, min_d))); };
  // seeds are pruned against the bound only where the bound cannot grow again
  const bool prune_ok = eps >= 0.f && eps <= 3.402823466e38f && fabsf(min_d) <= 3.402823466e38f;
  auto cut_of = [&](float b) { return prune_ok && rc >= k ? (uint64_t)fkey(b) << 32 : ~0ull; };

  // ---- unconditional pushes of a list of candidate ids (leaves, random fill) ----
  auto push_all = [&](int32_t my_id, bool have) {
    const bool fresh = !visited_mark(V, my_id, have, overflow) && have;
    const float d = fresh ? dist_to<QUANT>(ix, q, q8, qinv, my_id) : 0.f;
    unsigned m = __ballot_sync(0xffffffffu, fresh);
    evals += __popc(m);
    uint64_t bkey = fresh ? rkey(d, my_id) : ~0ull;
    unsigned mm = m;
    while (mm) {
      int j = __ffs(mm) - 1;
      mm &= mm - 1;
      float dj = __shfl_sync(0xffffffffu, d, j);
      int32_t ij = __shfl_sync(0xffffffffu, my_id, j);
      result_push(res, rc, k, dj, ij);
    }
    uint64_t sorted = warp_sort32(bkey);
    seeds_push(sq, bbuf, sorted, __popc(m), ~0ull);
  };

  // ---- tree seeding (greedy.rs:70-146): the points of the leaves each tree's
  // search_leaves returns (flat_tree.rs:239-311), in leaf order ----
  // Margins: FP32 hyperplanes (dot in the reference order + offset, builder.rs:331),
  // or for quantized queries over int8 routing trees the reconstructed margin
  // dot(codes) * scale * tree_query_scale + offset (flat_tree.rs:96-103), with
  // tree_query_scale = max|q| / 127 of the FP32 query (lib.rs:283-296).
  const bool qtrees = QUANT && ix.tree_codes != nullptr;
  const float tqs = qtrees ? tree_query_scale(Qrow, ix.D) : 0.f;
  uint64_t* fr = reinterpret_cast<uint64_t*>(wsm + L.fr_off());
  for (int t = 0; t < ix.n_trees; ++t) {
    const int32_t* tidx = ix.tree_idx + (size_t)t * ix.N;
    tree_search_leaves(ix, ix.tree_roots[t], L.f > 0 ? ix.leaf_budget : 1, fr, L.f, rng, qtrees,
                       QUANT ? Qrow : q, q8, tqs, &stats[3], [&](int start, int end) {
                         for (int p0 = start; p0 < end; p0 += 32) {
                           int p = p0 + lane;
                           int32_t id = p < end ? tidx[p] : -1;
                           push_all(id, id >= 0);
                         }
                       });
  }
  // ---- fill_random (greedy.rs:148-163) ----
  {
    int need = k - (sq.tail - sq.head + sq.nback);
    for (int r0 = 0; r0 < need; r0 += 32) {
      int32_t id = -1;
      // draws in sequence order (every lane runs the stream); lane r takes draw r0 + r
      for (int r = 0; r < 32 && r0 + r < need; ++r) {
        uint32_t x = rng.next_index((uint32_t)ix.N);
        if (r == lane) id = (int32_t)x;
      }
      // mark in draw order so a repeated draw is skipped like check_and_mark
      bool fresh = false;
      for (int r = 0; r < 32 && r0 + r < need; ++r) {
        int32_t x = __shfl_sync(0xffffffffu, id, r);
        bool f = !visited_mark(V, x, lane == 0, overflow);
        f = __shfl_sync(0xffffffffu, f, 0);
        if (lane == r) fresh = f;
      }
      __syncwarp();
      float d = fresh ? dist_to<QUANT>(ix, q, q8, qinv, id) : 0.f;
      unsigned m = __ballot_sync(0xffffffffu, fresh);
      evals += __popc(m);
      unsigned mm = m;
      while (mm) {
        int j = __ffs(mm) - 1;
        mm &= mm - 1;
        result_push(res, rc, k, __shfl_sync(0xffffffffu, d, j), __shfl_sync(0xffffffffu, id, j));
      }
      uint64_t sorted = warp_sort32(fresh ? rkey(d, id) : ~0ull);
      seeds_push(sq, bbuf, sorted, __popc(m), ~0ull);
    }
  }
  // ---- traverse (greedy.rs:165-201) ----
  float mx = result_max(res, rc);
  float bound = bound_of(mx);
  bool stopped = false;
  int32_t pv = -1, pnb = -1;  // predicted next seed, this lane's first neighbor of it
  int ps = 0, pe = 0;         // its CSR range
  while (true) {
    if (sq.head == sq.tail) {
      if (sq.nback == 0) break;
      seeds_refill(sq, bbuf, cut_of(bound));
      if (sq.head == sq.tail) break;
    }
    const uint64_t top = sq.front[(size_t)sq.cur * sq.stride + sq.head];
    ++sq.head;
    float vd = fkey_inv((uint32_t)(top >> 32));
    int32_t v = (int32_t)(uint32_t)top;
    if (top > sq.min_drop) {  // the unbounded search reaches the dropped seed first
      if (!(rc >= k && fkey_inv((uint32_t)(sq.min_drop >> 32)) >= bound)) lost = true;
    }
    if (rc >= k && vd >= bound) {
      stopped = true;
      break;
    }
    // With an exact visited set every node is expanded at most once; the cap
    // only matters after a visited-table overflow, where it bounds the loop.
    if (expansions >= (unsigned long long)ix.N + 64) break;
    // a bounded pass stops as soon as its result is known to need the re-run
    if (!W.bits && (lost || V.lost)) break;
    ++expansions;
    int s, e;
    int32_t nb_first;
    if (v == pv) {  // loaded one expansion ahead
      s = ps;
      e = pe;
      nb_first = pnb;
    } else {
      s = ix.indptr[v];
      e = ix.indptr[v + 1];
      nb_first = s + lane < e ? ix.indices[s + lane] : -1;
    }
    // the likely next seed (the front's first key, unless this expansion
    // pushes a smaller one): its CSR range now, its first neighbors after the
    // expansion, so that their latency overlaps this expansion
    pv = sq.head < sq.tail ? (int32_t)(uint32_t)sq.front[(size_t)sq.cur * sq.stride + sq.head] : -1;
    if (pv >= 0) {
      ps = ix.indptr[pv];
      pe = ix.indptr[pv + 1];
    }
    for (int c0 = s; c0 < e; c0 += 32) {
      int c = c0 + lane;
      int32_t nb = c0 == s ? nb_first : (c < e ? ix.indices[c] : -1);
      const bool fresh = !visited_mark(V, nb, nb >= 0, overflow) && nb >= 0;
      float d = fresh ? dist_to<QUANT>(ix, q, q8, qinv, nb) : 0.f;
      unsigned m = __ballot_sync(0xffffffffu, fresh);
      evals += __popc(m);
      unsigned acc_mask = 0;
      if (rc >= k) {
        // With a full result list the maximum and the bound only shrink, and a
        // neighbor enters the list only below the current maximum: those run in
        // order; every neighbor is accepted against the bound left by the
        // insertions of the neighbors before it (the reference's sequential test).
        float my_bound = bound;
        unsigned ins = __ballot_sync(0xffffffffu, fresh && d < mx);
        while (ins) {
          const int j = __ffs(ins) - 1;
          ins &= ins - 1;
          const float dj = __shfl_sync(0xffffffffu, d, j);
          if (dj < bound && result_push(res, rc, k, dj, __shfl_sync(0xffffffffu, nb, j))) {
            mx = result_max(res, rc);
            bound = bound_of(mx);
            if (lane > j) my_bound = bound;
          }
        }
        acc_mask = __ballot_sync(0xffffffffu, fresh && d < my_bound);
      } else {
        unsigned mm = m;
        while (mm) {
          int j = __ffs(mm) - 1;
          mm &= mm - 1;
          float dj = __shfl_sync(0xffffffffu, d, j);
          if (dj < bound) {
            int32_t ij = __shfl_sync(0xffffffffu, nb, j);
            acc_mask |= 1u << j;
            if (result_push(res, rc, k, dj, ij)) {
              mx = result_max(res, rc);
              bound = bound_of(mx);
            }
          }
        }
      }
      bool acc = (acc_mask >> lane) & 1u;
      uint64_t sorted = warp_sort32(acc ? rkey(d, nb) : ~0ull);
      seeds_push(sq, bbuf, sorted, __popc(acc_mask), cut_of(bound));
    }
    if (pv >= 0) pnb = ps + lane < pe ? ix.indices[ps + lane] : -1;
  }
  // seeds ran out: the unbounded search would go on with a dropped seed
  // within the bound
  if (!stopped && sq.min_drop != ~0ull && !(rc >= k && fkey_inv((uint32_t)(sq.min_drop >> 32)) >= bound))
    lost = true;
  // ---- exact rerank of the first `rerank` results (index.rs:103-126): exact
  // FP32 distance to the FP32 query, sorted by (distance, id) ----
  int nres = rc;
  if (QUANT && rerank > 0) {
    const int m = min(rc, rerank);
    uint64_t* tmp = seeds;  // the front's arrays (2 S >= 512 entries) are free after the traversal
    for (int e = lane; e < m; e += 32) {
      const int32_t id = (int32_t)(uint32_t)res[e];
      tmp[e] = rkey(exact_distance(ix.kind, Qrow, ix.X + (size_t)id * ix.Dp, ix.D), id);
    }
    __syncwarp();
    for (int e = lane; e < m; e += 32) {  // ids are distinct, so ranks are too
      const uint64_t key = tmp[e];
      int r = 0;
      for (int j = 0; j < m; ++j) r += tmp[j] < key;
      res[r] = key;
    }
    __syncwarp();
    nres = m;
  }
  // ---- output (index.rs:182-199, :324-333) ----
  for (int j = lane; j < k_out; j += 32) {
    if (j < nres) {
      uint64_t key = res[j];
      int32_t id = (int32_t)(uint32_t)key;
      float d = fkey_inv((uint32_t)(key >> 32));
      oi[j] = ix.vertex_order ? ix.vertex_order[id] : id;
      od[j] = QUANT ? d : apply_correction(ix.corr, d);
    } else {
      oi[j] = -1;
      od[j] = __int_as_float(0x7f800000);
    }
  }
  if (lane == 0) {
    atomicAdd(&stats[0], evals);
    atomicAdd(&stats[1], expansions);
    if (V.tab2_live) atomicAdd(&stats[6], 1ull);
    if (sq.spilled) atomicAdd(&stats[7], 1ull);
  }
  __syncwarp();
  return __any_sync(0xffffffffu, lost || V.lost);
}

// One pass of the search over a set of queries: all nq (list_in null) or
// list_in[0, *count_in); warps take queries from the counter `next` one at a
// time.  A query whose bounded state could have changed its result is
// appended to (count_out, list_out) for the next pass (none in the exact
// pass).  Per-warp global state: first-level visited tables of vis1_cap ids
// (null: the layout's shared-memory table), second-level tables of vis2_cap
// ids (null: none), seed back stores of back_cap keys and, in the exact pass,
// visited bitsets of `words` words.
struct PassState {
  const unsigned int* count_in;
  const int32_t* list_in;
  unsigned int* count_out;
  int32_t* list_out;
  unsigned int* next;
  int32_t* vis1;
  int vis1_cap;
  int32_t* vis2;
  int vis2_cap;
  uint64_t* back;
  int back_cap;
  uint32_t* bits;
  long long words;
};

template <bool QUANT>
__global__ void __launch_bounds__(WPB * 32)
    k_search(SearchIndex ix, const float* Q, const int8_t* Q8, const float* qinv, int nq, int k, int k_out,
             int rerank, float eps, uint64_t qid_base, QueryMeta meta, WarpLayout L, PassState P,
             int32_t* out_idx, float* out_dist, unsigned long long* stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int w = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  unsigned char* wsm = smem + (size_t)w * L.bytes();
  const size_t gw = (size_t)blockIdx.x * (blockDim.x >> 5) + w;  // the re-runs launch one-warp blocks
  WarpScratch W{P.vis1 ? P.vis1 + gw * P.vis1_cap : nullptr, P.vis1_cap,
                P.vis2 ? P.vis2 + gw * P.vis2_cap : nullptr, P.vis2_cap,
                P.back + gw * P.back_cap, P.back_cap,
                P.bits ? P.bits + gw * P.words : nullptr};
  const int n_run = P.list_in ? (int)min((unsigned int)nq, *P.count_in) : nq;
  for (;;) {
    int t = 0;
    if (lane == 0) t = (int)atomicAdd(P.next, 1u);
    t = __shfl_sync(0xffffffffu, t, 0);
    if (t >= n_run) break;
    const int qi = P.list_in ? P.list_in[t] : t;
    int qk = k, qko = k_out, qr = rerank;
    float qe = eps;
    // FP32 queries seed with seed + query index (index.rs:165); quantized
    // queries all use the seed alone (index.rs:298)
    uint64_t stream = QUANT ? 0ull : qid_base + (uint64_t)qi;
    int64_t off = (int64_t)qi * k_out;
    if (meta.width) {  // per-query parameters of a packed batch
      qk = meta.width[qi];
      qko = meta.kout[qi];
      qr = meta.rerank ? meta.rerank[qi] : 0;
      qe = meta.eps[qi];
      stream = QUANT ? 0ull : meta.stream[qi];
      off = meta.out_off[qi];
    }
    const bool lost = search_one<QUANT>(ix, Q + (size_t)qi * ix.Dp, QUANT ? Q8 + (size_t)qi * ix.Dq : nullptr,
                                        QUANT ? qinv[qi] : 0.f, ix.seed + stream, qk, qko, qr, qe, L, wsm, W,
                                        out_idx + off, out_dist + off, stats);
    if (lost && P.list_out && lane == 0) P.list_out[atomicAdd(P.count_out, 1u)] = qi;
  }
}

// search_leaves of one tree for a batch of queries (warp per query), with the
// search kernel's own routing code: leaves (start, end) in order into
// out[q * budget * 2 ...], their count into cnt[q].  Random sides of tied
// margins use the query's search stream (seed + qid_base + q; quantized
// queries the seed alone).
__global__ void __launch_bounds__(WPB * 32)
    k_tree_leaves(SearchIndex ix, const float* Q, const int8_t* Q8, int nq, int tree, int budget, int fcap,
                  uint64_t qid_base, int32_t* out, int32_t* cnt, unsigned long long* stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* fr = reinterpret_cast<uint64_t*>(smem) + (size_t)w * fcap;
  const bool qtrees = Q8 != nullptr;
  for (int qi = blockIdx.x * WPB + w; qi < nq; qi += gridDim.x * WPB) {
    const float* qf = Q + (size_t)qi * ix.Dp;
    const int8_t* q8 = qtrees ? Q8 + (size_t)qi * ix.Dq : nullptr;
    QRng rng(ix.seed + (qtrees ? 0ull : qid_base + (uint64_t)qi));
    const float tqs = qtrees ? tree_query_scale(qf, ix.D) : 0.f;
    int n = 0;
    int32_t* o = out + (size_t)qi * budget * 2;
    tree_search_leaves(ix, ix.tree_roots[tree], budget, fr, fcap, rng, qtrees, qf, q8, tqs, &stats[3],
                       [&](int start, int end) {
                         if (lane == 0 && n < budget) {
                           o[2 * n] = start;
                           o[2 * n + 1] = end;
                         }
                         ++n;
                       });
    if (lane == 0) cnt[qi] = n < budget ? n : budget;
    __syncwarp();
  }
}

WarpLayout layout_for(const SearchIndex& ix, int k) {
  if (k > 256) throw std::invalid_argument("k must be <= 256");
  WarpLayout L;
  L.dp = std::max(ix.Dp, ix.Dq / 4);
  L.kmax = k <= 32 ? 32 : (k <= 128 ? 128 : 256);
  L.s = seed_capacity(L.kmax);
  L.h = L.kmax <= 32 ? visited_capacity(L.kmax) : 0;  // wider searches use a global-memory table
  L.f = ix.leaf_budget > 1 ? ix.frontier_cap : 0;
  set_smem_limit_once(reinterpret_cast<const void*>(k_search<false>), 200 * 1024);
  set_smem_limit_once(reinterpret_cast<const void*>(k_search<true>), 200 * 1024);
  if (L.bytes() * WPB > 200 * 1024)
    throw std::invalid_argument("query dimension and search_tree_leaf_budget too large for search shared memory");
  return L;
}

// Blocks of `kernel` resident on the current device at once (cached).
int resident_blocks(const void* kernel, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, size_t, int>, int> cache;
  int dev = 0;
  RINND_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_tuple(kernel, threads, smem, dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int per_sm = 0, sms = 0;
  RINND_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  RINND_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int r = std::max(1, per_sm) * std::max(1, sms);
  cache[key] = r;
  return r;
}

// Per-warp global state of the passes.  Bounded pass: as many warps as are
// resident (at most FIRST_BYTES of state), a second-level visited table of
// 16x the shared table (4x the global first-level table for widths above 32)
// and a back store of 64 S seeds.  Wide pass (queries the bounded pass lost):
// WIDE_WARPS one-warp blocks with the same front (a merge costs S / 32 steps
// a lane, so a larger front slows every expansion) and a visited table of
// WIDE_VIS1 ids in shared memory, a second-level table of WIDE_VIS2 ids and a
// back store of WIDE_BACK seeds.  Exact pass (queries the wide pass
// lost): a visited bitset of N bits and a back store of N seeds per warp, as
// many warps as fit EXACT_BYTES (at least one, at most EXACT_MAX_WARPS).
constexpr size_t FIRST_BYTES = 1024ull << 20;
constexpr int WIDE_WARPS = 148;
constexpr int WIDE_VIS1 = 1 << 13;
constexpr int WIDE_VIS2 = 1 << 17;
constexpr int WIDE_BACK = 1 << 15;
constexpr size_t EXACT_BYTES = 256ull << 20;
constexpr int EXACT_MAX_WARPS = 128;

// stats[4] += queries re-run in the wide pass, stats[5] += in the exact pass
__global__ void k_count_reruns(const unsigned int* counts, unsigned long long* stats) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    atomicAdd(&stats[4], (unsigned long long)counts[0]);
    atomicAdd(&stats[5], (unsigned long long)counts[1]);
  }
}

// The bounded launch over all queries; the wide launch over the queries it
// recorded; the exact launch over the queries the wide launch recorded (their
// outputs are overwritten).  All are enqueued on `st`; each re-run finds its
// query count on the device.
template <bool QUANT>
void run_search(const SearchIndex& ix, const float* Q, const int8_t* Q8, const float* qinv, int nq, int k, int k_out,
                int rerank, float eps, uint64_t qid_base, const QueryMeta& meta, const WarpLayout& L,
                int32_t* out_idx, float* out_dist, cudaStream_t st, unsigned long long* dstats) {
  const void* kern = reinterpret_cast<const void*>(k_search<QUANT>);
  // counts: [0] wide list, [1] exact list, [2..4] work counters of the passes
  DVec<unsigned int> counts(8, st);
  counts.fill_bytes(0);
  DVec<int32_t> list1((size_t)nq, st), list2((size_t)nq, st);

  // bounded pass
  const int vis1 = L.h > 0 ? 0 : visited_capacity(L.kmax);
  const int vis2 = L.h > 0 ? 16 * L.h : 4 * vis1;
  const int back = 64 * L.s;
  const size_t per_warp = (size_t)vis1 * 4 + (size_t)vis2 * 4 + (size_t)back * 8;
  int blocks = std::min((nq + WPB - 1) / WPB, resident_blocks(kern, WPB * 32, L.bytes() * WPB));
  blocks = std::max(1, std::min<int>(blocks, (int)(FIRST_BYTES / (per_warp * WPB))));
  const size_t warps = (size_t)blocks * WPB;
  DVec<int32_t> v1(warps * vis1, st), v2(warps * vis2, st);
  DVec<uint64_t> bk(warps * back, st);
  PassState p1{nullptr, nullptr, counts.p, list1.p, counts.p + 2, v1.p, vis1, v2.p, vis2, bk.p, back, nullptr, 0};
  k_search<QUANT><<<blocks, WPB * 32, L.bytes() * WPB, st>>>(ix, Q, Q8, qinv, nq, k, k_out, rerank, eps, qid_base,
                                                             meta, L, p1, out_idx, out_dist, dstats);
  RINND_LAUNCH_CHECK();

  // wide pass
  WarpLayout Lw = L;
  Lw.h = WIDE_VIS1;
  const int wwarps = std::min(WIDE_WARPS, nq);
  DVec<int32_t> wv2((size_t)wwarps * WIDE_VIS2, st);
  DVec<uint64_t> wbk((size_t)wwarps * WIDE_BACK, st);
  PassState p2{counts.p, list1.p, counts.p + 1, list2.p, counts.p + 3, nullptr, 0, wv2.p, WIDE_VIS2,
               wbk.p, WIDE_BACK, nullptr, 0};
  k_search<QUANT><<<wwarps, 32, Lw.bytes(), st>>>(ix, Q, Q8, qinv, nq, k, k_out, rerank, eps, qid_base, meta, Lw,
                                                  p2, out_idx, out_dist, dstats);
  RINND_LAUNCH_CHECK();

  // exact pass
  WarpLayout Lx = L;
  Lx.h = 0;
  const long long words = ((long long)(ix.N + 31) / 32 + 3) / 4 * 4;  // 16-byte multiple per warp
  const size_t x_per_warp = (size_t)words * 4 + (size_t)ix.N * 8;
  const int xwarps =
      std::min(nq, (int)std::max<size_t>(1, std::min<size_t>(EXACT_BYTES / x_per_warp, EXACT_MAX_WARPS)));
  DVec<uint32_t> xbits((size_t)xwarps * words, st);
  DVec<uint64_t> xbk((size_t)xwarps * ix.N, st);
  PassState p3{counts.p + 1, list2.p, nullptr, nullptr, counts.p + 4, nullptr, 0, nullptr, 0,
               xbk.p, ix.N, xbits.p, words};
  k_search<QUANT><<<xwarps, 32, Lx.bytes(), st>>>(ix, Q, Q8, qinv, nq, k, k_out, rerank, eps, qid_base, meta, Lx,
                                                  p3, out_idx, out_dist, dstats);
  RINND_LAUNCH_CHECK();
  k_count_reruns<<<1, 32, 0, st>>>(counts.p, dstats);
  RINND_LAUNCH_CHECK();
}

}  // namespace

void greedy_search(const SearchIndex& ix, const float* Q, int nq, int k, float eps,
                   uint64_t qid_base, int32_t* out_idx, float* out_dist, cudaStream_t st,
                   unsigned long long* dstats) {
  if (nq <= 0) return;
  const WarpLayout L = layout_for(ix, k);
  run_search<false>(ix, Q, nullptr, nullptr, nq, k, k, 0, eps, qid_base, QueryMeta{}, L, out_idx, out_dist, st,
                    dstats);
}

void greedy_search_packed(const SearchIndex& ix, const float* Q, const int8_t* Q8, const float* qinv, int nq,
                          int max_width, const QueryMeta& meta, int32_t* out_idx, float* out_dist, cudaStream_t st,
                          unsigned long long* dstats) {
  if (nq <= 0) return;
  if (!meta.width || !meta.kout || !meta.eps || !meta.stream || !meta.out_off)
    throw std::invalid_argument("packed search needs every per-query array");
  const bool quant = Q8 != nullptr;
  if (quant && (!ix.codes || ix.Dq % 16 != 0)) throw std::invalid_argument("index has no int8 codes");
  const WarpLayout L = layout_for(ix, max_width);
  if (quant)
    run_search<true>(ix, Q, Q8, qinv, nq, 0, 0, 0, 0.f, 0, meta, L, out_idx, out_dist, st, dstats);
  else
    run_search<false>(ix, Q, nullptr, nullptr, nq, 0, 0, 0, 0.f, 0, meta, L, out_idx, out_dist, st, dstats);
}

void greedy_search_quantized(const SearchIndex& ix, const float* Q, const int8_t* Q8, const float* qinv, int nq,
                             int width, int k_out, int rerank, float eps, int32_t* out_idx, float* out_dist,
                             cudaStream_t st, unsigned long long* dstats) {
  if (nq <= 0) return;
  if (!ix.codes || ix.Dq % 16 != 0) throw std::invalid_argument("index has no int8 codes");
  if (k_out > width || rerank > width) throw std::invalid_argument("invalid quantized widths");
  const WarpLayout L = layout_for(ix, width);
  run_search<true>(ix, Q, Q8, qinv, nq, width, k_out, rerank, eps, 0, QueryMeta{}, L, out_idx, out_dist, st, dstats);
}

void tree_leaves(const SearchIndex& ix, const float* Q, const int8_t* Q8, int nq, int tree, int budget,
                 uint64_t qid_base, int32_t* out_leaves, int32_t* out_counts, cudaStream_t st,
                 unsigned long long* dstats) {
  if (nq <= 0) return;
  if (tree < 0 || tree >= ix.n_trees) throw std::invalid_argument("tree index out of range");
  if (budget < 1) throw std::invalid_argument("leaf budget must be >= 1");
  if (Q8 && !ix.tree_codes) throw std::invalid_argument("the index has no int8 routing trees");
  const int fcap = budget > 1 ? budget * std::max(ix.tree_depth, 1) + 2 : 3;
  const size_t smem = (size_t)WPB * fcap * 8;
  if (smem > 200 * 1024) throw std::invalid_argument("search_tree_leaf_budget too large for this forest");
  set_smem_limit_once(reinterpret_cast<const void*>(k_tree_leaves), 200 * 1024);
  const int blocks = std::min((nq + WPB - 1) / WPB, 148 * 8);
  k_tree_leaves<<<blocks, WPB * 32, smem, st>>>(ix, Q, Q8, nq, tree, budget, fcap, qid_base, out_leaves, out_counts,
                                                dstats);
  RINND_LAUNCH_CHECK();
}

}  // namespace rinnd
