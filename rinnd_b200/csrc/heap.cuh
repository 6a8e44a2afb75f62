// heap.cuh -- device-resident bounded neighbor rows with lock-free insertion.
//
// Restates NeighborHeap::checked_flagged_push (core/heap/neighbor_heap.rs:149-177)
// and checked_heap_push_flat (core/nndescent/candidates.rs:433-484) for many
// concurrent writers.  A row is k unordered 64-bit slots, key = (fkey(value) << 32) | id
// (flag in bit 31 of the low word for neighbor rows), stored with a stride that
// is a multiple of ROW_ALIGN slots (128 bytes) so a row spans whole cache lines.
// A push of (v, id):
//   1. is rejected if v >= the row's cached upper bound `thr[row]`,
//   2. reads a snapshot of all k slots (each 8-byte read is single-copy atomic;
//      all loads are issued before any is used), rejects if id is present or
//      v >= max slot value (the reference's `distance >= root`),
//   3. CASes the max slot (lowest index among equal keys) from its snapshot
//      value to the new key; on CAS failure it retries from 2.
// Slot values only ever decrease (a CAS always installs a strictly smaller key)
// and the max slot is chosen deterministically from the snapshot, which makes
// two concurrent pushes of the same id into one row impossible to both succeed:
// a successful CAS on slot m certifies that m held its snapshot value, and the
// monotonicity of slots forces both writers onto the same max slot unless one of
// them observed the other's id.  Retries are bounded (no unbounded spin).
#pragma once
#include "common.cuh"

namespace rinnd {

constexpr int PUSH_MAX_RETRY = 256;
constexpr int ROW_ALIGN = 16;  // slots per 128-byte line group

__host__ __device__ __forceinline__ int row_stride(int k) { return (k + ROW_ALIGN - 1) / ROW_ALIGN * ROW_ALIGN; }

// The order a push evicts by: distance, then id -- the new/old flag (bit 31)
// takes no part, so among equally distant entries a new one is not evicted
// before an old one (which would starve the next candidate samples on data
// with many tied distances).
constexpr uint64_t EVICT_MASK = ~(1ull << 31);

struct RowScan {
  uint64_t vmax;  // the slot value to evict: largest (distance, id), lowest index among equal
  uint64_t v2;    // largest key among the other slots
  int m;
  bool dup;
};

// Scans the k valid slots of a row whose storage holds row_stride(k) slots
// (16-byte aligned).  Loads are issued 16 slots at a time, unconditionally
// within the padded stride, and masked afterwards.
__device__ __forceinline__ RowScan scan_row(const uint64_t* row, int k, uint32_t id) {
  RowScan r{0, 0, 0, false};
  const ulonglong2* r2 = reinterpret_cast<const ulonglong2*>(row);
  bool first = true;
  for (int j0 = 0; j0 < k; j0 += ROW_ALIGN) {
    ulonglong2 v[ROW_ALIGN / 2];
#pragma unroll
    for (int t = 0; t < ROW_ALIGN / 2; ++t) v[t] = __ldcg(r2 + j0 / 2 + t);
#pragma unroll
    for (int t = 0; t < ROW_ALIGN; ++t) {
      int j = j0 + t;
      if (j < k) {
        uint64_t x = (t & 1) ? v[t >> 1].y : v[t >> 1].x;
        r.dup |= (((uint32_t)x) & 0x7FFFFFFFu) == id;
        if (first || (x & EVICT_MASK) > (r.vmax & EVICT_MASK)) {
          r.v2 = first ? 0 : r.vmax;
          r.vmax = x;
          r.m = j;
          first = false;
        } else if (x > r.v2) {
          r.v2 = x;
        }
      }
    }
  }
  return r;
}

// row_push for rows of at most KP (16 or 32) slots: the whole snapshot is held
// in registers, the scan tracks only the duplicate flag and the max slot, and
// the runner-up (for the bound update) is computed only after a successful CAS.
// Same decisions as the general form below.
template <int KP>
__device__ __forceinline__ int row_push_small(uint64_t* row, int k, uint32_t* thr, uint64_t key,
                                              unsigned long long* contention) {
  const uint32_t vk = (uint32_t)(key >> 32);
  const uint32_t id = ((uint32_t)key) & 0x7FFFFFFFu;
  const ulonglong2* r2 = reinterpret_cast<const ulonglong2*>(row);
  for (int attempt = 0; attempt < PUSH_MAX_RETRY; ++attempt) {
    uint64_t v[KP];
#pragma unroll
    for (int t = 0; t < KP / 2; ++t) {
      const ulonglong2 q = __ldcg(r2 + t);
      v[2 * t] = q.x;
      v[2 * t + 1] = q.y;
    }
    bool dup = false;
    uint64_t vmax = v[0];
    int m = 0;
#pragma unroll
    for (int j = 0; j < KP; ++j) {
      if (j < k) {
        dup |= (((uint32_t)v[j]) & 0x7FFFFFFFu) == id;
        if (j > 0 && (v[j] & EVICT_MASK) > (vmax & EVICT_MASK)) {
          vmax = v[j];
          m = j;
        }
      }
    }
    if (dup) return 0;
    if (vk >= (uint32_t)(vmax >> 32)) {
      if (thr != nullptr) atomicMin(thr, (uint32_t)(vmax >> 32));
      return 0;
    }
    unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(row + m), (unsigned long long)vmax,
                                       (unsigned long long)key);
    if (old == vmax) {
      if (thr != nullptr) {
        uint64_t v2 = 0;
#pragma unroll
        for (int j = 0; j < KP; ++j)
          if (j < k && j != m && v[j] > v2) v2 = v[j];
        const uint64_t nm = v2 > key ? v2 : key;
        atomicMin(thr, (uint32_t)(nm >> 32));
      }
      return 1;
    }
  }
  if (contention) atomicAdd(contention, 1ull);
  return 0;
}

// Returns 1 if inserted.  `key` = (fkey(v) << 32) | lo, lo's low 31 bits = id.
// `thr` (may be null) holds an upper bound of fkey(row max value).  This form
// scans the row in 16-slot chunks and keeps few registers: kernels whose push
// is a rare fallback (the join kernels' update-buffer overflow) use it.
__device__ __forceinline__ int row_push(uint64_t* row, int k, uint32_t* thr, uint64_t key,
                                        unsigned long long* contention) {
  const uint32_t vk = (uint32_t)(key >> 32);
  if (thr != nullptr && vk >= __ldcg(thr)) return 0;
  const uint32_t id = ((uint32_t)key) & 0x7FFFFFFFu;
  for (int attempt = 0; attempt < PUSH_MAX_RETRY; ++attempt) {
    RowScan s = scan_row(row, k, id);
    if (s.dup) return 0;
    if (vk >= (uint32_t)(s.vmax >> 32)) {
      if (thr != nullptr) atomicMin(thr, (uint32_t)(s.vmax >> 32));
      return 0;
    }
    unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(row + s.m),
                                       (unsigned long long)s.vmax, (unsigned long long)key);
    if (old == s.vmax) {
      if (thr != nullptr) {
        // Upper bound of the new row max: snapshot values are >= the current
        // ones, so max(runner-up of the snapshot, key) bounds the true max.
        uint64_t nm = s.v2 > key ? s.v2 : key;
        atomicMin(thr, (uint32_t)(nm >> 32));
      }
      return 1;
    }
  }
  if (contention) atomicAdd(contention, 1ull);
  return 0;
}

// The join kernels' rare direct push (an update beyond a full update-buffer
// region): the reject test (d >= the row's max, neighbor_heap.rs:156) on the
// rows' high words first, then a push whose eviction compares whole slot
// values (so among equally distant entries a new one goes first).  This form
// is kept as measured: the push's code is inlined into the join's pair loop
// and changes to it moved the 1M-point FP32 join between 67 and 101 ms.
__device__ __forceinline__ int row_push_raw(uint64_t* row, int k, uint32_t* thr, uint64_t key,
                                            unsigned long long* contention) {
  const uint32_t vk = (uint32_t)(key >> 32);
  const uint32_t id = ((uint32_t)key) & 0x7FFFFFFFu;
  const ulonglong2* r2 = reinterpret_cast<const ulonglong2*>(row);
  for (int attempt = 0; attempt < PUSH_MAX_RETRY; ++attempt) {
    uint64_t vmax = 0, v2 = 0;
    int m = 0;
    bool dup = false, first = true;
    for (int j0 = 0; j0 < k; j0 += ROW_ALIGN) {
      ulonglong2 v[ROW_ALIGN / 2];
#pragma unroll
      for (int t = 0; t < ROW_ALIGN / 2; ++t) v[t] = __ldcg(r2 + j0 / 2 + t);
#pragma unroll
      for (int t = 0; t < ROW_ALIGN; ++t) {
        const int j = j0 + t;
        if (j < k) {
          const uint64_t x = (t & 1) ? v[t >> 1].y : v[t >> 1].x;
          dup |= (((uint32_t)x) & 0x7FFFFFFFu) == id;
          if (first || x > vmax) {
            v2 = first ? 0 : vmax;
            vmax = x;
            m = j;
            first = false;
          } else if (x > v2) {
            v2 = x;
          }
        }
      }
    }
    if (dup) return 0;
    if (vk >= (uint32_t)(vmax >> 32)) {
      if (thr != nullptr) atomicMin(thr, (uint32_t)(vmax >> 32));
      return 0;
    }
    const unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(row + m),
                                             (unsigned long long)vmax, (unsigned long long)key);
    if (old == vmax) {
      if (thr != nullptr) {
        const uint64_t nm = v2 > key ? v2 : key;
        atomicMin(thr, (uint32_t)(nm >> 32));
      }
      return 1;
    }
  }
  if (contention) atomicAdd(contention, 1ull);
  return 0;
}

__device__ __forceinline__ int row_push_hi_first(uint64_t* row, int k, uint32_t* thr, uint64_t key,
                                                 unsigned long long* contention) {
  const uint32_t vk = (uint32_t)(key >> 32);
  if (thr != nullptr && vk >= __ldcg(thr)) return 0;
  const uint4* r4 = reinterpret_cast<const uint4*>(row);  // (lo, hi) word pairs
  uint32_t mx = 0;
  for (int j0 = 0; j0 < k; j0 += ROW_ALIGN) {
    uint4 v[ROW_ALIGN / 2];
#pragma unroll
    for (int t = 0; t < ROW_ALIGN / 2; ++t) v[t] = __ldcg(r4 + j0 / 2 + t);
#pragma unroll
    for (int t = 0; t < ROW_ALIGN / 2; ++t) {
      if (j0 + 2 * t < k) mx = max(mx, v[t].y);
      if (j0 + 2 * t + 1 < k) mx = max(mx, v[t].w);
    }
  }
  if (vk >= mx) {
    if (thr != nullptr) atomicMin(thr, mx);
    return 0;
  }
  return row_push_raw(row, k, thr, key, contention);
}

// The push of the reverse candidate offers and of the update application: rows
// of up to 32 slots take the register-snapshot form, longer rows the chunked
// scan.
__device__ __forceinline__ int row_push_fast(uint64_t* row, int k, uint32_t* thr, uint64_t key,
                                             unsigned long long* contention) {
  if (thr != nullptr && (uint32_t)(key >> 32) >= __ldcg(thr)) return 0;
  if (k <= 16) return row_push_small<16>(row, k, thr, key, contention);
  if (k <= 32) return row_push_small<32>(row, k, thr, key, contention);
  return row_push(row, k, thr, key, contention);
}

// Pushes that passed their row's bound, compacted per warp so that the row
// scans of row_push_fast start together on 32 queued updates instead of on
// whichever lanes of a 32-update slice passed.  `t` and `key` are this warp's
// 64 entries in shared memory.  append() queues the lanes whose `pass` is set
// and, once 32 are queued, hands one entry to every lane (returns true,
// warp-uniformly); drain() hands the rest to lanes below n.  Call both with
// the whole warp.
struct WarpQueue {
  uint32_t* t;
  uint64_t* key;
  int n;
  __device__ __forceinline__ bool append(bool pass, uint32_t ti, uint64_t ki, uint32_t& to, uint64_t& ko) {
    const int lane = threadIdx.x & 31;
    const unsigned bal = __ballot_sync(0xffffffffu, pass);
    if (pass) {
      const int pos = n + __popc(bal & ((1u << lane) - 1));
      t[pos] = ti;
      key[pos] = ki;
    }
    n += __popc(bal);
    __syncwarp();
    if (n < 32) return false;
    n -= 32;
    to = t[n + lane];
    ko = key[n + lane];
    __syncwarp();
    return true;
  }
  __device__ __forceinline__ bool drain(uint32_t& to, uint64_t& ko) const {
    const int lane = threadIdx.x & 31;
    if (lane >= n) return false;
    to = t[lane];
    ko = key[lane];
    return true;
  }
};

// Per-index accounting of a grouped build (several indices' rows in one set of
// heaps): an accepted push into row r adds 1 to changes[row_item[r]].  Both
// pointers are null outside grouped builds.
struct ItemCount {
  const int32_t* row_item;
  unsigned long long* changes;
  __device__ __forceinline__ void add(uint32_t row) const {
    if (changes != nullptr) atomicAdd(&changes[row_item[row]], 1ull);
  }
};

// Rows of indices that have finished iterating in a grouped build: frozen rows
// sample no candidates, so the join neither reads nor changes them.
struct GroupRows {
  const int32_t* row_item;
  const uint8_t* item_active;
  __device__ __forceinline__ bool frozen(int row) const {
    return item_active != nullptr && item_active[row_item[row]] == 0;
  }
};

// Run-length form for kernels that apply many pushes in row order: counts are
// held per thread while consecutive rows belong to one item.
struct ItemTally {
  int item = -1;
  unsigned int n = 0;
  __device__ __forceinline__ void add(const ItemCount& ic, uint32_t row) {
    if (ic.changes == nullptr) return;
    const int it = ic.row_item[row];
    if (it != item) {
      flush(ic);
      item = it;
    }
    ++n;
  }
  __device__ __forceinline__ void flush(const ItemCount& ic) {
    if (n) atomicAdd(&ic.changes[item], (unsigned long long)n);
    n = 0;
  }
};

}  // namespace rinnd
