// heap.cuh -- device-resident bounded neighbor rows with lock-free insertion.
//
// Restates NeighborHeap::checked_flagged_push (core/heap/neighbor_heap.rs:149-177)
// and checked_heap_push_flat (core/nndescent/candidates.rs:433-484) for many
// concurrent writers.  A row is k unordered 64-bit slots, key = (fkey(value) << 32) | id
// (flag in bit 31 of the low word for neighbor rows).  A push of (v, id):
//   1. is rejected if v >= the row's cached upper bound `thr[row]`,
//   2. reads a snapshot of all k slots (each 8-byte read is single-copy atomic),
//      rejects if id is present or v >= max slot value (the reference's
//      `distance >= root`),
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

__device__ __forceinline__ uint64_t ld_slot(const uint64_t* p) { return __ldcg(p); }

// Scan `k` slots; returns max slot index (lowest index among equal keys) and
// value; sets *dup if the low 31 bits of some slot equal `id`.
__device__ __forceinline__ int scan_row(const uint64_t* row, int k, uint32_t id, uint64_t* vmax,
                                        bool* dup) {
  uint64_t best = 0;
  int m = 0;
  bool d = false;
  if ((k & 1) == 0 && ((reinterpret_cast<uintptr_t>(row) & 15) == 0)) {
    const ulonglong2* r2 = reinterpret_cast<const ulonglong2*>(row);
    for (int j = 0; j < (k >> 1); ++j) {
      ulonglong2 v = __ldcg(r2 + j);
      d |= (((uint32_t)v.x) & 0x7FFFFFFFu) == id;
      d |= (((uint32_t)v.y) & 0x7FFFFFFFu) == id;
      if (j == 0 || v.x > best) { best = v.x; m = 2 * j; }
      if (v.y > best) { best = v.y; m = 2 * j + 1; }
    }
  } else {
    for (int j = 0; j < k; ++j) {
      uint64_t v = ld_slot(row + j);
      d |= (((uint32_t)v) & 0x7FFFFFFFu) == id;
      if (j == 0 || v > best) { best = v; m = j; }
    }
  }
  *vmax = best;
  *dup = d;
  return m;
}

// Returns 1 if inserted.  `key` = (fkey(v) << 32) | lo, lo's low 31 bits = id.
// `thr` (may be null) holds an upper bound of fkey(row max value).
__device__ __forceinline__ int row_push(uint64_t* row, int k, uint32_t* thr, uint64_t key,
                                        unsigned long long* contention) {
  const uint32_t vk = (uint32_t)(key >> 32);
  if (thr != nullptr && vk >= __ldcg(thr)) return 0;
  const uint32_t id = ((uint32_t)key) & 0x7FFFFFFFu;
  for (int attempt = 0; attempt < PUSH_MAX_RETRY; ++attempt) {
    uint64_t vmax;
    bool dup;
    int m = scan_row(row, k, id, &vmax, &dup);
    if (dup) return 0;
    if (vk >= (uint32_t)(vmax >> 32)) {
      if (thr != nullptr) atomicMin(thr, (uint32_t)(vmax >> 32));
      return 0;
    }
    unsigned long long old = atomicCAS(reinterpret_cast<unsigned long long*>(row + m),
                                       (unsigned long long)vmax, (unsigned long long)key);
    if (old == vmax) {
      if (thr != nullptr) {
        // Upper bound of the new row max: snapshot values can only be >= the
        // current ones, so max(snapshot without m, key) bounds the true max.
        uint64_t nm = key;
        for (int j = 0; j < k; ++j)
          if (j != m) {
            uint64_t v = ld_slot(row + j);
            nm = v > nm ? v : nm;
          }
        atomicMin(thr, (uint32_t)(nm >> 32));
      }
      return 1;
    }
  }
  if (contention) atomicAdd(contention, 1ull);
  return 0;
}

}  // namespace rinnd
