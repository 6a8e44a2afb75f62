// noalloc.cu -- concurrent neighbor-row pushes without any device allocation.
//
// Some callers cannot allocate device memory: a host that owns all device
// memory through its own budget (a plugin inside a larger engine), or code
// that must not call cudaMalloc/cudaFree at all.  For them,
// rinnd_heap_push_batch_noalloc performs the same operation as
// rinnd_heap_push_batch -- apply (row, id, distance, flag) pushes concurrently
// to an empty n x k neighbor heap, then sort every row -- with caller-owned
// device inputs/outputs and the heap rows in the file-scope scratch arrays below
// (fixed size, held by every GPU that loads this library until the process exits).
//
// Scratch addresses: in host code the array names are host-side stand-ins, not
// device addresses, so once per device, with that device current, the first
// call looks them up with cudaGetSymbolAddress and caches them; that first call
// on a device should therefore happen before any stream capture.  Every call
// also waits for its stream to finish before it returns, to read its counters
// back.  Every call shares the arrays and clears the rows, bounds and counters it
// uses; calls that overlap on the GPU (other streams, other host threads) race on
// them.  Pushes are validated like rinnd_heap_push_batch's (row in [0, n), id in
// [0, 2^31 - 2)), but on the device: an invalid push makes the call fail after the
// outputs were written from the valid pushes.
#include <mutex>
#include <string>

#include "../../include/rinnd.h"
#include "engine.h"
#include "heap.cuh"

namespace rinnd {
namespace {

constexpr long long NOALLOC_MAX_SLOTS = 1ll << 20;  // 8 MiB of 64-bit row slots
constexpr int NOALLOC_MAX_ROWS = 1 << 16;           // 256 KiB of row bounds
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) uint64_t g_noalloc_slots[NOALLOC_MAX_SLOTS];
static __device__ __align__(256) uint32_t g_noalloc_thr[NOALLOC_MAX_ROWS];
static __device__ __align__(256) unsigned long long g_noalloc_counters[4];  // accepted, contention, invalid

struct ScratchAddrs {
  uint64_t* slots = nullptr;
  uint32_t* thr = nullptr;
  unsigned long long* counters = nullptr;
};
ScratchAddrs g_addrs[NOALLOC_MAX_DEVICES];
std::mutex g_addrs_mu;

ScratchAddrs scratch_for_current_device() {
  int dev = 0;
  RINND_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) throw std::invalid_argument("device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_addrs_mu);
  ScratchAddrs& a = g_addrs[dev];
  if (!a.slots) {
    void* p = nullptr;
    RINND_CUDA(cudaGetSymbolAddress(&p, g_noalloc_slots));
    a.slots = static_cast<uint64_t*>(p);
    RINND_CUDA(cudaGetSymbolAddress(&p, g_noalloc_thr));
    a.thr = static_cast<uint32_t*>(p);
    RINND_CUDA(cudaGetSymbolAddress(&p, g_noalloc_counters));
    a.counters = static_cast<unsigned long long*>(p);
  }
  return a;
}

__global__ void k_noalloc_clear(uint64_t* slots, long long n_slots, uint32_t* thr, int n_rows) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_slots;
       i += (long long)gridDim.x * blockDim.x) {
    slots[i] = SLOT_EMPTY;
    if (i < n_rows) thr[i] = KEY_INF;
  }
}

// Pushes with device-side range checks (inputs are device memory the host cannot
// inspect); the bounds are rinnd_heap_push_batch's: rows in [0, n), ids in
// [0, INT32_MAX - 1).
__global__ void k_noalloc_push(uint64_t* slots, uint32_t* thr, int n, int k, int kp, long long n_ops,
                               const int32_t* rows, const int32_t* ids, const float* dists,
                               const uint8_t* flags, unsigned long long* counters) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n_ops;
       i += (long long)gridDim.x * blockDim.x) {
    int32_t r = rows[i], id = ids[i];
    if (r < 0 || r >= n || id < 0 || id >= 0x7FFFFFFE) {
      atomicAdd(&counters[2], 1ull);
      continue;
    }
    uint64_t key = slot_pack(dists[i], id, flags ? flags[i] : 0);
    if (row_push(slots + (size_t)r * kp, k, thr + r, key, &counters[1])) atomicAdd(&counters[0], 1ull);
  }
}

}  // namespace
}  // namespace rinnd

using namespace rinnd;

extern "C" int rinnd_heap_push_batch_noalloc(int32_t n, int32_t k, int64_t n_ops, const int32_t* d_rows,
                                             const int32_t* d_ids, const float* d_dists, const uint8_t* d_flags,
                                             int32_t* d_out_idx, float* d_out_dist, uint8_t* d_out_flags,
                                             int64_t* n_accepted, void* stream) {
  try {
    if (n < 1 || n > NOALLOC_MAX_ROWS)
      return api_fail(RINND_ERR_INVALID, "n must be in [1, 65536] for the allocation-free push batch");
    if (k < 1 || k > 512) return api_fail(RINND_ERR_INVALID, "k must be in [1, 512]");
    const int kp = row_stride(k);
    if ((long long)n * kp > NOALLOC_MAX_SLOTS)
      return api_fail(RINND_ERR_INVALID,
                      "n * round_up(k, 16) exceeds the 1048576-slot scratch of the allocation-free push batch");
    if (n_ops < 0) return api_fail(RINND_ERR_INVALID, "n_ops must be >= 0");
    if (n_ops > 0 && (!d_rows || !d_ids || !d_dists))
      return api_fail(RINND_ERR_INVALID, "push input pointers must not be null");
    if (!d_out_idx || !d_out_dist) return api_fail(RINND_ERR_INVALID, "output pointers must not be null");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return api_fail(RINND_ERR_NO_DEVICE, "no CUDA device is available: the B200 engine has no CPU fallback");
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    ScratchAddrs s = scratch_for_current_device();
    const long long n_slots = (long long)n * kp;
    k_noalloc_clear<<<grid_for(n_slots, 256, 148 * 8), 256, 0, st>>>(s.slots, n_slots, s.thr, n);
    RINND_LAUNCH_CHECK();
    RINND_CUDA(cudaMemsetAsync(s.counters, 0, 4 * sizeof(unsigned long long), st));
    if (n_ops > 0) {
      k_noalloc_push<<<grid_for(n_ops, 256, 148 * 32), 256, 0, st>>>(s.slots, s.thr, n, k, kp, n_ops, d_rows, d_ids,
                                                                    d_dists, d_flags, s.counters);
      RINND_LAUNCH_CHECK();
    }
    finalize_rows(s.slots, n, k, kp, d_out_idx, d_out_dist, d_out_flags, st);
    unsigned long long h[4] = {0, 0, 0, 0};
    RINND_CUDA(cudaMemcpyAsync(h, s.counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    RINND_CUDA(cudaStreamSynchronize(st));
    if (h[2]) return api_fail(RINND_ERR_INVALID, "push row or id out of range (" + std::to_string(h[2]) + " pushes)");
    if (n_accepted) *n_accepted = (int64_t)h[0];
    return RINND_OK;
  } catch (const std::invalid_argument& e) {
    return api_fail(RINND_ERR_INVALID, e.what());
  } catch (const std::exception& e) {
    return api_fail(RINND_ERR_CUDA, e.what());
  }
}
