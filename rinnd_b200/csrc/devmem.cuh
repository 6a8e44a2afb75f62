// devmem.cuh -- stream-ordered device buffers and CUB temp storage helpers.
#pragma once
#include <cuda_runtime.h>

#include <utility>
#include <vector>

#include "common.cuh"

namespace rinnd {

// Device allocation failures become CudaError; the C ABI maps them to RINND_ERR_OOM.
template <class T>
struct DVec {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = 0;
  DVec() = default;
  DVec(size_t count, cudaStream_t s) { alloc(count, s); }
  DVec(const DVec&) = delete;
  DVec& operator=(const DVec&) = delete;
  DVec(DVec&& o) noexcept : p(o.p), n(o.n), st(o.st) { o.p = nullptr; o.n = 0; }
  DVec& operator=(DVec&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; st = o.st;
      o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DVec() { release(); }
  void alloc(size_t count, cudaStream_t s) {
    release();
    st = s;
    n = count;
    if (count) RINND_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), count * sizeof(T), s));
  }
  // Grow to at least `count` elements preserving the first `keep` elements.
  void grow(size_t count, size_t keep, cudaStream_t s) {
    if (count <= n) return;
    size_t cap = n ? n : 1;
    while (cap < count) cap *= 2;
    T* q = nullptr;
    RINND_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&q), cap * sizeof(T), s));
    if (p && keep) RINND_CUDA(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, s));
    release();
    p = q;
    n = cap;
    st = s;
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    n = 0;
  }
  void fill_bytes(int v) {
    if (n) RINND_CUDA(cudaMemsetAsync(p, v, n * sizeof(T), st));
  }
  void to_host(T* h, size_t count) const {
    if (count) RINND_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, st));
  }
  void from_host(const T* h, size_t count) {
    if (count) RINND_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  T* get() const { return p; }
};

// Reusable CUB temp storage.
struct TempStorage {
  DVec<unsigned char> buf;
  void* ensure(size_t bytes, cudaStream_t s) {
    if (bytes > buf.n) buf.alloc(bytes + (bytes >> 2) + 256, s);
    return buf.p;
  }
};

inline int grid_for(long long n, int block, int cap = 1 << 30) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (int)g;
}

}  // namespace rinnd
