// join_tma.cu -- NN-Descent local join with bulk-copy row gathers (sm_100a).
//
// Same pairs and push semantics as the chunked join in nndescent.cu (the
// reference's update_iteration, core/nndescent/mod.rs:383-446): per vertex,
// new x new (q after p) and new x old (q != p) candidate pairs, each pushed to
// an endpoint's row when it beats that row's threshold.
//
// Persistent CTAs walk a strided vertex sequence through a two-stage shared
// memory pipeline.  Warp 0 prepares the next vertex: it compacts the candidate
// ids, caches their thresholds/norms and issues one cp.async.bulk (TMA engine)
// copy per candidate row (Dp floats) into a padded slot of the free stage,
// completing on that stage's mbarrier; meanwhile every warp computes the current
// vertex from the other stage.  A thread owns (4 A rows) x (1 B row) and
// accumulates 4 distances with 5 shared loads per 4 dimensions; consecutive
// lanes take consecutive B rows (row stride Dp + 4 floats: conflict-free).
// Updates that pass a threshold are appended to the device update buffer
// (one atomic per warp) and applied by k_apply_updates.
//
// Waits are bounded: a stage that does not complete within the poll limit sets
// the error flag, waits (bounded) for the other stage's copies, and the CTA
// leaves; the host turns the flag into an error.
#include "async_copy.cuh"
#include "dist.cuh"
#include "engine.h"
#include "heap.cuh"

namespace rinnd {
namespace {

constexpr uint32_t WAIT_POLLS = 1u << 22;

struct StageHdr {
  int na, nb, v, pad;
};

struct StageLayout {
  int maxc, dp, rs;  // rs = row stride in floats
  __host__ __device__ size_t ids_off() const { return sizeof(StageHdr); }
  __host__ __device__ size_t thr_off() const { return ids_off() + (size_t)2 * maxc * 4; }
  __host__ __device__ size_t nrm_off() const { return thr_off() + (size_t)2 * maxc * 4; }
  __host__ __device__ size_t rows_off() const { return (nrm_off() + (size_t)2 * maxc * 4 + 15) / 16 * 16; }
  __host__ __device__ size_t bytes() const {
    return (rows_off() + (size_t)(2 * maxc + 4) * rs * 4 + 15) / 16 * 16;
  }
};

template <int MAXC>
__device__ __forceinline__ void produce(unsigned char* stage, const StageLayout& L, uint64_t* bar,
                                        const uint64_t* cand_new, const uint64_t* cand_old, int v, int c,
                                        int cp, const float* __restrict__ X, int Dp, const uint32_t* thr,
                                        const float* norms) {
  const int lane = threadIdx.x & 31;
  StageHdr* hdr = reinterpret_cast<StageHdr*>(stage);
  int32_t* ids = reinterpret_cast<int32_t*>(stage + L.ids_off());
  uint32_t* sthr = reinterpret_cast<uint32_t*>(stage + L.thr_off());
  float* snrm = reinterpret_cast<float*>(stage + L.nrm_off());
  float* rows = reinterpret_cast<float*>(stage + L.rows_off());
  int base = 0;
  for (int t0 = 0; t0 < c; t0 += 32) {
    int t = t0 + lane;
    int32_t id = t < c ? slot_id(cand_new[(size_t)v * cp + t]) : -1;
    unsigned m = __ballot_sync(0xffffffffu, id >= 0);
    if (id >= 0) ids[base + __popc(m & ((1u << lane) - 1))] = id;
    base += __popc(m);
  }
  const int na = base;
  if (na > 0) {  // a vertex without new candidates contributes no pairs
    for (int t0 = 0; t0 < c; t0 += 32) {
      int t = t0 + lane;
      int32_t id = t < c ? slot_id(cand_old[(size_t)v * cp + t]) : -1;
      unsigned m = __ballot_sync(0xffffffffu, id >= 0);
      if (id >= 0) ids[base + __popc(m & ((1u << lane) - 1))] = id;
      base += __popc(m);
    }
  }
  const int nb = base;
  __syncwarp();
  for (int r = lane; r < nb; r += 32) {
    int32_t id = ids[r];
    sthr[r] = __ldcg(thr + id);
    if (norms) snrm[r] = norms[id];
  }
  if (lane == 0) {
    hdr->na = na;
    hdr->nb = nb;
    hdr->v = v;
  }
  fence_proxy_async_smem();  // earlier generic reads of this stage before the async writes
  __syncwarp();
  if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)nb * (uint32_t)Dp * 4u);
  __syncwarp();
  for (int r = lane; r < nb; r += 32)
    bulk_g2s(rows + (size_t)r * L.rs, X + (size_t)ids[r] * Dp, (uint32_t)Dp * 4u, bar);
}

template <int MAXC, int NT>
__global__ void __launch_bounds__(NT)
    k_join_tma(const uint64_t* cand_new, const uint64_t* cand_old, int v0, int v1, int c, int cp,
               const float* __restrict__ X, int Dp, int kind, const float* norms, uint64_t* slots,
               uint32_t* thr, int k, int kp, StageLayout L, uint32_t* urow_buf, uint64_t* ukey_buf,
               unsigned long long* ucount, unsigned long long ucap, unsigned long long* counters, int* err) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
  unsigned char* const stage0 = smem + 16;
  const size_t stage_bytes = L.bytes();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool is_dot = kind_is_dot(kind);
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const int first = v0 + blockIdx.x;
  if (first >= v1) return;
  if (warp == 0)
    produce<MAXC>(stage0, L, &bars[0], cand_new, cand_old, first, c, cp, X, Dp, thr, is_dot ? norms : nullptr);
  unsigned int pairs_total = 0, rows_total = 0;
  for (int it = 0;; ++it) {
    const int v = first + it * gridDim.x;
    if (v >= v1) break;
    const int s = it & 1;
    const int vn = v + gridDim.x;
    if (warp == 0 && vn < v1)
      produce<MAXC>(stage0 + (size_t)(s ^ 1) * stage_bytes, L, &bars[s ^ 1], cand_new, cand_old, vn, c, cp, X, Dp, thr,
                    is_dot ? norms : nullptr);
    const uint32_t parity = (uint32_t)(it >> 1) & 1u;
    bool ok = true;
    if (tid == 0) ok = mbar_wait_bounded(&bars[s], parity, WAIT_POLLS);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicExch(err, 1);
        if (vn < v1) mbar_wait_bounded(&bars[s ^ 1], parity ^ ((s ^ 1) < s ? 1u : 0u), WAIT_POLLS);
      }
      return;
    }
    mbar_try_wait(&bars[s], parity);  // acquire the completed phase in every thread
    unsigned char* st = stage0 + (size_t)s * stage_bytes;
    const StageHdr hdr = *reinterpret_cast<const StageHdr*>(st);
    const int32_t* ids = reinterpret_cast<const int32_t*>(st + L.ids_off());
    const uint32_t* sthr = reinterpret_cast<const uint32_t*>(st + L.thr_off());
    const float* snrm = reinterpret_cast<const float*>(st + L.nrm_off());
    const float* rows = reinterpret_cast<const float*>(st + L.rows_off());
    const int na = hdr.na, nb = hdr.nb;
    const int nq = (na + 3) >> 2;
    const int items = nq * nb;
    for (int b0 = 0; b0 < items; b0 += NT) {
      const int item = b0 + tid;
      const bool active = item < items;
      int iq = 0, j = 0;
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      if (active) {
        iq = item / nb;
        j = item - iq * nb;
        const float4* pb = reinterpret_cast<const float4*>(rows + (size_t)j * L.rs);
        const float4* pa = reinterpret_cast<const float4*>(rows + (size_t)(4 * iq) * L.rs);
        const int ars = L.rs / 4;
        if (kind == DK_SQEUCLIDEAN) {
#pragma unroll 4
          for (int q = 0; q < Dp / 4; ++q) {
            float4 b = pb[q];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              float4 a = pa[u * ars + q];
              float d0 = a.x - b.x, d1 = a.y - b.y, d2 = a.z - b.z, d3 = a.w - b.w;
              acc[u] = fmaf(d0, d0, acc[u]);
              acc[u] = fmaf(d1, d1, acc[u]);
              acc[u] = fmaf(d2, d2, acc[u]);
              acc[u] = fmaf(d3, d3, acc[u]);
            }
          }
        } else if (kind == DK_MANHATTAN) {
#pragma unroll 4
          for (int q = 0; q < Dp / 4; ++q) {
            float4 b = pb[q];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              float4 a = pa[u * ars + q];
              acc[u] += fabsf(a.x - b.x) + fabsf(a.y - b.y) + fabsf(a.z - b.z) + fabsf(a.w - b.w);
            }
          }
        } else {
#pragma unroll 4
          for (int q = 0; q < Dp / 4; ++q) {
            float4 b = pb[q];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              float4 a = pa[u * ars + q];
              acc[u] = fmaf(a.x, b.x, acc[u]);
              acc[u] = fmaf(a.y, b.y, acc[u]);
              acc[u] = fmaf(a.z, b.z, acc[u]);
              acc[u] = fmaf(a.w, b.w, acc[u]);
            }
          }
        }
      }
      // validity, thresholds -> emit masks (bit u: push to row of A[4iq+u]; bit 4+u: to B[j])
      uint32_t kd[4];
      unsigned emit = 0;
      int n_emit = 0;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        kd[u] = 0;
        const int i = 4 * iq + u;
        if (active && i < na) {
          bool valid = (j < na) ? (j > i) : (ids[j] != ids[i]);  // mod.rs:396, :424
          if (valid) {
            ++pairs_total;
            float d = acc[u];
            if (is_dot) d = finalize_dot(kind, d, snrm[i], snrm[j]);
            kd[u] = fkey(d);
            if (kd[u] < sthr[i]) { emit |= 1u << u; ++n_emit; }
            if (kd[u] < sthr[j]) { emit |= 16u << u; ++n_emit; }
          }
        }
      }
      int incl = n_emit;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
      }
      const int warp_total = __shfl_sync(0xffffffffu, incl, 31);
      unsigned long long base = 0;
      if (lane == 0 && warp_total) base = atomicAdd(ucount, (unsigned long long)warp_total);
      base = __shfl_sync(0xffffffffu, base, 0) + (unsigned long long)(incl - n_emit);
      if (emit) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = 4 * iq + u;
#pragma unroll
          for (int side = 0; side < 2; ++side) {
            if (!(emit & ((side ? 16u : 1u) << u))) continue;
            const int32_t row = side ? ids[j] : ids[i];
            const int32_t other = side ? ids[i] : ids[j];
            const uint64_t key = ((uint64_t)kd[u] << 32) | (uint32_t)other | 0x80000000u;
            if (base < ucap) {
              urow_buf[base] = (uint32_t)row;
              ukey_buf[base] = key;
            } else if (row_push(slots + (size_t)row * kp, k, thr + row, key, &counters[1])) {
              atomicAdd(&counters[0], 1ull);
            }
            ++base;
          }
        }
      }
    }
    if (tid == 0) rows_total += nb;
    __syncthreads();  // stage s fully consumed before warp 0 refills it
  }
  for (int o = 16; o; o >>= 1) pairs_total += __shfl_xor_sync(0xffffffffu, pairs_total, o);
  if (lane == 0 && pairs_total) atomicAdd(&counters[2], (unsigned long long)pairs_total);
  if (tid == 0 && rows_total) atomicAdd(&counters[3], (unsigned long long)rows_total);
}

template <int MAXC, int NT>
void launch_join(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, cudaStream_t st,
                 const StageLayout& L, int* err) {
  size_t smem = 16 + 2 * L.bytes();
  static bool attr[2] = {false, false};
  bool& done = attr[MAXC == 64];
  if (!done) {
    RINND_CUDA(cudaFuncSetAttribute(k_join_tma<MAXC, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    done = true;
  }
  int per_sm = std::max(1, (int)((220 * 1024) / smem));
  int grid = std::min(v1 - v0, 148 * per_sm);
  if (grid <= 0) return;
  k_join_tma<MAXC, NT><<<grid, NT, smem, st>>>(s.cand_new.p, s.cand_old.p, v0, v1, s.c, s.cp, X, Dp, kind,
                                               s.norms.p, s.slots.p, s.thr.p, s.k, s.kp, L, s.urow.p, s.ukey.p,
                                               s.counters.p + 4, s.ucap, s.counters.p, err);
  RINND_LAUNCH_CHECK();
}

}  // namespace

bool join_tma_supported(int c, int Dp) {
  StageLayout L{c <= 32 ? 32 : 64, Dp, Dp + 4};
  return 16 + 2 * L.bytes() <= 200 * 1024;
}

void join_tma_batch(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, int* err, cudaStream_t st) {
  if (s.c <= 32) launch_join<32, 128>(s, X, Dp, kind, v0, v1, st, StageLayout{32, Dp, Dp + 4}, err);
  else launch_join<64, 256>(s, X, Dp, kind, v0, v1, st, StageLayout{64, Dp, Dp + 4}, err);
}

}  // namespace rinnd
