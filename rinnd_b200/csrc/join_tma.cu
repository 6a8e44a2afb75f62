// join_tma.cu -- warp-specialized NN-Descent local join with bulk-copy gathers (sm_100a).
//
// Same pairs and push semantics as the chunked join in nndescent.cu (the
// reference's update_iteration, core/nndescent/mod.rs:383-446): per vertex,
// new x new (q after p) and new x old (q != p) candidate pairs, each pushed to
// an endpoint's row when it beats that row's threshold.
//
// Work decomposition.  A prepass (k_cand_describe) writes one descriptor per
// vertex: counts, the compacted candidate ids (new first), their norms, and a
// prefix table of the work items.  An item is (4 consecutive new
// rows) x (1 candidate row j); items entirely on or below the new x new
// diagonal are never generated.  Persistent CTAs of 1 producer warp + 8
// consumer warps walk a strided vertex sequence:
//   producer: keeps NDESC descriptors in flight (one cp.async.bulk each into a
//     ring, completing on per-slot mbarriers) and loads the next vertex's
//     candidate ids and current row thresholds one vertex ahead; a vertex with
//     pairs takes the next free row stage (empty mbarrier, armed by the
//     consumer warps): the producer copies the descriptor and the thresholds
//     into the stage and issues one cp.async.bulk per candidate row (Dp floats)
//     into a padded slot, completing on the stage's full mbarrier.  Vertices
//     without pairs take no stage; a stage with nb = -1 ends the work;
//   consumers: wait for the stage; each thread computes one item per round --
//     4 distances with packed FP32x2 arithmetic from 5 conflict-free 16-byte
//     shared loads per 4 dimensions -- and appends threshold-passing updates to
//     its CTA's region of the device update buffer (one shared-memory atomic
//     per warp and round; an update beyond the region is pushed directly) for
//     k_apply_regions.
// Every wait is bounded.  A wait that runs out sets the device error flag and a
// shared abort flag; all warps leave, the producer first waiting (bounded) for
// every copy it issued.  The host turns the flag into an error.
#include <map>
#include <mutex>
#include <tuple>

#include "engine.h"
#include "join_common.cuh"

namespace rinnd {
namespace {

using namespace joinc;

// Tile shape (JoinTile, chosen per build by join_tune): NSTAGE row stages in
// flight per CTA (pipeline depth), JB candidate rows per work item (each
// against 4 new rows), and the CTAs launched per SM.
constexpr int NCONS = 8;    // consumer warps
constexpr int NT = 32 * (1 + NCONS);

struct Layout {
  int maxc, dp, rs, dstride;  // rs: row stride (floats); dstride: descriptor stride (ints)
  int ns;                     // row stages (the kernel's NSTAGE)
  __host__ __device__ size_t bar_bytes() const { return 8 * (2 * ns + NDESC) + 16; }
  __host__ __device__ size_t desc_off() const { return (bar_bytes() + 15) / 16 * 16; }
  __host__ __device__ size_t stage_off() const { return desc_off() + (size_t)NDESC * dstride * 4; }
  __host__ __device__ size_t rows_off() const { return (size_t)dstride * 4; }  // within a stage
  // rows read: B rows j < nb and A quads up to row na + 3 <= 2 * maxc - 1
  __host__ __device__ size_t stage_bytes() const { return rows_off() + (size_t)(2 * maxc) * rs * 4; }
  __host__ __device__ size_t bytes() const { return stage_off() + ns * stage_bytes(); }
};

Layout make_layout(int c, int Dp, int ns = 2) {
  const int maxc = c <= 32 ? 32 : 64;
  return Layout{maxc, Dp, Dp + 4, Desc::stride(maxc), ns};
}

__global__ void k_cand_describe(const uint64_t* cand_new, const uint64_t* cand_old, int N, int c, int cp, int maxc,
                                int dstride, int JB, const float* norms, int32_t* desc) {
  const int v = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (v >= N) return;
  int32_t* d = desc + (size_t)v * dstride;
  int32_t* ids = d + Desc::ids(maxc);
  int base = 0;
  for (int t0 = 0; t0 < c; t0 += 32) {
    int t = t0 + lane;
    int32_t id = t < c ? slot_id(cand_new[(size_t)v * cp + t]) : -1;
    unsigned m = __ballot_sync(0xffffffffu, id >= 0);
    if (id >= 0) ids[base + __popc(m & ((1u << lane) - 1))] = id;
    base += __popc(m);
  }
  const int na = base;
  if (na > 0)  // a vertex without new candidates contributes no pairs
    for (int t0 = 0; t0 < c; t0 += 32) {
      int t = t0 + lane;
      int32_t id = t < c ? slot_id(cand_old[(size_t)v * cp + t]) : -1;
      unsigned m = __ballot_sync(0xffffffffu, id >= 0);
      if (id >= 0) ids[base + __popc(m & ((1u << lane) - 1))] = id;
      base += __popc(m);
    }
  const int nb = base;
  __syncwarp();
  if (norms)
    for (int r = lane; r < nb; r += 32) reinterpret_cast<float*>(d)[Desc::nrm(maxc) + r] = norms[ids[r]];
  // items of quad iq: JB consecutive candidate rows each, starting at row 4 iq + 1
  const int nq = (na + 3) >> 2;
  int cnt = (lane < nq) ? (max(0, nb - (4 * lane + 1)) + JB - 1) / JB : 0;
  int incl = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  if (lane < NQMAX) d[4 + lane] = incl - cnt;
  if (lane == 0) {
    d[0] = na;
    d[1] = nb;
    d[2] = nq;
    d[3] = total;
  }
}

struct Bars {
  uint64_t* full;   // [NSTAGE]
  uint64_t* empty;  // [NSTAGE]
  uint64_t* desc;   // [NDESC]
  int* abort_flag;
};

// GROUPED: rows of several indices (per-index accounting of direct pushes).
// (No minimum-blocks bound: asking for 3 CTAs per SM gave the same 72
// registers but a 20 % slower one-row tile on the 1M build.)
template <int MAXC, bool GROUPED, int NSTAGE, int JB>
__global__ void __launch_bounds__(NT)
    k_join_ws(const int32_t* __restrict__ desc, int v0, int v1, const float* __restrict__ X, int Dp, int kind,
              uint64_t* slots, uint32_t* thr, int k, int kp, Layout L, uint32_t* urow_buf, uint64_t* ukey_buf,
              unsigned long long* ucount, uint32_t* rcnt, unsigned int rsize, unsigned long long* counters,
              int* err, ItemCount ic) {
  extern __shared__ __align__(16) unsigned char smem[];
  Bars B{reinterpret_cast<uint64_t*>(smem), reinterpret_cast<uint64_t*>(smem) + NSTAGE,
         reinterpret_cast<uint64_t*>(smem) + 2 * NSTAGE,
         reinterpret_cast<int*>(smem + 8 * (2 * NSTAGE + NDESC))};
  // this CTA's region of the update buffer and its fill count (shared memory)
  unsigned int* s_ucnt = reinterpret_cast<unsigned int*>(B.abort_flag + 1);
  unsigned int* s_done = s_ucnt + 1;  // consumer warps finished
  uint32_t* urow_reg = urow_buf + (size_t)blockIdx.x * rsize;
  uint64_t* ukey_reg = ukey_buf + (size_t)blockIdx.x * rsize;
  // (offsets with the stage count as a constant; the launch's L.ns is NSTAGE)
  constexpr size_t kDescOff = (8 * (2 * NSTAGE + NDESC) + 16 + 15) / 16 * 16;
  int32_t* dring = reinterpret_cast<int32_t*>(smem + kDescOff);
  unsigned char* stage0 = smem + kDescOff + (size_t)NDESC * L.dstride * 4;
  const size_t sbytes = L.stage_bytes();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&B.full[s], 1);
      mbar_init(&B.empty[s], NCONS);
    }
    for (int s = 0; s < NDESC; ++s) mbar_init(&B.desc[s], 1);
    *B.abort_flag = 0;
    *s_ucnt = 0;
    *s_done = 0;
    fence_mbar_init();
  }
  __syncthreads();
  const int first = v0 + (int)blockIdx.x;
  if (first >= v1) return;
  const int stride = gridDim.x;
  const int nv = (v1 - first + stride - 1) / stride;  // vertices of this CTA
  volatile int* abort_flag = B.abort_flag;
  const int dstride = L.dstride;

  if (warp == 0) {
    // ------------------------------ producer ------------------------------
    const uint32_t dbytes = (uint32_t)dstride * 4u;
    if (lane == 0)
      for (int i = 0; i < NDESC && i < nv; ++i) {
        mbar_arrive_expect_tx(&B.desc[i], dbytes);
        bulk_g2s(dring + (size_t)i * dstride, desc + (size_t)(first + i * stride) * dstride, dbytes, &B.desc[i]);
      }
    constexpr int TPL = (2 * MAXC + 31) / 32;  // candidate rows per lane
    bool ok = true;
    int i = 0, jobs = 0;                        // vertices walked, stages filled
    int desc_issued = nv < NDESC ? nv : NDESC;  // descriptors issued for vertices [0, desc_issued)
    // Candidate ids and current row thresholds of the next vertex, loaded one
    // vertex ahead so the threshold loads overlap the previous vertex's copies.
    int32_t nx_ids[TPL];
    uint32_t nx_thr[TPL];
    auto prefetch = [&](int v) {
      const bool got = wait_or_abort(&B.desc[v % NDESC], (uint32_t)(v / NDESC) & 1u, abort_flag);
      const int32_t* dn = dring + (size_t)(v % NDESC) * dstride;
      const int nbn = got ? dn[1] : 0;
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        const int r = lane + 32 * t;
        nx_ids[t] = r < nbn ? dn[Desc::ids(MAXC) + r] : 0;
        nx_thr[t] = r < nbn ? __ldcg(thr + nx_ids[t]) : 0u;
      }
      return got;
    };
    if (nv > 0) ok = prefetch(0);
    for (; ok && i < nv; ++i) {
      const int ds = i % NDESC;
      int32_t my_ids[TPL];
      uint32_t my_thr[TPL];
#pragma unroll
      for (int t = 0; t < TPL; ++t) {
        my_ids[t] = nx_ids[t];
        my_thr[t] = nx_thr[t];
      }
      if (i + 1 < nv) {
        ok = prefetch(i + 1);
        if (!ok) break;
      }
      const int32_t* dsc = dring + (size_t)ds * dstride;
      const int nb = dsc[1], items = dsc[3];
      if (items > 0) {  // vertices without pairs take no stage
        const int s = jobs % NSTAGE;
        if (jobs >= NSTAGE) {
          ok = wait_or_abort(&B.empty[s], (uint32_t)((jobs / NSTAGE) - 1) & 1u, abort_flag);
          if (!ok) break;
        }
        unsigned char* st = stage0 + (size_t)s * sbytes;
        int32_t* sd = reinterpret_cast<int32_t*>(st);
        for (int t = lane; t < dstride; t += 32)  // descriptor -> stage header (thresholds below)
          if (t < Desc::thr(MAXC) || t >= Desc::nrm(MAXC)) sd[t] = dsc[t];
        uint32_t* sthr = reinterpret_cast<uint32_t*>(sd + Desc::thr(MAXC));
#pragma unroll
        for (int t = 0; t < TPL; ++t) {
          const int r = lane + 32 * t;
          if (r < nb) sthr[r] = my_thr[t];
        }
        float* rows = reinterpret_cast<float*>(st + L.rows_off());
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(&B.full[s], (uint32_t)nb * (uint32_t)Dp * 4u);
        __syncwarp();
#pragma unroll
        for (int t = 0; t < TPL; ++t) {
          const int r = lane + 32 * t;
          if (r < nb) bulk_g2s(rows + (size_t)r * L.rs, X + (size_t)my_ids[t] * Dp, (uint32_t)Dp * 4u, &B.full[s]);
        }
        ++jobs;
      }
      // descriptor slot consumed: refill it NDESC vertices ahead
      fence_proxy_async_smem();
      __syncwarp();
      if (i + NDESC < nv) {
        desc_issued = i + NDESC + 1;
        if (lane == 0) {
          mbar_arrive_expect_tx(&B.desc[ds], dbytes);
          bulk_g2s(dring + (size_t)ds * dstride, desc + (size_t)(first + (i + NDESC) * stride) * dstride, dbytes,
                   &B.desc[ds]);
        }
      }
    }
    if (ok) {  // end-of-work stage (nb = -1)
      const int s = jobs % NSTAGE;
      if (jobs >= NSTAGE) ok = wait_or_abort(&B.empty[s], (uint32_t)((jobs / NSTAGE) - 1) & 1u, abort_flag);
      if (ok && lane == 0) {
        reinterpret_cast<int32_t*>(stage0 + (size_t)s * sbytes)[1] = -1;
        mbar_arrive(&B.full[s]);
      }
    }
    if (!ok && lane == 0) {
      *abort_flag = 1;
      atomicExch(err, 1);
      // drain: wait (bounded) for every descriptor and row copy this warp issued
      for (int j = i; j < desc_issued; ++j)
        mbar_wait_bounded(&B.desc[j % NDESC], (uint32_t)(j / NDESC) & 1u, WAIT_POLLS);
      for (int j = (jobs > NSTAGE ? jobs - NSTAGE : 0); j < jobs; ++j)
        mbar_wait_bounded(&B.full[j % NSTAGE], (uint32_t)(j / NSTAGE) & 1u, WAIT_POLLS);
    }
    return;
  }

  // ------------------------------ consumers ------------------------------
  const int ct = tid - 32;
  const bool is_dot = kind_is_dot(kind);
  unsigned int pairs_total = 0;
  unsigned long long rows_total = 0;
  for (int i = 0;; ++i) {  // stages in fill order, up to the end-of-work stage
    const int s = i % NSTAGE;
    if (!__all_sync(0xffffffffu, wait_or_abort(&B.full[s], (uint32_t)(i / NSTAGE) & 1u, abort_flag))) {
      if (lane == 0) {
        *abort_flag = 1;
        atomicExch(err, 1);
      }
      return;
    }
    const unsigned char* st = stage0 + (size_t)s * sbytes;
    const int32_t* sd = reinterpret_cast<const int32_t*>(st);
    const int na = sd[0], nb = sd[1], nq = sd[2], items = sd[3];
    if (nb < 0) break;
    const int32_t* ids = sd + Desc::ids(MAXC);
    const uint32_t* sthr = reinterpret_cast<const uint32_t*>(sd + Desc::thr(MAXC));
    const float* snrm = reinterpret_cast<const float*>(sd + Desc::nrm(MAXC));
    const float* rows = reinterpret_cast<const float*>(st + L.rows_off());
    if (ct == 0) rows_total += (unsigned long long)nb;
    if constexpr (JB == 1) {  // one candidate row per item
      for (int b0 = 0; b0 < items; b0 += 32 * NCONS) {
        const int item = b0 + ct;
        const bool active = item < items;
        int iq = 0, j = 0;
        unsigned long long acc[4] = {0ull, 0ull, 0ull, 0ull};
        if (active) {
          for (int q = 1; q < nq; ++q) iq += (sd[4 + q] <= item);
          j = 4 * iq + 1 + (item - sd[4 + iq]);
          const ulonglong2* pb = reinterpret_cast<const ulonglong2*>(rows + (size_t)j * L.rs);
          const ulonglong2* pa = reinterpret_cast<const ulonglong2*>(rows + (size_t)(4 * iq) * L.rs);
          const int ars = L.rs / 4;
          if (kind == DK_SQEUCLIDEAN) {
  #pragma unroll 4
            for (int q = 0; q < Dp / 4; ++q) {
              const ulonglong2 b = pb[q];
  #pragma unroll
              for (int u = 0; u < 4; ++u) {
                const ulonglong2 a = pa[u * ars + q];
                const unsigned long long d01 = f2_sub(a.x, b.x), d23 = f2_sub(a.y, b.y);
                acc[u] = f2_fma(d01, d01, acc[u]);
                acc[u] = f2_fma(d23, d23, acc[u]);
              }
            }
          } else if (kind == DK_MANHATTAN) {
            const unsigned long long absmask = 0x7FFFFFFF7FFFFFFFull;
  #pragma unroll 4
            for (int q = 0; q < Dp / 4; ++q) {
              const ulonglong2 b = pb[q];
  #pragma unroll
              for (int u = 0; u < 4; ++u) {
                const ulonglong2 a = pa[u * ars + q];
                acc[u] = f2_add(acc[u], f2_sub(a.x, b.x) & absmask);
                acc[u] = f2_add(acc[u], f2_sub(a.y, b.y) & absmask);
              }
            }
          } else {
  #pragma unroll 4
            for (int q = 0; q < Dp / 4; ++q) {
              const ulonglong2 b = pb[q];
  #pragma unroll
              for (int u = 0; u < 4; ++u) {
                const ulonglong2 a = pa[u * ars + q];
                acc[u] = f2_fma(a.x, b.x, acc[u]);
                acc[u] = f2_fma(a.y, b.y, acc[u]);
              }
            }
          }
        }
        // validity and thresholds -> emit bits (u: push into A row; 4+u: into B row)
        uint32_t kd[4];
        unsigned emit = 0;
        int n_emit = 0;
        const int32_t bid = active ? ids[j] : -1;
        const uint32_t bthr = active ? sthr[j] : 0u;
  #pragma unroll
        for (int u = 0; u < 4; ++u) {
          kd[u] = 0;
          const int ia = 4 * iq + u;
          if (active && ia < na) {
            const bool valid = (j < na) ? (j > ia) : (bid != ids[ia]);  // mod.rs:396, :424
            if (valid) {
              ++pairs_total;
              float d = f2_sum(acc[u]);
              if (is_dot) d = finalize_dot(kind, d, snrm[ia], snrm[j]);
              kd[u] = fkey(d);
              if (kd[u] < sthr[ia]) { emit |= 1u << u; ++n_emit; }
              if (kd[u] < bthr) { emit |= 16u << u; ++n_emit; }
            }
          }
        }
        int incl = n_emit;
  #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        const int warp_total = __shfl_sync(0xffffffffu, incl, 31);
        unsigned int base = 0;
        if (lane == 0 && warp_total) base = atomicAdd(s_ucnt, (unsigned int)warp_total);
        base = __shfl_sync(0xffffffffu, base, 0) + (unsigned int)(incl - n_emit);
        if (emit) {
  #pragma unroll
          for (int u = 0; u < 4; ++u) {
  #pragma unroll
            for (int side = 0; side < 2; ++side) {
              if (!(emit & ((side ? 16u : 1u) << u))) continue;
              const int32_t aid = ids[4 * iq + u];
              const int32_t row = side ? bid : aid;
              const int32_t other = side ? aid : bid;
              const uint64_t key = ((uint64_t)kd[u] << 32) | (uint32_t)other | 0x80000000u;
              if (base < rsize) {
                urow_reg[base] = (uint32_t)row;
                ukey_reg[base] = key;
              } else if (row_push_hi_first(slots + (size_t)row * kp, k, thr + row, key, &counters[1])) {
                atomicAdd(&counters[0], 1ull);
                if constexpr (GROUPED) ic.add((uint32_t)row);
              }
              ++base;
            }
          }
        }
      }
    } else {  // JB candidate rows per item
      for (int b0 = 0; b0 < items; b0 += 32 * NCONS) {
        const int item = b0 + ct;
        const bool active = item < items;
        int iq = 0, j = 0;
        unsigned long long acc[4 * JB];
  #pragma unroll
        for (int p = 0; p < 4 * JB; ++p) acc[p] = 0ull;
        if (active) {
          for (int q = 1; q < nq; ++q) iq += (sd[4 + q] <= item);
          j = 4 * iq + 1 + JB * (item - sd[4 + iq]);
          // candidate rows j .. j + JB - 1 (a row past nb repeats row nb - 1; its results are discarded)
          const ulonglong2* pb[JB];
  #pragma unroll
          for (int v = 0; v < JB; ++v)
            pb[v] = reinterpret_cast<const ulonglong2*>(rows + (size_t)min(j + v, nb - 1) * L.rs);
          const ulonglong2* pa = reinterpret_cast<const ulonglong2*>(rows + (size_t)(4 * iq) * L.rs);
          const int ars = L.rs / 4;
          if (kind == DK_SQEUCLIDEAN) {
  #pragma unroll(JB == 1 ? 4 : 2)
            for (int q = 0; q < Dp / 4; ++q) {
              ulonglong2 b[JB];
  #pragma unroll
              for (int v = 0; v < JB; ++v) b[v] = pb[v][q];
  #pragma unroll
              for (int u = 0; u < 4; ++u) {
                const ulonglong2 a = pa[u * ars + q];
  #pragma unroll
                for (int v = 0; v < JB; ++v) {
                  const unsigned long long d01 = f2_sub(a.x, b[v].x), d23 = f2_sub(a.y, b[v].y);
                  acc[4 * v + u] = f2_fma(d01, d01, acc[4 * v + u]);
                  acc[4 * v + u] = f2_fma(d23, d23, acc[4 * v + u]);
                }
              }
            }
          } else if (kind == DK_MANHATTAN) {
            const unsigned long long absmask = 0x7FFFFFFF7FFFFFFFull;
  #pragma unroll(JB == 1 ? 4 : 2)
            for (int q = 0; q < Dp / 4; ++q) {
              ulonglong2 b[JB];
  #pragma unroll
              for (int v = 0; v < JB; ++v) b[v] = pb[v][q];
  #pragma unroll
              for (int u = 0; u < 4; ++u) {
                const ulonglong2 a = pa[u * ars + q];
  #pragma unroll
                for (int v = 0; v < JB; ++v) {
                  acc[4 * v + u] = f2_add(acc[4 * v + u], f2_sub(a.x, b[v].x) & absmask);
                  acc[4 * v + u] = f2_add(acc[4 * v + u], f2_sub(a.y, b[v].y) & absmask);
                }
              }
            }
          } else {
  #pragma unroll(JB == 1 ? 4 : 2)
            for (int q = 0; q < Dp / 4; ++q) {
              ulonglong2 b[JB];
  #pragma unroll
              for (int v = 0; v < JB; ++v) b[v] = pb[v][q];
  #pragma unroll
              for (int u = 0; u < 4; ++u) {
                const ulonglong2 a = pa[u * ars + q];
  #pragma unroll
                for (int v = 0; v < JB; ++v) {
                  acc[4 * v + u] = f2_fma(a.x, b[v].x, acc[4 * v + u]);
                  acc[4 * v + u] = f2_fma(a.y, b[v].y, acc[4 * v + u]);
                }
              }
            }
          }
        }
        // validity and thresholds -> emit bits (bit p = 4 v + u: push into A row; 16 + p: into B row)
        uint32_t kd[4 * JB];
        unsigned emit = 0;
        int n_emit = 0;
  #pragma unroll
        for (int v = 0; v < JB; ++v) {
          const int jv = j + v;
          const bool have = active && jv < nb;
          const int32_t bid = have ? ids[jv] : -1;
          const uint32_t bthr = have ? sthr[jv] : 0u;
  #pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int p = 4 * v + u;
            kd[p] = 0;
            const int ia = 4 * iq + u;
            if (have && ia < na) {
              const bool valid = (jv < na) ? (jv > ia) : (bid != ids[ia]);  // mod.rs:396, :424
              if (valid) {
                ++pairs_total;
                float d = f2_sum(acc[p]);
                if (is_dot) d = finalize_dot(kind, d, snrm[ia], snrm[jv]);
                kd[p] = fkey(d);
                if (kd[p] < sthr[ia]) { emit |= 1u << p; ++n_emit; }
                if (kd[p] < bthr) { emit |= 0x10000u << p; ++n_emit; }
              }
            }
          }
        }
        int incl = n_emit;
  #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        const int warp_total = __shfl_sync(0xffffffffu, incl, 31);
        unsigned int base = 0;
        if (lane == 0 && warp_total) base = atomicAdd(s_ucnt, (unsigned int)warp_total);
        base = __shfl_sync(0xffffffffu, base, 0) + (unsigned int)(incl - n_emit);
        if (emit) {
  #pragma unroll
          for (int p = 0; p < 4 * JB; ++p) {
  #pragma unroll
            for (int side = 0; side < 2; ++side) {
              if (!(emit & ((side ? 0x10000u : 1u) << p))) continue;
              const int32_t aid = ids[4 * iq + (p & 3)];
              const int32_t bid = ids[j + (p >> 2)];
              const int32_t row = side ? bid : aid;
              const int32_t other = side ? aid : bid;
              const uint64_t key = ((uint64_t)kd[p] << 32) | (uint32_t)other | 0x80000000u;
              if (base < rsize) {
                urow_reg[base] = (uint32_t)row;
                ukey_reg[base] = key;
              } else if (row_push_hi_first(slots + (size_t)row * kp, k, thr + row, key, &counters[1])) {
                atomicAdd(&counters[0], 1ull);
                if constexpr (GROUPED) ic.add((uint32_t)row);
              }
              ++base;
            }
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&B.empty[s]);  // this warp is done with stage s
  }
  // The last consumer warp to finish publishes the region's fill count (capped
  // at the region size; the rest were pushed directly) and adds the CTA's
  // appended updates to the launch total.  An aborted CTA publishes nothing:
  // its region count stays 0.
  __syncwarp();
  if (lane == 0) {
    __threadfence_block();
    if (atomicAdd(s_done, 1u) == NCONS - 1) {
      const unsigned int total = atomicAdd(s_ucnt, 0u);
      rcnt[blockIdx.x] = total < rsize ? total : rsize;
      atomicAdd(ucount, (unsigned long long)total);
    }
  }
  for (int o = 16; o; o >>= 1) pairs_total += __shfl_xor_sync(0xffffffffu, pairs_total, o);
  if (lane == 0 && pairs_total) atomicAdd(&counters[2], (unsigned long long)pairs_total);
  if (ct == 0 && rows_total) atomicAdd(&counters[3], rows_total);
}

using JoinKernel = void (*)(const int32_t*, int, int, const float*, int, int, uint64_t*, uint32_t*, int, int, Layout,
                           uint32_t*, uint64_t*, unsigned long long*, uint32_t*, unsigned int, unsigned long long*, int*,
                           ItemCount);

// The tile shapes the tuner chooses among (candidate lists of <= 32; longer
// lists run the default shape).
template <int MAXC, bool G>
JoinKernel pick_kernel(int ns, int jb) {
  if constexpr (MAXC == 32) {
    if (ns == 3) return jb == 1 ? k_join_ws<MAXC, G, 3, 1> : k_join_ws<MAXC, G, 3, 2>;
    return jb == 1 ? k_join_ws<MAXC, G, 2, 1> : k_join_ws<MAXC, G, 2, 2>;
  } else {
    (void)ns;
    (void)jb;
    return k_join_ws<MAXC, G, 2, 1>;
  }
}

JoinTile effective_tile(const KnnState& s) {
  JoinTile t = s.tile;
  if (t.nstage != 2 && t.nstage != 3) t.nstage = 2;
  if (t.jb != 1 && t.jb != 2) t.jb = 1;
  if (s.c > 32) {  // one shape for long lists
    t.nstage = 2;
    t.jb = 1;
  }
  return t;
}

JoinKernel join_kernel(const KnnState& s, const JoinTile& t) {
  const bool grouped = s.item_changes.p != nullptr;
  if (s.c <= 32) return grouped ? pick_kernel<32, true>(t.nstage, t.jb) : pick_kernel<32, false>(t.nstage, t.jb);
  return grouped ? pick_kernel<64, true>(t.nstage, t.jb) : pick_kernel<64, false>(t.nstage, t.jb);
}

void launch_join(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, cudaStream_t st, int* err) {
  const JoinTile t = effective_tile(s);
  const Layout L = make_layout(s.c, Dp, t.nstage);
  const size_t smem = L.bytes();
  JoinKernel kern = join_kernel(s, t);
  set_smem_limit_once(reinterpret_cast<const void*>(kern), 227 * 1024);
  int per_sm = std::max(1, (int)((227 * 1024) / (smem + 1024)));
  if (t.per_sm > 0) per_sm = std::min(per_sm, t.per_sm);
  const int grid = std::min(v1 - v0, 148 * per_sm);
  if (grid <= 0) return;
  // one region of the update buffer per CTA (k_apply_regions reads them back)
  if (s.rcnt.n < (size_t)grid) s.rcnt.alloc((size_t)grid, st);
  RINND_CUDA(cudaMemsetAsync(s.rcnt.p, 0, sizeof(uint32_t) * grid, st));
  s.nreg = grid;
  s.rsize = (unsigned int)std::min<unsigned long long>(s.ucap / (unsigned long long)grid, 0xFFFFFFFFull);
  kern<<<grid, NT, smem, st>>>(s.desc.p, v0, v1, X, Dp, kind, s.slots.p, s.thr.p, s.k, s.kp, L, s.urow.p, s.ukey.p,
                               s.counters.p + 4, s.rcnt.p, s.rsize, s.counters.p, err, s.item_count());
  RINND_LAUNCH_CHECK();
}

}  // namespace

bool join_tma_supported(int c, int Dp) { return make_layout(c, Dp, 2).bytes() <= 220 * 1024; }
bool join_tile_fits(int c, int Dp, const JoinTile& t) { return make_layout(c, Dp, t.nstage).bytes() <= 220 * 1024; }

void join_describe_reserve(KnnState& s) {
  const Layout L = make_layout(s.c, 4);
  if (s.desc.n < (size_t)s.N * L.dstride) s.desc.alloc((size_t)s.N * L.dstride, s.slots.st);
}

void join_tma_reserve(const KnnState& s, int Dp) {
  (void)Dp;
  set_smem_limit_once(reinterpret_cast<const void*>(join_kernel(s, effective_tile(s))), 227 * 1024);
}

void join_describe(KnnState& s, int kind, cudaStream_t st) {
  const Layout L = make_layout(s.c, 4);
  if (s.desc.n < (size_t)s.N * L.dstride) s.desc.alloc((size_t)s.N * L.dstride, st);
  k_cand_describe<<<grid_for((long long)s.N * 32, 256), 256, 0, st>>>(
      s.cand_new.p, s.cand_old.p, s.N, s.c, s.cp, L.maxc, L.dstride, effective_tile(s).jb,
      kind_is_dot(kind) ? s.norms.p : nullptr, s.desc.p);
  RINND_LAUNCH_CHECK();
}

void join_tma_batch(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, int* err, cudaStream_t st) {
  launch_join(s, X, Dp, kind, v0, v1, st, err);
}

// ---- tile tuner -------------------------------------------------------------
// Tuned shapes are kept per (device, Dp, list class, metric class, grouped) for
// the life of the process.
namespace {
using TileKey = std::tuple<int, int, int, int, int>;
std::mutex g_tile_mu;
std::map<TileKey, JoinTile> g_tiles;

TileKey tile_key(const KnnState& s, int Dp, int kind) {
  int dev = 0;
  RINND_CUDA(cudaGetDevice(&dev));
  const int kclass = kind == DK_SQEUCLIDEAN ? 0 : kind == DK_MANHATTAN ? 1 : 2;
  return TileKey{dev, Dp, s.c <= 32 ? 32 : 64, kclass, s.item_changes.p != nullptr ? 1 : 0};
}
}  // namespace

bool join_tile_lookup(KnnState& s, int Dp, int kind) {
  std::lock_guard<std::mutex> lock(g_tile_mu);
  auto it = g_tiles.find(tile_key(s, Dp, kind));
  if (it == g_tiles.end()) return false;
  s.tile = it->second;
  return true;
}

std::vector<std::array<int, 8>> join_tile_table() {
  std::lock_guard<std::mutex> lock(g_tile_mu);
  std::vector<std::array<int, 8>> out;
  for (const auto& kv : g_tiles) {
    const TileKey& k = kv.first;
    out.push_back({std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k), std::get<4>(k), kv.second.nstage,
                   kv.second.jb, kv.second.per_sm});
  }
  return out;
}

void join_tile_store(int device, int Dp, int list_class, int metric_class, int grouped, const JoinTile& t) {
  std::lock_guard<std::mutex> lock(g_tile_mu);
  g_tiles[TileKey{device, Dp, list_class, metric_class, grouped}] = t;
}

void join_tile_table_clear() {
  std::lock_guard<std::mutex> lock(g_tile_mu);
  g_tiles.clear();
}

// Times every tile shape on the same vertex sample of the current candidate
// lists (built by the caller) and keeps the fastest in s.tile and the table.
// Trials append to the update buffer but their updates are never applied, and
// the few pushes a full buffer region sends directly are undone by restoring
// the rows and thresholds afterwards, so the heaps are those the caller had.
JoinTile join_tune(KnnState& s, const float* X, int Dp, int kind, long long sample, cudaStream_t st,
                   std::vector<TileTrial>* trials) {
  const size_t nslots = (size_t)s.N * s.kp;
  DVec<uint64_t> slots0(nslots, st);
  DVec<uint32_t> thr0((size_t)s.N, st);
  DVec<unsigned long long> cnt0(8, st);
  RINND_CUDA(cudaMemcpyAsync(slots0.p, s.slots.p, sizeof(uint64_t) * nslots, cudaMemcpyDeviceToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(thr0.p, s.thr.p, sizeof(uint32_t) * s.N, cudaMemcpyDeviceToDevice, st));
  RINND_CUDA(cudaMemcpyAsync(cnt0.p, s.counters.p, sizeof(unsigned long long) * 8, cudaMemcpyDeviceToDevice, st));
  const int v1 = (int)std::min<long long>(s.N, std::max<long long>(1, sample));
  std::vector<JoinTile> cands;
  for (int ns : {2, 3})
    for (int jb : {2, 1})
      for (int per_sm : {0, 2}) {
        JoinTile t{ns, jb, per_sm};
        if (s.c > 32 && !(ns == 2 && jb == 1)) continue;
        if (!join_tile_fits(s.c, Dp, t)) continue;
        cands.push_back(t);
      }
  const JoinTile saved = s.tile;
  std::vector<float> best(cands.size(), 1e30f);
  cudaEvent_t e0, e1;
  RINND_CUDA(cudaEventCreate(&e0));
  RINND_CUDA(cudaEventCreate(&e1));
  for (int round = 0; round < 2; ++round)
    for (size_t i = 0; i < cands.size(); ++i) {
      s.tile = cands[i];
      join_tma_reserve(s, Dp);
      join_describe(s, kind, st);
      RINND_CUDA(cudaMemsetAsync(s.counters.p + 4, 0, sizeof(unsigned long long), st));
      RINND_CUDA(cudaEventRecord(e0, st));
      join_tma_batch(s, X, Dp, kind, 0, v1, s.err.p, st);
      RINND_CUDA(cudaEventRecord(e1, st));
      s.nreg = 0;  // the trial's updates are dropped
      RINND_CUDA(cudaMemcpyAsync(s.slots.p, slots0.p, sizeof(uint64_t) * nslots, cudaMemcpyDeviceToDevice, st));
      RINND_CUDA(cudaMemcpyAsync(s.thr.p, thr0.p, sizeof(uint32_t) * s.N, cudaMemcpyDeviceToDevice, st));
      RINND_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      RINND_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (round > 0) best[i] = std::min(best[i], ms);
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  RINND_CUDA(cudaMemcpyAsync(s.counters.p, cnt0.p, sizeof(unsigned long long) * 8, cudaMemcpyDeviceToDevice, st));
  int herr = 0;
  RINND_CUDA(cudaMemcpyAsync(&herr, s.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  if (herr) throw CudaError("join tuning: a shared-memory pipeline stage did not complete within its wait limit");
  size_t pick = 0;
  for (size_t i = 0; i < cands.size(); ++i) {
    if (best[i] < best[pick]) pick = i;
    if (trials) trials->push_back(TileTrial{cands[i], best[i], v1});
  }
  JoinTile chosen = cands.empty() ? saved : cands[pick];
  s.tile = chosen;
  join_tma_reserve(s, Dp);
  std::lock_guard<std::mutex> lock(g_tile_mu);
  g_tiles[tile_key(s, Dp, kind)] = chosen;
  return chosen;
}

}  // namespace rinnd
