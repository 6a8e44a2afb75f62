// join_tc.cu -- local join on the tensor cores: BF16 Gram tiles (tcgen05.mma,
// FP32 accumulate in tensor memory) filter the candidate pairs, and every pair
// that may beat its row's threshold is recomputed in exact FP32 before it is
// pushed, so heap order is always decided in FP32.
//
// Same pairs and push semantics as the FP32 joins (the reference's
// update_iteration, core/nndescent/mod.rs:383-446): per vertex, new x new and
// new x old candidate pairs, each pushed into an endpoint's row when its
// distance beats that row's threshold.
//
// Data.  A BF16 copy of the rows (N x Kp, Kp = round_up(D, 16), zero padded)
// and per row r: bn_r = |b_r|^2 of its BF16 row b_r and e_r >= |b_r - x_r|, the
// rounding error of the copy (both FP32, k_bf16_rows).
//
// Work.  A job is two vertices of a CTA's strided vertex sequence (vertices
// without pairs are skipped).  Its tile holds 128 BF16 rows: the new candidates
// of vertex 0 and of vertex 1, then the old candidates of vertex 0 and of vertex
// 1, 32 rows each, K-major in the tcgen05 no-swizzle core-matrix layout.  One
// M = 128, N = 64 Gram product (A = all 128 rows, B = the first 64: the two
// vertices' new rows) gives every pair a vertex needs: tile row t times the new
// rows of t's own vertex.  K is streamed in chunks of 128 through two tile stages,
// so rows of any width fit.
// Warp roles (6 warps):
//   warp 0, producer: keeps vertex descriptors in flight (a bulk copy each),
//     writes a job header (ids, thresholds, row terms) and gathers the rows of
//     each K chunk with 16-byte cp.async copies straight into the core-matrix
//     layout (8 lanes fill one 128-byte core matrix), a stage's copies are
//     waited for one stage later, fenced to the async proxy and signalled;
//   warp 1, MMA: allocates 128 tensor-memory columns (two 64-column
//     accumulators) and, from one thread, issues the chunk's MMAs and commits
//     them to the stage's empty barrier and, after the last chunk, to the
//     accumulator's barrier;
//   warps 2-5, epilogue: warp w reads tensor-memory lane quadrant w % 4 = tile
//     rows 32 (w % 4) ...: one candidate row per thread, the 32 Gram columns of
//     its vertex's new rows, then releases the accumulator; it keeps each valid
//     pair whose distance LOWER BOUND beats a threshold, recomputes the kept
//     pairs in exact FP32 from the rows in global memory (the FP32 join's
//     arithmetic, so both joins push identical distances) and appends the
//     updates to its CTA's region of the update buffer (k_apply_regions).
// Lower bounds.  G = b_i . b_j is exact products accumulated in FP32: |G - b_i.b_j|
// <= Kp 2^-20 |b_i||b_j| (a factor 16 over sequential FP32 rounding).
//   Squared Euclidean: |b_i - b_j|^2 >= bn_i + bn_j - 2G - E with E = (Kp 2^-19 +
//   2^-20)(bn_i + bn_j) (the Gram error, the FP32 sums bn and the final
//   subtraction), and |x_i - x_j| >= |b_i - b_j| - e_i - e_j.  A pair can beat
//   threshold T only if sqrt(max(0, bn_i + bn_j - 2G - E)) < sqrt(T (1 + 2^-11))
//   + e_i + e_j (the factor covers the rounding of the FP32 recheck).
//   Dot-form metrics: x_i.x_j <= G + e_i |b_j| + e_j (|b_i| + e_i) + Kp 2^-20
//   |b_i||b_j|; every such metric is non-increasing in the dot, so the metric of
//   that bound, less 2^-11 of itself, is a lower bound of the distance.
// Every wait is bounded; a wait that runs out sets the device error flag and a
// shared abort flag, all warps leave their loops, the producer waits for its
// copies, the MMA thread for its last commit, and the tensor memory is freed.
#include <cuda_bf16.h>

#include "engine.h"
#include "join_common.cuh"
#include "tcgen05.cuh"

namespace rinnd {
namespace {

using namespace joinc;

constexpr int NSTAGE = 2;          // tile stages
constexpr int NHDR = 3;            // job headers
constexpr int NEPI = 4;            // epilogue warps (one per tensor-memory lane quadrant)
constexpr int NT = 32 * (2 + NEPI);
constexpr int MAXC = 32;           // new and old lists of <= 32 ids
constexpr int KC = 128;            // K elements per tile stage
constexpr int TROWS = 128;         // tile rows: new(v0), new(v1), old(v0), old(v1)
constexpr int SBO = (KC / 8) * 128;  // bytes between 8-row core-matrix groups
constexpr int TILE_BYTES = TROWS * KC * 2;
constexpr uint32_t TMEM_COLS = 128;  // two 64-column accumulators
constexpr int SURV = 1024;         // survivor entries per epilogue warp (32 rows x 32 new rows)

struct VertexHdr {
  int na, no, pad0, pad1;
  int32_t id[64];   // slots 0..31: new candidates, 32..63: old candidates
  uint32_t thr[64]; // row thresholds (fkey) read when the job was set up
  float s[64];      // squared Euclidean: sqrt(T (1 + 2^-11)); dot forms: T
  float e[64];      // BF16 rounding error bound of the row
  float bn[64];     // |BF16 row|^2
  float xn[64];     // FP32 squared norm (dot-form metrics)
};
struct JobHdr {
  int nvert, pad[3];
  VertexHdr v[2];
};

struct TcLayout {
  int kp, dstride, nchunk;
  // mbarriers: tile_full[2], tile_empty[2], hdr_full[3], hdr_empty[3], mma_done[2],
  // tmem_empty[2], desc[NDESC], drain; then 8 ints
  __host__ __device__ static constexpr int n_bars() { return 2 * NSTAGE + 2 * NHDR + 4 + NDESC + 1; }
  __host__ __device__ size_t ints_off() const { return (size_t)n_bars() * 8; }
  __host__ __device__ size_t desc_off() const { return (ints_off() + 32 + 15) / 16 * 16; }
  __host__ __device__ size_t hdr_off() const { return desc_off() + (size_t)NDESC * dstride * 4; }
  __host__ __device__ size_t surv_off() const { return hdr_off() + (size_t)NHDR * sizeof(JobHdr); }
  __host__ __device__ size_t tile_off() const {
    return (surv_off() + (size_t)NEPI * SURV * 4 + 1023) / 1024 * 1024;
  }
  __host__ __device__ size_t bytes() const { return tile_off() + (size_t)NSTAGE * TILE_BYTES; }
};

TcLayout make_tc_layout(int D) {
  TcLayout L;
  L.kp = round_up(D, 16);
  L.dstride = Desc::stride(MAXC);
  L.nchunk = (L.kp + KC - 1) / KC;
  return L;
}

// BF16 copy of the rows and the per-row terms of the lower bounds, one warp per row.
__global__ void k_bf16_rows(const float* __restrict__ X, int N, int D, int Dp, int Kp, __nv_bfloat16* __restrict__ Xb,
                            float2* __restrict__ rinfo) {
  const long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (r >= N) return;
  float bn = 0.f, ee = 0.f;
  for (int k = lane; k < Kp; k += 32) {
    const float x = k < D ? X[r * Dp + k] : 0.f;
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    const float bf = __bfloat162float(b);
    Xb[r * Kp + k] = b;
    bn = fmaf(bf, bf, bn);
    const float d = bf - x;  // exact: b is x rounded to 8 significant bits
    ee = fmaf(d, d, ee);
  }
  for (int o = 16; o; o >>= 1) {
    bn += __shfl_xor_sync(0xffffffffu, bn, o);
    ee += __shfl_xor_sync(0xffffffffu, ee, o);
  }
  // e: the FP32 sum of squares is within Kp 2^-24 of its value; 2^-10 covers it and the sqrt
  if (lane == 0) rinfo[r] = make_float2(bn, sqrtf(ee) * 1.0009765625f + 1e-30f);
}

struct Bars {
  uint64_t *tile_full, *tile_empty, *hdr_full, *hdr_empty, *mma_done, *tmem_empty, *desc, *drain;
};

// Bounded wait whose outcome is the same in every lane of the warp.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  return __all_sync(0xffffffffu, wait_or_abort(bar, parity, abort_flag));
}

template <bool SQ>
__global__ void __launch_bounds__(NT)
    k_join_tc(const int32_t* __restrict__ desc, int v0, int v1, const __nv_bfloat16* __restrict__ Xb,
              const float2* __restrict__ rinfo, const float* __restrict__ X, int Dp, int kind, uint64_t* slots,
              uint32_t* thr, int k, int kp, TcLayout L, uint32_t* urow_buf, uint64_t* ukey_buf,
              unsigned long long* ucount, uint32_t* rcnt, unsigned int rsize, unsigned long long* counters,
              int* err, ItemCount ic) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  Bars B{bar, bar + NSTAGE, bar + 2 * NSTAGE, bar + 2 * NSTAGE + NHDR, bar + 2 * NSTAGE + 2 * NHDR,
         bar + 2 * NSTAGE + 2 * NHDR + 2, bar + 2 * NSTAGE + 2 * NHDR + 4, bar + 2 * NSTAGE + 2 * NHDR + 4 + NDESC};
  int* ints = reinterpret_cast<int*>(smem + L.ints_off());
  volatile int* abort_flag = ints;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(ints + 1);
  unsigned int* s_ucnt = reinterpret_cast<unsigned int*>(ints + 2);
  unsigned int* s_done = reinterpret_cast<unsigned int*>(ints + 3);
  volatile int* stage_end = ints + 4;  // [NSTAGE]: 1 = end-of-work stage
  int32_t* dring = reinterpret_cast<int32_t*>(smem + L.desc_off());
  JobHdr* hdr = reinterpret_cast<JobHdr*>(smem + L.hdr_off());
  uint32_t* surv_all = reinterpret_cast<uint32_t*>(smem + L.surv_off());
  unsigned char* tiles = smem + L.tile_off();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int dstride = L.dstride, Kp = L.kp, nchunk = L.nchunk;

  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&B.tile_full[s], 32);
      mbar_init(&B.tile_empty[s], 1);
    }
    for (int h = 0; h < NHDR; ++h) {
      mbar_init(&B.hdr_full[h], 32);
      mbar_init(&B.hdr_empty[h], NEPI);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&B.mma_done[b], 1);
      mbar_init(&B.tmem_empty[b], NEPI);
    }
    for (int s = 0; s < NDESC; ++s) mbar_init(&B.desc[s], 1);
    mbar_init(B.drain, 1);
    *abort_flag = 0;
    *s_ucnt = 0;
    *s_done = 0;
    fence_mbar_init();
  }
  if (warp == 1) umma::tmem_alloc(tmem_slot, TMEM_COLS);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t taddr = *tmem_slot;
  const int first = v0 + (int)blockIdx.x;
  const int stride = gridDim.x;
  const int nv = first < v1 ? (v1 - first + stride - 1) / stride : 0;

  if (warp == 0) {
    // ------------------------------ producer ------------------------------
    const uint32_t dbytes = (uint32_t)dstride * 4u;
    if (lane == 0)
      for (int i = 0; i < NDESC && i < nv; ++i) {
        mbar_arrive_expect_tx(&B.desc[i], dbytes);
        bulk_g2s(dring + (size_t)i * dstride, desc + (size_t)(first + i * stride) * dstride, dbytes, &B.desc[i]);
      }
    bool ok = true;
    int i = 0;                                  // vertices walked
    int desc_issued = nv < NDESC ? nv : NDESC;  // descriptors issued for vertices [0, desc_issued)
    int jobs = 0, cs = 0;                       // jobs set up, tile stages filled
    int pending = -1;                           // stage whose copies are issued but not yet signalled
    const int r8 = lane & 7, qsub = lane >> 3;
    auto signal_pending = [&]() {               // every copy of this lane but the newest group landed
      if (pending >= 0) {
        cp_async_wait<1>();
        fence_proxy_async_smem();
        mbar_arrive(&B.tile_full[pending]);
        pending = -1;
      }
    };
    while (ok) {
      const int h = jobs % NHDR;
      if (jobs >= NHDR) ok = warp_wait(&B.hdr_empty[h], (uint32_t)((jobs / NHDR) - 1) & 1u, abort_flag);
      if (!ok) break;
      JobHdr* H = hdr + h;
      int nvert = 0;
      while (nvert < 2 && i < nv) {
        const int ds = i % NDESC;
        ok = warp_wait(&B.desc[ds], (uint32_t)(i / NDESC) & 1u, abort_flag);
        if (!ok) break;
        const int32_t* dsc = dring + (size_t)ds * dstride;
        if (dsc[3] > 0) {  // vertices without pairs take no job slot
          VertexHdr& V = H->v[nvert];
          const int na = dsc[0], nb = dsc[1];
          const int32_t* ids = dsc + Desc::ids(MAXC);
          const float* nrm = reinterpret_cast<const float*>(dsc + Desc::nrm(MAXC));
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            const int slot = half * 32 + lane;
            const int src = half ? na + lane : lane;
            const bool have = half ? (na + lane < nb) : (lane < na);
            int32_t id = -1;
            uint32_t th = 0u;
            float2 ri = make_float2(0.f, 0.f);
            float xn = 0.f;
            if (have) {
              id = ids[src];
              th = __ldcg(thr + id);
              ri = rinfo[id];
              if (!SQ) xn = nrm[src];
            }
            const float T = fkey_inv(th);
            V.id[slot] = id;
            V.thr[slot] = th;
            V.s[slot] = SQ ? sqrtf(T * 1.00048828125f) : T;
            V.e[slot] = ri.y;
            V.bn[slot] = ri.x;
            V.xn[slot] = xn;
          }
          if (lane == 0) {
            V.na = na;
            V.no = nb - na;
          }
          ++nvert;
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
        ++i;
      }
      if (!ok) break;
      if (nvert == 1 && lane == 0) {
        H->v[1].na = 0;
        H->v[1].no = 0;
      }
      if (lane == 0) H->nvert = nvert;
      __syncwarp();
      mbar_arrive(&B.hdr_full[h]);  // every lane: its header writes are released
      ++jobs;
      if (nvert == 0) {  // end of work: an end stage for the MMA thread
        const int s = cs % NSTAGE;
        if (cs >= NSTAGE) ok = warp_wait(&B.tile_empty[s], (uint32_t)((cs / NSTAGE) - 1) & 1u, abort_flag);
        if (!ok) break;
        if (pending >= 0) {  // no newer copy group: wait for all of them
          cp_async_wait<0>();
          fence_proxy_async_smem();
          mbar_arrive(&B.tile_full[pending]);
          pending = -1;
        }
        if (lane == 0) stage_end[s] = 1;
        __syncwarp();
        mbar_arrive(&B.tile_full[s]);
        ++cs;
        break;
      }
      // the job's K chunks
      for (int c = 0; c < nchunk && ok; ++c) {
        const int s = cs % NSTAGE;
        if (cs >= NSTAGE) ok = warp_wait(&B.tile_empty[s], (uint32_t)((cs / NSTAGE) - 1) & 1u, abort_flag);
        if (!ok) break;
        if (lane == 0) stage_end[s] = 0;
        unsigned char* tile = tiles + (size_t)s * TILE_BYTES;
        const int k0 = c * KC;
        const int nq = min(KC, Kp - k0) / 8;  // 16-byte pieces per row in this chunk
        for (int g = 0; g < TROWS / 8; ++g) {
          const int t = 8 * g + r8;  // tile row: block t / 32 = new(v0), new(v1), old(v0), old(v1)
          const int blk = t >> 5;
          const int32_t id = H->v[blk & 1].id[((blk >> 1) << 5) + (t & 31)];
          if (!__any_sync(0xffffffffu, id >= 0)) continue;
          const __nv_bfloat16* src = Xb + (size_t)(id >= 0 ? id : 0) * Kp + k0;
          unsigned char* dst = tile + (size_t)g * SBO + r8 * 16;
          for (int q0 = 0; q0 < nq; q0 += 4) {
            const int q = q0 + qsub;
            if (id >= 0 && q < nq) cp_async_16(dst + (size_t)q * 128, src + 8 * q);
          }
        }
        cp_async_commit();
        signal_pending();
        pending = s;
        ++cs;
      }
    }
    if (ok) {
      if (pending >= 0) {
        cp_async_wait<0>();
        fence_proxy_async_smem();
        mbar_arrive(&B.tile_full[pending]);
      }
    } else {
      cp_async_wait<0>();  // copies always complete; none may land after the CTA exits
      if (lane == 0) {
        *abort_flag = 1;
        atomicExch(err, 1);
        for (int j = i; j < desc_issued; ++j)  // drain (bounded) the descriptor copies in flight
          mbar_wait_bounded(&B.desc[j % NDESC], (uint32_t)(j / NDESC) & 1u, WAIT_POLLS);
      }
    }
  } else if (warp == 1) {
    // ------------------------------ MMA issuer ------------------------------
    if (lane == 0) {
      bool ok = true;
      int cs = 0, jobs = 0, committed = -1;  // committed: last job whose accumulator commit was issued
      const uint32_t idesc = umma::idesc_bf16_f32(128, 64);
      const uint32_t tile0 = smem_addr(tiles);
      for (;; ++jobs) {
        const int b = jobs & 1;
        if (jobs >= 2) ok = wait_or_abort(&B.tmem_empty[b], (uint32_t)((jobs / 2) - 1) & 1u, abort_flag);
        if (!ok) break;
        bool end = false;
        for (int c = 0; c < nchunk; ++c) {
          const int s = cs % NSTAGE;
          ok = wait_or_abort(&B.tile_full[s], (uint32_t)(cs / NSTAGE) & 1u, abort_flag);
          if (!ok) break;
          if (stage_end[s]) {
            end = true;
            break;
          }
          umma::fence_after_sync();
          const int nk = min(KC, Kp - c * KC) / 16;
          const uint32_t base = tile0 + (uint32_t)s * TILE_BYTES;
          for (int kk = 0; kk < nk; ++kk) {
            const uint64_t d = umma::smem_desc(base + 256u * kk, 128u, (uint32_t)SBO);
            umma::mma_bf16(taddr + (uint32_t)(64 * b), d, d, idesc, c > 0 || kk > 0);
          }
          umma::commit(&B.tile_empty[s]);  // the stage is free once these MMAs completed
          ++cs;
        }
        if (!ok || end) break;
        umma::commit(&B.mma_done[b]);
        committed = jobs;
      }
      if (!ok) {
        *abort_flag = 1;
        atomicExch(err, 1);
      }
      // no MMA may run once the tensor memory is freed: a last commit tracks every MMA issued
      (void)committed;
      umma::commit(B.drain);
      mbar_wait_bounded(B.drain, 0u, WAIT_POLLS);
    }
    __syncwarp();
  } else {
    // ------------------------------ epilogue ------------------------------
    const int q = warp & 3;                // tensor-memory lane quadrant = tile-row block
    const int vs = q & 1;                  // the block's vertex
    const bool is_new = q < 2;
    uint32_t* surv = surv_all + (size_t)(warp - 2) * SURV;
    const float gam = SQ ? (float)Kp * 1.9073486328125e-06f + 9.5367431640625e-07f   // Kp 2^-19 + 2^-20
                         : (float)Kp * 9.5367431640625e-07f + 9.5367431640625e-07f;  // Kp 2^-20 + 2^-20
    unsigned int pairs_total = 0;
    unsigned long long rows_total = 0;
    for (int job = 0;; ++job) {
      const int h = job % NHDR, b = job & 1;
      if (!warp_wait(&B.hdr_full[h], (uint32_t)(job / NHDR) & 1u, abort_flag)) {
        if (lane == 0) {
          *abort_flag = 1;
          atomicExch(err, 1);
        }
        break;
      }
      const JobHdr* H = hdr + h;
      if (H->nvert == 0) break;  // end of work
      const VertexHdr& V = H->v[vs];
      const int na = V.na;
      const int cnt = is_new ? na : V.no;
      if (!warp_wait(&B.mma_done[b], (uint32_t)(job / 2) & 1u, abort_flag)) {
        if (lane == 0) {
          *abort_flag = 1;
          atomicExch(err, 1);
        }
        break;
      }
      umma::fence_after_sync();
      float g[32];
      if (cnt > 0 && na > 0) {  // warp-uniform
        uint32_t r[32];
        const uint32_t ta = taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)(64 * b + 32 * vs);
        umma::ld_32x32b_x16(ta, r);
        umma::ld_32x32b_x16(ta + 16u, r + 16);
        umma::wait_ld();
#pragma unroll
        for (int j = 0; j < 32; ++j) g[j] = __uint_as_float(r[j]);
      }
      umma::fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&B.tmem_empty[b]);  // this warp's reads of the accumulator are done
      if (lane == 0 && is_new) rows_total += (unsigned long long)(na + V.no);
      // pairs of this warp's rows -> survivors (row lane, new row j, directions)
      const bool rv = lane < cnt;
      const int slot = (is_new ? 0 : 32) + lane;
      const int32_t idt = rv ? V.id[slot] : -1;
      const float st = V.s[slot], et = V.e[slot], bnt = V.bn[slot], xnt = V.xn[slot];
      int nsurv = 0;
      if (cnt > 0 && na > 0) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          if (j < na) {
            const bool valid = rv && (is_new ? (j < lane) : (V.id[j] != idt));  // mod.rs:396, :424
            bool kt = false, kj = false;
            if (valid) {
              ++pairs_total;
              const float G = g[j];
              const float bnj = V.bn[j], ej = V.e[j];
              if (SQ) {
                const float sum = bnt + bnj;
                const float lb = sqrtf(fmaxf(sum - 2.0f * G - gam * sum, 0.f));
                const float ee = et + ej;
                kt = lb < st + ee;
                kj = lb < V.s[j] + ee;
              } else {
                const float bt = sqrtf(bnt), bj = sqrtf(bnj);
                const float ub = G + et * bj + ej * (bt + et) + gam * bt * bj;
                float lb = finalize_dot(kind, ub, V.xn[j], xnt);
                lb = lb - fabsf(lb) * 4.8828125e-4f - 1e-30f;
                kt = lb < st;
                kj = lb < V.s[j];
              }
            }
            const bool keep = kt || kj;
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (keep)
              surv[nsurv + __popc(m & ((1u << lane) - 1))] =
                  ((uint32_t)lane << 8) | ((uint32_t)j << 2) | (kt ? 1u : 0u) | (kj ? 2u : 0u);
            nsurv += __popc(m);
          }
        }
      }
      __syncwarp();
      // exact FP32 recheck of the survivors (the FP32 join's arithmetic: new row first)
      for (int e0 = 0; e0 < nsurv; e0 += 32) {
        const int e = e0 + lane;
        uint32_t rowa = 0, rowb = 0;
        uint64_t keya = 0, keyb = 0;
        bool ea = false, eb = false;
        if (e < nsurv) {
          const uint32_t pr = surv[e];
          const int ts = (is_new ? 0 : 32) + (int)(pr >> 8), j = (int)((pr >> 2) & 63u);
          const int32_t it = V.id[ts], ij = V.id[j];
          float d = join_dist_fp32(kind, X + (size_t)ij * Dp, X + (size_t)it * Dp, Dp);
          if (!SQ) d = finalize_dot(kind, d, V.xn[j], V.xn[ts]);
          const uint32_t kd = fkey(d);
          ea = (pr & 1u) && kd < V.thr[ts];
          eb = (pr & 2u) && kd < V.thr[j];
          rowa = (uint32_t)it;
          rowb = (uint32_t)ij;
          keya = ((uint64_t)kd << 32) | rowb | 0x80000000u;
          keyb = ((uint64_t)kd << 32) | rowa | 0x80000000u;
        }
        const int n_emit = (ea ? 1 : 0) + (eb ? 1 : 0);
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
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          if (!(side ? eb : ea)) continue;
          const uint32_t row = side ? rowb : rowa;
          const uint64_t key = side ? keyb : keya;
          if (base < rsize) {
            urow_buf[(size_t)blockIdx.x * rsize + base] = row;
            ukey_buf[(size_t)blockIdx.x * rsize + base] = key;
          } else if (row_push(slots + (size_t)row * kp, k, thr + row, key, &counters[1])) {
            atomicAdd(&counters[0], 1ull);
            ic.add(row);
          }
          ++base;
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&B.hdr_empty[h]);  // this warp is done with the job's header
    }
    // The last epilogue warp to finish publishes the region's fill count (capped
    // at the region size; the rest were pushed directly) and adds the CTA's
    // appended updates to the launch total.
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(s_done, 1u) == NEPI - 1) {
        const unsigned int total = atomicAdd(s_ucnt, 0u);
        rcnt[blockIdx.x] = total < rsize ? total : rsize;
        atomicAdd(ucount, (unsigned long long)total);
      }
    }
    for (int o = 16; o; o >>= 1) pairs_total += __shfl_xor_sync(0xffffffffu, pairs_total, o);
    if (lane == 0 && pairs_total) atomicAdd(&counters[2], (unsigned long long)pairs_total);
    if (lane == 0 && rows_total) atomicAdd(&counters[3], rows_total);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 1) umma::tmem_dealloc(taddr, TMEM_COLS);
}

template <bool SQ>
void launch_tc(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, cudaStream_t st, const TcLayout& L,
               int* err) {
  const size_t smem = L.bytes();
  set_smem_limit_once(reinterpret_cast<const void*>(k_join_tc<SQ>), 227 * 1024);
  // resident CTAs per SM: shared memory, and at most 4 x 128 of the 512 tensor-memory columns
  const int per_sm = std::max(1, std::min(4, (int)((227 * 1024) / (smem + 1024))));
  const int grid = std::min(v1 - v0, 148 * per_sm);
  if (grid <= 0) return;
  // one region of the update buffer per CTA (k_apply_regions reads them back)
  if (s.rcnt.n < (size_t)grid) s.rcnt.alloc((size_t)grid, st);
  RINND_CUDA(cudaMemsetAsync(s.rcnt.p, 0, sizeof(uint32_t) * grid, st));
  s.nreg = grid;
  s.rsize = (unsigned int)std::min<unsigned long long>(s.ucap / (unsigned long long)grid, 0xFFFFFFFFull);
  k_join_tc<SQ><<<grid, NT, smem, st>>>(s.desc.p, v0, v1, reinterpret_cast<const __nv_bfloat16*>(s.xb.p),
                                        reinterpret_cast<const float2*>(s.rinfo.p), X, Dp, kind, s.slots.p, s.thr.p,
                                        s.k, s.kp, L, s.urow.p, s.ukey.p, s.counters.p + 4, s.rcnt.p, s.rsize,
                                        s.counters.p, err, s.item_count());
  RINND_LAUNCH_CHECK();
}

}  // namespace

bool join_tc_supported(int kind, int c, int Dp) {
  (void)Dp;  // K is streamed in chunks: any row width
  return kind != DK_MANHATTAN && c <= MAXC;
}

void join_tc_reserve(int kind) {
  const void* kern = kind == DK_SQEUCLIDEAN ? reinterpret_cast<const void*>(k_join_tc<true>)
                                            : reinterpret_cast<const void*>(k_join_tc<false>);
  set_smem_limit_once(kern, 227 * 1024);
}

void join_tc_prepare(KnnState& s, const float* X, int D, int Dp, cudaStream_t st) {
  const TcLayout L = make_tc_layout(D);
  if (s.xb.n == (size_t)s.N * L.kp && s.rinfo.n == 2 * (size_t)s.N) return;
  s.xb.alloc((size_t)s.N * L.kp, st);
  s.rinfo.alloc(2 * (size_t)s.N, st);
  s.kpb = L.kp;
  k_bf16_rows<<<grid_for((long long)s.N * 32, 256), 256, 0, st>>>(X, s.N, D, Dp, L.kp,
                                                                  reinterpret_cast<__nv_bfloat16*>(s.xb.p),
                                                                  reinterpret_cast<float2*>(s.rinfo.p));
  RINND_LAUNCH_CHECK();
}

void join_tc_batch(KnnState& s, const float* X, int D, int Dp, int kind, int v0, int v1, int* err, cudaStream_t st) {
  const TcLayout L = make_tc_layout(D);
  if (kind == DK_SQEUCLIDEAN) launch_tc<true>(s, X, Dp, kind, v0, v1, st, L, err);
  else launch_tc<false>(s, X, Dp, kind, v0, v1, st, L, err);
}

}  // namespace rinnd
