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
// Per vertex (candidate lists of <= 32 new + 32 old ids, so nb <= 64 rows):
//   producer warp: one cp.async.bulk per candidate row (FP32, Dp floats) plus,
//     for squared Euclidean, the vertex's own row, into a shared-memory stage
//     (the FP32 join's descriptor/stage pipeline, two stages; vertices without
//     pairs take no stage, and a stage with nb = -1 ends the work);
//   4 compute warps (one per tensor-memory lane quadrant):
//     1. convert the rows to BF16 into a K-major tile; squared Euclidean rows
//        are centered on the vertex's own row first (distances are translation
//        invariant and the centered norms are of the order of the distances,
//        which keeps the BF16 error small next to them);
//     2. one thread issues Kp/16 tcgen05.mma (M = 64, N = round_up(nb, 16))
//        computing the Gram matrix G = T T^T into tensor memory;
//     3. the threads of the leading (new) rows read their Gram rows and keep
//        each valid join pair (i < j) whose distance LOWER BOUND (below) beats
//        the threshold of row i, of row j, or both;
//     4. the kept pairs are recomputed exactly in FP32 from the staged rows with
//        the FP32 join's arithmetic and appended as updates (one per row whose
//        threshold the exact distance beats).
// Lower bounds.  BF16 keeps 8 significant bits: t = bf16(fl(x - c)) has
// |t - (x - c)| <= (2^-8 + 2^-24)|x - c| elementwise and in norm.
// Squared Euclidean: with g = G_ij and G_ii, G_jj the diagonal, the rounded rows
// satisfy |t_i - t_j|^2 >= G_ii + G_jj - 2 g - e, e = Kp 2^-22 (G_ii + G_jj) (FP32
// accumulation), and |x_i - x_j| >= |t_i - t_j| - 2^-7 (sqrt G_ii + sqrt G_jj)
// (a factor 2 over the rounding bound).  So a pair can beat threshold T only if
// G_ii + G_jj - 2 g - e < (sqrt(T (1 + 2^-12)) + 2^-7 (sqrt G_ii + sqrt G_jj))^2,
// the test applied (no square root per pair).
// Dot-form metrics (no centering): |g - x_i.x_j| <= (2^-7 + Kp 2^-23) |x_i||x_j|
// (rounding of both factors); with a factor 2, b = (2^-6 + Kp 2^-22) |x_i||x_j|,
// and as each metric is non-increasing in the dot product, finalize(g + b) is a
// lower bound.  The relative slack 2^-12 covers the rounding of the FP32
// recheck itself.
#include "engine.h"
#include "join_common.cuh"
#include "tcgen05.cuh"

namespace rinnd {
namespace {

using namespace joinc;

constexpr int NSTAGE = 2;
constexpr int NCOMP = 4;  // compute warps: one per TMEM lane quadrant
constexpr int NT = 32 * (1 + NCOMP);
constexpr int MAXC = 32;  // new and old lists of <= 32 ids: <= 64 rows, one M = 64 tile
constexpr int TROWS = 2 * MAXC;
constexpr uint32_t TMEM_COLS = 64;
constexpr int CBAR = 1;  // named barrier of the compute warps

struct TcLayout {
  int dp, rs, kp, dstride;
  // mbarriers: full[NSTAGE], empty[NSTAGE], desc[NDESC], mma; then 4 ints
  __host__ __device__ size_t bar_bytes() const { return 8 * (2 * NSTAGE + NDESC + 1) + 16; }
  __host__ __device__ size_t desc_off() const { return (bar_bytes() + 15) / 16 * 16; }
  __host__ __device__ size_t stage_off() const { return desc_off() + (size_t)NDESC * dstride * 4; }
  __host__ __device__ size_t rows_off() const { return (size_t)dstride * 4; }
  // TROWS candidate rows + the vertex's own row
  __host__ __device__ size_t stage_bytes() const { return rows_off() + (size_t)(TROWS + 1) * rs * 4; }
  __host__ __device__ size_t tile_off() const { return (stage_off() + NSTAGE * stage_bytes() + 127) / 128 * 128; }
  // per row: Gram diagonal, its square root (or the row norm), threshold term
  __host__ __device__ size_t diag_off() const { return tile_off() + (size_t)TROWS * kp * 2; }
  __host__ __device__ size_t surv_off() const { return diag_off() + 3 * TROWS * 4; }
  __host__ __device__ size_t bytes() const { return surv_off() + (size_t)TROWS * TROWS * 4; }
};

TcLayout make_tc_layout(int Dp) { return TcLayout{Dp, Dp + 4, round_up(Dp, 16), Desc::stride(MAXC)}; }

__device__ __forceinline__ void cbar_sync() { asm volatile("bar.sync %0, %1;" ::"n"(CBAR), "n"(NCOMP * 32) : "memory"); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  uint32_t r;
  asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));  // first source -> upper half
  return r;
}

// Dot-form metrics: lower bound of the distance from the BF16 Gram entry g
// (see the file comment); sni, snj are the rows' FP32 norms.
__device__ __forceinline__ float dot_lower_bound(int kind, float g, float ni, float nj, float sni, float snj,
                                                 float kerr) {
  const float lb = finalize_dot(kind, g + (0.015625f + kerr) * sni * snj, ni, nj);
  return lb - fabsf(lb) * 0.000244140625f - 1e-30f;
}

template <bool SQ>
__global__ void __launch_bounds__(NT)
    k_join_tc(const int32_t* __restrict__ desc, int v0, int v1, const float* __restrict__ X, int Dp, int kind,
              uint64_t* slots, uint32_t* thr, int k, int kp, TcLayout L, uint32_t* urow_buf, uint64_t* ukey_buf,
              unsigned long long* ucount, unsigned long long ucap, unsigned long long* counters, int* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + NSTAGE;
  uint64_t* dbar = empty + NSTAGE;
  uint64_t* mma_bar = dbar + NDESC;
  int* ints = reinterpret_cast<int*>(mma_bar + 1);
  volatile int* abort_flag = ints;
  volatile int* go_flag = ints + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(ints + 2);
  int* nsurv = ints + 3;
  int32_t* dring = reinterpret_cast<int32_t*>(smem + L.desc_off());
  unsigned char* stage0 = smem + L.stage_off();
  unsigned char* tile = smem + L.tile_off();
  float* diag = reinterpret_cast<float*>(smem + L.diag_off());
  uint32_t* surv = reinterpret_cast<uint32_t*>(smem + L.surv_off());
  const size_t sbytes = L.stage_bytes();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int dstride = L.dstride;

  if (tid == 0) {
    for (int s = 0; s < NSTAGE; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCOMP);
    }
    for (int s = 0; s < NDESC; ++s) mbar_init(&dbar[s], 1);
    mbar_init(mma_bar, 1);
    *abort_flag = 0;
    *nsurv = 0;
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
        mbar_arrive_expect_tx(&dbar[i], dbytes);
        bulk_g2s(dring + (size_t)i * dstride, desc + (size_t)(first + i * stride) * dstride, dbytes, &dbar[i]);
      }
    bool ok = true;
    int i = 0, jobs = 0;  // vertices walked, stages filled
    int desc_issued = nv < NDESC ? nv : NDESC;
    for (; i < nv; ++i) {
      const int ds = i % NDESC;
      const int v = first + i * stride;
      ok = wait_or_abort(&dbar[ds], (uint32_t)(i / NDESC) & 1u, abort_flag);
      if (!ok) break;
      const int32_t* dsc = dring + (size_t)ds * dstride;
      const int nb = dsc[1], items = dsc[3];
      if (items > 0) {  // vertices without pairs take no stage
        const int s = jobs % NSTAGE;
        if (jobs >= NSTAGE) {
          ok = wait_or_abort(&empty[s], (uint32_t)((jobs / NSTAGE) - 1) & 1u, abort_flag);
          if (!ok) break;
        }
        unsigned char* st = stage0 + (size_t)s * sbytes;
        int32_t* sd = reinterpret_cast<int32_t*>(st);
        for (int t = lane; t < dstride; t += 32)  // descriptor -> stage header (thresholds below)
          if (t < Desc::thr(MAXC) || t >= Desc::nrm(MAXC)) sd[t] = dsc[t];
        // row thresholds as of now (pushes applied by earlier batches tighten them)
        int32_t my_ids[2];
        uint32_t* sthr = reinterpret_cast<uint32_t*>(sd + Desc::thr(MAXC));
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int r = lane + 32 * t;
          my_ids[t] = r < nb ? dsc[Desc::ids(MAXC) + r] : 0;
          if (r < nb) sthr[r] = __ldcg(thr + my_ids[t]);
        }
        float* rows = reinterpret_cast<float*>(st + L.rows_off());
        const int ncopy = nb + (SQ ? 1 : 0);
        __syncwarp();
        if (lane == 0) mbar_arrive_expect_tx(&full[s], (uint32_t)ncopy * (uint32_t)Dp * 4u);
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 2; ++t) {
          const int r = lane + 32 * t;
          if (r < nb) bulk_g2s(rows + (size_t)r * L.rs, X + (size_t)my_ids[t] * Dp, (uint32_t)Dp * 4u, &full[s]);
        }
        if (SQ && lane == 0)
          bulk_g2s(rows + (size_t)TROWS * L.rs, X + (size_t)v * Dp, (uint32_t)Dp * 4u, &full[s]);
        ++jobs;
      }
      // descriptor slot consumed: refill it NDESC vertices ahead
      fence_proxy_async_smem();
      __syncwarp();
      if (i + NDESC < nv) {
        desc_issued = i + NDESC + 1;
        if (lane == 0) {
          mbar_arrive_expect_tx(&dbar[ds], dbytes);
          bulk_g2s(dring + (size_t)ds * dstride, desc + (size_t)(first + (i + NDESC) * stride) * dstride, dbytes,
                   &dbar[ds]);
        }
      }
    }
    if (ok) {  // end-of-work stage (nb = -1)
      const int s = jobs % NSTAGE;
      if (jobs >= NSTAGE) ok = wait_or_abort(&empty[s], (uint32_t)((jobs / NSTAGE) - 1) & 1u, abort_flag);
      if (ok && lane == 0) {
        reinterpret_cast<int32_t*>(stage0 + (size_t)s * sbytes)[1] = -1;
        mbar_arrive(&full[s]);
      }
    }
    if (!ok && lane == 0) {
      *abort_flag = 1;
      atomicExch(err, 1);
      // drain: wait (bounded) for every descriptor and row copy this warp issued
      for (int j = i; j < desc_issued; ++j)
        mbar_wait_bounded(&dbar[j % NDESC], (uint32_t)(j / NDESC) & 1u, WAIT_POLLS);
      for (int j = (jobs > NSTAGE ? jobs - NSTAGE : 0); j < jobs; ++j)
        mbar_wait_bounded(&full[j % NSTAGE], (uint32_t)(j / NSTAGE) & 1u, WAIT_POLLS);
    }
    return;
  }

  // ------------------------------ compute warps ------------------------------
  // Every decision that ends the loop is taken by one thread and published
  // through shared memory behind a named barrier, so the four warps always
  // leave together and reach the tensor-memory release below.
  const int ct = tid - 32;
  const int quad = warp & 3;            // TMEM lanes 32*quad .. 32*quad+31
  const uint32_t sbo = (uint32_t)(L.kp / 8) * 128u;
  const uint32_t tile_addr = smem_addr(tile);
  const float kerr = (float)L.kp * 2.384185791015625e-07f;  // Kp 2^-22
  unsigned int pairs_total = 0;
  unsigned long long rows_total = 0;
  int nmma = 0;
  for (int i = 0;; ++i) {  // stages in fill order, up to the end-of-work stage
    const int s = i % NSTAGE;
    if (ct == 0) {
      const bool ok = wait_or_abort(&full[s], (uint32_t)(i / NSTAGE) & 1u, abort_flag);
      if (!ok) {
        *abort_flag = 1;
        atomicExch(err, 1);
      }
      *go_flag = ok;
    }
    cbar_sync();
    if (!*go_flag) break;
    if (ct == 0) *nsurv = 0;  // every compute thread is past the previous vertex's survivor list
    mbar_try_wait(&full[s], (uint32_t)(i / NSTAGE) & 1u);  // acquire the completed phase in every thread
    const unsigned char* st = stage0 + (size_t)s * sbytes;
    const int32_t* sd = reinterpret_cast<const int32_t*>(st);
    const int na = sd[0], nb = sd[1];
    if (nb < 0) break;  // read by every compute thread after the same barrier
    const int32_t* ids = sd + Desc::ids(MAXC);
    const uint32_t* sthr = reinterpret_cast<const uint32_t*>(sd + Desc::thr(MAXC));
    const float* snrm = reinterpret_cast<const float*>(sd + Desc::nrm(MAXC));
    const float* rows = reinterpret_cast<const float*>(st + L.rows_off());
    if (ct == 0) rows_total += (unsigned long long)nb;
    if (na > 0) {
      // 1. rows -> BF16 K-major tile (centered on the vertex's row for squared Euclidean)
      const float* cen = rows + (size_t)TROWS * L.rs;
      const int nchunk = L.kp / 8;
      for (int e = ct; e < nb * nchunk; e += NCOMP * 32) {
        const int r = e % nb, kc = e / nb, k0 = 8 * kc;
        float v[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) v[t] = 0.f;
        const float* src = rows + (size_t)r * L.rs + k0;
        if (k0 + 4 <= Dp) {
          const float4 a = *reinterpret_cast<const float4*>(src);
          v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
          if (SQ) {
            const float4 c = *reinterpret_cast<const float4*>(cen + k0);
            v[0] -= c.x; v[1] -= c.y; v[2] -= c.z; v[3] -= c.w;
          }
        }
        if (k0 + 8 <= Dp) {
          const float4 a = *reinterpret_cast<const float4*>(src + 4);
          v[4] = a.x; v[5] = a.y; v[6] = a.z; v[7] = a.w;
          if (SQ) {
            const float4 c = *reinterpret_cast<const float4*>(cen + k0 + 4);
            v[4] -= c.x; v[5] -= c.y; v[6] -= c.z; v[7] -= c.w;
          }
        }
        uint4 packed;
        packed.x = pack_bf16x2(v[0], v[1]);
        packed.y = pack_bf16x2(v[2], v[3]);
        packed.z = pack_bf16x2(v[4], v[5]);
        packed.w = pack_bf16x2(v[6], v[7]);
        *reinterpret_cast<uint4*>(tile + (size_t)(r >> 3) * sbo + (size_t)kc * 128 + (r & 7) * 16) = packed;
      }
      fence_proxy_async_smem();  // generic tile writes -> tensor-core (async proxy) reads
      cbar_sync();
      // 2. Gram tile into tensor memory
      const int N = round_up(nb, 16);
      if (ct == 0) {
        umma::fence_after_sync();
        const uint32_t idesc = umma::idesc_bf16_f32(64, N);
        for (int ks = 0; ks < L.kp / 16; ++ks) {
          const uint64_t d = umma::smem_desc(tile_addr + 256u * ks, 128u, sbo);
          umma::mma_bf16(taddr, d, d, idesc, ks > 0);
        }
        umma::commit(mma_bar);
        const bool ok = wait_or_abort(mma_bar, (uint32_t)nmma & 1u, abort_flag);
        if (!ok) {
          *abort_flag = 1;
          atomicExch(err, 1);
        }
        *go_flag = ok;
      }
      cbar_sync();
      if (!*go_flag) break;
      mbar_try_wait(mma_bar, (uint32_t)nmma & 1u);
      ++nmma;
      umma::fence_after_sync();
      // 3. Gram entries -> candidate pairs.  A pair (ia < j) needs ia new (new rows
      // come first), so only rows < na <= 32 lead pairs.  Lane l and l + 16 share
      // row 16*quad + (l & 15); each TMEM chunk of 16 columns is split between them.
      const uint32_t ta = taddr + ((uint32_t)(32 * quad) << 16);
      const int row = 16 * quad + (lane & 15);
      const bool row_ok = row < nb;
      {
        uint32_t r[16];
        umma::ld_32x32b_x16(ta + 16u * quad, r);  // the chunk holding this warp's diagonal
        umma::wait_ld();
        float gii = 0.f;
#pragma unroll
        for (int t = 0; t < 16; ++t)
          if (t == (lane & 15)) gii = __uint_as_float(r[t]);
        if (lane < 16 && row_ok) {
          diag[row] = gii;
          if (SQ) {
            diag[TROWS + row] = sqrtf(fmaxf(gii, 0.f));
            diag[2 * TROWS + row] = sqrtf(fkey_inv(sthr[row]) * 1.000244140625f);
          } else {
            diag[TROWS + row] = sqrtf(snrm[row]);
            diag[2 * TROWS + row] = fkey_inv(sthr[row]);
          }
        }
      }
      umma::fence_before_sync();
      cbar_sync();  // per-row terms complete
      if (16 * quad < na) {  // warp-uniform: tcgen05.ld and the shuffles need the whole warp
        const bool lead = row < na;
        const int32_t aid = lead ? ids[row] : -1;
        const float gi = lead ? diag[row] : 0.f, si = lead ? diag[TROWS + row] : 0.f;
        const float ti = lead ? diag[2 * TROWS + row] : 0.f;
        const float ni = (SQ || !lead) ? 0.f : snrm[row];
        unsigned int my_pairs = 0;
        for (int c0 = 16 * quad; c0 < nb; c0 += 16) {  // chunks on or right of the diagonal block
          uint32_t r[16];
          umma::ld_32x32b_x16(ta + (uint32_t)c0, r);
          umma::wait_ld();
          const int half = (lane >> 4) * 8;  // this lane's 8 columns: c0 + half + t
          uint32_t keep = 0;
#pragma unroll
          for (int t = 0; t < 8; ++t) {
            const uint32_t hi = __shfl_sync(0xffffffffu, r[t + 8], lane & 15);
            const float g = __uint_as_float(half ? hi : r[t]);
            const int j = c0 + half + t;
            if (lead && j > row && j < nb && (j < na || ids[j] != aid)) {  // mod.rs:396, :424
              ++my_pairs;
              if (SQ) {
                const float gj = diag[j], sj = diag[TROWS + j], tj = diag[2 * TROWS + j];
                const float d2 = (gi + gj) * (1.0f - kerr) - 2.0f * g;
                const float dl = 0.0078125f * (si + sj);
                const float bi = ti + dl, bj = tj + dl;
                keep |= (d2 < bi * bi ? 1u : 0u) << (2 * t);
                keep |= (d2 < bj * bj ? 2u : 0u) << (2 * t);
              } else {
                const float lb = dot_lower_bound(kind, g, ni, snrm[j], si, diag[TROWS + j], kerr);
                keep |= (lb < ti ? 1u : 0u) << (2 * t);
                keep |= (lb < diag[2 * TROWS + j] ? 2u : 0u) << (2 * t);
              }
            }
          }
          if (keep) {
            int cnt = 0;
#pragma unroll
            for (int t = 0; t < 8; ++t) cnt += ((keep >> (2 * t)) & 3u) != 0;
            int base = atomicAdd(nsurv, cnt);
#pragma unroll
            for (int t = 0; t < 8; ++t) {
              const uint32_t dirs = (keep >> (2 * t)) & 3u;
              if (dirs) surv[base++] = ((uint32_t)row << 16) | ((uint32_t)(c0 + half + t) << 2) | dirs;
            }
          }
        }
        pairs_total += my_pairs;
      }
      // every thread's tensor-memory reads are complete (wait_ld) before this barrier
      umma::fence_before_sync();
      cbar_sync();
      // 4. exact FP32 recheck of the kept pairs -> updates (one distance, up to two pushes)
      const int ns = *nsurv;
      for (int e0 = 0; e0 < ns; e0 += NCOMP * 32) {
        const int e = e0 + ct;
        uint32_t rowa = 0, rowb = 0;
        uint64_t keya = 0, keyb = 0;
        bool ea = false, eb = false;
        if (e < ns) {
          const uint32_t pr = surv[e];
          const int ia = (int)(pr >> 16), jb = (int)((pr >> 2) & 0x3FFFu);
          float d = join_dist_fp32(kind, rows + (size_t)ia * L.rs, rows + (size_t)jb * L.rs, Dp);
          if (!SQ) d = finalize_dot(kind, d, snrm[ia], snrm[jb]);
          const uint32_t kd = fkey(d);
          ea = (pr & 1u) && kd < sthr[ia];
          eb = (pr & 2u) && kd < sthr[jb];
          rowa = (uint32_t)ids[ia];
          rowb = (uint32_t)ids[jb];
          keya = ((uint64_t)kd << 32) | rowb | 0x80000000u;
          keyb = ((uint64_t)kd << 32) | rowa | 0x80000000u;
        }
#pragma unroll
        for (int side = 0; side < 2; ++side) {
          const bool emit = side ? eb : ea;
          const uint32_t urow = side ? rowb : rowa;
          const uint64_t key = side ? keyb : keya;
          const unsigned m = __ballot_sync(0xffffffffu, emit);
          if (m) {
            unsigned long long base = 0;
            if (lane == __ffs(m) - 1) base = atomicAdd(ucount, (unsigned long long)__popc(m));
            base = __shfl_sync(0xffffffffu, base, __ffs(m) - 1) + (unsigned long long)__popc(m & ((1u << lane) - 1));
            if (emit) {
              if (base < ucap) {
                urow_buf[base] = urow;
                ukey_buf[base] = key;
              } else if (row_push(slots + (size_t)urow * kp, k, thr + urow, key, &counters[1])) {
                atomicAdd(&counters[0], 1ull);
              }
            }
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s
  }
  for (int o = 16; o; o >>= 1) pairs_total += __shfl_xor_sync(0xffffffffu, pairs_total, o);
  if (lane == 0 && pairs_total) atomicAdd(&counters[2], (unsigned long long)pairs_total);
  if (ct == 0 && rows_total) atomicAdd(&counters[3], rows_total);
  umma::fence_before_sync();
  cbar_sync();
  if (warp == 1) umma::tmem_dealloc(taddr, TMEM_COLS);
}

template <bool SQ>
void launch_tc(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, cudaStream_t st, const TcLayout& L,
               int* err) {
  const size_t smem = L.bytes();
  set_smem_limit_once(reinterpret_cast<const void*>(k_join_tc<SQ>), 227 * 1024);
  // resident CTAs per SM: shared memory, and at most 4 x 64 of the 512 TMEM columns
  const int per_sm = std::max(1, std::min(4, (int)((227 * 1024) / (smem + 1024))));
  const int grid = std::min(v1 - v0, 148 * per_sm);
  if (grid <= 0) return;
  k_join_tc<SQ><<<grid, NT, smem, st>>>(s.desc.p, v0, v1, X, Dp, kind, s.slots.p, s.thr.p, s.k, s.kp, L, s.urow.p,
                                        s.ukey.p, s.counters.p + 4, s.ucap, s.counters.p, err);
  RINND_LAUNCH_CHECK();
}

}  // namespace

bool join_tc_supported(int kind, int c, int Dp) {
  return kind != DK_MANHATTAN && c <= MAXC && make_tc_layout(Dp).bytes() <= 220 * 1024;
}

void join_tc_batch(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, int* err, cudaStream_t st) {
  const TcLayout L = make_tc_layout(Dp);
  if (kind == DK_SQEUCLIDEAN) launch_tc<true>(s, X, Dp, kind, v0, v1, st, L, err);
  else launch_tc<false>(s, X, Dp, kind, v0, v1, st, L, err);
}

}  // namespace rinnd
