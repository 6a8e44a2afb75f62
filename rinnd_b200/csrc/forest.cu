// forest.cu -- batched random-projection forest, all trees level by level.
//
// Restates TreeBuilder::build_recursive / make_split / partition_inplace
// (core/tree/builder.rs:172-348) and build_rp_forest (:89-118) as a
// level-synchronous GPU algorithm:
//   per level, every active segment (size > leaf_size, depth < max_depth) of
//   every tree picks two random points and forms the reference's hyperplane
//   (euclidean perpendicular bisector, or angular normalized difference), all
//   member points compute margins with the reference's dot order, and a
//   device-wide scan performs a stable left|right partition.  A split that sends
//   everything to one side becomes a leaf, as in the reference (:198-210).
// The stable in-place partition leaves each tree's `perm` slice in DFS leaf
// order, which is what the reference's `indices` array holds.  Point order
// inside a leaf and the random streams differ from the reference's two-pointer
// partition and Xoshiro streams; the tree distribution is the same.
#include <cub/cub.cuh>

#include "dist.cuh"
#include "engine.h"

namespace rinnd {
namespace {

struct Seg {
  int tree, start, end, node;
};

__global__ void k_init_perm(int32_t* perm, int N, int T) {
  long long total = (long long)N * T;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    perm[i] = (int32_t)(i % N);
}

// builder.rs:228-308 make_split (+ euclidean / angular hyperplanes).
__global__ void k_split_params(const Seg* segs, int S, const int32_t* perm, int N, const float* X,
                               int D, int Dp, bool angular, uint64_t seed, float* hp, float* off,
                               int32_t* piv) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  Seg g = segs[s];
  uint32_t size = (uint32_t)(g.end - g.start);
  const int32_t* P = perm + (size_t)g.tree * N + g.start;
  uint64_t h = hash3(seed, 0x51u + (uint64_t)g.tree, ((uint64_t)g.start << 32) | (uint32_t)g.end);
  uint32_t i1 = (uint32_t)(((h & 0xffffffffull) * size) >> 32);
  uint32_t i2 = i1;
  for (int r = 1; r < 64 && i2 == i1 && size > 1; ++r)
    i2 = (uint32_t)(((mix64(h + (uint64_t)r) & 0xffffffffull) * size) >> 32);
  if (i2 == i1 && size > 1) i2 = (i1 + 1) % size;
  const float* p1 = X + (size_t)P[i1] * Dp;
  const float* p2 = X + (size_t)P[i2] * Dp;
  piv[2 * s] = P[i1];
  piv[2 * s + 1] = P[i2];
  float* H = hp + (size_t)s * Dp;
  float o = 0.f;
  if (angular) {
    float n1 = 0.f, n2 = 0.f;
    for (int i = 0; i < D; ++i) n1 = __fadd_rn(n1, __fmul_rn(p1[i], p1[i]));
    for (int i = 0; i < D; ++i) n2 = __fadd_rn(n2, __fmul_rn(p2[i], p2[i]));
    n1 = __fsqrt_rn(n1);
    n2 = __fsqrt_rn(n2);
    if (n1 < 1e-8f || n2 < 1e-8f) {
      for (int i = 0; i < Dp; ++i) H[i] = 0.f;
    } else {
      float nn = 0.f;
      for (int i = 0; i < D; ++i) {
        float v = __fsub_rn(__fdiv_rn(p2[i], n2), __fdiv_rn(p1[i], n1));
        H[i] = v;
        nn = __fadd_rn(nn, __fmul_rn(v, v));
      }
      nn = __fsqrt_rn(nn);
      if (nn > 1e-8f)
        for (int i = 0; i < D; ++i) H[i] = __fdiv_rn(H[i], nn);
      for (int i = D; i < Dp; ++i) H[i] = 0.f;
    }
  } else {
    float norm_sq = 0.f, dot_nm = 0.f;
    for (int i = 0; i < D; ++i) {
      float hh = __fsub_rn(p2[i], p1[i]);
      float m = __fmul_rn(__fadd_rn(p1[i], p2[i]), 0.5f);
      H[i] = hh;
      norm_sq = __fadd_rn(norm_sq, __fmul_rn(hh, hh));
      dot_nm = __fadd_rn(dot_nm, __fmul_rn(hh, m));
    }
    float norm = __fsqrt_rn(norm_sq);
    if (norm > 1e-8f) {
      float inv = __fdiv_rn(1.0f, norm);
      for (int i = 0; i < D; ++i) H[i] = __fmul_rn(H[i], inv);
      o = __fmul_rn(-dot_nm, inv);
    }
    for (int i = D; i < Dp; ++i) H[i] = 0.f;
  }
  off[s] = o;
}

// Position -> active segment map for this level (-1 outside active segments).
__global__ void k_fill_segmap(const long long* seg_gstart, const long long* seg_gend, int S,
                              int32_t* seg_of) {
  for (int s = blockIdx.x; s < S; s += gridDim.x)
    for (long long g = seg_gstart[s] + threadIdx.x; g < seg_gend[s]; g += blockDim.x)
      seg_of[g] = s;
}

// builder.rs:312-348 partition_inplace side decision for every tree's position
// of a point: margin = dot(point, hyperplane) + offset in the reference's dot
// order (builder.rs:11-60, exact_dot_a); |margin| < 1e-8 -> random side; else
// margin < 0 -> left.  Two lanes per (point, tree) pair, a warp over 16
// consecutive pairs (a point's trees are neighbors, so its row is read once
// from DRAM per level): lane q carries the reference's accumulator chains
// 4q .. 4q + 3 (elements 8c + 4q + i, c in order) with 16-byte loads of the
// row and the hyperplane (rows are 4-float padded and 16-byte aligned), the
// pair's lanes combine the eight chains in the reference's horizontal-sum tree
// ((s4 + s0) + (s5 + s1)) + ((s6 + s2) + (s7 + s3)) and lane 0 adds the
// remainder -- the margins are bit-identical to exact_dot_a's.  inv[t N + p] is
// point p's position in tree t; positions of finished leaves (segment -1) get
// side 0.
__global__ void k_margins(const int32_t* seg_of, const int32_t* inv, int N, int T, const float* X, int D, int Dp,
                          const float* hp, const float* off, uint64_t seed, int depth, int32_t* is_left) {
  const int lane = threadIdx.x & 31, q = lane & 1;
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const int chunks = D >> 3;
  const long long total = (long long)N * T;
  for (long long u0 = warp * 16; u0 < total; u0 += nwarps * 16) {
    const long long u = u0 + (lane >> 1);
    long long g = -1;
    int sg = -1, pid = 0, t = 0;
    if (u < total) {
      pid = (int)(u / T);
      t = (int)(u - (long long)pid * T);
      g = (long long)t * N + inv[(size_t)t * N + pid];
      sg = seg_of[g];
    }
    const float* x = X + (size_t)pid * Dp;
    const float* h = hp + (size_t)(sg >= 0 ? sg : 0) * Dp;
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
    if (sg >= 0) {
      const float4* x4 = reinterpret_cast<const float4*>(x) + q;
      const float4* h4 = reinterpret_cast<const float4*>(h) + q;
      for (int c = 0; c < chunks; ++c) {
        const float4 xa = __ldg(x4 + 2 * c), ha = __ldg(h4 + 2 * c);
        s0 = __fmaf_rn(xa.x, ha.x, s0);
        s1 = __fmaf_rn(xa.y, ha.y, s1);
        s2 = __fmaf_rn(xa.z, ha.z, s2);
        s3 = __fmaf_rn(xa.w, ha.w, s3);
      }
    }
    // lane 0 of the pair receives chains 4..7 from lane 1
    const float p0 = __shfl_xor_sync(0xffffffffu, s0, 1), p1 = __shfl_xor_sync(0xffffffffu, s1, 1);
    const float p2 = __shfl_xor_sync(0xffffffffu, s2, 1), p3 = __shfl_xor_sync(0xffffffffu, s3, 1);
    if (q == 0 && g >= 0) {
      int left = 0;
      if (sg >= 0) {
        const float a0 = __fadd_rn(p0, s0), a1 = __fadd_rn(p1, s1), a2 = __fadd_rn(p2, s2), a3 = __fadd_rn(p3, s3);
        float r = __fadd_rn(__fadd_rn(a0, a1), __fadd_rn(a2, a3));
        for (int i = chunks * 8; i < D; ++i) r = __fadd_rn(r, __fmul_rn(x[i], h[i]));
        const float margin = __fadd_rn(r, off[sg]);
        if (fabsf(margin) < 1e-8f)
          left = (int)(hash3(seed ^ 0x7a11u, ((uint64_t)t << 32) | (uint32_t)depth, (uint64_t)pid) >> 63);
        else
          left = margin < 0.f;
      }
      is_left[g] = left;
    }
  }
}

__global__ void k_scatter(const int32_t* seg_of, const long long* seg_gstart,
                          const long long* seg_gend, const int32_t* scan, const int32_t* is_left,
                          const int32_t* perm, int32_t* perm_next, int32_t* inv, int N, long long total) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < total;
       g += (long long)gridDim.x * blockDim.x) {
    int s = seg_of[g];
    if (s < 0) continue;
    long long gs = seg_gstart[s], ge = seg_gend[s];
    int lrank = scan[g] - scan[gs];
    int nl = scan[ge] - scan[gs];
    long long dst = is_left[g] ? gs + lrank : gs + nl + ((g - gs) - lrank);
    const int32_t pid = perm[g];
    perm_next[dst] = pid;
    const long long base = (g / N) * N;  // the tree's first position
    inv[base + pid] = (int32_t)(dst - base);
  }
}

__global__ void k_seg_bounds(const Seg* segs, int S, int N, long long* gs, long long* ge) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  Seg g = segs[s];
  gs[s] = (long long)g.tree * N + g.start;
  ge[s] = (long long)g.tree * N + g.end;
}

__global__ void k_outcome(const Seg* segs, int S, const long long* gs, const int32_t* scan,
                          int leaf_size, int depth, int max_depth, int32_t* nleft, int32_t* n_next,
                          int32_t* n_node) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  Seg g = segs[s];
  int size = g.end - g.start;
  int nl = scan[gs[s] + size] - scan[gs[s]];
  nleft[s] = nl;
  bool ok = nl > 0 && nl < size;
  auto cont = [&](int sz) { return (sz > leaf_size && depth + 1 < max_depth) ? 1 : 0; };
  n_next[s] = ok ? cont(nl) + cont(size - nl) : 0;
  n_node[s] = ok ? 2 : 0;
}

__device__ __forceinline__ void emit_leaf(int tree, int start, int end, int node, int32_t* children,
                                          float* offsets, int32_t* pivots, int4* leaves,
                                          unsigned long long* counters) {
  offsets[node] = 0.f;
  pivots[2 * (size_t)node] = -1;
  pivots[2 * (size_t)node + 1] = -1;
  children[2 * (size_t)node] = -start;
  children[2 * (size_t)node + 1] = -end;
  unsigned long long li = atomicAdd(&counters[0], 1ull);
  leaves[li] = make_int4(tree, start, end, node);
  atomicMax(reinterpret_cast<unsigned long long*>(&counters[1]), (unsigned long long)(end - start));
}

__global__ void k_finalize(const Seg* segs, int S, const int32_t* nleft, const int32_t* next_off,
                           const int32_t* node_off, long long node_base, const float* hp,
                           const float* off, const int32_t* piv, int Dp, int leaf_size, int depth,
                           int max_depth, int32_t* children, float* offsets, float* hyperplanes,
                           int32_t* pivots, Seg* next, int4* leaves, unsigned long long* counters) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  Seg g = segs[s];
  int size = g.end - g.start;
  int nl = nleft[s];
  if (!(nl > 0 && nl < size)) {  // builder.rs:198-210 degenerate split -> leaf
    emit_leaf(g.tree, g.start, g.end, g.node, children, offsets, pivots, leaves, counters);
    return;
  }
  int c0 = (int)(node_base + node_off[s]);
  int c1 = c0 + 1;
  children[2 * (size_t)g.node] = c0;
  children[2 * (size_t)g.node + 1] = c1;
  offsets[g.node] = off[s];
  pivots[2 * (size_t)g.node] = piv[2 * s];
  pivots[2 * (size_t)g.node + 1] = piv[2 * s + 1];
  const float4* src = reinterpret_cast<const float4*>(hp + (size_t)s * Dp);
  float4* dst = reinterpret_cast<float4*>(hyperplanes + (size_t)g.node * Dp);
  for (int i = 0; i < Dp / 4; ++i) dst[i] = src[i];
  int o = next_off[s];
  int cs[2] = {g.start, g.start + nl}, ce[2] = {g.start + nl, g.end}, cid[2] = {c0, c1};
  for (int j = 0; j < 2; ++j) {
    int sz = ce[j] - cs[j];
    if (sz > leaf_size && depth + 1 < max_depth) {
      next[o++] = Seg{g.tree, cs[j], ce[j], cid[j]};
    } else {
      emit_leaf(g.tree, cs[j], ce[j], cid[j], children, offsets, pivots, leaves, counters);
    }
  }
}

// Roots that are leaves already (an item of at most leaf_size points, or max_depth 0).
__global__ void k_root_leaves(const int4* roots, int n, int32_t* children, float* offsets, int32_t* pivots,
                              int4* leaves, unsigned long long* counters) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int4 g = roots[r];
  emit_leaf(g.x, g.y, g.z, g.w, children, offsets, pivots, leaves, counters);
}

template <class T>
void exclusive_scan(const T* in, T* out, long long n, TempStorage& tmp, cudaStream_t st) {
  size_t bytes = 0;
  RINND_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st));
  void* p = tmp.ensure(bytes, st);
  RINND_CUDA(cub::DeviceScan::ExclusiveSum(p, bytes, in, out, n, st));
}

}  // namespace

void build_forest(const float* X, int N, int D, int Dp, int T, int leaf_size, bool angular,
                  int max_depth, uint64_t seed, cudaStream_t st, TempStorage& tmp, Forest& f,
                  const ForestItems* items) {
  ForestItems one;
  if (items == nullptr) {
    one.off = {0, (int64_t)N};
    one.trees = {T};
    items = &one;
  }
  const int n_items = (int)items->trees.size();
  f.T = T;
  f.N = N;
  f.Dp = Dp;
  if (leaf_size < 1) leaf_size = 1;
  long long total = (long long)N * T;
  f.perm.alloc((size_t)total, st);
  DVec<int32_t> perm_next((size_t)total, st);
  DVec<int32_t> inv((size_t)total, st);  // inv[t N + p]: position of point p in tree t
  k_init_perm<<<grid_for(total, 256, 148 * 64), 256, 0, st>>>(f.perm.p, N, T);
  RINND_LAUNCH_CHECK();
  k_init_perm<<<grid_for(total, 256, 148 * 64), 256, 0, st>>>(inv.p, N, T);  // identity is its own inverse
  RINND_LAUNCH_CHECK();

  // Root of (tree t, item i) is node t * n_items + i (node t for a single item);
  // roots of trees an item does not have stay unused.
  const size_t n_roots = (size_t)T * n_items;
  size_t node_cap = std::max<size_t>(n_roots * 64, 64);
  f.children.alloc(2 * node_cap, st);
  f.children.fill_bytes(0);
  f.offsets.alloc(node_cap, st);
  f.pivots.alloc(2 * node_cap, st);
  f.hyperplanes.alloc(node_cap * (size_t)Dp, st);
  f.hyperplanes.fill_bytes(0);
  f.n_nodes = (int64_t)n_roots;
  size_t leaf_cap = std::max<size_t>(n_roots * 64, 64);
  f.leaves.alloc(leaf_cap, st);
  DVec<unsigned long long> counters(2, st);  // [0] n_leaves, [1] max leaf size
  counters.fill_bytes(0);

  std::vector<Seg> h_roots;
  std::vector<int4> h_root_leaves;
  for (int t = 0; t < T; ++t)
    for (int i = 0; i < n_items; ++i) {
      if (t >= items->trees[i]) continue;
      const int s0 = (int)items->off[i], s1 = (int)items->off[i + 1], node = t * n_items + i;
      if (s1 - s0 > leaf_size && max_depth > 0) h_roots.push_back(Seg{t, s0, s1, node});
      else h_root_leaves.push_back(make_int4(t, s0, s1, node));
    }
  if (!h_root_leaves.empty()) {
    const int nr = (int)h_root_leaves.size();
    DVec<int4> rl((size_t)nr, st);
    rl.from_host(h_root_leaves.data(), (size_t)nr);
    k_root_leaves<<<grid_for(nr, 128), 128, 0, st>>>(rl.p, nr, f.children.p, f.offsets.p, f.pivots.p, f.leaves.p,
                                                     counters.p);
    RINND_LAUNCH_CHECK();
  }
  int S = (int)h_roots.size();
  DVec<Seg> segs(std::max(S, 1), st);
  segs.from_host(h_roots.data(), (size_t)S);
  DVec<int32_t> is_left((size_t)total + 1, st), scan((size_t)total + 1, st);
  DVec<int32_t> seg_of((size_t)total, st);
  RINND_CUDA(cudaMemsetAsync(is_left.p + total, 0, sizeof(int32_t), st));
  unsigned long long h_counters[2] = {0, 0};
  int depth = 0;
  while (S > 0) {
    DVec<long long> gs((size_t)S, st), ge((size_t)S, st);
    k_seg_bounds<<<grid_for(S, 256), 256, 0, st>>>(segs.p, S, N, gs.p, ge.p);
    DVec<float> hp((size_t)S * Dp, st), off((size_t)S, st);
    DVec<int32_t> piv(2 * (size_t)S, st);
    k_split_params<<<grid_for(S, 128), 128, 0, st>>>(segs.p, S, f.perm.p, N, X, D, Dp, angular,
                                                     seed, hp.p, off.p, piv.p);
    RINND_LAUNCH_CHECK();
    RINND_CUDA(cudaMemsetAsync(seg_of.p, 0xFF, sizeof(int32_t) * (size_t)total, st));
    k_fill_segmap<<<std::min(S, 148 * 16), 256, 0, st>>>(gs.p, ge.p, S, seg_of.p);
    RINND_LAUNCH_CHECK();
    k_margins<<<grid_for((long long)N * 32, 256, 148 * 32), 256, 0, st>>>(seg_of.p, inv.p, N, T, X, D, Dp, hp.p,
                                                                         off.p, seed, depth, is_left.p);
    RINND_LAUNCH_CHECK();
    exclusive_scan(is_left.p, scan.p, total + 1, tmp, st);
    RINND_CUDA(cudaMemcpyAsync(perm_next.p, f.perm.p, sizeof(int32_t) * (size_t)total,
                               cudaMemcpyDeviceToDevice, st));
    k_scatter<<<grid_for(total, 256, 148 * 32), 256, 0, st>>>(seg_of.p, gs.p, ge.p, scan.p,
                                                             is_left.p, f.perm.p, perm_next.p, inv.p, N,
                                                             total);
    RINND_LAUNCH_CHECK();
    std::swap(f.perm.p, perm_next.p);

    DVec<int32_t> nleft((size_t)S, st), n_next((size_t)S + 1, st), n_node((size_t)S + 1, st);
    DVec<int32_t> next_off((size_t)S + 1, st), node_off((size_t)S + 1, st);
    RINND_CUDA(cudaMemsetAsync(n_next.p + S, 0, sizeof(int32_t), st));
    RINND_CUDA(cudaMemsetAsync(n_node.p + S, 0, sizeof(int32_t), st));
    k_outcome<<<grid_for(S, 256), 256, 0, st>>>(segs.p, S, gs.p, scan.p, leaf_size, depth,
                                                max_depth, nleft.p, n_next.p, n_node.p);
    RINND_LAUNCH_CHECK();
    exclusive_scan(n_next.p, next_off.p, (long long)S + 1, tmp, st);
    exclusive_scan(n_node.p, node_off.p, (long long)S + 1, tmp, st);
    int32_t h_tot[2];
    RINND_CUDA(cudaMemcpyAsync(&h_tot[0], next_off.p + S, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    RINND_CUDA(cudaMemcpyAsync(&h_tot[1], node_off.p + S, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    RINND_CUDA(cudaMemcpyAsync(h_counters, counters.p, sizeof(h_counters), cudaMemcpyDeviceToHost, st));
    RINND_CUDA(cudaStreamSynchronize(st));
    int S_next = h_tot[0];
    long long new_nodes = h_tot[1];
    // capacity for nodes and leaves emitted by this level
    size_t need_nodes = (size_t)(f.n_nodes + new_nodes);
    if (need_nodes > f.offsets.n) {
      f.children.grow(2 * need_nodes, 2 * (size_t)f.n_nodes, st);
      f.offsets.grow(need_nodes, (size_t)f.n_nodes, st);
      f.pivots.grow(2 * need_nodes, 2 * (size_t)f.n_nodes, st);
      f.hyperplanes.grow(f.offsets.n * (size_t)Dp, (size_t)f.n_nodes * Dp, st);
      RINND_CUDA(cudaMemsetAsync(f.hyperplanes.p + (size_t)f.n_nodes * Dp, 0,
                                 sizeof(float) * (f.hyperplanes.n - (size_t)f.n_nodes * Dp), st));
    }
    size_t need_leaves = (size_t)h_counters[0] + 3 * (size_t)S;
    if (need_leaves > f.leaves.n) f.leaves.grow(need_leaves, (size_t)h_counters[0], st);
    DVec<Seg> next((size_t)std::max(S_next, 1), st);
    k_finalize<<<grid_for(S, 128), 128, 0, st>>>(segs.p, S, nleft.p, next_off.p, node_off.p,
                                                 f.n_nodes, hp.p, off.p, piv.p, Dp, leaf_size, depth,
                                                 max_depth, f.children.p, f.offsets.p,
                                                 f.hyperplanes.p, f.pivots.p, next.p, f.leaves.p, counters.p);
    RINND_LAUNCH_CHECK();
    f.n_nodes += new_nodes;
    segs = std::move(next);
    S = S_next;
    ++depth;
  }
  RINND_CUDA(cudaMemcpyAsync(h_counters, counters.p, sizeof(h_counters), cudaMemcpyDeviceToHost, st));
  RINND_CUDA(cudaStreamSynchronize(st));
  f.n_leaves = (int64_t)h_counters[0];
  f.max_leaf = (int)h_counters[1];
  f.levels = depth;
}

}  // namespace rinnd
