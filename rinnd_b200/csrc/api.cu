// api.cu -- C ABI and host orchestration of the B200 NN-Descent engine.
//
// rinnd_build follows NNDescentBuilder::build_with_distance (core/index.rs:601-733):
// parameter defaults (:617-625), RP forest + leaf init + NN-Descent iterations
// with the delta convergence test (core/nndescent/mod.rs:137-163), sorted kNN
// rows (:653), the diversified CSR (:656-666), corrected neighbor distances
// (:669-673) and the physical reorder by the first tree's leaf order (:679-715).
// Everything stays resident on the device; host copies are made only for
// exports.  There is no CPU fallback: without a CUDA device every entry point
// fails with RINND_ERR_NO_DEVICE.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <utility>
#include <new>
#include <string>
#include <vector>

#include "../../include/rinnd.h"
#include "common.cuh"
#include "engine.h"
#include "server.h"

using namespace rinnd;

namespace rinnd {
std::atomic<unsigned long long>& launch_counter() {
  static std::atomic<unsigned long long> n{0};
  return n;
}
}  // namespace rinnd

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace rinnd {
int api_fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
}  // namespace rinnd

namespace {

struct NoDevice : std::runtime_error {
  using std::runtime_error::runtime_error;
};

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <class F>
int guarded(F&& f) {
  try {
    f();
    return RINND_OK;
  } catch (const std::invalid_argument& e) {
    return fail(RINND_ERR_INVALID, e.what());
  } catch (const ServerBusy& e) {
    return fail(RINND_ERR_BUSY, e.what());
  } catch (const NoDevice& e) {
    return fail(RINND_ERR_NO_DEVICE, e.what());
  } catch (const std::bad_alloc& e) {
    return fail(RINND_ERR_OOM, "host allocation failed");
  } catch (const CudaError& e) {
    std::string m = e.what();
    int code = (m.find("out of memory") != std::string::npos) ? RINND_ERR_OOM : RINND_ERR_CUDA;
    return fail(code, m);
  } catch (const std::exception& e) {
    return fail(RINND_ERR_INTERNAL, e.what());
  }
}

void require(bool cond, const std::string& msg) {
  if (!cond) throw std::invalid_argument(msg);
}

void ensure_device(int dev) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw NoDevice("no CUDA device is available: the B200 engine has no CPU fallback");
  }
  require(dev >= 0 && dev < n, "device ordinal out of range");
  RINND_CUDA(cudaSetDevice(dev));
  // Keep freed stream-ordered allocations cached in the device pool instead of
  // returning them to the driver at every synchronization: builds allocate and
  // free large temporaries per level / per iteration.
  static std::mutex mu;
  static bool pool_set[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (dev < 64 && !pool_set[dev]) {
    cudaMemPool_t pool;
    RINND_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t threshold = UINT64_MAX;
    RINND_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    pool_set[dev] = true;
  }
}

// Grows the device's stream-ordered pool once to `bytes` (a single mapping) when
// this library has not yet reserved that much on the device.  Growing the pool
// piecemeal, one new mapping per large block a build asks for, stalled 1M-point
// builds by 0.1-1.5 s until the pool's segments happened to fit the build's
// allocation pattern; one reservation of the working set removes the stalls.
// The reservation is best effort: a failed allocation leaves the pool as it was.
void reserve_pool(int dev, size_t bytes, cudaStream_t st) {
  static std::mutex mu;
  static size_t reserved[64] = {};
  if (dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (bytes <= reserved[dev]) return;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  bytes = std::min(bytes, free_b / 10 * 9);
  void* p = nullptr;
  if (cudaMallocAsync(&p, bytes, st) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  RINND_CUDA(cudaFreeAsync(p, st));
  reserved[dev] = bytes;
}

// Device working set of one build: rows (input copy and search layout), forest,
// neighbor rows, candidate lists, join descriptors, update buffer, sorted rows and
// search-graph temporaries, plus a quarter for fragmentation.
size_t build_working_set(int64_t n, int Dp, int k, int c, int n_trees) {
  const double N = (double)n;
  const int kp = round_up(k, 16), cp = round_up(c, 16), maxc = c <= 32 ? 32 : 64;
  double b = N * Dp * 4.0 * 2 + N * std::max(n_trees, 1) * 4.0 * 2 + N * kp * 8.0 + 2 * N * cp * 8.0 +
             N * (20 + 6 * maxc) * 4.0 + std::max(4194304.0, 96 * N) * 12.0 + N * k * 8.0 * 3 + 256.0 * (1 << 20);
  return (size_t)(b * 1.25);
}

}  // namespace

void rinnd::set_smem_limit_once(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  RINND_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({kernel, dev})) return;
  RINND_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  done.insert({kernel, dev});
}

namespace {

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct StreamGuard {
  cudaStream_t s = nullptr;
  StreamGuard() { RINND_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~StreamGuard() {
    if (s) cudaStreamDestroy(s);
  }
};

// Copies n rows of d floats (row stride ld) into a zero-padded n x Dp device buffer.
void load_rows(const float* src, bool src_device, int64_t n, int d, int64_t ld, int Dp, DVec<float>& dst,
               cudaStream_t st) {
  dst.alloc((size_t)n * Dp, st);
  if (Dp != d) dst.fill_bytes(0);
  RINND_CUDA(cudaMemcpy2DAsync(dst.p, sizeof(float) * Dp, src, sizeof(float) * ld, sizeof(float) * d,
                               (size_t)n, src_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               st));
}

bool kind_uses_norms(int kind) { return kind != DK_SQEUCLIDEAN && kind != DK_MANHATTAN && kind < DK_FIRST_GENERIC; }

__global__ void k_tree_idx(const int32_t* perm, const int32_t* inverse, long long total, int32_t* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = inverse[perm[i]];
}

__global__ void k_iota(int32_t* p, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = i;
}

}  // namespace

struct rinnd_index {
  int device = 0;
  cudaStream_t st = nullptr;
  bool own_stream = true;
  int64_t N = 0;
  int D = 0, Dp = 0, k = 0;
  rinnd_build_params p{};
  int kind = 0, corr = 0;
  bool normalize = false;
  DVec<float> X;                 // internal order, N x Dp
  DVec<int32_t> vertex_order;    // internal -> original
  DVec<int32_t> inverse;         // original -> internal
  Csr graph_int, graph_orig;
  Forest forest;
  DVec<int32_t> tree_idx, tree_roots;
  int n_search_trees = 0;
  DVec<int32_t> knn_idx;
  DVec<float> knn_dist;          // corrected
  float min_distance = 0.f;
  rinnd_build_info info{};
  DVec<unsigned long long> search_stats;
  // int8 serving
  int encoding = -1;
  DVec<int8_t> codes;
  DVec<float> inv_norms;
  DVec<float> dim_scales;        // per-dimension encoding: Dq scales
  // int8 routing trees (tree_quantization="int8", lib.rs:681-704): codes and scales of every forest node
  DVec<int8_t> tree_codes;
  DVec<float> tree_scales;
  bool fp32_released = false;    // rows X freed (retain_fp32_data=False): no FP32 search or rerank
  float global_mult = 0.f;
  int Dq = 0;
  double encode_seconds = 0.0;
  std::mutex mu;
  ~rinnd_index() {
    if (st) {
      cudaSetDevice(device);
      cudaStreamSynchronize(st);
    }
  }
  void destroy_stream() {
    if (st && own_stream) cudaStreamDestroy(st);
    st = nullptr;
  }
  SearchIndex search_view() const {
    SearchIndex s;
    s.N = (int)N;
    s.D = D;
    s.Dp = Dp;
    s.kind = kind;
    s.corr = corr;
    s.X = X.p;
    s.indptr = graph_int.indptr.p;
    s.indices = graph_int.indices.p;
    s.min_distance = min_distance;
    s.n_trees = n_search_trees;
    s.tree_roots = tree_roots.p;
    s.children = forest.children.p;
    s.offsets = forest.offsets.p;
    s.hyperplanes = forest.hyperplanes.p;
    s.tree_idx = tree_idx.p;
    s.leaf_budget = p.search_tree_leaf_budget;
    s.tree_depth = forest.levels;
    s.frontier_cap = s.leaf_budget > 1 ? s.leaf_budget * std::max(forest.levels, 1) + 2 : 0;
    s.tree_codes = tree_codes.p;
    s.tree_scales = tree_scales.p;
    s.vertex_order = vertex_order.p;
    s.seed = p.random_seed;
    s.codes = codes.p;
    s.inv_norms = inv_norms.p;
    s.dim_scales = encoding == Q8_PER_DIMENSION ? dim_scales.p : nullptr;
    s.Dq = Dq;
    return s;
  }
};

namespace {

void validate_params(const rinnd_build_params* p, int64_t n, int d) {
  require(p != nullptr, "params must not be null");
  require(n >= 1, "data must contain at least one point");
  require(n < (int64_t)INT32_MAX - 1, "at most 2^31-2 points are supported");
  require(d >= 1, "data dimension must be positive");
  require(p->n_neighbors >= 1 && p->n_neighbors <= 128, "n_neighbors must be in [1, 128]");
  require(p->n_trees >= 0 && p->n_trees <= 64, "n_trees must be in [0, 64]");
  require(p->n_search_trees >= 0, "n_search_trees must be >= 0");
  require(p->search_tree_leaf_budget <= 256, "search_tree_leaf_budget must be <= 256");
  require(p->distance_kind >= 0 && p->distance_kind < DK_COUNT, "unknown distance kind");
  require(p->correction >= 0 && p->correction <= CK_ALT_IP, "unknown correction");
  require(p->diversify_prob == p->diversify_prob, "diversify_prob must not be NaN");
  require(p->pruning_degree_multiplier > 0.f, "pruning_degree_multiplier must be positive");
  require(p->precision == RINND_PRECISION_FP32 || p->precision == RINND_PRECISION_BF16, "unknown precision");
  require(p->join_tuning >= RINND_TUNE_TABLE && p->join_tuning <= RINND_TUNE_RETUNE, "unknown join_tuning mode");
}

// The index from its sorted kNN rows (ids local to the index, raw distances):
// diversified CSR (index.rs:656-666) on the original order, corrected neighbor
// distances (:669-673), vertex order = the first retained tree's leaf order and
// the rows gathered in it (:679-715), search trees.  X0 = the index's rows in
// original order (N x Dp); ix->forest holds the trees (perm: tree t's leaf
// order at t * N), of which the first n_search_trees are kept.  Runs on ix->st
// and synchronizes it.
void finish_index(rinnd_index* ix, const float* X0, DVec<int32_t>&& knn_idx, DVec<float>&& knn_raw,
                  TempStorage& tmp) {
  const rinnd_build_params* pin = &ix->p;
  cudaStream_t st = ix->st;
  const int N = (int)ix->N, D = ix->D, Dp = ix->Dp, k = ix->k;
  // diversified CSR (index.rs:656-666) on the original order
  float min_d = 0.f;
  build_search_graph(knn_idx.p, knn_raw.p, X0, N, k, D, Dp, ix->kind, pin->pruning_degree_multiplier, st,
                     tmp, ix->graph_orig, &min_d, pin->diversify_prob, pin->random_seed);
  ix->min_distance = min_d;
  // corrected neighbor distances (index.rs:669-673)
  apply_correction_dev(knn_raw.p, (int64_t)N * k, ix->corr, st);
  ix->knn_idx = std::move(knn_idx);
  ix->knn_dist = std::move(knn_raw);
  // vertex order = first retained tree's leaf order (index.rs:679-715)
  ix->n_search_trees = std::min(std::max(pin->n_search_trees, 0), std::max(pin->n_trees, 0));
  ix->vertex_order.alloc((size_t)N, st);
  if (ix->n_search_trees > 0) {
    RINND_CUDA(cudaMemcpyAsync(ix->vertex_order.p, ix->forest.perm.p, sizeof(int32_t) * N,
                               cudaMemcpyDeviceToDevice, st));
  } else {
    k_iota<<<grid_for(N, 256), 256, 0, st>>>(ix->vertex_order.p, N);
    RINND_LAUNCH_CHECK();
  }
  ix->inverse.alloc((size_t)N, st);
  invert_permutation(ix->vertex_order.p, N, ix->inverse.p, st);
  ix->X.alloc((size_t)N * Dp, st);
  gather_rows(X0, ix->vertex_order.p, N, Dp, ix->X.p, st);
  reorder_csr(ix->graph_orig, ix->vertex_order.p, ix->inverse.p, st, tmp, ix->graph_int);
  if (ix->n_search_trees > 0) {
    long long tot = (long long)ix->n_search_trees * N;
    ix->tree_idx.alloc((size_t)tot, st);
    k_tree_idx<<<grid_for(tot, 256, 148 * 64), 256, 0, st>>>(ix->forest.perm.p, ix->inverse.p, tot,
                                                              ix->tree_idx.p);
    RINND_LAUNCH_CHECK();
    std::vector<int32_t> roots(ix->n_search_trees);
    for (int t = 0; t < ix->n_search_trees; ++t) roots[t] = t;
    ix->tree_roots.alloc(roots.size(), st);
    ix->tree_roots.from_host(roots.data(), roots.size());
  }
  ix->forest.perm.release();
  ix->forest.leaves.release();
  ix->search_stats.alloc(8, st);
  ix->search_stats.fill_bytes(0);
  RINND_CUDA(cudaStreamSynchronize(st));
}

void build_impl(const float* data, bool on_device, int64_t n, int d, int64_t ld,
                const rinnd_build_params* pin, cudaStream_t user_st, rinnd_index** out) {
  require(out != nullptr, "out must not be null");
  require(data != nullptr, "data must not be null");
  validate_params(pin, n, d);
  require(ld >= d, "row stride must be >= dimension");
  ensure_device(pin->device);
  double t_start = now_ms();
  std::unique_ptr<rinnd_index> ix(new rinnd_index());
  ix->device = pin->device;
  ix->p = *pin;
  if (user_st) {
    ix->st = user_st;
    ix->own_stream = false;
  } else {
    RINND_CUDA(cudaStreamCreateWithFlags(&ix->st, cudaStreamNonBlocking));
  }
  cudaStream_t st = ix->st;
  const unsigned long long launches0 = launch_counter();
  const int N = (int)n, D = d, Dp = round_up(d, 4), k = pin->n_neighbors;
  ix->N = n;
  ix->D = D;
  ix->Dp = Dp;
  ix->k = k;
  ix->kind = pin->distance_kind;
  ix->corr = pin->correction;
  ix->normalize = pin->normalize != 0;
  // index.rs:617-625 defaults
  int leaf_size = pin->leaf_size > 0 ? pin->leaf_size : std::max(60, std::min(5 * k, 256));
  int max_cand = pin->max_candidates > 0 ? pin->max_candidates : std::min(k, 60);
  int n_iters = pin->n_iters > 0 ? pin->n_iters : std::max(5, (int)std::ceil(std::log2((double)N)));
  int c = std::min(std::min(max_cand, 60), k);  // nndescent/mod.rs:89
  ix->p.leaf_size = leaf_size;
  ix->p.max_candidates = max_cand;
  ix->p.n_iters = n_iters;
  ix->p.search_tree_leaf_budget = std::max(1, pin->search_tree_leaf_budget);

  // (the BF16 precision form adds its BF16 copy of the rows and two floats per row)
  reserve_pool(pin->device,
               build_working_set(n, Dp, k, c, pin->n_trees) +
                   (pin->precision == RINND_PRECISION_BF16 ? (size_t)n * (round_up(d, 16) * 2 + 8) : 0),
               st);
  TempStorage tmp;
  DVec<float> X0;
  load_rows(data, on_device, n, d, ld, Dp, X0, st);
  if (ix->normalize) normalize_rows(X0.p, n, D, Dp, st);
  KnnState ks;
  ks.precision = pin->precision;
  if (kind_uses_norms(ix->kind)) {
    ks.norms.alloc((size_t)N, st);
    compute_norms(X0.p, N, D, Dp, ks.norms.p, st);
  }
  RINND_CUDA(cudaStreamSynchronize(st));
  double t0 = now_ms();
  build_forest(X0.p, N, D, Dp, std::max(pin->n_trees, 0), leaf_size, pin->angular != 0, 200,
               pin->random_seed, st, tmp, ix->forest);
  RINND_CUDA(cudaStreamSynchronize(st));
  double t1 = now_ms();
  knn_init(ks, N, k, c, st);
  leaf_init(ks, ix->forest, X0.p, D, Dp, ix->kind, st);
  RINND_CUDA(cudaStreamSynchronize(st));
  double t2 = now_ms();
  bool tile_tuned = false;
  choose_join_tile(ks, X0.p, D, Dp, ix->kind, pin->random_seed, pin->join_tuning, st, &tile_tuned);
  const size_t conv = (size_t)(pin->delta * (float)k * (float)N);  // mod.rs:157
  uint64_t pairs_total = 0, pushes_total = 0, rows_total = 0;
  double ms_cand = 0, ms_join = 0, ms_join_kernel = 0;
  uint64_t join_launches = 0, join_updates = 0;
  int join_form = RINND_JOIN_CHUNKED_FP32;
  int iters = 0;
  for (int it = 0; it < n_iters; ++it) {
    iters = it + 1;
    double a = now_ms();
    build_candidates(ks, pin->random_seed, it, st);
    RINND_CUDA(cudaStreamSynchronize(st));
    double b = now_ms();
    JoinStats js = local_join(ks, X0.p, D, Dp, ix->kind, st);
    double e = now_ms();
    ms_cand += b - a;
    ms_join += e - b;
    ms_join_kernel += js.kernel_ms;
    join_launches += (uint64_t)js.launches;
    join_updates += js.appended;
    join_form = js.form;
    pairs_total += js.pairs;
    pushes_total += js.changes;
    rows_total += js.rows;
    if (pin->verbose)
      std::printf("Iteration %d: %llu updates (%llu pairs, %llu rows, %llu buffered of %llu, %d join launches "
                  "%.3f ms, join step %.3f ms)\n",
                  it + 1, js.changes, js.pairs, js.rows, js.updates, js.appended, js.launches, js.kernel_ms,
                  js.total_ms);
    if ((size_t)js.changes <= conv) break;
  }
  double t3 = now_ms();
  // sorted kNN rows (index.rs:653)
  DVec<int32_t> knn_idx((size_t)N * k, st);
  DVec<float> knn_raw((size_t)N * k, st);
  finalize_knn(ks, knn_idx.p, knn_raw.p, st);
  unsigned long long hc[4];
  RINND_CUDA(cudaMemcpyAsync(hc, ks.counters.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
  const JoinTile tile = ks.tile;
  ks = KnnState();  // release heap and candidate rows
  RINND_CUDA(cudaStreamSynchronize(st));
  double t4 = now_ms();
  finish_index(ix.get(), X0.p, std::move(knn_idx), std::move(knn_raw), tmp);
  X0.release();
  double t5 = now_ms();
  rinnd_build_info& inf = ix->info;
  inf.iterations = iters;
  inf.forest_levels = ix->forest.levels;
  inf.n_leaves = ix->forest.n_leaves;
  inf.ms_forest = t1 - t0;
  inf.ms_leaf_init = t2 - t1;
  inf.ms_iterations = t3 - t2;
  inf.ms_candidates = ms_cand;
  inf.ms_join = ms_join;
  inf.ms_sort = t4 - t3;
  inf.ms_graph = t5 - t4;
  inf.ms_total = t5 - t_start;
  inf.pairs_evaluated = pairs_total;
  inf.join_rows_gathered = rows_total;
  inf.ms_join_kernel = ms_join_kernel;
  inf.join_kernel_launches = join_launches;
  inf.join_updates = join_updates;
  inf.join_form = join_form;
  inf.kernel_launches = launch_counter() - launches0;
  inf.pushes_accepted = pushes_total;
  inf.push_contention = hc[1];
  inf.search_graph_nnz = ix->graph_orig.nnz;
  inf.min_distance = ix->min_distance;
  inf.group_items = 1;
  inf.join_tile_stages = tile.nstage;
  inf.join_tile_rows = tile.jb;
  inf.join_tile_ctas_per_sm = tile.per_sm;
  inf.join_tile_tuned = tile_tuned ? 1 : 0;
  *out = ix.release();
}

// ---- grouped batched build --------------------------------------------------
// rinnd_build_many puts indices that share the shape of their NN-Descent state
// (device, d, metric, normalization, tree kind, k, candidate-list length, leaf
// size, precision) into groups and builds each group's NN-Descent as ONE set of
// device rows: one forest pass (every index's trees are root segments of the
// same level-synchronous split), one leaf initialization, and per iteration one
// candidate pass and one join whose persistent CTAs walk the vertices of all the
// group's indices.  Each index keeps its own delta test and iteration cap: its
// rows are frozen (sample no candidates) once it stops, so its graph is the one
// its own NN-Descent run would produce from the same trees.  Random streams are
// keyed by the group's first index's seed and the rows' positions in the group.
// The search graph, reorder and search trees are then made per index.

// Parameters a build resolves from its inputs (index.rs:617-625, nndescent/mod.rs:89).
struct Resolved {
  int leaf_size, max_cand, n_iters, c;
};
Resolved resolve_params(const rinnd_build_params* p, int64_t n) {
  const int k = p->n_neighbors;
  Resolved r;
  r.leaf_size = p->leaf_size > 0 ? p->leaf_size : std::max(60, std::min(5 * k, 256));
  r.max_cand = p->max_candidates > 0 ? p->max_candidates : std::min(k, 60);
  r.n_iters = p->n_iters > 0 ? p->n_iters : std::max(5, (int)std::ceil(std::log2((double)n)));
  r.c = std::min(std::min(r.max_cand, 60), k);
  return r;
}

struct BatchMember {
  int32_t item;                 // position in the caller's batch
  const rinnd_batch_item* it;
  Resolved r;
};

struct GroupKey {
  int device, d, kind, normalize, angular, k, c, leaf_size, precision;
  bool operator<(const GroupKey& o) const {
    const int a[9] = {device, d, kind, normalize, angular, k, c, leaf_size, precision};
    const int b[9] = {o.device, o.d, o.kind, o.normalize, o.angular, o.k, o.c, o.leaf_size, o.precision};
    return std::lexicographical_compare(a, a + 9, b, b + 9);
  }
};

// row -> item by binary search over the item offsets
__global__ void k_row_items(const int64_t* off, int n_items, int N, int32_t* out) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (off[mid] <= r) lo = mid;
      else hi = mid - 1;
    }
    out[r] = lo;
  }
}

// group row ids -> ids local to the row's index
__global__ void k_localize_ids(int32_t* idx, long long total, int k, const int32_t* row_item, const int64_t* off) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int32_t id = idx[e];
    if (id >= 0) idx[e] = id - (int32_t)off[row_item[e / k]];
  }
}

// Copies the nodes src[0..cnt) of the group forest into an index's own forest
// (point ids made local); children were remapped on the host.
__global__ void k_gather_nodes(const int32_t* src, long long cnt, int Dp, const float* offsets, const float* hp,
                               const int32_t* pivots, int32_t base, float* o_offsets, float* o_hp,
                               int32_t* o_pivots) {
  const long long total = cnt * (long long)Dp;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long j = e / Dp;
    const int t = (int)(e - j * Dp);
    const int32_t s = src[j];
    o_hp[e] = hp[(size_t)s * Dp + t];
    if (t == 0) {
      o_offsets[j] = offsets[s];
      const int32_t p0 = pivots[2 * (size_t)s], p1 = pivots[2 * (size_t)s + 1];
      o_pivots[2 * j] = p0 >= 0 ? p0 - base : -1;
      o_pivots[2 * j + 1] = p1 >= 0 ? p1 - base : -1;
    }
  }
}

// tree t's leaf order of the index's rows: perm[t * Ntot + base + p] - base
__global__ void k_local_perm(const int32_t* perm, long long Ntot, int T, int32_t base, int n, int32_t* out) {
  const long long total = (long long)T * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / n, p = e - t * n;
    out[e] = perm[t * Ntot + base + p] - base;
  }
}

// The index's own forest from the group forest (children on the host): its
// first `keep` trees renumbered with roots 0..keep-1 followed by the other
// nodes in breadth-first order; leaf bounds and pivots made local.  levels and
// n_leaves count all `trees` trees of the index.
void extract_forest(const Forest& g, const std::vector<int32_t>& ch, int n_items, int item, int trees, int keep,
                    int64_t base, int n, cudaStream_t st, Forest& out) {
  std::vector<int32_t> src, lch;
  std::vector<std::pair<int32_t, int>> q;  // (group node, depth)
  int64_t n_leaves = 0;
  int levels = 0;
  for (int t = 0; t < trees; ++t) {
    const bool kept = t < keep;
    q.clear();
    q.push_back({(int32_t)(t * n_items + item), 0});
    if (kept) {
      // roots first: reserve slot t
      if (src.size() < (size_t)keep) src.resize((size_t)keep, -1);
      src[(size_t)t] = q[0].first;
    }
    for (size_t h = 0; h < q.size(); ++h) {
      const int32_t nd = q[h].first;
      const int dep = q[h].second;
      const int32_t c0 = ch[2 * (size_t)nd], c1 = ch[2 * (size_t)nd + 1];
      if (c1 <= 0) {
        ++n_leaves;
        continue;
      }
      levels = std::max(levels, dep + 1);
      q.push_back({c0, dep + 1});
      q.push_back({c1, dep + 1});
    }
    if (!kept) continue;
    for (size_t h = 1; h < q.size(); ++h) src.push_back(q[h].first);
  }
  // group node -> local id
  std::vector<std::pair<int32_t, int32_t>> map;
  map.reserve(src.size());
  for (size_t j = 0; j < src.size(); ++j) map.push_back({src[j], (int32_t)j});
  std::sort(map.begin(), map.end());
  auto local = [&](int32_t nd) {
    auto itr = std::lower_bound(map.begin(), map.end(), std::make_pair(nd, (int32_t)INT32_MIN));
    return itr->second;
  };
  lch.resize(2 * src.size());
  for (size_t j = 0; j < src.size(); ++j) {
    const int32_t c0 = ch[2 * (size_t)src[j]], c1 = ch[2 * (size_t)src[j] + 1];
    if (c1 <= 0) {  // leaf: {-start, -end} within the tree's slice
      lch[2 * j] = c0 + (int32_t)base;
      lch[2 * j + 1] = c1 + (int32_t)base;
    } else {
      lch[2 * j] = local(c0);
      lch[2 * j + 1] = local(c1);
    }
  }
  const long long cnt = (long long)src.size();
  out.T = keep;
  out.N = n;
  out.Dp = g.Dp;
  out.n_nodes = cnt;
  out.n_leaves = n_leaves;
  out.levels = levels;
  out.max_leaf = g.max_leaf;
  out.children.alloc(std::max<size_t>(lch.size(), 2), st);
  out.offsets.alloc(std::max<size_t>(src.size(), 1), st);
  out.pivots.alloc(std::max<size_t>(2 * src.size(), 2), st);
  out.hyperplanes.alloc(std::max<size_t>(src.size(), 1) * (size_t)g.Dp, st);
  out.perm.alloc(std::max<size_t>((size_t)keep * n, 1), st);
  if (cnt > 0) {
    out.children.from_host(lch.data(), lch.size());
    DVec<int32_t> d_src((size_t)cnt, st);
    d_src.from_host(src.data(), (size_t)cnt);
    k_gather_nodes<<<grid_for(cnt * g.Dp, 256, 148 * 32), 256, 0, st>>>(
        d_src.p, cnt, g.Dp, g.offsets.p, g.hyperplanes.p, g.pivots.p, (int32_t)base, out.offsets.p,
        out.hyperplanes.p, out.pivots.p);
    RINND_LAUNCH_CHECK();
    k_local_perm<<<grid_for((long long)keep * n, 256, 148 * 32), 256, 0, st>>>(g.perm.p, g.N, keep, (int32_t)base,
                                                                            n, out.perm.p);
    RINND_LAUNCH_CHECK();
    RINND_CUDA(cudaStreamSynchronize(st));  // host arrays and d_src are released at scope exit
  }
}

// Builds one group; out[m.item] / codes[m.item] / msgs[m.item] receive each
// member's index or error.
void build_group(const std::vector<BatchMember>& mem, bool capture, rinnd_index** out, std::vector<int32_t>& codes,
                 std::vector<std::string>& msgs) {
  const rinnd_build_params& gp = *mem[0].it->params;
  const int n_items = (int)mem.size();
  auto fail_all = [&](int code) {
    for (const BatchMember& m : mem) {
      codes[(size_t)m.item] = code;
      msgs[(size_t)m.item] = g_last_error;
    }
  };
  // the group's rows and NN-Descent state live in this scope
  std::vector<int64_t> off((size_t)n_items + 1, 0);
  for (int i = 0; i < n_items; ++i) off[(size_t)i + 1] = off[(size_t)i] + mem[(size_t)i].it->n;
  const int64_t Ntot = off.back();
  const int D = mem[0].it->d, Dp = round_up(D, 4), k = gp.n_neighbors;
  const Resolved R0 = mem[0].r;
  StreamGuard sg;
  cudaStream_t st = sg.s;
  TempStorage tmp;
  DVec<float> X0;
  DVec<int32_t> gidx;
  DVec<float> graw;
  DVec<int64_t> d_off;
  DVec<int32_t> row_item;
  Forest gf;
  std::vector<int32_t> iters((size_t)n_items, 0);
  std::vector<int32_t> ch;
  double ms_forest = 0, ms_leaf = 0, ms_iters = 0, ms_cand = 0, ms_join = 0, ms_join_kernel = 0, ms_sort = 0;
  uint64_t pairs_total = 0, pushes_total = 0, rows_total = 0, join_launches = 0, join_updates = 0;
  unsigned long long hc[4] = {0, 0, 0, 0};
  int join_form = RINND_JOIN_CHUNKED_FP32;
  JoinTile tile;
  bool tile_tuned = false;
  const unsigned long long launches0 = launch_counter();
  const double t_start = now_ms();
  int code = guarded([&] {
    ensure_device(gp.device);
    require(Ntot < (int64_t)INT32_MAX - 1, "a group holds at most 2^31-2 points");
    const int N = (int)Ntot;
    int T = 0;
    for (const BatchMember& m : mem) T = std::max(T, std::max(m.it->params->n_trees, 0));
    reserve_pool(gp.device,
                 build_working_set(Ntot, Dp, k, R0.c, T) +
                     (gp.precision == RINND_PRECISION_BF16 ? (size_t)Ntot * (round_up(D, 16) * 2 + 8) : 0),
                 st);
    X0.alloc((size_t)Ntot * Dp, st);
    if (Dp != D) X0.fill_bytes(0);
    for (int i = 0; i < n_items; ++i) {
      const rinnd_batch_item& it = *mem[(size_t)i].it;
      const int64_t ld = it.ld > 0 ? it.ld : it.d;
      RINND_CUDA(cudaMemcpy2DAsync(X0.p + (size_t)off[(size_t)i] * Dp, sizeof(float) * Dp, it.data,
                                   sizeof(float) * ld, sizeof(float) * D, (size_t)it.n,
                                   it.data_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    }
    if (gp.normalize) normalize_rows(X0.p, Ntot, D, Dp, st);
    KnnState ks;
    ks.precision = gp.precision;
    if (kind_uses_norms(gp.distance_kind)) {
      ks.norms.alloc((size_t)N, st);
      compute_norms(X0.p, N, D, Dp, ks.norms.p, st);
    }
    d_off.alloc(off.size(), st);
    d_off.from_host(off.data(), off.size());
    row_item.alloc((size_t)N, st);
    k_row_items<<<grid_for(N, 256, 148 * 16), 256, 0, st>>>(d_off.p, n_items, N, row_item.p);
    RINND_LAUNCH_CHECK();
    RINND_CUDA(cudaStreamSynchronize(st));
    double t0 = now_ms();
    ForestItems fi;
    fi.off = off;
    for (const BatchMember& m : mem) fi.trees.push_back(std::max(m.it->params->n_trees, 0));
    build_forest(X0.p, N, D, Dp, T, R0.leaf_size, gp.angular != 0, 200, gp.random_seed, st, tmp, gf, &fi);
    RINND_CUDA(cudaStreamSynchronize(st));
    double t1 = now_ms();
    knn_init(ks, N, k, R0.c, st);
    leaf_init(ks, gf, X0.p, D, Dp, gp.distance_kind, st);
    ks.row_item.alloc((size_t)N, st);
    RINND_CUDA(cudaMemcpyAsync(ks.row_item.p, row_item.p, sizeof(int32_t) * N, cudaMemcpyDeviceToDevice, st));
    ks.item_active.alloc((size_t)n_items, st);
    ks.item_changes.alloc((size_t)n_items, st);
    RINND_CUDA(cudaStreamSynchronize(st));
    double t2 = now_ms();
    choose_join_tile(ks, X0.p, D, Dp, gp.distance_kind, gp.random_seed, gp.join_tuning, st, &tile_tuned);
    std::vector<uint8_t> active((size_t)n_items, 1);
    std::vector<unsigned long long> changes((size_t)n_items, 0);
    int max_iters = 0;
    for (const BatchMember& m : mem) max_iters = std::max(max_iters, m.r.n_iters);
    IterationGraph ig;
    for (int it = 0; it < max_iters; ++it) {
      int n_active = 0;
      for (int i = 0; i < n_items; ++i) n_active += active[(size_t)i];
      if (n_active == 0) break;
      RINND_CUDA(cudaMemcpyAsync(ks.item_active.p, active.data(), (size_t)n_items, cudaMemcpyHostToDevice, st));
      JoinStats js;
      const double a = now_ms();
      if (capture) {  // candidates + join + applications as one CUDA graph
        js = iteration_graph(ks, ig, gp.random_seed, it, X0.p, D, Dp, gp.distance_kind, st, changes.data(),
                             n_items);
        ms_join += now_ms() - a;
      } else {
        ks.item_changes.fill_bytes(0);
        build_candidates(ks, gp.random_seed, it, st);
        RINND_CUDA(cudaStreamSynchronize(st));
        const double b = now_ms();
        js = local_join(ks, X0.p, D, Dp, gp.distance_kind, st);
        const double e = now_ms();
        RINND_CUDA(cudaMemcpyAsync(changes.data(), ks.item_changes.p, sizeof(unsigned long long) * n_items,
                                   cudaMemcpyDeviceToHost, st));
        RINND_CUDA(cudaStreamSynchronize(st));
        ms_cand += b - a;
        ms_join += e - b;
      }
      ms_join_kernel += js.kernel_ms;
      join_launches += (uint64_t)js.launches;
      join_updates += js.appended;
      join_form = js.form;
      pairs_total += js.pairs;
      pushes_total += js.changes;
      rows_total += js.rows;
      if (gp.verbose)
        std::printf("Group of %d: iteration %d, %d indices active, %llu updates (%llu pairs)\n", n_items, it + 1,
                    n_active, js.changes, js.pairs);
      for (int i = 0; i < n_items; ++i) {
        if (!active[(size_t)i]) continue;
        const BatchMember& m = mem[(size_t)i];
        iters[(size_t)i] = it + 1;
        // mod.rs:157 delta test per index
        const size_t conv = (size_t)(m.it->params->delta * (float)k * (float)m.it->n);
        if ((size_t)changes[(size_t)i] <= conv || it + 1 >= m.r.n_iters) active[(size_t)i] = 0;
      }
    }
    double t3 = now_ms();
    gidx.alloc((size_t)N * k, st);
    graw.alloc((size_t)N * k, st);
    finalize_knn(ks, gidx.p, graw.p, st);
    k_localize_ids<<<grid_for((long long)N * k, 256, 148 * 32), 256, 0, st>>>(gidx.p, (long long)N * k, k,
                                                                             row_item.p, d_off.p);
    RINND_LAUNCH_CHECK();
    RINND_CUDA(cudaMemcpyAsync(hc, ks.counters.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
    tile = ks.tile;
    ks = KnnState();
    ch.resize(2 * (size_t)gf.n_nodes);
    gf.children.to_host(ch.data(), ch.size());
    gf.leaves.release();
    RINND_CUDA(cudaStreamSynchronize(st));
    double t4 = now_ms();
    ms_forest = t1 - t0;
    ms_leaf = t2 - t1;
    ms_iters = t3 - t2;
    ms_sort = t4 - t3;
  });
  if (code != RINND_OK) {
    fail_all(code);
    return;
  }
  // per index: kNN rows, own forest, search graph, reorder, trees
  for (int i = 0; i < n_items; ++i) {
    const BatchMember& m = mem[(size_t)i];
    const rinnd_build_params* pin = m.it->params;
    const int32_t n = (int32_t)m.it->n;
    const double ti = now_ms();
    codes[(size_t)m.item] = guarded([&] {
      std::unique_ptr<rinnd_index> ix(new rinnd_index());
      ix->device = pin->device;
      ix->p = *pin;
      ix->p.leaf_size = m.r.leaf_size;
      ix->p.max_candidates = m.r.max_cand;
      ix->p.n_iters = m.r.n_iters;
      ix->p.search_tree_leaf_budget = std::max(1, pin->search_tree_leaf_budget);
      RINND_CUDA(cudaStreamCreateWithFlags(&ix->st, cudaStreamNonBlocking));
      cudaStream_t is = ix->st;
      ix->N = n;
      ix->D = D;
      ix->Dp = Dp;
      ix->k = k;
      ix->kind = pin->distance_kind;
      ix->corr = pin->correction;
      ix->normalize = pin->normalize != 0;
      const int64_t base = off[(size_t)i];
      DVec<int32_t> kidx((size_t)n * k, is);
      DVec<float> kraw((size_t)n * k, is);
      RINND_CUDA(cudaMemcpyAsync(kidx.p, gidx.p + (size_t)base * k, sizeof(int32_t) * (size_t)n * k,
                                 cudaMemcpyDeviceToDevice, is));
      RINND_CUDA(cudaMemcpyAsync(kraw.p, graw.p + (size_t)base * k, sizeof(float) * (size_t)n * k,
                                 cudaMemcpyDeviceToDevice, is));
      const int trees = std::max(pin->n_trees, 0);
      const int keep = std::min(std::max(pin->n_search_trees, 0), trees);
      extract_forest(gf, ch, n_items, i, trees, keep, base, n, is, ix->forest);
      TempStorage itmp;
      finish_index(ix.get(), X0.p + (size_t)base * Dp, std::move(kidx), std::move(kraw), itmp);
      rinnd_build_info& inf = ix->info;
      inf.iterations = iters[(size_t)i];
      inf.forest_levels = ix->forest.levels;
      inf.n_leaves = ix->forest.n_leaves;
      inf.ms_forest = ms_forest;
      inf.ms_leaf_init = ms_leaf;
      inf.ms_iterations = ms_iters;
      inf.ms_candidates = ms_cand;
      inf.ms_join = ms_join;
      inf.ms_sort = ms_sort;
      inf.ms_graph = now_ms() - ti;
      inf.ms_total = now_ms() - t_start;
      inf.pairs_evaluated = pairs_total;
      inf.join_rows_gathered = rows_total;
      inf.ms_join_kernel = ms_join_kernel;
      inf.join_kernel_launches = join_launches;
      inf.join_updates = join_updates;
      inf.join_form = join_form;
      inf.kernel_launches = launch_counter() - launches0;
      inf.pushes_accepted = pushes_total;
      inf.push_contention = hc[1];
      inf.search_graph_nnz = ix->graph_orig.nnz;
      inf.min_distance = ix->min_distance;
      inf.group_items = n_items;
      inf.join_tile_stages = tile.nstage;
      inf.join_tile_rows = tile.jb;
      inf.join_tile_ctas_per_sm = tile.per_sm;
      inf.join_tile_tuned = tile_tuned ? 1 : 0;
      out[m.item] = ix.release();
    });
    if (codes[(size_t)m.item] != RINND_OK) msgs[(size_t)m.item] = g_last_error;
  }
}

void check_index(const rinnd_index* idx) { require(idx != nullptr, "index must not be null"); }

void query_impl(rinnd_index* ix, const float* q, bool on_device, int64_t nq, int64_t ld, int k, float eps,
                uint64_t qid_base, int32_t* out_idx, float* out_dist, bool out_device, cudaStream_t user_st) {
  check_index(ix);
  require(nq >= 0, "number of queries must be >= 0");
  require(k >= 1 && k <= 256, "k must be in [1, 256]");
  if (nq == 0) return;
  require(q != nullptr && out_idx != nullptr && out_dist != nullptr, "query/output pointers must not be null");
  require(!ix->fp32_released, "FP32 search is unavailable because FP32 vector data was released");
  std::lock_guard<std::mutex> lock(ix->mu);
  RINND_CUDA(cudaSetDevice(ix->device));
  cudaStream_t st = user_st ? user_st : ix->st;
  DVec<float> Q;
  load_rows(q, on_device, nq, ix->D, ld, ix->Dp, Q, st);
  if (ix->normalize) normalize_rows(Q.p, nq, ix->D, ix->Dp, st);
  SearchIndex sv = ix->search_view();
  if (out_device) {
    greedy_search(sv, Q.p, (int)nq, k, eps, qid_base, out_idx, out_dist, st, ix->search_stats.p);
  } else {
    DVec<int32_t> oi((size_t)nq * k, st);
    DVec<float> od((size_t)nq * k, st);
    greedy_search(sv, Q.p, (int)nq, k, eps, qid_base, oi.p, od.p, st, ix->search_stats.p);
    oi.to_host(out_idx, (size_t)nq * k);
    od.to_host(out_dist, (size_t)nq * k);
    RINND_CUDA(cudaStreamSynchronize(st));
  }
  Q.release();
}

}  // namespace

extern "C" {

int rinnd_params_default(rinnd_build_params* p) {
  if (!p) return fail(RINND_ERR_INVALID, "params must not be null");
  std::memset(p, 0, sizeof(*p));
  p->n_neighbors = 30;  // index.rs:475-494
  p->n_trees = 8;
  p->n_search_trees = 1;
  p->search_tree_leaf_budget = 1;
  p->delta = 0.001f;
  p->random_seed = 42;
  p->diversify_prob = 1.0f;
  p->pruning_degree_multiplier = 1.5f;
  p->distance_kind = RINND_DIST_SQEUCLIDEAN;
  p->correction = RINND_CORR_SQRT;
  return RINND_OK;
}

int rinnd_build(const float* data, int64_t n, int32_t d, const rinnd_build_params* p, rinnd_index** out) {
  return guarded([&] { build_impl(data, false, n, d, d, p, nullptr, out); });
}

int rinnd_build_device(const float* d_data, int64_t n, int32_t d, int64_t ld, const rinnd_build_params* p,
                       rinnd_index** out) {
  return guarded([&] { build_impl(d_data, true, n, d, ld, p, nullptr, out); });
}

int rinnd_build_on_stream(const float* data, int32_t data_on_device, int64_t n, int32_t d, int64_t ld,
                          const rinnd_build_params* p, void* stream, rinnd_index** out) {
  return guarded([&] {
    build_impl(data, data_on_device != 0, n, d, ld, p, reinterpret_cast<cudaStream_t>(stream), out);
  });
}

int rinnd_batch_options_default(rinnd_batch_options* o) {
  if (!o) return fail(RINND_ERR_INVALID, "options must not be null");
  std::memset(o, 0, sizeof(*o));
  o->grouped = 1;
  o->max_group_points = 8 << 20;
  o->capture_iterations = 1;
  return RINND_OK;
}

int rinnd_build_many_ex(const rinnd_batch_item* items, int32_t n_items, const rinnd_batch_options* opt,
                        rinnd_index** out, int32_t* status) {
  if (n_items < 0 || (n_items > 0 && (!items || !out)))
    return fail(RINND_ERR_INVALID, "items and out must not be null and n_items >= 0");
  rinnd_batch_options o;
  rinnd_batch_options_default(&o);
  if (opt) o = *opt;
  if (n_items == 0) return RINND_OK;
  for (int32_t i = 0; i < n_items; ++i) out[i] = nullptr;
  std::vector<int32_t> codes((size_t)n_items, RINND_OK);
  std::vector<std::string> msgs((size_t)n_items);
  // validation first: an invalid item fails alone
  std::vector<BatchMember> valid;
  for (int32_t i = 0; i < n_items; ++i) {
    const rinnd_batch_item& it = items[i];
    codes[(size_t)i] = guarded([&] {
      require(it.data != nullptr && it.params != nullptr, "batch item data and params must not be null");
      validate_params(it.params, it.n, it.d);
      require((it.ld > 0 ? it.ld : it.d) >= it.d, "row stride must be >= dimension");
      valid.push_back(BatchMember{i, &it, resolve_params(it.params, it.n)});
    });
    if (codes[(size_t)i] != RINND_OK) msgs[(size_t)i] = g_last_error;
  }
  // tasks: groups of compatible items (or single items), longest first
  struct Task {
    std::vector<BatchMember> mem;
    double cost = 0;
  };
  std::vector<Task> tasks;
  auto cost = [](const BatchMember& m) {
    return (double)m.it->n * (double)std::max(m.it->d, 1) * (double)std::max(m.it->params->n_neighbors, 1);
  };
  if (o.grouped) {
    std::map<GroupKey, std::vector<BatchMember>> groups;
    for (const BatchMember& m : valid) {
      const rinnd_build_params& p = *m.it->params;
      GroupKey key{p.device, m.it->d, p.distance_kind, p.normalize != 0, p.angular != 0, p.n_neighbors, m.r.c,
                   m.r.leaf_size, p.precision};
      groups[key].push_back(m);
    }
    const int64_t cap = o.max_group_points > 0 ? o.max_group_points : ((int64_t)INT32_MAX - 2);
    for (auto& kv : groups) {
      std::vector<BatchMember>& v = kv.second;
      std::stable_sort(v.begin(), v.end(), [&](const BatchMember& a, const BatchMember& b) { return cost(a) > cost(b); });
      Task cur;
      int64_t pts = 0;
      for (const BatchMember& m : v) {
        if (!cur.mem.empty() && pts + m.it->n > cap) {
          tasks.push_back(std::move(cur));
          cur = Task();
          pts = 0;
        }
        cur.mem.push_back(m);
        cur.cost += cost(m);
        pts += m.it->n;
      }
      if (!cur.mem.empty()) tasks.push_back(std::move(cur));
    }
  } else {
    for (const BatchMember& m : valid) {
      Task t;
      t.mem.push_back(m);
      t.cost = cost(m);
      tasks.push_back(std::move(t));
    }
  }
  std::stable_sort(tasks.begin(), tasks.end(), [](const Task& a, const Task& b) { return a.cost > b.cost; });
  const int n_tasks = (int)tasks.size();
  const int workers = std::max(1, std::min<int>(o.n_workers > 0 ? o.n_workers : 16, std::max(n_tasks, 1)));
  std::atomic<int32_t> next{0};
  auto work = [&]() {
    for (;;) {
      const int32_t t = next.fetch_add(1);
      if (t >= n_tasks) return;
      const std::vector<BatchMember>& mem = tasks[(size_t)t].mem;
      if (mem.size() == 1) {
        const BatchMember& m = mem[0];
        const rinnd_batch_item& it = *m.it;
        codes[(size_t)m.item] = guarded([&] {
          build_impl(it.data, it.data_on_device != 0, it.n, it.d, it.ld > 0 ? it.ld : it.d, it.params, nullptr,
                     &out[m.item]);
        });
        if (codes[(size_t)m.item] != RINND_OK) msgs[(size_t)m.item] = g_last_error;
      } else {
        build_group(mem, o.capture_iterations != 0, out, codes, msgs);
      }
    }
  };
  std::vector<std::thread> pool;
  for (int w = 1; w < workers; ++w) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  int rc = RINND_OK;
  for (int32_t i = 0; i < n_items; ++i) {
    if (status) status[i] = codes[(size_t)i];
    if (rc == RINND_OK && codes[(size_t)i] != RINND_OK) {
      rc = codes[(size_t)i];
      g_last_error = "batch item " + std::to_string(i) + ": " + msgs[(size_t)i];
    }
  }
  return rc;
}

int rinnd_build_many(const rinnd_batch_item* items, int32_t n_items, int32_t n_workers, rinnd_index** out,
                     int32_t* status) {
  rinnd_batch_options o;
  rinnd_batch_options_default(&o);
  o.n_workers = n_workers;
  return rinnd_build_many_ex(items, n_items, &o, out, status);
}

int rinnd_join_tile_table(int32_t* rows, int32_t cap, int32_t* n_rows) {
  return guarded([&] {
    require(cap >= 0, "cap must be >= 0");
    const std::vector<std::array<int, 8>> t = join_tile_table();
    if (n_rows) *n_rows = (int32_t)t.size();
    if (rows)
      for (size_t i = 0; i < t.size() && (int32_t)i < cap; ++i)
        for (int j = 0; j < 8; ++j) rows[8 * i + j] = t[i][(size_t)j];
  });
}

int rinnd_join_tile_table_clear(void) {
  return guarded([&] { join_tile_table_clear(); });
}

int rinnd_join_tile_set(const int32_t* row) {
  return guarded([&] {
    require(row != nullptr, "row must not be null");
    require(row[2] == 32 || row[2] == 64, "list class must be 32 or 64");
    require(row[3] >= 0 && row[3] <= 2 && (row[4] == 0 || row[4] == 1), "unknown metric class or grouped flag");
    JoinTile t{row[5], row[6], row[7]};
    require((t.nstage == 2 || t.nstage == 3) && (t.jb == 1 || t.jb == 2) && t.per_sm >= 0,
            "stages must be 2 or 3, rows per item 1 or 2, CTAs per SM >= 0");
    require(row[2] == 32 || (t.nstage == 2 && t.jb == 1), "lists longer than 32 run the default shape only");
    require(join_tile_fits(row[2], row[1], t), "the tile shape does not fit shared memory at this dimension");
    join_tile_store(row[0], row[1], row[2], row[3], row[4], t);
  });
}

int rinnd_search_counters(rinnd_index* idx, uint64_t* out, int32_t reset) {
  return guarded([&] {
    check_index(idx);
    require(out != nullptr, "out must not be null");
    RINND_CUDA(cudaSetDevice(idx->device));
    unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    RINND_CUDA(cudaDeviceSynchronize());
    RINND_CUDA(cudaMemcpy(h, idx->search_stats.p, sizeof(h), cudaMemcpyDeviceToHost));
    for (int i = 0; i < 8; ++i) out[i] = h[i];
    if (reset) RINND_CUDA(cudaMemset(idx->search_stats.p, 0, sizeof(h)));
  });
}

int rinnd_search_stats_get(rinnd_index* idx, uint64_t* evaluations, uint64_t* expansions,
                           uint64_t* visited_overflows, int32_t reset) {
  return guarded([&] {
    check_index(idx);
    RINND_CUDA(cudaSetDevice(idx->device));
    unsigned long long h[4] = {0, 0, 0, 0};
    RINND_CUDA(cudaDeviceSynchronize());
    RINND_CUDA(cudaMemcpy(h, idx->search_stats.p, sizeof(h), cudaMemcpyDeviceToHost));
    if (evaluations) *evaluations = h[0];
    if (expansions) *expansions = h[1];
    if (visited_overflows) *visited_overflows = h[2];
    if (reset) RINND_CUDA(cudaMemset(idx->search_stats.p, 0, 8 * sizeof(unsigned long long)));
  });
}

int rinnd_server_params_default(rinnd_server_params* p) {
  if (!p) return fail(RINND_ERR_INVALID, "params must not be null");
  std::memset(p, 0, sizeof(*p));
  p->max_batch_queries = 32768;
  p->max_inflight = 8;
  p->max_k = 256;
  p->max_pending_queries = 1ll << 22;
  return RINND_OK;
}

int rinnd_server_create(rinnd_index* idx, const rinnd_server_params* p, rinnd_server** out) {
  return guarded([&] {
    check_index(idx);
    require(p != nullptr && out != nullptr, "params and out must not be null");
    require(p->max_batch_queries >= 1 && p->max_batch_queries <= (1 << 20), "max_batch_queries must be in [1, 2^20]");
    require(p->max_inflight >= 1 && p->max_inflight <= 64, "max_inflight must be in [1, 64]");
    require(p->max_k >= 1 && p->max_k <= 256, "max_k must be in [1, 256]");
    require(p->max_pending_queries >= p->max_batch_queries, "max_pending_queries must be >= max_batch_queries");
    require(p->quantized || !idx->fp32_released, "FP32 search is unavailable because FP32 vector data was released");
    if (p->quantized) {
      require(idx->encoding >= 0, "a quantized server needs a quantized index (rinnd_quantize)");
      require(!(idx->fp32_released && p->rerank_width > 0),
              "exact reranking is unavailable because FP32 vector data was released");
      require(p->candidate_width >= 0 && p->rerank_width >= 0, "quantized widths must be >= 0");
      require(quantized_width(1, p->candidate_width, p->rerank_width) <= 256, "candidate width must be <= 256");
    }
    ServerIndexView v;
    v.index = idx->search_view();
    v.device = idx->device;
    v.D = idx->D;
    v.Dp = idx->Dp;
    v.normalize = idx->normalize;
    v.quantized = p->quantized != 0;
    v.encoding = idx->encoding;
    v.global_mult = idx->global_mult;
    v.stats = idx->search_stats.p;
    *out = reinterpret_cast<rinnd_server*>(server_create(v, *p));
  });
}

int rinnd_server_submit(rinnd_server* s, const float* queries, int64_t nq, int32_t k, float epsilon,
                        int64_t* request_id) {
  return guarded([&] {
    require(s != nullptr && request_id != nullptr, "server and request_id must not be null");
    Server* sv = reinterpret_cast<Server*>(s);
    require(nq >= 1 && nq <= (int64_t)INT32_MAX, "nq must be >= 1");
    require(queries != nullptr, "queries must not be null");
    const rinnd_server_params& p = server_params(sv);
    require(k >= 1 && k <= p.max_k, "k must be in [1, max_k]");
    if (p.quantized) {
      require(quantized_width(k, p.candidate_width, p.rerank_width) >= k, "quantized candidate width must be at least k");
      require(quantized_width(k, p.candidate_width, p.rerank_width) <= 256, "quantized candidate width must be <= 256");
      require(p.candidate_width == 0 || p.rerank_width == 0 || p.rerank_width >= k,
              "quantized rerank width must be zero or at least k");
    }
    *request_id = server_submit(sv, queries, nq, k, epsilon);
  });
}

int rinnd_server_poll(rinnd_server* s, int64_t request_id, int32_t wait_ms, int32_t* out_idx, float* out_dist,
                      int32_t* done) {
  return guarded([&] {
    require(s != nullptr && done != nullptr, "server and done must not be null");
    *done = server_poll(reinterpret_cast<Server*>(s), request_id, wait_ms, out_idx, out_dist) ? 1 : 0;
  });
}

int rinnd_server_stats_get(rinnd_server* s, rinnd_server_stats* out) {
  return guarded([&] {
    require(s != nullptr && out != nullptr, "server and out must not be null");
    server_stats(reinterpret_cast<Server*>(s), out);
  });
}

int rinnd_server_destroy(rinnd_server* s) {
  return guarded([&] {
    if (s) server_destroy(reinterpret_cast<Server*>(s));
  });
}

int rinnd_kernel_target(int32_t* binary_version, int32_t* ptx_version) {
  return guarded([&] {
    require(binary_version != nullptr, "binary_version must not be null");
    int dev = 0;
    {
      int n = 0;
      cudaError_t e = cudaGetDeviceCount(&n);
      if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw NoDevice("no CUDA device is available: the B200 engine has no CPU fallback");
      }
      RINND_CUDA(cudaGetDevice(&dev));
    }
    cudaFuncAttributes a{};
    RINND_CUDA(cudaFuncGetAttributes(&a, reinterpret_cast<const void*>(k_iota)));
    *binary_version = a.binaryVersion;
    if (ptx_version) *ptx_version = a.ptxVersion;
  });
}

int rinnd_kernel_launches(uint64_t* count) {
  return guarded([&] {
    require(count != nullptr, "count must not be null");
    *count = launch_counter();
  });
}

int rinnd_free(rinnd_index* idx) {
  return guarded([&] {
    if (idx) {
      cudaSetDevice(idx->device);
      cudaStream_t st = idx->st;
      bool own = idx->own_stream;
      delete idx;  // device buffers are freed stream-ordered on st
      if (st && own) cudaStreamDestroy(st);
    }
  });
}

int rinnd_build_info_get(const rinnd_index* idx, rinnd_build_info* info) {
  return guarded([&] {
    check_index(idx);
    require(info != nullptr, "info must not be null");
    *info = idx->info;
  });
}

int rinnd_index_shape(const rinnd_index* idx, int64_t* n, int32_t* d, int32_t* k) {
  return guarded([&] {
    check_index(idx);
    if (n) *n = idx->N;
    if (d) *d = idx->D;
    if (k) *k = idx->k;
  });
}

int rinnd_query(rinnd_index* idx, const float* queries, int64_t nq, int32_t k, float epsilon,
                int32_t* out_idx, float* out_dist) {
  return guarded([&] {
    check_index(idx);
    query_impl(idx, queries, false, nq, idx->D, k, epsilon, 0, out_idx, out_dist, false, nullptr);
  });
}

int rinnd_query_one(rinnd_index* idx, const float* query, int32_t k, float epsilon, int32_t* out_idx,
                    float* out_dist) {
  return guarded([&] {
    check_index(idx);
    query_impl(idx, query, false, 1, idx->D, k, epsilon, 0, out_idx, out_dist, false, nullptr);
  });
}

int rinnd_query_device(rinnd_index* idx, const float* d_queries, int64_t nq, int64_t ld, int32_t k,
                       float epsilon, uint64_t qid_base, int32_t* d_out_idx, float* d_out_dist, void* stream) {
  return guarded([&] {
    check_index(idx);
    require(ld >= idx->D, "query row stride must be >= dimension");
    query_impl(idx, d_queries, true, nq, ld, k, epsilon, qid_base, d_out_idx, d_out_dist, true,
               reinterpret_cast<cudaStream_t>(stream));
  });
}

int rinnd_neighbor_graph(const rinnd_index* idx, int32_t* out_idx, float* out_dist) {
  return guarded([&] {
    check_index(idx);
    RINND_CUDA(cudaSetDevice(idx->device));
    size_t nk = (size_t)idx->N * idx->k;
    if (out_idx) idx->knn_idx.to_host(out_idx, nk);
    if (out_dist) idx->knn_dist.to_host(out_dist, nk);
    RINND_CUDA(cudaStreamSynchronize(idx->st));
  });
}

int rinnd_search_graph_nnz(const rinnd_index* idx, int64_t* nnz) {
  return guarded([&] {
    check_index(idx);
    require(nnz != nullptr, "nnz must not be null");
    *nnz = idx->graph_orig.nnz;
  });
}

int rinnd_search_graph(const rinnd_index* idx, int32_t* indptr, int32_t* indices, float* min_distance) {
  return guarded([&] {
    check_index(idx);
    RINND_CUDA(cudaSetDevice(idx->device));
    if (indptr) idx->graph_orig.indptr.to_host(indptr, (size_t)idx->N + 1);
    if (indices) idx->graph_orig.indices.to_host(indices, (size_t)idx->graph_orig.nnz);
    if (min_distance) *min_distance = idx->min_distance;
    RINND_CUDA(cudaStreamSynchronize(idx->st));
  });
}

int rinnd_vertex_order(const rinnd_index* idx, int32_t* out) {
  return guarded([&] {
    check_index(idx);
    require(out != nullptr, "out must not be null");
    RINND_CUDA(cudaSetDevice(idx->device));
    idx->vertex_order.to_host(out, (size_t)idx->N);
    RINND_CUDA(cudaStreamSynchronize(idx->st));
  });
}

int rinnd_export_search_tree(rinnd_index* idx, int64_t* n_nodes, float* hyperplanes, float* offsets,
                             int32_t* children, int32_t* indices, int32_t* pivots) {
  return guarded([&] {
    check_index(idx);
    require(idx->n_search_trees >= 1, "no retained search tree is available");
    std::lock_guard<std::mutex> lock(idx->mu);
    RINND_CUDA(cudaSetDevice(idx->device));
    cudaStream_t st = idx->st;
    const Forest& f = idx->forest;
    const size_t total = (size_t)f.n_nodes;
    std::vector<int32_t> ch(2 * total);
    f.children.to_host(ch.data(), 2 * total);
    RINND_CUDA(cudaStreamSynchronize(st));
    // the first tree (root node 0) in depth-first preorder, the reference's node
    // numbering (tree/builder.rs:172-226 assigns ids on entry, left subtree first)
    std::vector<int32_t> order;
    std::vector<int32_t> local(total, -1);
    std::vector<int32_t> stack{0};
    while (!stack.empty()) {
      const int32_t g = stack.back();
      stack.pop_back();
      local[(size_t)g] = (int32_t)order.size();
      order.push_back(g);
      if (ch[2 * (size_t)g] > 0) {
        stack.push_back(ch[2 * (size_t)g + 1]);
        stack.push_back(ch[2 * (size_t)g]);
      }
    }
    const size_t m = order.size();
    if (n_nodes) *n_nodes = (int64_t)m;
    if (!hyperplanes && !offsets && !children && !indices && !pivots) return;
    if (children)
      for (size_t i = 0; i < m; ++i) {
        const size_t g = (size_t)order[i];
        const bool leaf = ch[2 * g] <= 0;
        children[2 * i] = leaf ? ch[2 * g] : local[(size_t)ch[2 * g]];
        children[2 * i + 1] = leaf ? ch[2 * g + 1] : local[(size_t)ch[2 * g + 1]];
      }
    if (offsets || pivots) {
      std::vector<float> off(total);
      std::vector<int32_t> pv(2 * total);
      f.offsets.to_host(off.data(), total);
      f.pivots.to_host(pv.data(), 2 * total);
      RINND_CUDA(cudaStreamSynchronize(st));
      for (size_t i = 0; i < m; ++i) {
        const size_t g = (size_t)order[i];
        if (offsets) offsets[i] = off[g];
        if (pivots) {
          pivots[2 * i] = pv[2 * g];
          pivots[2 * i + 1] = pv[2 * g + 1];
        }
      }
    }
    if (hyperplanes) {
      DVec<int32_t> ord(m, st);
      ord.from_host(order.data(), m);
      DVec<float> rows(m * (size_t)idx->Dp, st);
      gather_rows(f.hyperplanes.p, ord.p, (int64_t)m, idx->Dp, rows.p, st);
      RINND_CUDA(cudaMemcpy2DAsync(hyperplanes, sizeof(float) * idx->D, rows.p, sizeof(float) * idx->Dp,
                                   sizeof(float) * idx->D, m, cudaMemcpyDeviceToHost, st));
      RINND_CUDA(cudaStreamSynchronize(st));
    }
    if (indices) {  // leaf order of the first tree in original ids (index.rs:145-154)
      const size_t N = (size_t)idx->N;
      std::vector<int32_t> ti(N), vo(N);
      idx->tree_idx.to_host(ti.data(), N);
      idx->vertex_order.to_host(vo.data(), N);
      RINND_CUDA(cudaStreamSynchronize(st));
      for (size_t i = 0; i < N; ++i) indices[i] = vo[(size_t)ti[i]];
    }
  });
}

int rinnd_storage_info_get(const rinnd_index* idx, rinnd_storage_info* info) {
  return guarded([&] {
    check_index(idx);
    require(info != nullptr, "info must not be null");
    std::memset(info, 0, sizeof(*info));
    static const char* names[] = {"int8_per_vector_cosine", "sq8u_global_symmetric", "sq8p_per_vector_symmetric",
                                  "sq8d_per_dimension_symmetric"};
    const char* enc = idx->encoding >= 0 ? names[idx->encoding] : "fp32";
    std::snprintf(info->encoding, sizeof(info->encoding), "%s", enc);
    if (idx->encoding >= 0) {
      // QuantizedI8Index::storage_info / quantized_tree_storage_info (lib.rs:474-539),
      // retained_fp32_bytes (core/index.rs:94-101): rows (unless released), neighbor
      // distances and the FP32 search trees' hyperplanes and offsets (unless quantized)
      const int64_t N = idx->N, D = idx->D;
      int64_t nodes = 0;
      if (idx->n_search_trees > 0) {
        std::vector<int32_t> ch(2 * (size_t)idx->forest.n_nodes);
        RINND_CUDA(cudaSetDevice(idx->device));
        idx->forest.children.to_host(ch.data(), ch.size());
        RINND_CUDA(cudaStreamSynchronize(idx->st));
        for (int t = 0; t < idx->n_search_trees; ++t) {  // nodes of each retained tree
          std::vector<int32_t> stack{t};
          while (!stack.empty()) {
            const int32_t g = stack.back();
            stack.pop_back();
            ++nodes;
            if (ch[2 * (size_t)g] > 0) {
              stack.push_back(ch[2 * (size_t)g]);
              stack.push_back(ch[2 * (size_t)g + 1]);
            }
          }
        }
      }
      const int64_t topo = nodes * 8 + (int64_t)idx->n_search_trees * N * 4;
      const bool qtrees = idx->tree_codes.p != nullptr;
      info->code_bytes = N * D;
      info->metadata_bytes = idx->encoding == Q8_PER_DIMENSION ? D * 4 : N * 4;
      info->retained_fp32_bytes =
          (idx->fp32_released ? 0 : N * D * 4) + N * idx->k * 4 + (qtrees ? 0 : nodes * (D + 1) * 4);
      info->encode_seconds = idx->encode_seconds;
      if (qtrees) {
        info->tree_code_bytes = nodes * D;
        info->tree_scale_bytes = nodes * 4;
        info->tree_offset_bytes = nodes * 4;
        info->tree_topology_bytes = topo;
        info->released_fp32_tree_bytes = nodes * D * 4 + nodes * 4 + topo;
      } else {
        info->retained_fp32_tree_topology_bytes = topo;
      }
      info->released_fp32_data_bytes = idx->fp32_released ? N * D * 4 : 0;
    } else {
      info->code_bytes = (int64_t)idx->N * idx->D * 4;
    }
    info->device_bytes = (int64_t)(idx->X.n * 4 + idx->graph_int.indices.n * 4 + idx->graph_orig.indices.n * 4 +
                                   idx->knn_idx.n * 4 + idx->knn_dist.n * 4 + idx->codes.n + idx->inv_norms.n * 4 +
                                   idx->forest.hyperplanes.n * 4 + idx->tree_idx.n * 4);
  });
}

int rinnd_distance_pairs(int32_t kind, const float* a, const float* b, int64_t n_pairs, int32_t d, float* out) {
  return guarded([&] {
    require(kind >= 0 && kind < DK_COUNT, "unknown distance kind");
    require(d >= 1 && n_pairs >= 0, "invalid shape");
    if (n_pairs == 0) return;
    require(a && b && out, "pointers must not be null");
    ensure_device(0);
    StreamGuard sg;
    int Dp = round_up(d, 4);
    DVec<float> A, B;
    load_rows(a, false, n_pairs, d, d, Dp, A, sg.s);
    load_rows(b, false, n_pairs, d, d, Dp, B, sg.s);
    DVec<float> O((size_t)n_pairs, sg.s);
    distance_pairs(kind, A.p, B.p, n_pairs, d, Dp, O.p, sg.s);
    O.to_host(out, (size_t)n_pairs);
    RINND_CUDA(cudaStreamSynchronize(sg.s));
  });
}

int rinnd_brute_force_knn(const float* data, int64_t n, int64_t ld_data, const float* queries, int64_t nq,
                          int64_t ld_queries, int32_t d, int32_t k, int32_t distance_kind, int32_t precision,
                          const int32_t* exclude_ids, int32_t on_device, int32_t* out_idx, float* out_dist) {
  return guarded([&] {
    require(n >= 1 && nq >= 0 && d >= 1, "invalid shape");
    require(n < (int64_t)INT32_MAX - 1 && nq < (int64_t)INT32_MAX, "too many rows");
    require(ld_data >= d && ld_queries >= d, "row stride smaller than the dimension");
    require(k >= 1 && k <= 128, "k must be in [1, 128]");
    require(precision == RINND_BRUTE_FP32 || precision == RINND_BRUTE_BF16 || precision == RINND_BRUTE_FP64,
            "precision must be FP32, BF16 or FP64");
    require(distance_kind >= 0 && distance_kind < DK_COUNT && brute_supported(distance_kind),
            "brute force supports squared Euclidean, Manhattan, inner product, cosine and direct cosine");
    if (nq == 0) return;
    require(data && queries && out_idx && out_dist, "pointers must not be null");
    int dev = 0;
    if (on_device) RINND_CUDA(cudaGetDevice(&dev));
    ensure_device(dev);
    StreamGuard sg;
    const int Dp = round_up(d, 4);
    DVec<float> X, Q;
    load_rows(data, on_device != 0, n, d, ld_data, Dp, X, sg.s);
    load_rows(queries, on_device != 0, nq, d, ld_queries, Dp, Q, sg.s);
    DVec<int32_t> ex, oi;
    DVec<float> od;
    const int32_t* excl = nullptr;
    if (exclude_ids) {
      if (on_device) {
        excl = exclude_ids;
      } else {
        ex.alloc((size_t)nq, sg.s);
        RINND_CUDA(cudaMemcpyAsync(ex.p, exclude_ids, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, sg.s));
        excl = ex.p;
      }
    }
    int32_t* pi = out_idx;
    float* pd = out_dist;
    if (!on_device) {
      oi.alloc((size_t)nq * k, sg.s);
      od.alloc((size_t)nq * k, sg.s);
      pi = oi.p;
      pd = od.p;
    }
    brute_force_knn(Q.p, (int)nq, X.p, n, Dp, k, distance_kind, precision, excl, pi, pd, sg.s);
    if (!on_device) {
      oi.to_host(out_idx, (size_t)nq * k);
      od.to_host(out_dist, (size_t)nq * k);
    }
    RINND_CUDA(cudaStreamSynchronize(sg.s));
  });
}

int rinnd_search_graph_from_knn(const int32_t* knn_idx, const float* knn_dist, const float* data, int32_t n,
                                int32_t k, int32_t d, int32_t kind, float mult, int32_t* indptr,
                                int32_t* indices, int64_t* nnz, float* min_distance) {
  return guarded([&] {
    require(n >= 1 && k >= 1 && d >= 1, "invalid shape");
    require(kind >= 0 && kind < DK_COUNT, "unknown distance kind");
    require(knn_idx && knn_dist && data && indptr && indices, "pointers must not be null");
    ensure_device(0);
    StreamGuard sg;
    cudaStream_t st = sg.s;
    int Dp = round_up(d, 4);
    DVec<float> X;
    load_rows(data, false, n, d, d, Dp, X, st);
    DVec<int32_t> ki((size_t)n * k, st);
    DVec<float> kd((size_t)n * k, st);
    ki.from_host(knn_idx, (size_t)n * k);
    kd.from_host(knn_dist, (size_t)n * k);
    TempStorage tmp;
    Csr g;
    float md = 0.f;
    build_search_graph(ki.p, kd.p, X.p, n, k, d, Dp, kind, mult, st, tmp, g, &md);
    g.indptr.to_host(indptr, (size_t)n + 1);
    g.indices.to_host(indices, (size_t)g.nnz);
    RINND_CUDA(cudaStreamSynchronize(st));
    if (nnz) *nnz = g.nnz;
    if (min_distance) *min_distance = md;
  });
}

int rinnd_heap_push_batch(int32_t n, int32_t k, int64_t n_ops, const int32_t* rows, const int32_t* ids,
                          const float* dists, const uint8_t* flags, int32_t* out_idx, float* out_dist,
                          uint8_t* out_flags, int64_t* n_accepted) {
  return guarded([&] {
    require(n >= 1 && k >= 1 && k <= 512 && n_ops >= 0, "invalid shape");
    require(out_idx && out_dist, "output pointers must not be null");
    std::vector<int32_t> hr(rows, rows + n_ops), hi(ids, ids + n_ops);
    for (int64_t i = 0; i < n_ops; ++i) {
      require(hr[(size_t)i] >= 0 && hr[(size_t)i] < n, "push row out of range");
      require(hi[(size_t)i] >= 0 && hi[(size_t)i] < INT32_MAX - 1, "push id out of range");
    }
    ensure_device(0);
    StreamGuard sg;
    cudaStream_t st = sg.s;
    KnnState s;
    knn_init(s, n, k, 1, st);
    DVec<int32_t> dr((size_t)std::max<int64_t>(n_ops, 1), st), di((size_t)std::max<int64_t>(n_ops, 1), st);
    DVec<float> dd((size_t)std::max<int64_t>(n_ops, 1), st);
    DVec<uint8_t> df((size_t)std::max<int64_t>(n_ops, 1), st);
    dr.from_host(rows, (size_t)n_ops);
    di.from_host(ids, (size_t)n_ops);
    dd.from_host(dists, (size_t)n_ops);
    if (flags) df.from_host(flags, (size_t)n_ops);
    else df.fill_bytes(0);
    unsigned long long acc = n_ops ? heap_push_batch(s, n_ops, dr.p, di.p, dd.p, df.p, st) : 0ull;
    DVec<int32_t> oi((size_t)n * k, st);
    DVec<float> od((size_t)n * k, st);
    DVec<uint8_t> of((size_t)n * k, st);
    finalize_rows(s.slots.p, n, k, s.kp, oi.p, od.p, of.p, st);
    oi.to_host(out_idx, (size_t)n * k);
    od.to_host(out_dist, (size_t)n * k);
    if (out_flags) of.to_host(out_flags, (size_t)n * k);
    RINND_CUDA(cudaStreamSynchronize(st));
    if (n_accepted) *n_accepted = (int64_t)acc;
  });
}

int rinnd_nndescent_step(const float* data, int64_t n, int32_t d, int32_t k, int32_t max_candidates, int32_t kind,
                         int32_t precision, uint64_t seed, int32_t iteration, int32_t* idx, float* dist,
                         uint8_t* flags, int64_t* changes, int32_t* join_form) {
  return guarded([&] {
    require(n >= 2 && n < (int64_t)INT32_MAX - 1 && d >= 1, "invalid shape");
    require(k >= 1 && k <= 128, "k must be in [1, 128]");
    require(kind >= 0 && kind < DK_COUNT, "unknown distance kind");
    require(precision == RINND_PRECISION_FP32 || precision == RINND_PRECISION_BF16, "unknown precision");
    require(data && idx && dist && flags, "pointers must not be null");
    const int N = (int)n, Dp = round_up(d, 4);
    const int c = std::min(std::min(max_candidates > 0 ? max_candidates : std::min(k, 60), 60), k);  // mod.rs:89
    std::vector<int32_t> hr, hi;
    std::vector<float> hd;
    std::vector<uint8_t> hf;
    for (int64_t r = 0; r < n; ++r)
      for (int j = 0; j < k; ++j) {
        const int32_t id = idx[r * k + j];
        if (id < 0) continue;
        require(id < N, "neighbor id out of range");
        hr.push_back((int32_t)r);
        hi.push_back(id);
        hd.push_back(dist[r * k + j]);
        hf.push_back(flags[r * k + j] ? 1 : 0);
      }
    ensure_device(0);
    StreamGuard sg;
    cudaStream_t st = sg.s;
    DVec<float> X;
    load_rows(data, false, n, d, d, Dp, X, st);
    KnnState ks;
    knn_init(ks, N, k, c, st);
    ks.precision = precision;
    if (kind_uses_norms(kind)) {
      ks.norms.alloc((size_t)N, st);
      compute_norms(X.p, N, d, Dp, ks.norms.p, st);
    }
    const size_t m = std::max<size_t>(hr.size(), 1);
    DVec<int32_t> dr(m, st), di(m, st);
    DVec<float> dd(m, st);
    DVec<uint8_t> df(m, st);
    dr.from_host(hr.data(), hr.size());
    di.from_host(hi.data(), hi.size());
    dd.from_host(hd.data(), hd.size());
    df.from_host(hf.data(), hf.size());
    if (!hr.empty()) heap_push_batch(ks, (long long)hr.size(), dr.p, di.p, dd.p, df.p, st);
    join_tile_lookup(ks, Dp, kind);  // the table's tile shape for this key, if any (else the default)
    build_candidates(ks, seed, iteration, st);
    JoinStats js = local_join(ks, X.p, d, Dp, kind, st);
    DVec<int32_t> oi((size_t)N * k, st);
    DVec<float> od((size_t)N * k, st);
    DVec<uint8_t> of((size_t)N * k, st);
    finalize_rows(ks.slots.p, N, k, ks.kp, oi.p, od.p, of.p, st);
    oi.to_host(idx, (size_t)N * k);
    od.to_host(dist, (size_t)N * k);
    of.to_host(flags, (size_t)N * k);
    RINND_CUDA(cudaStreamSynchronize(st));
    if (changes) *changes = (int64_t)js.changes;
    if (join_form) *join_form = js.form;
  });
}

const char* rinnd_last_error(void) { return g_last_error.c_str(); }

const char* rinnd_version(void) { return "0.1.0-b200"; }

int rinnd_device_count(int32_t* count) {
  return guarded([&] {
    require(count != nullptr, "count must not be null");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
      cudaGetLastError();
      n = 0;
    }
    *count = n;
  });
}

int rinnd_quantize(rinnd_index* idx, int32_t encoding) {
  return guarded([&] {
    check_index(idx);
    require(encoding >= RINND_Q8_PER_VECTOR_COSINE && encoding <= RINND_Q8_PER_DIMENSION, "unknown int8 encoding");
    require(idx->kind == DK_DIRECT_COSINE,
            "int8 quantization requires an index built with the direct cosine distance on normalized rows");
    require(!idx->fp32_released, "the FP32 rows were released: the index can no longer be encoded");
    std::lock_guard<std::mutex> lock(idx->mu);
    RINND_CUDA(cudaSetDevice(idx->device));
    cudaStream_t st = idx->st;
    RINND_CUDA(cudaStreamSynchronize(st));
    const double t0 = now_ms();
    const int Dq = round_up(idx->D, 16);
    const float gm = quant_global_multiplier(idx->X.p, (long long)idx->N * idx->Dp, st);
    idx->codes.alloc((size_t)idx->N * Dq, st);
    if (encoding == Q8_PER_DIMENSION) {
      idx->inv_norms.release();
      idx->dim_scales.alloc((size_t)Dq, st);
      quant_dim_scales(idx->X.p, idx->N, idx->D, idx->Dp, Dq, idx->dim_scales.p, st);
    } else {
      idx->dim_scales.release();
      idx->inv_norms.alloc((size_t)idx->N, st);
    }
    quantize_rows(idx->X.p, idx->N, idx->D, idx->Dp, Dq, encoding, gm, idx->dim_scales.p, idx->codes.p,
                  idx->inv_norms.p, st);
    RINND_CUDA(cudaStreamSynchronize(st));
    idx->Dq = Dq;
    idx->global_mult = gm;
    idx->encoding = encoding;
    idx->encode_seconds = (now_ms() - t0) / 1000.0;
  });
}

int rinnd_query_quantized(rinnd_index* idx, const float* queries, int64_t nq, int32_t k, float epsilon,
                          int32_t candidate_width, int32_t rerank_width, int32_t* out_idx, float* out_dist) {
  return guarded([&] {
    check_index(idx);
    require(idx->encoding >= 0, "index has no int8 codes: call rinnd_quantize first");
    require(nq >= 0, "number of queries must be >= 0");
    require(k >= 1, "k must be >= 1");
    require(candidate_width >= 0 && rerank_width >= 0, "quantized widths must be >= 0");
    // resolve_quantized_candidate_width / should_rerank_quantized (index.rs:55-89)
    const int resolved = candidate_width == 0 ? std::max(k, rerank_width) : candidate_width;
    require(resolved >= k, "quantized candidate width must be at least k");
    require(rerank_width <= resolved, "quantized rerank width must not exceed candidate width");
    require(candidate_width == 0 || rerank_width == 0 || rerank_width >= k,
            "quantized rerank width must be zero or at least k");
    require(resolved <= 256, "quantized candidate width must be <= 256");
    const bool rerank = candidate_width == 0 ? rerank_width > k : rerank_width > 0;
    require(!(rerank && idx->fp32_released), "exact reranking is unavailable because FP32 vector data was released");
    if (nq == 0) return;
    require(queries && out_idx && out_dist, "query/output pointers must not be null");
    std::lock_guard<std::mutex> lock(idx->mu);
    RINND_CUDA(cudaSetDevice(idx->device));
    cudaStream_t st = idx->st;
    DVec<float> Q;
    load_rows(queries, false, nq, idx->D, idx->D, idx->Dp, Q, st);
    if (idx->normalize) normalize_rows(Q.p, nq, idx->D, idx->Dp, st);
    DVec<int8_t> Q8((size_t)nq * idx->Dq, st);
    DVec<float> qs((size_t)nq, st);
    quantize_rows(Q.p, nq, idx->D, idx->Dp, idx->Dq, idx->encoding, idx->global_mult, idx->dim_scales.p, Q8.p, qs.p,
                  st);
    DVec<int32_t> oi((size_t)nq * k, st);
    DVec<float> od((size_t)nq * k, st);
    greedy_search_quantized(idx->search_view(), Q.p, Q8.p, qs.p, (int)nq, resolved, k, rerank ? rerank_width : 0,
                            epsilon, oi.p, od.p, st, idx->search_stats.p);
    oi.to_host(out_idx, (size_t)nq * k);
    od.to_host(out_dist, (size_t)nq * k);
    RINND_CUDA(cudaStreamSynchronize(st));
  });
}

int rinnd_quantize_rows(const float* data, int64_t n, int32_t d, int32_t encoding, int8_t* codes, float* scales,
                        float* global_multiplier) {
  return guarded([&] {
    require(n >= 0 && d >= 1, "invalid shape");
    require(encoding >= RINND_Q8_PER_VECTOR_COSINE && encoding <= RINND_Q8_PER_VECTOR_SYMMETRIC,
            "unknown int8 encoding (per-dimension codes: rinnd_quantize_rows_per_dimension)");
    if (n == 0) {
      if (global_multiplier) *global_multiplier = 0.f;
      return;
    }
    require(data && codes && scales, "pointers must not be null");
    ensure_device(0);
    StreamGuard sg;
    const int Dp = round_up(d, 4), Dq = round_up(d, 16);
    DVec<float> X;
    load_rows(data, false, n, d, d, Dp, X, sg.s);
    const float gm = quant_global_multiplier(X.p, n * Dp, sg.s);
    DVec<int8_t> C((size_t)n * Dq, sg.s);
    DVec<float> S((size_t)n, sg.s);
    quantize_rows(X.p, n, d, Dp, Dq, encoding, gm, nullptr, C.p, S.p, sg.s);
    RINND_CUDA(cudaMemcpy2DAsync(codes, (size_t)d, C.p, (size_t)Dq, (size_t)d, (size_t)n, cudaMemcpyDeviceToHost,
                                 sg.s));
    S.to_host(scales, (size_t)n);
    RINND_CUDA(cudaStreamSynchronize(sg.s));
    if (global_multiplier) *global_multiplier = gm;
  });
}

}  // extern "C"

namespace {

// ---- index file (no counterpart in the reference, whose indices live in memory
// only): a header, then every resident array as (element count u64, bytes).
constexpr char kFileMagic[8] = {'R', 'I', 'N', 'N', 'D', 'B', '2', '\0'};
constexpr uint32_t kFileVersion = 1;

struct FileHeader {
  char magic[8];
  uint32_t version, header_bytes;
  int64_t N, n_nodes, graph_int_nnz, graph_orig_nnz;
  int32_t D, Dp, k, kind, corr, normalize, encoding, Dq, n_search_trees, forest_levels, fp32_released, pad;
  float global_mult, min_distance;
  double encode_seconds;
  rinnd_build_params params;
  rinnd_build_info info;
};

struct File {
  FILE* f = nullptr;
  std::string path;
  ~File() {
    if (f) std::fclose(f);
  }
  void write(const void* p, size_t bytes) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes) throw std::invalid_argument("cannot write index file " + path);
  }
  void read(void* p, size_t bytes) {
    if (bytes && std::fread(p, 1, bytes, f) != bytes)
      throw std::invalid_argument("index file " + path + " is truncated or unreadable");
  }
};

template <class T>
void save_array(File& F, const DVec<T>& v, size_t count, cudaStream_t st) {
  const uint64_t c = v.p ? (uint64_t)count : 0;
  F.write(&c, sizeof(c));
  if (!c) return;
  std::vector<T> h((size_t)c);
  v.to_host(h.data(), (size_t)c);
  RINND_CUDA(cudaStreamSynchronize(st));
  F.write(h.data(), sizeof(T) * (size_t)c);
}

template <class T>
void load_array(File& F, DVec<T>& v, cudaStream_t st, size_t expect_max) {
  uint64_t c = 0;
  F.read(&c, sizeof(c));
  require(c <= expect_max, "index file " + F.path + " has an array larger than its header allows");
  if (!c) return;
  std::vector<T> h((size_t)c);
  F.read(h.data(), sizeof(T) * (size_t)c);
  v.alloc((size_t)c, st);
  v.from_host(h.data(), (size_t)c);
  RINND_CUDA(cudaStreamSynchronize(st));
}

}  // namespace

extern "C" {

int rinnd_save(rinnd_index* idx, const char* path, const char* meta) {
  return guarded([&] {
    check_index(idx);
    require(path != nullptr, "path must not be null");
    std::lock_guard<std::mutex> lock(idx->mu);
    RINND_CUDA(cudaSetDevice(idx->device));
    cudaStream_t st = idx->st;
    RINND_CUDA(cudaStreamSynchronize(st));
    File F;
    F.path = path;
    F.f = std::fopen(path, "wb");
    require(F.f != nullptr, std::string("cannot open index file ") + path + " for writing");
    FileHeader h{};
    std::memcpy(h.magic, kFileMagic, 8);
    h.version = kFileVersion;
    h.header_bytes = sizeof(FileHeader);
    h.N = idx->N;
    h.n_nodes = idx->forest.n_nodes;
    h.graph_int_nnz = idx->graph_int.nnz;
    h.graph_orig_nnz = idx->graph_orig.nnz;
    h.D = idx->D;
    h.Dp = idx->Dp;
    h.k = idx->k;
    h.kind = idx->kind;
    h.corr = idx->corr;
    h.normalize = idx->normalize ? 1 : 0;
    h.encoding = idx->encoding;
    h.Dq = idx->Dq;
    h.n_search_trees = idx->n_search_trees;
    h.forest_levels = idx->forest.levels;
    h.fp32_released = idx->fp32_released ? 1 : 0;
    h.global_mult = idx->global_mult;
    h.min_distance = idx->min_distance;
    h.encode_seconds = idx->encode_seconds;
    h.params = idx->p;
    h.info = idx->info;
    F.write(&h, sizeof(h));
    const std::string m = meta ? meta : "";
    const uint64_t mlen = m.size();
    F.write(&mlen, sizeof(mlen));
    F.write(m.data(), m.size());
    const size_t N = (size_t)idx->N, nn = (size_t)idx->forest.n_nodes;
    save_array(F, idx->X, N * idx->Dp, st);
    save_array(F, idx->vertex_order, N, st);
    save_array(F, idx->graph_orig.indptr, N + 1, st);
    save_array(F, idx->graph_orig.indices, (size_t)idx->graph_orig.nnz, st);
    save_array(F, idx->graph_int.indptr, N + 1, st);
    save_array(F, idx->graph_int.indices, (size_t)idx->graph_int.nnz, st);
    save_array(F, idx->knn_idx, N * idx->k, st);
    save_array(F, idx->knn_dist, N * idx->k, st);
    save_array(F, idx->forest.children, 2 * nn, st);
    save_array(F, idx->forest.offsets, nn, st);
    save_array(F, idx->forest.hyperplanes, nn * idx->Dp, st);
    save_array(F, idx->forest.pivots, 2 * nn, st);
    save_array(F, idx->tree_idx, (size_t)idx->n_search_trees * N, st);
    save_array(F, idx->tree_roots, (size_t)idx->n_search_trees, st);
    save_array(F, idx->codes, N * idx->Dq, st);
    save_array(F, idx->inv_norms, N, st);
    save_array(F, idx->dim_scales, (size_t)idx->Dq, st);
    save_array(F, idx->tree_codes, nn * idx->Dq, st);
    save_array(F, idx->tree_scales, nn, st);
    require(std::fflush(F.f) == 0, std::string("cannot write index file ") + path);
  });
}

int rinnd_load(const char* path, int32_t device, rinnd_index** out, char* meta, int64_t meta_cap,
               int64_t* meta_len) {
  return guarded([&] {
    require(path != nullptr && out != nullptr, "path and out must not be null");
    *out = nullptr;
    File F;
    F.path = path;
    F.f = std::fopen(path, "rb");
    require(F.f != nullptr, std::string("cannot open index file ") + path);
    FileHeader h{};
    F.read(&h, sizeof(h));
    require(std::memcmp(h.magic, kFileMagic, 8) == 0, std::string(path) + " is not a rinnd_b200 index file");
    require(h.version == kFileVersion && h.header_bytes == sizeof(FileHeader),
            std::string(path) + " was written by an incompatible version");
    require(h.N >= 1 && h.D >= 1 && h.Dp == round_up(h.D, 4) && h.k >= 1 && h.n_nodes >= 0 &&
                h.n_search_trees >= 0 && h.graph_orig_nnz >= 0 && h.graph_int_nnz >= 0,
            std::string(path) + " has an invalid header");
    uint64_t mlen = 0;
    F.read(&mlen, sizeof(mlen));
    require(mlen < (1ull << 30), std::string(path) + " has an invalid header");
    std::string m((size_t)mlen, '\0');
    F.read(&m[0], (size_t)mlen);
    ensure_device(device);
    std::unique_ptr<rinnd_index> ix(new rinnd_index());
    ix->device = device;
    RINND_CUDA(cudaStreamCreateWithFlags(&ix->st, cudaStreamNonBlocking));
    cudaStream_t st = ix->st;
    ix->N = h.N;
    ix->D = h.D;
    ix->Dp = h.Dp;
    ix->k = h.k;
    ix->kind = h.kind;
    ix->corr = h.corr;
    ix->normalize = h.normalize != 0;
    ix->encoding = h.encoding;
    ix->Dq = h.Dq;
    ix->n_search_trees = h.n_search_trees;
    ix->fp32_released = h.fp32_released != 0;
    ix->global_mult = h.global_mult;
    ix->min_distance = h.min_distance;
    ix->encode_seconds = h.encode_seconds;
    ix->p = h.params;
    ix->p.device = device;
    ix->info = h.info;
    const size_t N = (size_t)h.N, nn = (size_t)h.n_nodes;
    load_array(F, ix->X, st, N * h.Dp);
    load_array(F, ix->vertex_order, st, N);
    load_array(F, ix->graph_orig.indptr, st, N + 1);
    load_array(F, ix->graph_orig.indices, st, (size_t)h.graph_orig_nnz);
    load_array(F, ix->graph_int.indptr, st, N + 1);
    load_array(F, ix->graph_int.indices, st, (size_t)h.graph_int_nnz);
    load_array(F, ix->knn_idx, st, N * h.k);
    load_array(F, ix->knn_dist, st, N * h.k);
    load_array(F, ix->forest.children, st, 2 * nn);
    load_array(F, ix->forest.offsets, st, nn);
    load_array(F, ix->forest.hyperplanes, st, nn * h.Dp);
    load_array(F, ix->forest.pivots, st, 2 * nn);
    load_array(F, ix->tree_idx, st, (size_t)h.n_search_trees * N);
    load_array(F, ix->tree_roots, st, (size_t)h.n_search_trees);
    load_array(F, ix->codes, st, N * (size_t)std::max(h.Dq, 0));
    load_array(F, ix->inv_norms, st, N);
    load_array(F, ix->dim_scales, st, (size_t)std::max(h.Dq, 0));
    load_array(F, ix->tree_codes, st, nn * (size_t)std::max(h.Dq, 0));
    load_array(F, ix->tree_scales, st, nn);
    require(ix->vertex_order.n == N && ix->graph_int.indptr.n == N + 1 && ix->knn_idx.n == N * h.k &&
                (ix->fp32_released || ix->X.n == N * h.Dp),
            std::string(path) + " is missing index arrays");
    ix->graph_orig.N = ix->graph_int.N = (int)N;
    ix->graph_orig.nnz = h.graph_orig_nnz;
    ix->graph_int.nnz = h.graph_int_nnz;
    ix->forest.n_nodes = h.n_nodes;
    ix->forest.levels = h.forest_levels;
    ix->forest.T = h.params.n_trees;
    ix->forest.N = (int)N;
    ix->forest.Dp = h.Dp;
    ix->inverse.alloc(N, st);
    invert_permutation(ix->vertex_order.p, (int)N, ix->inverse.p, st);
    ix->search_stats.alloc(8, st);
    ix->search_stats.fill_bytes(0);
    RINND_CUDA(cudaStreamSynchronize(st));
    if (meta_len) *meta_len = (int64_t)m.size();
    if (meta && meta_cap > 0) {
      const size_t n = std::min((size_t)meta_cap - 1, m.size());
      std::memcpy(meta, m.data(), n);
      meta[n] = '\0';
    }
    *out = ix.release();
  });
}

int rinnd_quantize_trees(rinnd_index* idx) {
  return guarded([&] {
    check_index(idx);
    require(idx->encoding >= 0, "tree_quantization='int8' is available only with a quantized cosine_distance_mode");
    require(idx->encoding != Q8_GLOBAL_SYMMETRIC,
            "tree_quantization='int8' is incompatible with cosine_distance_mode='sq8u'; use tree_quantization='none'");
    require(idx->encoding != Q8_PER_DIMENSION,
            "tree_quantization='int8' is incompatible with cosine_distance_mode='sq8d'; use tree_quantization='none'");
    std::lock_guard<std::mutex> lock(idx->mu);
    RINND_CUDA(cudaSetDevice(idx->device));
    cudaStream_t st = idx->st;
    const long long nn = (long long)idx->forest.n_nodes;
    const int Dq = round_up(idx->D, 16);
    idx->tree_codes.alloc((size_t)std::max<long long>(nn, 1) * Dq, st);
    idx->tree_scales.alloc((size_t)std::max<long long>(nn, 1), st);
    quantize_tree_hyperplanes(idx->forest.hyperplanes.p, nn, idx->D, idx->Dp, Dq, idx->tree_codes.p,
                              idx->tree_scales.p, st);
    RINND_CUDA(cudaStreamSynchronize(st));
  });
}

int rinnd_release_fp32(rinnd_index* idx) {
  return guarded([&] {
    check_index(idx);
    require(idx->encoding >= 0, "only a quantized index can release its FP32 rows");
    std::lock_guard<std::mutex> lock(idx->mu);
    RINND_CUDA(cudaSetDevice(idx->device));
    idx->X.release();
    idx->fp32_released = true;
    RINND_CUDA(cudaStreamSynchronize(idx->st));
  });
}

int rinnd_tree_search_leaves(rinnd_index* idx, const float* queries, int64_t nq, int32_t tree, int32_t budget,
                             int32_t quantized, int32_t* out_leaves, int32_t* out_counts) {
  return guarded([&] {
    check_index(idx);
    require(nq >= 0, "number of queries must be >= 0");
    require(tree >= 0 && tree < idx->n_search_trees, "tree index out of range of the retained search trees");
    require(budget >= 1 && budget <= 256, "leaf budget must be in [1, 256]");
    require(!quantized || idx->tree_codes.p != nullptr, "the index has no int8 routing trees");
    if (nq == 0) return;
    require(queries && out_leaves && out_counts, "pointers must not be null");
    std::lock_guard<std::mutex> lock(idx->mu);
    RINND_CUDA(cudaSetDevice(idx->device));
    cudaStream_t st = idx->st;
    DVec<float> Q;
    load_rows(queries, false, nq, idx->D, idx->D, idx->Dp, Q, st);
    if (idx->normalize) normalize_rows(Q.p, nq, idx->D, idx->Dp, st);
    DVec<int8_t> Q8;
    DVec<float> qs;
    if (quantized) {
      Q8.alloc((size_t)nq * idx->Dq, st);
      qs.alloc((size_t)nq, st);
      quantize_rows(Q.p, nq, idx->D, idx->Dp, idx->Dq, idx->encoding, idx->global_mult, idx->dim_scales.p, Q8.p,
                    qs.p, st);
    }
    DVec<int32_t> ol((size_t)nq * budget * 2, st), oc((size_t)nq, st);
    tree_leaves(idx->search_view(), Q.p, quantized ? Q8.p : nullptr, (int)nq, tree, budget, 0, ol.p, oc.p, st,
                idx->search_stats.p);
    ol.to_host(out_leaves, (size_t)nq * budget * 2);
    oc.to_host(out_counts, (size_t)nq);
    RINND_CUDA(cudaStreamSynchronize(st));
  });
}

int rinnd_quantize_rows_per_dimension(const float* data, int64_t n, int32_t d, int8_t* codes, float* dim_scales) {
  return guarded([&] {
    require(n >= 1 && d >= 1, "invalid shape");
    require(data && codes && dim_scales, "pointers must not be null");
    ensure_device(0);
    StreamGuard sg;
    const int Dp = round_up(d, 4), Dq = round_up(d, 16);
    DVec<float> X;
    load_rows(data, false, n, d, d, Dp, X, sg.s);
    DVec<float> S((size_t)Dq, sg.s);
    quant_dim_scales(X.p, n, d, Dp, Dq, S.p, sg.s);
    DVec<int8_t> C((size_t)n * Dq, sg.s);
    quantize_rows(X.p, n, d, Dp, Dq, Q8_PER_DIMENSION, 0.f, S.p, C.p, nullptr, sg.s);
    RINND_CUDA(cudaMemcpy2DAsync(codes, (size_t)d, C.p, (size_t)Dq, (size_t)d, (size_t)n, cudaMemcpyDeviceToHost,
                                 sg.s));
    S.to_host(dim_scales, (size_t)d);
    RINND_CUDA(cudaStreamSynchronize(sg.s));
  });
}

}  // extern "C"
