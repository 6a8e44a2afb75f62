// engine.h -- internal interfaces between the kernel files and the C ABI layer.
#pragma once
#include <stdint.h>

#include "devmem.cuh"
#include "heap.cuh"

#include <array>
#include <string>

namespace rinnd {

// Records msg as the thread's last error (rinnd_last_error) and returns code.
int api_fail(int code, const std::string& msg);

// ---- RP forest (forest.cu) -------------------------------------------------
// Level-synchronous batched construction of all trees at once.  Node ids are
// global across the forest; roots are 0..T-1.  children[2*node] = {left,right}
// for internal nodes (always > 0) and {-start, -end} (positions within the
// tree's `perm` slice) for leaves, the reference FlatTree encoding
// (core/tree/flat_tree.rs:14-28).
struct Forest {
  int T = 0, N = 0, Dp = 0;
  DVec<int32_t> perm;         // T*N, leaf order per tree
  DVec<int32_t> children;     // 2 * n_nodes
  DVec<float> offsets;        // n_nodes
  DVec<float> hyperplanes;    // n_nodes * Dp (zeros for leaves)
  DVec<int32_t> pivots;       // 2 * n_nodes: the two points whose split is the node's hyperplane (-1: leaf)
  DVec<int4> leaves;          // (tree, start, end, node)
  int64_t n_nodes = 0;
  int64_t n_leaves = 0;
  int max_leaf = 0;
  int levels = 0;
};
// Several indices' rows in one forest (a grouped build): item i owns rows
// [off[i], off[i+1]) and trees 0..trees[i]-1 (trees[i] <= T); the root of
// (tree t, item i) is node t * n_items + i.  Splits never cross item bounds.
struct ForestItems {
  std::vector<int64_t> off;  // n_items + 1
  std::vector<int> trees;    // n_items
};
void build_forest(const float* X, int N, int D, int Dp, int T, int leaf_size, bool angular,
                  int max_depth, uint64_t seed, cudaStream_t st, TempStorage& tmp, Forest& out,
                  const ForestItems* items = nullptr);

// Raises `kernel`'s dynamic shared-memory limit to `bytes` once per (kernel,
// current device); safe to call from concurrent host threads (api.cu).  Later
// calls for the same kernel are ignored, so pass the largest size any launch uses.
void set_smem_limit_once(const void* kernel, int bytes);

// ---- NN-Descent (nndescent.cu) ---------------------------------------------
struct BuildStats {
  int iterations = 0;
  unsigned long long changes[64] = {};
  unsigned long long pairs[64] = {};
  unsigned long long contention = 0;
  double ms_forest = 0, ms_leaf = 0, ms_iters = 0, ms_sort = 0, ms_graph = 0, ms_total = 0;
  double ms_candidates = 0, ms_join = 0;
};

// Tile shape of the pipelined FP32 join: row stages in flight per CTA (2 or 3),
// candidate rows per work item (1 or 2) and CTAs launched per SM (0 = as many
// as shared memory allows).  Candidate lists longer than 32 run (2, 1, 0).
struct JoinTile {
  int nstage = 2, jb = 1, per_sm = 0;
};

struct KnnState {
  int N = 0, k = 0, c = 0;
  int kp = 0, cp = 0;        // row strides (multiples of 16 slots)
  DVec<uint64_t> slots;      // N*kp neighbor slots (first k of each row used)
  DVec<uint32_t> thr;        // N upper bounds of fkey(row max)
  DVec<uint64_t> cand_new;   // N*cp
  DVec<uint64_t> cand_old;   // N*cp
  DVec<float> norms;         // N squared norms (dot-form metrics)
  // [0] changes, [1] contention, [2] pairs, [3] gathered rows, [4] buffered updates (batch),
  // [5] applied buffered updates (iteration), [6] appended updates incl. overflow (iteration)
  DVec<unsigned long long> counters;
  DVec<uint32_t> cthr;       // 2N candidate-list priority bounds (new, old)
  DVec<int> err;             // device error flag of pipelined kernels
  DVec<int32_t> desc;        // per-vertex join descriptors (counts, item prefix, ids, thresholds, norms)
  bool use_tma = true;       // bulk-copy pipelined join when shared memory allows
  JoinTile tile;             // tile shape of the pipelined FP32 join
  int precision = 0;         // 0: FP32 join tiles; 1: BF16 tensor-core filter + FP32 recheck
  DVec<uint32_t> urow;       // update buffer: destination rows
  DVec<uint64_t> ukey;       // update buffer: slot keys
  unsigned long long ucap = 0;
  // Region form of the update buffer (FP32 pipelined join): nreg regions of
  // rsize entries, region r holding rcnt[r] updates; nreg = 0 after they are applied.
  DVec<uint32_t> rcnt;
  int nreg = 0;
  unsigned int rsize = 0;
  // BF16 precision form: BF16 copy of the rows (N x kpb) and per-row (|b|^2, rounding error bound)
  DVec<uint16_t> xb;
  DVec<float> rinfo;         // 2N floats
  int kpb = 0;
  double upv_prev = -1.0;    // updates appended per vertex by the previous join (-1: none yet)
  bool seeded = false;       // rows initialized from tree leaves (their thresholds already filter)
  // Grouped build (several indices' rows in one state; empty otherwise):
  // row_item[r] = index of row r; item_active[i] = 0 once index i stopped
  // iterating; item_changes[i] = accepted pushes into index i's rows since reset.
  DVec<int32_t> row_item;
  DVec<uint8_t> item_active;
  DVec<unsigned long long> item_changes;
  ItemCount item_count() const { return ItemCount{row_item.p, item_changes.p}; }
  GroupRows group_rows() const { return GroupRows{row_item.p, item_active.p}; }
};

void knn_init(KnnState& s, int N, int k, int c, cudaStream_t st);
void ensure_update_buffer(KnnState& s, cudaStream_t st);
void compute_norms(const float* X, int N, int D, int Dp, float* norms, cudaStream_t st);
void leaf_init(KnnState& s, const Forest& f, const float* X, int D, int Dp, int kind,
               cudaStream_t st);
void build_candidates(KnnState& s, uint64_t seed, int iter, cudaStream_t st);
struct JoinStats {
  unsigned long long changes = 0, pairs = 0, rows = 0, updates = 0, appended = 0;
  float kernel_ms = 0.f;   // CUDA-event duration of the join kernel launches on their stream
  float total_ms = 0.f;    // CUDA-event duration of the whole join step (describe, joins, applies)
  int launches = 0;        // join kernel launches
  int form = 0;            // RINND_JOIN_* of the kernel that ran
};
// One local join: plan (host decisions and every allocation / kernel attribute
// the join needs), enqueue (stream work only: capturable in a CUDA graph), and
// collect (counters read back -> stats).  local_join does the three in order,
// timing each join kernel launch with events.
constexpr int JOIN_MAX_GRID = 148 * 64;  // upper bound of any join launch's grid
struct JoinPlan {
  bool generic = false, use_tc = false, use_tma = false;
  long long per_batch = 1;  // vertices per join launch (each followed by its update application)
};
JoinPlan join_plan(KnnState& s, const float* X, int D, int Dp, int kind, cudaStream_t st);
void join_enqueue(KnnState& s, const JoinPlan& p, const float* X, int D, int Dp, int kind, cudaStream_t st,
                  std::vector<cudaEvent_t>* kernel_events);
JoinStats join_collect(KnnState& s, const JoinPlan& p, const unsigned long long* counters, int err);
JoinStats local_join(KnnState& s, const float* X, int D, int Dp, int kind, cudaStream_t st);
void candidates_reserve(KnnState& s, cudaStream_t st);
// One NN-Descent iteration (candidate pass, join launches, update applications,
// counter read-back) captured by stream capture into a CUDA graph and launched;
// later iterations update the instantiated graph in place (cudaGraphExecUpdate)
// when its topology is unchanged.  item_changes_host (n_items) receives the
// grouped build's per-index change counts.
struct IterationGraph {
  cudaGraphExec_t exec = nullptr;
  unsigned long long* host = nullptr;  // pinned: 7 counters, error flag, per-index changes
  size_t host_words = 0;
  int launches = 0, updates = 0;       // graph launches; of them, in-place updates of the executable
  IterationGraph() = default;
  IterationGraph(const IterationGraph&) = delete;
  IterationGraph& operator=(const IterationGraph&) = delete;
  ~IterationGraph();
};
JoinStats iteration_graph(KnnState& s, IterationGraph& g, uint64_t seed, int iter, const float* X, int D, int Dp,
                          int kind, cudaStream_t st, unsigned long long* item_changes_host, int n_items);
bool join_tma_supported(int c, int Dp);
bool join_tile_fits(int c, int Dp, const JoinTile& t);
// Join tile tuner (join_tma.cu).  join_tune times every tile shape that fits on
// the vertices [0, sample) of the current candidate lists, leaves the heaps as
// they were, stores the fastest shape in s.tile and in the process-wide table,
// and returns it; join_tile_lookup loads a tuned shape for s's key from the
// table (false when none is stored).  Table rows: device, Dp, list class (32 or
// 64), metric class (0 squared Euclidean, 1 Manhattan, 2 dot forms), grouped,
// stages, rows per item, CTAs per SM.
struct TileTrial {
  JoinTile tile;
  float ms;         // best of the timed trials on the sample
  int vertices;     // sample size
};
JoinTile join_tune(KnnState& s, const float* X, int Dp, int kind, long long sample, cudaStream_t st,
                   std::vector<TileTrial>* trials = nullptr);
bool join_tile_lookup(KnnState& s, int Dp, int kind);
// The build's join tile by rinnd_build_params.join_tuning (RINND_TUNE_*): the
// fixed default, the table's shape for this key, or one tuned now on the
// first iteration's candidates (heaps left as they were).  Call before the
// first iteration; *tuned (may be null) tells whether trials ran.
JoinTile choose_join_tile(KnnState& s, const float* X, int D, int Dp, int kind, uint64_t seed, int mode,
                          cudaStream_t st, bool* tuned);
std::vector<std::array<int, 8>> join_tile_table();
void join_tile_table_clear();
void join_tile_store(int device, int Dp, int list_class, int metric_class, int grouped, const JoinTile& t);
void join_tma_batch(KnnState& s, const float* X, int Dp, int kind, int v0, int v1, int* err, cudaStream_t st);
void join_tma_reserve(const KnnState& s, int Dp);   // kernel attributes of join_tma_batch
void join_describe(KnnState& s, int kind, cudaStream_t st);
void join_describe_reserve(KnnState& s);           // descriptor storage of join_describe
// Tensor-core join (join_tc.cu): BF16 Gram filter + exact FP32 recheck.  prepare
// makes the BF16 copy of the rows once per build (s.xb, s.rinfo).
bool join_tc_supported(int kind, int c, int Dp);
void join_tc_prepare(KnnState& s, const float* X, int D, int Dp, cudaStream_t st);
void join_tc_reserve(int kind);                     // kernel attributes of join_tc_batch
void join_tc_batch(KnnState& s, const float* X, int D, int Dp, int kind, int v0, int v1, int* err, cudaStream_t st);
// Sorted output: idx (-1 empty), raw distance (+inf empty).
void finalize_knn(const KnnState& s, int32_t* out_idx, float* out_dist, cudaStream_t st);
void finalize_rows(const uint64_t* slots, int N, int k, int kp, int32_t* out_idx, float* out_dist,
                   uint8_t* out_flags, cudaStream_t st);
unsigned long long heap_push_batch(KnnState& s, long long n_ops, const int32_t* rows,
                                   const int32_t* ids, const float* dists, const uint8_t* flags,
                                   cudaStream_t st);

// ---- search graph (graph.cu) -----------------------------------------------
struct Csr {
  int N = 0;
  DVec<int32_t> indptr;   // N+1
  DVec<int32_t> indices;  // nnz
  int64_t nnz = 0;
};
// search_graph.rs:263-360 from a sorted dense kNN graph (raw distances); a
// qualifying prune is taken with probability prune_prob (diversify_prob, 1 = always).
void build_search_graph(const int32_t* knn_idx, const float* knn_dist, const float* X, int N,
                        int k, int D, int Dp, int kind, float mult, cudaStream_t st,
                        TempStorage& tmp, Csr& out, float* min_distance_host, float prune_prob = 1.0f,
                        uint64_t seed = 0);
// search_graph.rs:199-229: row new_v = old row order[new_v], neighbors mapped by inverse.
void reorder_csr(const Csr& in, const int32_t* order, const int32_t* inverse, cudaStream_t st,
                 TempStorage& tmp, Csr& out);

// ---- greedy search (search.cu) ----------------------------------------------
struct SearchIndex {
  int N = 0, D = 0, Dp = 0, kind = 0, corr = 0;
  const float* X = nullptr;              // internal order, N x Dp
  const int32_t* indptr = nullptr;
  const int32_t* indices = nullptr;
  float min_distance = 0.f;
  int n_trees = 0;
  const int32_t* tree_roots = nullptr;   // n_trees
  const int32_t* children = nullptr;
  const float* offsets = nullptr;
  const float* hyperplanes = nullptr;
  const int32_t* tree_idx = nullptr;     // n_trees * N leaf order (internal ids)
  int leaf_budget = 1;
  int frontier_cap = 0;                  // spill-frontier entries per query (leaf_budget > 1)
  int tree_depth = 0;                    // most internal nodes on a root-to-leaf path
  // int8 routing trees (QuantizedFlatTree, flat_tree.rs:35-183): per-node codes
  // (n_nodes x Dq) and scales; used by quantized queries when non-null
  const int8_t* tree_codes = nullptr;
  const float* tree_scales = nullptr;
  const int32_t* vertex_order = nullptr; // internal -> original id
  uint64_t seed = 42;
  // int8 codes (optional)
  const int8_t* codes = nullptr;         // N x Dq (Dq = round_up(D,16))
  const float* inv_norms = nullptr;
  const float* dim_scales = nullptr;     // per-dimension codes: Dq scales (null otherwise)
  int Dq = 0;
};
struct SearchStats {
  unsigned long long evals = 0, expansions = 0, visited_overflow = 0;
};
// Q: nq x Dp device queries.  Results already remapped to original ids.
void greedy_search(const SearchIndex& ix, const float* Q, int nq, int k, float eps,
                   uint64_t qid_base, int32_t* out_idx, float* out_dist, cudaStream_t st,
                   unsigned long long* dstats);
// Per-query parameters of a packed batch (device arrays of nq entries): result
// list width, entries written, exact-rerank width (quantized; may be null), epsilon,
// random stream (added to the index seed; unused by quantized queries, which all use
// the seed alone) and output offset (entries) into out_idx / out_dist.
struct QueryMeta {
  const int32_t* width = nullptr;
  const int32_t* kout = nullptr;
  const int32_t* rerank = nullptr;
  const float* eps = nullptr;
  const uint64_t* stream = nullptr;
  const int64_t* out_off = nullptr;
};
// Packed batch of queries with per-query parameters (Q8/qinv non-null: quantized).
void greedy_search_packed(const SearchIndex& ix, const float* Q, const int8_t* Q8, const float* qinv, int nq,
                          int max_width, const QueryMeta& meta, int32_t* out_idx, float* out_dist, cudaStream_t st,
                          unsigned long long* dstats);
// FlatTree::search_leaves of tree `tree` for nq device queries (nq x Dp FP32
// rows; with Q8, their int8 codes route over the int8 routing trees): up to
// `budget` leaves (start, end) per query into out_leaves (nq x budget x 2) and
// the count into out_counts.
// ---- brute-force exact kNN (brute.cu) ---------------------------------------
// Q: nq x Dp, X: n x Dp (device, Dp a multiple of 4); precision 0 FP32, 2 FP64;
// excl (nullable): per query a row to leave out.  out: nq x k, ascending.
bool brute_supported(int kind);
void brute_force_knn(const float* Q, int nq, const float* X, long long n, int Dp, int k, int kind, int precision,
                     const int32_t* excl, int32_t* out_idx, float* out_dist, cudaStream_t st);

void tree_leaves(const SearchIndex& ix, const float* Q, const int8_t* Q8, int nq, int tree, int budget,
                 uint64_t qid_base, int32_t* out_leaves, int32_t* out_counts, cudaStream_t st,
                 unsigned long long* dstats);
// Quantized search (index.rs:283-334): int8 query codes Q8 (nq x Dq) with scales
// qinv; the result list holds k_search entries; with rerank > 0 the first
// `rerank` results are re-ordered by their exact FP32 distance to Q (index.rs:103-126);
// k_out entries per query are written.  Every query uses the index seed alone.
void greedy_search_quantized(const SearchIndex& ix, const float* Q, const int8_t* Q8, const float* qinv, int nq,
                             int k_search, int k_out, int rerank, float eps, int32_t* out_idx, float* out_dist,
                             cudaStream_t st, unsigned long long* dstats);

// ---- int8 scalar quantization (quantize.cu) -------------------------------------
enum Q8Encoding : int {
  Q8_PER_VECTOR_COSINE = 0,
  Q8_GLOBAL_SYMMETRIC = 1,
  Q8_PER_VECTOR_SYMMETRIC = 2,
  Q8_PER_DIMENSION = 3  // one scale per dimension (quantized.rs:42-56)
};
// 127 / max |x| over `total` floats (0 if all zero), lib.rs:163-174.
float quant_global_multiplier(const float* X, long long total, cudaStream_t st);
// int8 routing-tree codes (n_nodes x Dq) and per-node scales of hyperplanes H
// (n_nodes x Dp), flat_tree.rs:47-64.
void quantize_tree_hyperplanes(const float* H, long long n_nodes, int D, int Dp, int Dq, int8_t* codes, float* scales,
                               cudaStream_t st);
// Per-dimension scales of rows X (n x Dp): dim_scales[j] = max_i |x_ij| / 127
// (0 for a zero column and for j >= D), Dq entries.
void quant_dim_scales(const float* X, long long n, int D, int Dp, int Dq, float* dim_scales, cudaStream_t st);
// Codes (n x Dq, zero-padded beyond D) and per-row scales of rows X (n x Dp);
// the per-dimension encoding takes its scales from dim_scales (device, Dq
// entries) and writes no row scales (scale may be null).
void quantize_rows(const float* X, long long n, int D, int Dp, int Dq, int encoding, float gmult,
                   const float* dim_scales, int8_t* codes, float* scale, cudaStream_t st);

// ---- utilities (util.cu) ------------------------------------------------------
void distance_pairs(int kind, const float* A, const float* B, int64_t n, int D, int Dp,
                    float* out, cudaStream_t st);
void pad_rows(const float* src, int64_t n, int D, int Dp, float* dst, cudaStream_t st);
void gather_rows(const float* src, const int32_t* order, int64_t n, int Dp, float* dst,
                 cudaStream_t st);
void normalize_rows(float* X, int64_t n, int D, int Dp, cudaStream_t st);
void invert_permutation(const int32_t* order, int N, int32_t* inverse, cudaStream_t st);
void apply_correction_dev(float* d, int64_t n, int corr, cudaStream_t st);

}  // namespace rinnd
