/*
 * rinnd.h -- C ABI of the B200-native NN-Descent engine (librinnd_b200.so).
 *
 * Drop-in boundary for lmcinnes/rinnd's build/query path.  Plain pointers and
 * sizes only.  Every call returns RINND_OK (0) or a negative RINND_ERR_* code;
 * rinnd_last_error() returns a thread-local message for the last failure.
 * Host pointers are read/written synchronously unless a name says "device".
 *
 * Reference interfaces replaced (paths relative to the reference root; core/ =
 * crates/rinnd-core/src/):
 *   NNDescentBuilder::new + setters + build_with_distance   core/index.rs:449-733
 *   NNDescentIndex::query / query_one                        core/index.rs:389-439
 *   NNDescentIndex::query_one_quantized_i8_with_workspace    core/index.rs:283-334
 *   RINND(...) constructor / query / neighbor_graph / search_graph / storage_info
 *                                                            crates/rinnd/src/lib.rs:616-1103
 */
#ifndef RINND_H
#define RINND_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RINND_EXPORT __attribute__((visibility("default")))
#else
#define RINND_EXPORT
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define RINND_OK 0
#define RINND_ERR_INVALID (-1)   /* bad argument (reference: ValueError / assert!) */
#define RINND_ERR_OOM (-2)       /* device allocation failed (MemoryError)          */
#define RINND_ERR_CUDA (-3)      /* CUDA runtime failure (RuntimeError)             */
#define RINND_ERR_NO_DEVICE (-4) /* no CUDA device visible                         */
#define RINND_ERR_INTERNAL (-5)
#define RINND_ERR_BUSY (-6)      /* server queue full: collect completed requests, retry */

/* ---- distance kinds: the reference's build distances and proxies -------- */
#define RINND_DIST_SQEUCLIDEAN 0        /* core/distance/euclidean.rs:14-93    */
#define RINND_DIST_MANHATTAN 1          /* core/distance/minkowski.rs:11-83    */
#define RINND_DIST_COSINE 2             /* core/distance/cosine.rs:20-113      */
#define RINND_DIST_ALT_COSINE 3         /* core/distance/alternatives.rs:200-231 */
#define RINND_DIST_ALT_DOT 4            /* core/distance/alternatives.rs:15-124  */
#define RINND_DIST_DIRECT_COSINE 5      /* core/distance/alternatives.rs:131-154 */
#define RINND_DIST_INNER_PRODUCT 6      /* core/distance/inner_product.rs:96-107 */
#define RINND_DIST_ALT_INNER_PRODUCT 7  /* core/distance/alternatives.rs:160-193 */
/* The reference's other metrics (built with their own distance, no correction,
 * crates/rinnd/src/lib.rs:1276-1293), evaluated per pair by generic kernels. */
#define RINND_DIST_CHEBYSHEV 8          /* core/distance/minkowski.rs:106-121 */
#define RINND_DIST_CANBERRA 9           /* core/distance/minkowski.rs:165-181 */
#define RINND_DIST_BRAYCURTIS 10        /* core/distance/minkowski.rs:191-212 */
#define RINND_DIST_CORRELATION 11       /* core/distance/angular.rs:13-52     */
#define RINND_DIST_TRUE_ANGULAR 12      /* core/distance/angular.rs:62-90     */
#define RINND_DIST_TSSS 13              /* core/distance/angular.rs:99-133    */
#define RINND_DIST_HAMMING 14           /* core/distance/binary.rs:13-32      */
#define RINND_DIST_JACCARD 15           /* core/distance/binary.rs:42-68      */
#define RINND_DIST_DICE 16              /* core/distance/binary.rs:142-167    */
#define RINND_DIST_MATCHING 17          /* core/distance/binary.rs:113-132    */
#define RINND_DIST_KULSINSKI 18         /* core/distance/binary.rs:177-203    */
#define RINND_DIST_ROGERSTANIMOTO 19    /* core/distance/binary.rs:213-229    */
#define RINND_DIST_RUSSELLRAO 20        /* core/distance/binary.rs:239-258    */
#define RINND_DIST_SOKALMICHENER 21     /* core/distance/binary.rs:268-276    */
#define RINND_DIST_SOKALSNEATH 22       /* core/distance/binary.rs:286-311    */
#define RINND_DIST_YULE 23              /* core/distance/binary.rs:321-353    */
#define RINND_DIST_HELLINGER 24         /* core/distance/hellinger.rs:16-44   */
#define RINND_DIST_JENSEN_SHANNON 25    /* core/distance/hellinger.rs:98-128  */
#define RINND_DIST_SYMMETRIC_KL 26      /* core/distance/hellinger.rs:137-166 */

/* ---- corrections applied to reported distances -------------------------- */
#define RINND_CORR_NONE 0
#define RINND_CORR_SQRT 1        /* index.rs:587                    */
#define RINND_CORR_ALT_COSINE 2  /* alternatives.rs:273-277          */
#define RINND_CORR_ALT_IP 3      /* alternatives.rs:279-287          */

/* ---- int8 encodings (crates/rinnd/src/lib.rs:151-156) ------------------- */
#define RINND_Q8_PER_VECTOR_COSINE 0  /* "int8"  */
#define RINND_Q8_GLOBAL_SYMMETRIC 1   /* "sq8u"  */
#define RINND_Q8_PER_VECTOR_SYMMETRIC 2 /* "sq8p" */
/* "sq8d" (no counterpart in the reference's encoders): one symmetric scale per
 * dimension, scale_j = max_i |x_ij| / 127 over the index rows, code =
 * clamp(round(x / scale_j), +-127); the search similarity is the reference's
 * quantized_i8_per_dimension_dot (core/distance/quantized.rs:42-56). */
#define RINND_Q8_PER_DIMENSION 3

/* Local-join tile arithmetic (no counterpart in the reference, whose join is FP32):
 * FP32 evaluates every candidate pair in FP32; BF16 filters the pairs with BF16
 * Gram tiles on the tensor cores (FP32 accumulate) and recomputes every pair
 * that may beat its row's threshold in exact FP32 before it is pushed.
 * Manhattan and candidate lists longer than 32 use the FP32 tiles. */
#define RINND_PRECISION_FP32 0
#define RINND_PRECISION_BF16 1

/* Mirrors NNDescentBuilder's fields (core/index.rs:449-494) plus the metric
 * dispatch decisions the Python layer makes (crates/rinnd/src/lib.rs:1175-1297). */
typedef struct rinnd_build_params {
  int32_t n_neighbors;              /* default 30                                  */
  int32_t n_trees;                  /* default 8                                   */
  int32_t n_search_trees;           /* default 1                                   */
  int32_t search_tree_leaf_budget;  /* default 1; leaves seeded per search tree (<= 256) */
  int32_t leaf_size;                /* <= 0: clamp(5k, 60, 256)  (index.rs:617-619) */
  int32_t max_candidates;           /* <= 0: min(k, 60)          (index.rs:620-622) */
  int32_t n_iters;                  /* <= 0: max(5, ceil(log2 N)) (index.rs:623-625) */
  float delta;                      /* default 0.001                               */
  uint64_t random_seed;             /* default 42                                  */
  float diversify_prob;             /* default 1.0: chance a qualifying prune is taken */
  float pruning_degree_multiplier;  /* default 1.5                                 */
  int32_t angular;                  /* angular RP splits (index.rs:606-614)        */
  int32_t distance_kind;            /* RINND_DIST_*                                */
  int32_t correction;               /* RINND_CORR_*                                */
  int32_t normalize;                /* L2-normalize rows before build (lib.rs:710-712) */
  int32_t verbose;
  int32_t device;                   /* CUDA device ordinal, default 0              */
  int32_t precision;                /* RINND_PRECISION_*: local-join tile arithmetic */
  int32_t join_tuning;              /* RINND_TUNE_*: tile shape of the pipelined FP32 join */
  int32_t reserved[5];
} rinnd_build_params;

/* Tile shape of the pipelined FP32 local join (row stages in flight per CTA,
 * candidate rows per work item, CTAs per SM).  RINND_TUNE_TABLE (default): the
 * shape tuned earlier in this process for the build's (device, padded
 * dimension, list length class, metric class, grouped) key, else one tuned now
 * by timing every shape on a sample of the first iteration's candidate lists
 * (the heaps are restored afterwards, so the build's result distribution does
 * not change); RINND_TUNE_FIXED: the default shape, no trials; RINND_TUNE_RETUNE:
 * trials even when the table has the key.  rinnd_join_tile_table lists the
 * table: 8 ints per row (device, Dp, list class 32|64, metric class 0 squared
 * Euclidean / 1 Manhattan / 2 dot forms, grouped, stages, rows per item, CTAs
 * per SM with 0 = as many as shared memory allows); rows = NULL just counts. */
#define RINND_TUNE_TABLE 0
#define RINND_TUNE_FIXED 1
#define RINND_TUNE_RETUNE 2
RINND_EXPORT int rinnd_join_tile_table(int32_t* rows, int32_t cap, int32_t* n_rows);
RINND_EXPORT int rinnd_join_tile_table_clear(void);
/* Stores one table row (8 ints as above): later builds of that key with
 * RINND_TUNE_TABLE (and rinnd_nndescent_step) run the shape without trials. */
RINND_EXPORT int rinnd_join_tile_set(const int32_t* row);

typedef struct rinnd_index rinnd_index;

/* Per-phase timings and counters of the last build. */
typedef struct rinnd_build_info {
  int32_t iterations;
  int32_t forest_levels;
  int64_t n_leaves;
  double ms_forest, ms_leaf_init, ms_iterations, ms_candidates, ms_join, ms_sort, ms_graph, ms_total;
  uint64_t pairs_evaluated;      /* local-join pair distances over all iterations */
  uint64_t pushes_accepted;      /* heap changes over all iterations              */
  uint64_t push_contention;      /* pushes abandoned after the bounded retry count */
  int64_t search_graph_nnz;
  float min_distance;
  uint64_t join_rows_gathered;   /* candidate rows gathered by the join kernel      */
  double ms_join_kernel;         /* CUDA-event time of the local-join kernel launches */
  uint64_t kernel_launches;      /* kernels this library launched during the build  */
  uint64_t join_kernel_launches; /* local-join kernel launches (ms_join_kernel covers these) */
  uint64_t join_updates;         /* updates the join kernels appended for the heap pushes */
  int32_t join_form;             /* RINND_JOIN_* of the last iteration's local join      */
  int32_t group_items;           /* indices built together with this one (1 = alone; see
                                    rinnd_build_many_ex): times and counters are the group's */
  int32_t join_tile_stages;      /* tile shape the pipelined FP32 join ran (RINND_TUNE_*) */
  int32_t join_tile_rows;
  int32_t join_tile_ctas_per_sm;
  int32_t join_tile_tuned;       /* 1: this build ran the tile trials                     */
} rinnd_build_info;

/* Local-join kernels (rinnd_build_info.join_form).  The pipelined FP32 join
 * holds a vertex's candidate rows in shared memory (rows padded to Dp =
 * round_up(D, 4) floats: Dp <= 424 with candidate lists of <= 32, Dp <= 204 with
 * longer lists); the tensor-core form (precision BF16) needs lists of <= 32 and
 * a non-Manhattan metric of the tiled family (any D: the Gram tiles stream K
 * in chunks); other builds use the chunked FP32 join (the generic metrics their
 * per-pair kernel). */
#define RINND_JOIN_CHUNKED_FP32 0
#define RINND_JOIN_PIPELINED_FP32 1
#define RINND_JOIN_TENSOR_BF16 2

/* ---- lifecycle ------------------------------------------------------------ */
RINND_EXPORT int rinnd_params_default(rinnd_build_params* p);
/* NNDescentBuilder::build_with_distance (core/index.rs:601-733) from host rows (n x d f32). */
RINND_EXPORT int rinnd_build(const float* data, int64_t n, int32_t d, const rinnd_build_params* p,
                rinnd_index** out);
/* Same, with the rows already on the device (row stride `ld` floats, ld >= d). */
RINND_EXPORT int rinnd_build_device(const float* d_data, int64_t n, int32_t d, int64_t ld,
                       const rinnd_build_params* p, rinnd_index** out);
/* General form: rows on host or device (`data_on_device`), all build work on
 * `stream` (a cudaStream_t; NULL = a stream owned by the index).  A caller
 * stream is adopted by the index for its later calls and must outlive it. */
RINND_EXPORT int rinnd_build_on_stream(const float* data, int32_t data_on_device, int64_t n, int32_t d,
                                       int64_t ld, const rinnd_build_params* p, void* stream,
                                       rinnd_index** out);
RINND_EXPORT int rinnd_free(rinnd_index* idx);
/* Index files (no counterpart in the reference, whose indices live in memory
 * only): rinnd_save writes every resident array of the index (rows in search
 * layout, graphs, trees, int8 codes) and `meta`, an opaque caller string (may
 * be NULL), to `path`; rinnd_load reads such a file onto `device` and returns
 * the index, whose queries then return exactly what the saved index's did.
 * meta (meta_cap bytes, may be NULL) receives the stored string NUL-terminated
 * and *meta_len (may be NULL) its full length.  A file of another format or
 * version, or a truncated one, fails with RINND_ERR_INVALID. */
RINND_EXPORT int rinnd_save(rinnd_index* idx, const char* path, const char* meta);
RINND_EXPORT int rinnd_load(const char* path, int32_t device, rinnd_index** out, char* meta, int64_t meta_cap,
                            int64_t* meta_len);
/* ---- batched form: many independent indices ------------------------------- */
/* One index of a batch: n x d f32 rows (row stride ld floats) on the host or,
 * with data_on_device, in device memory of params->device; params as for
 * rinnd_build (metric, k, precision, ... per index). */
typedef struct rinnd_batch_item {
  const float* data;
  int64_t n;
  int32_t d;
  int32_t data_on_device;
  int64_t ld;
  const rinnd_build_params* params;
} rinnd_batch_item;
/* Options of the batched form. */
typedef struct rinnd_batch_options {
  int32_t n_workers;          /* host threads driving groups (0 = min(tasks, 16))                 */
  int32_t grouped;            /* 1 (default): indices of one NN-Descent shape are built as a group */
  int64_t max_group_points;   /* rows per group at most (default 8 Mi; 0 = no cap)                  */
  int32_t capture_iterations; /* 1 (default): each grouped iteration runs as one CUDA graph          */
  int32_t reserved;
} rinnd_batch_options;
RINND_EXPORT int rinnd_batch_options_default(rinnd_batch_options* o);
/* Builds n_items independent indices (no counterpart in the reference, which
 * builds one index per call).  Grouped (the default): items with equal device,
 * d, distance kind, normalize, angular, n_neighbors, resolved candidate-list
 * length, resolved leaf size and precision form a group (split to at most
 * max_group_points rows) whose NN-Descent runs once over all its rows: one
 * forest pass with every index's trees as root segments, one leaf
 * initialization, and per iteration one candidate pass and one join launch
 * family whose persistent CTAs walk the vertices of every index in the group.
 * Each index keeps its own n_iters cap and delta test (its rows stop sampling
 * candidates once it stops); trees, candidate draws and priorities are keyed by
 * the group's first index's random_seed and the rows' positions in the group,
 * so an index's graph is a valid build of its parameters but not bit-identical
 * to its one-at-a-time build.  Search graph, reorder and search trees are made
 * per index; each index's build_info reports the group's phase times and
 * counters with group_items = the group's size.  With capture_iterations, a
 * group's iteration (candidate pass, join launches, update applications and
 * the counter read-back) is stream-captured into a CUDA graph and launched as
 * one unit; later iterations update the executable graph in place, and
 * ms_join then covers the whole iteration (ms_candidates and ms_join_kernel
 * are 0).  Items alone in their group,
 * or all items with grouped = 0, are built as by rinnd_build, concurrently on
 * one stream each.  n_workers host threads take groups longest first
 * (estimated n * d * k).  An item whose data or params are invalid fails
 * alone.  out[i] receives index i (NULL on failure) and status[i] (may be NULL)
 * its status code.  Returns RINND_OK when every item built, else the first
 * failing item's code with its message in rinnd_last_error(). */
RINND_EXPORT int rinnd_build_many_ex(const rinnd_batch_item* items, int32_t n_items,
                                     const rinnd_batch_options* options, rinnd_index** out, int32_t* status);
/* rinnd_build_many_ex with the default options and n_workers. */
RINND_EXPORT int rinnd_build_many(const rinnd_batch_item* items, int32_t n_items, int32_t n_workers,
                                  rinnd_index** out, int32_t* status);
RINND_EXPORT int rinnd_build_info_get(const rinnd_index* idx, rinnd_build_info* info);
RINND_EXPORT int rinnd_index_shape(const rinnd_index* idx, int64_t* n, int32_t* d, int32_t* k);

/* ---- queries -------------------------------------------------------------- */
/* NNDescentIndex::query (core/index.rs:406-439): nq x d host queries -> nq x k
 * results in original ids, corrected distances, (-1, +inf) padding.  Query i
 * uses random stream seed + qid_base + i (index.rs:165). */
RINND_EXPORT int rinnd_query(rinnd_index* idx, const float* queries, int64_t nq, int32_t k, float epsilon,
                int32_t* out_idx, float* out_dist);
/* NNDescentIndex::query_one (core/index.rs:390-392): stream seed + 0. */
RINND_EXPORT int rinnd_query_one(rinnd_index* idx, const float* query, int32_t k, float epsilon,
                    int32_t* out_idx, float* out_dist);
/* Device-resident queries/results (row stride d rounded up to 4 floats is NOT
 * required: rows are `ld` floats apart). */
RINND_EXPORT int rinnd_query_device(rinnd_index* idx, const float* d_queries, int64_t nq, int64_t ld,
                       int32_t k, float epsilon, uint64_t qid_base, int32_t* d_out_idx,
                       float* d_out_dist, void* stream);

/* ---- graph exports ----------------------------------------------------------- */
/* neighbor_graph property (crates/rinnd/src/lib.rs:1087-1103): n x k ids and
 * corrected distances sorted ascending. */
RINND_EXPORT int rinnd_neighbor_graph(const rinnd_index* idx, int32_t* out_idx, float* out_dist);
/* search_graph property (lib.rs:1013-1025, index.rs:137-141): CSR in original id order. */
RINND_EXPORT int rinnd_search_graph_nnz(const rinnd_index* idx, int64_t* nnz);
RINND_EXPORT int rinnd_search_graph(const rinnd_index* idx, int32_t* indptr, int32_t* indices,
                       float* min_distance);
/* Internal (search-layout) vertex order: vertex_order[internal] = original id (index.rs:679-715). */
RINND_EXPORT int rinnd_vertex_order(const rinnd_index* idx, int32_t* out);
/* export_search_tree (crates/rinnd/src/lib.rs:1105-1128, core/index.rs:145-154):
 * the first retained RP tree in the reference's FlatTree layout, nodes numbered
 * in depth-first preorder from the root (node 0): hyperplanes n_nodes x d
 * (zeros for leaves), offsets n_nodes, children n_nodes x 2 (child node ids for
 * an internal node, (-start, -end) into `indices` for a leaf), indices n leaf
 * order in original ids.  `pivots` (n_nodes x 2, no counterpart in the
 * reference) receives the two original points whose split gave each internal
 * node its hyperplane (-1 for leaves).  Call with every array NULL to get
 * *n_nodes first; any array may be NULL.  Fails with RINND_ERR_INVALID when the
 * index retains no search tree (n_search_trees = 0). */
RINND_EXPORT int rinnd_export_search_tree(rinnd_index* idx, int64_t* n_nodes, float* hyperplanes, float* offsets,
                                          int32_t* children, int32_t* indices, int32_t* pivots);

/* ---- int8 serving (crates/rinnd/src/lib.rs:159-416, core/index.rs:283-334) -- */
/* Encodes the index rows (must be built with RINND_DIST_DIRECT_COSINE on
 * normalized rows) with one of RINND_Q8_*. */
RINND_EXPORT int rinnd_quantize(rinnd_index* idx, int32_t encoding);
/* Quantized greedy search + optional exact FP32 rerank; width rules of
 * core/index.rs:55-89.  Uses random stream seed + 0 for every query (index.rs:298). */
RINND_EXPORT int rinnd_query_quantized(rinnd_index* idx, const float* queries, int64_t nq, int32_t k,
                          float epsilon, int32_t candidate_width, int32_t rerank_width,
                          int32_t* out_idx, float* out_dist);
/* tree_quantization="int8" (crates/rinnd/src/lib.rs:681-704, QuantizedFlatTree
 * core/tree/flat_tree.rs:35-183): int8 codes and one scale per node of the
 * search trees' hyperplanes; quantized queries then route with the
 * reconstructed margin dot(codes) * scale * tree_query_scale + offset.  Needs a
 * quantized index with a per-vector encoding (int8 or sq8p). */
RINND_EXPORT int rinnd_quantize_trees(rinnd_index* idx);
/* retain_fp32_data=False (lib.rs:712-716): frees the FP32 rows of a quantized
 * index; afterwards FP32 queries and exact reranks fail with RINND_ERR_INVALID. */
RINND_EXPORT int rinnd_release_fp32(rinnd_index* idx);
/* FlatTree::search_leaves (flat_tree.rs:239-311) of retained tree `tree` for nq
 * host queries (normalized like the index's queries) with the search kernel's
 * routing: up to `budget` leaves per query as (start, end) ranges into the
 * tree's leaf order (out_leaves, nq x budget x 2) and their count (out_counts).
 * quantized != 0 routes the queries' int8 codes over the int8 routing trees.
 * Tied margins (|m| < 1e-8) take a side from the query's search stream. */
RINND_EXPORT int rinnd_tree_search_leaves(rinnd_index* idx, const float* queries, int64_t nq, int32_t tree,
                                          int32_t budget, int32_t quantized, int32_t* out_leaves,
                                          int32_t* out_counts);
/* Per-dimension encoder (RINND_Q8_PER_DIMENSION) for host rows (n x d f32):
 * codes (n x d int8) and the d per-dimension scales. */
RINND_EXPORT int rinnd_quantize_rows_per_dimension(const float* data, int64_t n, int32_t d, int8_t* codes,
                                                   float* dim_scales);
/* Row encoder of QuantizedI8Index::new (lib.rs:159-223) on the GPU for host rows
 * (n x d f32): codes (n x d int8), per-row scales (inv_norms) and the global
 * multiplier 127 / max|x|. */
RINND_EXPORT int rinnd_quantize_rows(const float* data, int64_t n, int32_t d, int32_t encoding, int8_t* codes,
                                     float* scales, float* global_multiplier);

/* ---- serving form: continuous batching over one resident index ------------ */
/* No counterpart in the reference (one query call at a time, lib.rs:775-874).
 * A server owns a dispatcher thread that packs the queries of pending requests
 * (any mix of sizes, k and epsilon) into device batches of up to
 * max_batch_queries, keeps up to max_inflight batches on the device at once and
 * admits new queries into a batch slot as soon as it frees up.  Each query runs
 * with its own parameters and random stream (its index within its request), so
 * a request's results equal rinnd_query (quantized = 0) or rinnd_query_quantized
 * with the server's widths (quantized = 1, a quantized index) run alone.  The
 * index must outlive the server; submit and poll may be called from any thread. */
typedef struct rinnd_server_params {
  int32_t max_batch_queries;     /* queries per device batch, default 32768            */
  int32_t max_inflight;          /* batches on the device at once, default 8           */
  int32_t max_k;                 /* largest k accepted, default 256 (sizes the buffers) */
  int32_t quantized;             /* 1: int8 search (+ exact rerank) on a quantized index */
  int32_t candidate_width;       /* quantized widths, rules of core/index.rs:55-89      */
  int32_t rerank_width;
  int64_t max_pending_queries;   /* queued, undispatched queries; default 4,194,304    */
  int32_t reserved[8];
} rinnd_server_params;
typedef struct rinnd_server_stats {
  uint64_t completed_requests, completed_queries, batches, pending_queries;
  double mean_batch_queries;
  double p50_ms, p99_ms, max_ms;     /* request latency, submission to completion */
  int32_t peak_inflight;
  int32_t reserved[7];
} rinnd_server_stats;
typedef struct rinnd_server rinnd_server;
RINND_EXPORT int rinnd_server_params_default(rinnd_server_params* p);
RINND_EXPORT int rinnd_server_create(rinnd_index* idx, const rinnd_server_params* p, rinnd_server** out);
/* Copies the nq x d query rows; returns at once with the request id. */
RINND_EXPORT int rinnd_server_submit(rinnd_server* s, const float* queries, int64_t nq, int32_t k, float epsilon,
                                     int64_t* request_id);
/* Waits up to wait_ms for the request; *done = 1: nq x k results copied out and
 * the request released (its id is then unknown), 0: still running. */
RINND_EXPORT int rinnd_server_poll(rinnd_server* s, int64_t request_id, int32_t wait_ms, int32_t* out_idx,
                                   float* out_dist, int32_t* done);
RINND_EXPORT int rinnd_server_stats_get(rinnd_server* s, rinnd_server_stats* out);
/* Finishes the batches in flight and every queued request, then frees the server. */
RINND_EXPORT int rinnd_server_destroy(rinnd_server* s);

/* Search counters of an index since it was built (or last reset): distance
 * evaluations, node expansions and visited-table overflows (ids skipped because
 * their table had no free slot within the probe limit).  reset != 0 zeroes them. */
RINND_EXPORT int rinnd_search_stats_get(rinnd_index* idx, uint64_t* evaluations, uint64_t* expansions,
                                        uint64_t* visited_overflows, int32_t reset);
/* All search counters since the last reset (8 words): evaluations, expansions,
 * visited-table overflows, spill-frontier overflows, queries re-run with the
 * wide bounded state, queries re-run with the exact state, query runs that
 * used the second-level (global-memory) visited table, query runs that moved
 * seeds to the global-memory back store.  A query is re-run when its bounded
 * state could have changed its result (see rinnd_query); the re-run's result
 * is the one returned. */
RINND_EXPORT int rinnd_search_counters(rinnd_index* idx, uint64_t* out, int32_t reset);

/* ---- storage info (crates/rinnd/src/lib.rs:1028-1077) ---------------------- */
typedef struct rinnd_storage_info {
  char encoding[32];
  int64_t code_bytes, metadata_bytes, retained_fp32_bytes;
  double encode_seconds;
  int64_t device_bytes;           /* device memory the index holds (no counterpart) */
  /* quantized_tree_storage_info / released bytes (lib.rs:1037-1061) */
  int64_t tree_code_bytes, tree_scale_bytes, tree_offset_bytes, tree_topology_bytes;
  int64_t released_fp32_tree_bytes, released_fp32_data_bytes, retained_fp32_tree_topology_bytes;
} rinnd_storage_info;
RINND_EXPORT int rinnd_storage_info_get(const rinnd_index* idx, rinnd_storage_info* info);

/* ---- component entry points (parity tests, tools) -------------------------- */
/* out[i] = distance(kind, a[i], b[i]) over n_pairs row pairs (host, n x d each);
 * reference accumulation order, core/distance/*.rs. */
RINND_EXPORT int rinnd_distance_pairs(int32_t kind, const float* a, const float* b, int64_t n_pairs, int32_t d,
                         float* out);
/* Brute-force exact kNN.  No counterpart in the reference, which has no exact
 * pass; its recall criteria are measured against these neighbors.  For each of
 * nq query rows, the k data rows of smallest (distance, id), ascending, padded
 * with (-1, +inf) when n < k.  data: n x d floats with row stride ld_data,
 * queries: nq x d with stride ld_queries; on the current device when on_device
 * != 0 (outputs are then device pointers too), else host memory.
 * distance_kind: RINND_DIST_SQEUCLIDEAN, _MANHATTAN, _INNER_PRODUCT, _COSINE or
 * _DIRECT_COSINE.  precision: RINND_BRUTE_FP32 (the FP32 join's per-pair
 * arithmetic, so distances equal the build's), RINND_BRUTE_BF16 (BF16
 * tensor-core Gram tiles filter the pairs with a rigorous lower bound and the
 * survivors are recomputed in that FP32 arithmetic: the FP32 form's results,
 * for d <= 128, k <= 32 and squared Euclidean or a dot form; other shapes are
 * rejected) or RINND_BRUTE_FP64 (every term in double: the checker the FP32
 * form's ids are compared with).  exclude_ids
 * (nullable, nq entries): query i leaves out data row exclude_ids[i] (the kNN
 * graph of the data itself).  k in [1, 128]. */
#define RINND_BRUTE_FP32 0
#define RINND_BRUTE_BF16 1
#define RINND_BRUTE_FP64 2
RINND_EXPORT int rinnd_brute_force_knn(const float* data, int64_t n, int64_t ld_data, const float* queries,
                                       int64_t nq, int64_t ld_queries, int32_t d, int32_t k, int32_t distance_kind,
                                       int32_t precision, const int32_t* exclude_ids, int32_t on_device,
                                       int32_t* out_idx, float* out_dist);

/* SearchGraph::from_dense_diversified (core/graph/search_graph.rs:263-360) on a
 * host kNN graph (n x k, ascending rows, -1 padding) over host data (n x d).
 * indices must hold n * round(mult * k) entries; *nnz receives the edge count. */
RINND_EXPORT int rinnd_search_graph_from_knn(const int32_t* knn_idx, const float* knn_dist, const float* data,
                                int32_t n, int32_t k, int32_t d, int32_t kind, float mult,
                                int32_t* indptr, int32_t* indices, int64_t* nnz,
                                float* min_distance);
/* Concurrent NeighborHeap::checked_flagged_push (core/heap/neighbor_heap.rs:149-177):
 * applies n_ops pushes (row, id, dist, is_new) to an empty n x k heap on the
 * device, all at once, then sort_all (:293-320).  Returns accepted pushes. */
RINND_EXPORT int rinnd_heap_push_batch(int32_t n, int32_t k, int64_t n_ops, const int32_t* rows,
                          const int32_t* ids, const float* dists, const uint8_t* flags,
                          int32_t* out_idx, float* out_dist, uint8_t* out_flags,
                          int64_t* n_accepted);
/* One NN-Descent iteration (nndescent/mod.rs:101-155: candidate sampling,
 * candidates.rs:51-484, then the local join, mod.rs:321-491) on host arrays:
 * idx/dist/flags (n x k, -1 = empty) hold the neighbor heap rows on entry
 * (distances raw, of `kind`) and the sorted rows after the iteration; `changes`
 * receives the number of successful pushes.  `precision` selects the join tiles
 * (RINND_PRECISION_*); the candidate sample depends only on the rows' contents,
 * `seed` and `iteration`.  `join_form` (may be NULL) receives the RINND_JOIN_*
 * of the join kernel that ran. */
RINND_EXPORT int rinnd_nndescent_step(const float* data, int64_t n, int32_t d, int32_t k, int32_t max_candidates,
                                      int32_t kind, int32_t precision, uint64_t seed, int32_t iteration,
                                      int32_t* idx, float* dist, uint8_t* flags, int64_t* changes,
                                      int32_t* join_form);

/* No counterpart in the reference.  The same operation as rinnd_heap_push_batch
 * for callers that may not allocate device memory (a host engine that owns the
 * whole device budget, code that must not call cudaMalloc/cudaFree): every
 * pointer is caller-owned device memory (d_flags and d_out_flags may be NULL),
 * `stream` is a cudaStream_t (NULL = legacy default stream), and the n x k rows
 * live in a static device scratch of 1,048,576 slots that every device loading
 * the library holds until exit.  Limits: n <= 65536 and n * round_up(k, 16) <=
 * 1,048,576; larger requests fail with RINND_ERR_INVALID.  The first call on a
 * device resolves the scratch address and should come before any stream
 * capture.  Calls that overlap on the GPU race on the shared scratch.  Every
 * call synchronizes `stream` before it returns, to read back *n_accepted and
 * its validity count.  Pushes are validated on the device with the bounds of
 * rinnd_heap_push_batch (row in [0, n), id in [0, 2^31 - 2)); when any push is
 * invalid the call returns RINND_ERR_INVALID, and the outputs have already been
 * overwritten with the rows built from the valid pushes. */
RINND_EXPORT int rinnd_heap_push_batch_noalloc(int32_t n, int32_t k, int64_t n_ops, const int32_t* d_rows,
                                               const int32_t* d_ids, const float* d_dists,
                                               const uint8_t* d_flags, int32_t* d_out_idx,
                                               float* d_out_dist, uint8_t* d_out_flags,
                                               int64_t* n_accepted, void* stream);

/* ---- misc ------------------------------------------------------------------- */
RINND_EXPORT const char* rinnd_last_error(void);
RINND_EXPORT const char* rinnd_version(void);
RINND_EXPORT int rinnd_device_count(int32_t* count);
/* Compiled target of this library's kernels on the current device, from
 * cudaFuncGetAttributes: binaryVersion (100 for sm_100a code) and, when
 * ptx_version is not NULL, ptxVersion (the virtual architecture the code was
 * compiled from, 100 for compute_100a). */
RINND_EXPORT int rinnd_kernel_target(int32_t* binary_version, int32_t* ptx_version);
/* Number of kernels this library has launched in the process so far. */
RINND_EXPORT int rinnd_kernel_launches(uint64_t* count);

#ifdef __cplusplus
}
#endif
#endif /* RINND_H */
