/*
 * rinnd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of lmcinnes/rinnd's NN-Descent hot path (the Rust crate
 * rinnd-core), used as the parity checker and as the timed CPU baseline.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library; the product (rinnd_b200) never links or calls it.
 *
 * Every function cites the reference file:line it restates; paths are relative
 * to the reference project root (crates/rinnd-core/src/... = "core/...").
 */
#ifndef RINND_ORACLE_H
#define RINND_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Distance kinds (same numbering as include/rinnd.h). */
enum {
  ORC_SQEUCLIDEAN = 0,        /* core/distance/euclidean.rs:14-93            */
  ORC_MANHATTAN = 1,          /* core/distance/minkowski.rs:11-83            */
  ORC_COSINE = 2,             /* core/distance/cosine.rs:20-113              */
  ORC_ALT_COSINE = 3,         /* core/distance/alternatives.rs:200-231       */
  ORC_ALT_DOT = 4,            /* core/distance/alternatives.rs:15-124        */
  ORC_DIRECT_COSINE = 5,      /* core/distance/alternatives.rs:131-154       */
  ORC_INNER_PRODUCT = 6,      /* core/distance/inner_product.rs:96-107       */
  ORC_ALT_INNER_PRODUCT = 7   /* core/distance/alternatives.rs:160-193       */
};

/* Correction kinds applied to reported distances. */
enum {
  ORC_CORR_NONE = 0,
  ORC_CORR_SQRT = 1,          /* index.rs:587                                */
  ORC_CORR_ALT_COSINE = 2,    /* alternatives.rs:273-277                     */
  ORC_CORR_ALT_IP = 3         /* alternatives.rs:279-287                     */
};

typedef struct orc_params {
  int32_t n_neighbors;
  int32_t n_trees;
  int32_t n_search_trees;
  int32_t search_tree_leaf_budget;
  int32_t leaf_size;        /* <=0 : default clamp(5k,60,256)  index.rs:617-619 */
  int32_t max_candidates;   /* <=0 : default min(k,60)         index.rs:620-622 */
  int32_t n_iters;          /* <=0 : default max(5,ceil(log2N)) index.rs:623-625 */
  float delta;
  uint64_t random_seed;
  float diversify_prob;
  float pruning_degree_multiplier;
  int32_t angular;          /* tree split kind, index.rs:606-614 */
  int32_t distance_kind;    /* ORC_* */
  int32_t correction;       /* ORC_CORR_* */
  int32_t n_threads;        /* <=0 : all OpenMP threads */
  int32_t verbose;
} orc_params;

typedef struct orc_index orc_index;

/* ---- distances ---------------------------------------------------------- */
float orc_distance(int kind, const float* a, const float* b, int32_t dim);
void orc_distance_pairs(int kind, const float* a, const float* b, int64_t n_pairs,
                        int32_t dim, float* out);
float orc_correct(int correction, float d);
int32_t orc_i8_dot(const int8_t* x, const int8_t* y, int32_t dim);
float orc_i8_per_dimension_dot(const int8_t* x, const int8_t* y, const float* scales,
                               int32_t dim);

/* ---- rng (core/rng.rs:15-86, Xoshiro256++ seeded by SplitMix64) -------- */
void orc_rng_u64(uint64_t seed, int32_t n, uint64_t* out);
void orc_rng_float(uint64_t seed, int32_t n, float* out);
void orc_rng_index(uint64_t seed, uint64_t range, int32_t n, uint64_t* out);

/* ---- heaps --------------------------------------------------------------- */
/* Runs a sequence of pushes on a single NeighborHeap row of size k.
 * op: 0 simple_push, 1 checked_push, 2 checked_flagged_push, 3 unchecked_flagged_push.
 * results[i] = 1 if push i was accepted. Row state returned in out_*.
 * neighbor_heap.rs:99-243 */
void orc_neighbor_heap_sequence(int32_t k, int32_t n_ops, const int32_t* op,
                                const int32_t* ids, const float* dists,
                                const uint8_t* flags, int32_t* results,
                                int32_t* out_idx, float* out_dist, uint8_t* out_flags);
/* Applies pushes (row, id, dist, flag) in order to an n x k heap
 * (checked_flagged_push semantics), then returns rows sorted (sort_all). */
void orc_neighbor_heap_apply(int32_t n, int32_t k, int64_t n_ops, const int32_t* rows,
                             const int32_t* ids, const float* dists, const uint8_t* flags,
                             int32_t* out_idx, float* out_dist, uint8_t* out_flags,
                             int64_t* n_accepted);
/* checked_heap_push_flat sequence on one candidate row (candidates.rs:433-484). */
void orc_candidate_heap_sequence(int32_t size, int32_t n_ops, const float* priorities,
                                 const int32_t* ids, float* out_pri, int32_t* out_idx);
/* BoundedHeap (candidate_heap.rs:78-163): pushes then into_sorted. */
int32_t orc_bounded_heap_sequence(int32_t k, int32_t n_ops, const float* dists,
                                  const int32_t* ids, int32_t* accepted,
                                  int32_t* out_idx, float* out_dist);

/* ---- candidates (candidates.rs:51-417) --------------------------------- */
/* Builds new/old candidate lists from a heap (n x k, flags in/out). Uses the
 * parallel two-phase algorithm when n >= 256 and n_threads > 1, else the
 * sequential one (candidates.rs:51-65). */
void orc_build_candidates(int32_t n, int32_t k, const int32_t* heap_idx,
                          uint8_t* heap_flags, int32_t max_candidates, uint64_t seed,
                          int32_t n_threads, int32_t* new_idx, int32_t* old_idx);

/* ---- trees --------------------------------------------------------------- */
/* FlatTree::search_leaves on an explicit tree (flat_tree.rs:239-311).
 * Returns number of hyperplane evaluations; leaves written as (start,end). */
int32_t orc_tree_search_leaves(int32_t n_nodes, int32_t dim, const float* hyperplanes,
                               const float* offsets, const int32_t* children,
                               const float* point, uint64_t seed, int32_t leaf_budget,
                               int32_t* out_leaves, int32_t* n_leaves);

/* QuantizedFlatTree (flat_tree.rs:35-183): per-node int8 codes and scales of
 * the hyperplanes (:47-64), and search_leaves over them (:106-183) for a query's
 * int8 codes and tree_query_scale. */
void orc_quantize_tree_hyperplanes(int32_t n_nodes, int32_t dim, const float* hyperplanes, int8_t* codes,
                                   float* scales);
int32_t orc_tree_search_leaves_quantized(int32_t n_nodes, int32_t dim, const float* hyperplanes,
                                         const float* offsets, const int32_t* children, const int8_t* qcodes,
                                         float qscale, uint64_t seed, int32_t leaf_budget, int32_t* out_leaves,
                                         int32_t* n_leaves);
/* Hyperplane and offset of a split through points p1, p2 (builder.rs:249-308). */
float orc_tree_hyperplane(const float* p1, const float* p2, int32_t dim, int32_t angular, float* hp);
/* Leaf node reached by each of n points under the budget-1 routing rule
 * (flat_tree.rs:253-273); -1 where a margin on the path is a tie (|m| < 1e-8). */
void orc_tree_route_points(int32_t n_nodes, int32_t dim, const float* hyperplanes, const float* offsets,
                           const int32_t* children, const float* points, int64_t n, int32_t* leaf_node);

/* ---- search graph (search_graph.rs:263-567) ----------------------------- */
/* From a sorted dense kNN graph: returns nnz; indptr[n+1], indices[cap]. */
int64_t orc_search_graph_from_knn(const int32_t* knn_idx, const float* knn_dist,
                                  const float* data, int32_t n, int32_t k, int32_t dim,
                                  int kind, float diversify_prob, float mult,
                                  int32_t* indptr, int32_t* indices, int64_t cap,
                                  float* min_distance);
/* weighted_union_pruned on explicit rows (search_graph.rs:368-426). */
int64_t orc_weighted_union_pruned(int32_t n, const int32_t* fwd_ptr, const int32_t* fwd_idx,
                                  const float* fwd_dist, const int32_t* rev_ptr,
                                  const int32_t* rev_idx, const float* rev_dist,
                                  int32_t max_degree, int32_t* indptr, int32_t* indices);

/* ---- full index ---------------------------------------------------------- */
void orc_params_default(orc_params* p);
orc_index* orc_build(const float* data, int64_t n, int32_t dim, const orc_params* p);
orc_index* orc_index_from_parts(const float* data, int64_t n, int32_t dim, int32_t kind, int32_t corr,
                                const int32_t* indptr, const int32_t* indices, float min_distance, int32_t n_trees,
                                const int64_t* tree_nodes, const float* hyperplanes, const float* offsets,
                                const int32_t* children, const int32_t* tree_indices, int32_t leaf_budget,
                                const int32_t* vertex_order, uint64_t seed, int32_t n_threads);
void orc_free(orc_index* idx);
int32_t orc_index_k(const orc_index* idx);
void orc_neighbor_graph(const orc_index* idx, int32_t* out_idx, float* out_dist);
int64_t orc_search_graph_nnz(const orc_index* idx);
void orc_search_graph(const orc_index* idx, int32_t* indptr, int32_t* indices,
                      float* min_distance);
void orc_vertex_order(const orc_index* idx, int32_t* out);
int32_t orc_iterations(const orc_index* idx);
void orc_timings(const orc_index* idx, double* out5);
void orc_query(const orc_index* idx, const float* queries, int64_t nq, int32_t k,
               float epsilon, int32_t* out_idx, float* out_dist);
void orc_query_one(const orc_index* idx, const float* query, int32_t k, float epsilon,
                   int32_t* out_idx, float* out_dist);

/* ---- int8 serving (crates/rinnd/src/lib.rs:159-358, index.rs:283-334) -- */
/* encoding: 0 int8 per-vector cosine, 1 sq8u global symmetric, 2 sq8p per-vector
 * (orc_query_quantized also takes 3: per-dimension symmetric codes). */
void orc_quantize_rows(const float* data, int64_t n, int32_t dim, int32_t encoding,
                       int8_t* codes, float* inv_norms, float* global_mult);
/* quantize_query (lib.rs:325-358) with the index's global multiplier `global_mult`
 * (used by encoding 1 only): codes nq x dim, per-query scale (query_inv_norm). */
void orc_quantize_queries(const float* queries, int64_t nq, int32_t dim, int32_t encoding,
                          float global_mult, int8_t* codes, float* scales);
/* Per-dimension symmetric int8 codes for quantized_i8_per_dimension_dot
 * (quantized.rs:42-56): dim_scales[j] = max_i |x_ij| / 127, codes = clamp(round(x /
 * scale_j), +-127) (encoding 3 of orc_query_quantized).  The query form uses the
 * index's scales. */
void orc_quantize_per_dimension(const float* data, int64_t n, int32_t dim, int8_t* codes, float* dim_scales);
void orc_quantize_queries_per_dimension(const float* queries, int64_t nq, int32_t dim, const float* dim_scales,
                                        int8_t* codes);
/* orc_query_quantized with int8 routing trees when quantize_trees != 0
 * (tree_quantization="int8", lib.rs:681-704). */
int32_t orc_query_quantized_trees(const orc_index* idx, const float* queries, int64_t nq, int32_t k,
                                  float epsilon, int32_t encoding, int32_t candidate_width,
                                  int32_t rerank_width, int32_t quantize_trees, int32_t* out_idx, float* out_dist);
/* normalize_rows_inplace (lib.rs:1131-1146). */
void orc_normalize_rows(float* data, int64_t n, int32_t dim);
int32_t orc_query_quantized(const orc_index* idx, const float* queries, int64_t nq,
                            int32_t k, float epsilon, int32_t encoding,
                            int32_t candidate_width, int32_t rerank_width,
                            int32_t* out_idx, float* out_dist);

/* ---- exact kNN (FP64) ----------------------------------------------------- */
void orc_exact_knn_f64(int kind, const float* data, int64_t n, const float* queries,
                       int64_t nq, int32_t dim, int32_t k, int32_t exclude_self,
                       int32_t* out_idx, double* out_dist);

int32_t orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
