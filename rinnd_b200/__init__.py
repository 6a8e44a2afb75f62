"""rinnd_b200 -- B200-native NN-Descent engine behind the reference's ``rinnd.RINND`` API.

``RINND`` mirrors the PyO3 class of lmcinnes/rinnd (crates/rinnd/src/lib.rs:61-1103):
the same constructor keywords and defaults, metric dispatch, ``ValueError``
messages, output dtypes (int32 ids, float32 distances) and methods.  All compute
runs in librinnd_b200.so (hand-written sm_100a CUDA) through the C ABI in
include/rinnd.h; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import threading
import time

import numpy as np

from . import _lib as L

__all__ = ["RINND", "Server", "build_many", "load", "version", "simd_info", "device_count"]

# Metric::from_str aliases (core/distance/mod.rs:203-247).
_ALIASES = {
    "euclidean": "euclidean", "l2": "euclidean",
    "sqeuclidean": "sqeuclidean", "squared_euclidean": "sqeuclidean",
    "manhattan": "manhattan", "taxicab": "manhattan", "l1": "manhattan",
    "cosine": "cosine", "inner_product": "inner_product", "ip": "inner_product", "dot": "dot",
    "chebyshev": "chebyshev", "linfinity": "chebyshev", "linfty": "chebyshev", "linf": "chebyshev",
    "canberra": "canberra", "braycurtis": "braycurtis", "correlation": "correlation",
    "true_angular": "true_angular", "tsss": "tsss", "hamming": "hamming", "jaccard": "jaccard", "dice": "dice",
    "matching": "matching", "kulsinski": "kulsinski", "rogerstanimoto": "rogerstanimoto",
    "russellrao": "russellrao", "sokalsneath": "sokalsneath", "sokalmichener": "sokalmichener", "yule": "yule",
    "hellinger": "hellinger", "jensen_shannon": "jensen_shannon", "jensen-shannon": "jensen_shannon",
    "symmetric_kl": "symmetric_kl", "symmetric-kl": "symmetric_kl", "symmetric_kullback_liebler": "symmetric_kl",
}
# lib.rs:1276-1293: the metrics without a fast alternative are built with their
# own distance and no correction (evaluated per pair by the generic kernels)
_DIRECT = {
    "chebyshev": L.DIST_CHEBYSHEV, "canberra": L.DIST_CANBERRA, "braycurtis": L.DIST_BRAYCURTIS,
    "correlation": L.DIST_CORRELATION, "true_angular": L.DIST_TRUE_ANGULAR, "tsss": L.DIST_TSSS,
    "hamming": L.DIST_HAMMING, "jaccard": L.DIST_JACCARD, "dice": L.DIST_DICE, "matching": L.DIST_MATCHING,
    "kulsinski": L.DIST_KULSINSKI, "rogerstanimoto": L.DIST_ROGERSTANIMOTO, "russellrao": L.DIST_RUSSELLRAO,
    "sokalmichener": L.DIST_SOKALMICHENER, "sokalsneath": L.DIST_SOKALSNEATH, "yule": L.DIST_YULE,
    "hellinger": L.DIST_HELLINGER, "jensen_shannon": L.DIST_JENSEN_SHANNON, "symmetric_kl": L.DIST_SYMMETRIC_KL,
}
# index.rs:606-614: angular RP splits
_ANGULAR = {"cosine", "inner_product", "dot", "correlation", "true_angular", "tsss"}

# Local-join tile arithmetic (an addition of the B200 engine): "bf16" filters
# pairs with tensor-core BF16 Gram tiles and recomputes survivors in FP32.
_PRECISIONS = {"fp32": L.PRECISION_FP32, "bf16": L.PRECISION_BF16}
# tile shape of the pipelined FP32 join: the process's tuned table (tuning a new
# key on first use), the fixed default shape, or fresh trials
_TUNINGS = {"table": L.TUNE_TABLE, "fixed": L.TUNE_FIXED, "retune": L.TUNE_RETUNE}
_ENCODINGS = {"int8": L.Q8_PER_VECTOR_COSINE, "sq8u": L.Q8_GLOBAL_SYMMETRIC, "sq8p": L.Q8_PER_VECTOR_SYMMETRIC,
              # an addition of the B200 engine: per-dimension scales (quantized.rs:42-56)
              "sq8d": L.Q8_PER_DIMENSION}


def version() -> str:
    """Library version (crates/rinnd/src/lib.rs:1301-1304)."""
    return L.lib.rinnd_version().decode()


def simd_info() -> str:
    """Compute backend description (crates/rinnd/src/lib.rs:1307-1336)."""
    n = L.device_count()
    return f"CUDA sm_100a ({n} device{'s' if n != 1 else ''})"


def device_count() -> int:
    return L.device_count()


_BRUTE_METRICS = {"sqeuclidean": (L.DIST_SQEUCLIDEAN, False), "euclidean": (L.DIST_SQEUCLIDEAN, True),
                  "l2": (L.DIST_SQEUCLIDEAN, True), "manhattan": (L.DIST_MANHATTAN, False),
                  "l1": (L.DIST_MANHATTAN, False), "taxicab": (L.DIST_MANHATTAN, False),
                  "cosine": (L.DIST_COSINE, False), "inner_product": (L.DIST_INNER_PRODUCT, False),
                  "dot": (L.DIST_INNER_PRODUCT, False)}


def brute_force_knn(data, queries, k=10, metric="sqeuclidean", precision="auto", exclude_self=False):
    """Exact k nearest data rows of every query row, by (distance, id) ascending
    (no counterpart in the reference; its recall criteria are measured against
    these).  precision "fp32" computes each distance with the build's FP32 join
    arithmetic; "bf16" filters the pairs on the tensor cores (BF16 Gram tiles,
    a rigorous lower bound) and recomputes the survivors in that FP32
    arithmetic, giving the FP32 results (dimension <= 128, k <= 32, not
    Manhattan); "auto" (default) takes "bf16" where it applies and "fp32"
    elsewhere -- the same results either way; "fp64" computes in double (the
    checker).  exclude_self leaves out data
    row i for query i (queries must then be the data rows themselves).
    Returns (int32[nq, k], float32[nq, k]), padded with (-1, inf) when k > n."""
    if metric not in _BRUTE_METRICS:
        raise ValueError(f"Unknown metric for brute force: {metric}")
    kind, take_sqrt = _BRUTE_METRICS[metric]
    X = np.ascontiguousarray(_as_f32_2d(data, "data"))
    Q = np.ascontiguousarray(_as_f32_2d(queries, "queries"))
    if Q.shape[1] != X.shape[1]:
        raise ValueError(f"Query dimension {Q.shape[1]} does not match data dimension {X.shape[1]}")
    precisions = {"fp32": L.BRUTE_FP32, "bf16": L.BRUTE_BF16, "fp64": L.BRUTE_FP64}
    if precision == "auto":
        precision = "bf16" if (X.shape[1] <= 128 and int(k) <= 32 and kind != L.DIST_MANHATTAN) else "fp32"
    if precision not in precisions:
        raise ValueError("precision must be 'auto', 'fp32', 'bf16' or 'fp64'")
    nq = Q.shape[0]
    excl = None
    if exclude_self:
        if nq > X.shape[0]:
            raise ValueError("exclude_self needs the queries to be the first rows of the data")
        excl = np.arange(nq, dtype=np.int32)
    oi = np.empty((nq, int(k)), np.int32)
    od = np.empty((nq, int(k)), np.float32)
    L.check(L.lib.rinnd_brute_force_knn(L.ptr(X), X.shape[0], X.shape[1], L.ptr(Q), nq, Q.shape[1], X.shape[1],
                                        int(k), kind, precisions[precision],
                                        L.ptr(excl) if excl is not None else None, 0, L.ptr(oi), L.ptr(od)))
    if take_sqrt:
        od = np.sqrt(od)
    return oi, od


def _as_f32_2d(a, what="data") -> np.ndarray:
    a = np.asarray(a)
    if a.dtype != np.float32:
        raise TypeError(f"{what} must be a float32 array, got {a.dtype}")
    if a.ndim != 2:
        raise ValueError(f"{what} must be 2-dimensional")
    return np.ascontiguousarray(a)


def _validate_quantized_widths(k: int, candidate_width: int, rerank_width: int) -> None:
    """crates/rinnd/src/lib.rs:1148-1172."""
    if candidate_width == 0:
        return
    if candidate_width < k:
        raise ValueError(f"candidate_width {candidate_width} must be at least k ({k})")
    if rerank_width > candidate_width:
        raise ValueError(f"rerank_width {rerank_width} must not exceed candidate_width {candidate_width}")
    if 0 < rerank_width < k:
        raise ValueError(f"rerank_width {rerank_width} must be zero or at least k ({k})")


def _prepare(data, *, metric, n_neighbors, n_trees, n_search_trees, search_tree_leaf_budget, leaf_size,
             max_candidates, n_iters, delta, random_state, diversify_prob, pruning_degree_multiplier, verbose,
             normalize, cosine_distance_mode, quantized_candidate_width, quantized_rerank_width, tree_quantization,
             retain_fp32_data, device, precision, join_tuning="table"):
    """Validates the constructor arguments (lib.rs:616-755) and maps them to
    build parameters; returns (rows, params, state for RINND._attach)."""
    if precision not in _PRECISIONS:
        raise ValueError(f"Unknown precision: {precision}; expected 'fp32' or 'bf16'")
    if join_tuning not in _TUNINGS:
        raise ValueError(f"Unknown join_tuning: {join_tuning}; expected 'table', 'fixed' or 'retune'")
    data = _as_f32_2d(data)
    n_points, dim = data.shape
    if quantized_candidate_width > 0 and quantized_rerank_width > quantized_candidate_width:
        raise ValueError("quantized_rerank_width must not exceed quantized_candidate_width when candidate "
                         "width is explicit")
    name = metric.lower()
    if name not in _ALIASES:
        raise ValueError(f"Unknown metric: {metric}")
    name = _ALIASES[name]
    normalize_cosine = bool(normalize) and name == "cosine"
    modes = {"log": (False, None), "direct": (True, None)}
    modes.update({m: (True, e) for m, e in _ENCODINGS.items()})
    if cosine_distance_mode not in modes:
        raise ValueError(f"Unknown cosine_distance_mode: {cosine_distance_mode}; expected 'log', 'direct', "
                         "'int8', 'sq8u', 'sq8p', or 'sq8d'")
    direct_cosine, encoding = modes[cosine_distance_mode]
    if tree_quantization not in ("none", "int8"):
        raise ValueError(f"Unknown tree_quantization: {tree_quantization}; expected 'none' or 'int8'")
    quantize_trees = tree_quantization == "int8"
    if quantize_trees and encoding is None:
        raise ValueError("tree_quantization='int8' is available only with a quantized cosine_distance_mode")
    if quantize_trees and encoding == L.Q8_GLOBAL_SYMMETRIC:
        raise ValueError("tree_quantization='int8' is incompatible with cosine_distance_mode='sq8u'; use "
                         "tree_quantization='none'")
    if quantize_trees and encoding == L.Q8_PER_DIMENSION:
        raise ValueError("tree_quantization='int8' is incompatible with cosine_distance_mode='sq8d'; use "
                         "tree_quantization='none'")
    if direct_cosine and not normalize_cosine:
        raise ValueError("direct and quantized cosine modes require metric='cosine' and normalize=True")
    if retain_fp32_data is None:
        retain_fp32_data = (not quantize_trees) or quantized_rerank_width > 0

    # lib.rs:1200-1204 n_trees default: clamp(round(2 log10 N), 3, 12)
    if n_trees is None:
        v = 2.0 * math.log10(n_points) if n_points > 0 else float("-inf")
        n_trees = int(min(max(math.floor(v + 0.5) if math.isfinite(v) else 0, 3), 12))

    # lib.rs:1239-1294 metric -> build distance + correction
    if name == "euclidean":
        kind, corr = L.DIST_SQEUCLIDEAN, L.CORR_SQRT
    elif name == "sqeuclidean":
        kind, corr = L.DIST_SQEUCLIDEAN, L.CORR_NONE
    elif name == "manhattan":
        kind, corr = L.DIST_MANHATTAN, L.CORR_NONE
    elif name == "cosine":
        if normalize_cosine:
            if encoding is not None or direct_cosine:
                kind, corr = L.DIST_DIRECT_COSINE, L.CORR_NONE
            else:
                kind, corr = L.DIST_ALT_DOT, L.CORR_ALT_COSINE
        else:
            kind, corr = L.DIST_ALT_COSINE, L.CORR_ALT_COSINE
    elif name == "dot":
        kind, corr = L.DIST_ALT_DOT, L.CORR_ALT_COSINE
    elif name == "inner_product":
        kind, corr = L.DIST_ALT_INNER_PRODUCT, L.CORR_ALT_IP
    else:
        kind, corr = _DIRECT[name], L.CORR_NONE

    p = L.BuildParams()
    L.check(L.lib.rinnd_params_default(ctypes.byref(p)))
    p.n_neighbors = int(n_neighbors)
    p.n_trees = int(n_trees)
    p.n_search_trees = int(n_search_trees)
    p.search_tree_leaf_budget = max(int(search_tree_leaf_budget), 1)
    p.leaf_size = int(leaf_size) if leaf_size is not None else 0
    p.max_candidates = int(max_candidates) if max_candidates is not None else 0
    p.n_iters = int(n_iters) if n_iters is not None else 0
    p.delta = float(delta)
    p.random_seed = int(random_state) if random_state is not None else 42
    p.diversify_prob = float(diversify_prob)
    p.pruning_degree_multiplier = float(pruning_degree_multiplier)
    p.angular = int(name in _ANGULAR)
    p.distance_kind = kind
    p.correction = corr
    p.normalize = int(normalize_cosine)
    p.verbose = int(bool(verbose))
    p.device = int(device)
    p.precision = _PRECISIONS[precision]
    p.join_tuning = _TUNINGS[join_tuning]

    state = {"n_points": n_points, "dim": dim, "n_neighbors": int(n_neighbors), "metric": metric,
             "encoding": encoding, "candidate_width": int(quantized_candidate_width),
             "rerank_width": int(quantized_rerank_width), "retain_fp32": bool(retain_fp32_data),
             "quantize_trees": quantize_trees, "leaf_budget": max(int(search_tree_leaf_budget), 1)}
    return data, p, state


class RINND:
    """NNDescent index built and queried on the GPU (crates/rinnd/src/lib.rs:616-755)."""

    def __init__(self, data, metric="euclidean", n_neighbors=30, n_trees=None, n_search_trees=1,
                 search_tree_leaf_budget=1, leaf_size=None, max_candidates=None, n_iters=None, delta=0.001,
                 random_state=None, diversify_prob=1.0, pruning_degree_multiplier=1.5, verbose=False,
                 normalize=False, cosine_distance_mode="log", quantized_candidate_width=0,
                 quantized_rerank_width=0, tree_quantization="none", retain_fp32_data=None, device=0,
                 precision="fp32", join_tuning="table"):
        self._h = None
        data, p, state = _prepare(data, metric=metric, n_neighbors=n_neighbors, n_trees=n_trees,
                                  n_search_trees=n_search_trees, search_tree_leaf_budget=search_tree_leaf_budget,
                                  leaf_size=leaf_size, max_candidates=max_candidates, n_iters=n_iters, delta=delta,
                                  random_state=random_state, diversify_prob=diversify_prob,
                                  pruning_degree_multiplier=pruning_degree_multiplier, verbose=verbose,
                                  normalize=normalize, cosine_distance_mode=cosine_distance_mode,
                                  quantized_candidate_width=quantized_candidate_width,
                                  quantized_rerank_width=quantized_rerank_width, tree_quantization=tree_quantization,
                                  retain_fp32_data=retain_fp32_data, device=device, precision=precision,
                                  join_tuning=join_tuning)
        h = ctypes.c_void_p()
        L.check(L.lib.rinnd_build(L.ptr(data), data.shape[0], data.shape[1], ctypes.byref(p), ctypes.byref(h)))
        self._attach(h, state)

    def _attach(self, h, state, encode=True):
        self._h = h
        self._state = dict(state)
        self.n_points, self.dim, self.n_neighbors = state["n_points"], state["dim"], state["n_neighbors"]
        self.metric = state["metric"]
        self._encoding = state["encoding"]
        self._candidate_width = state["candidate_width"]
        self._rerank_width = state["rerank_width"]
        self._retain_fp32 = state["retain_fp32"]
        self._leaf_budget = state["leaf_budget"]
        if not encode:
            return
        if self._encoding is not None:
            # QuantizedI8Index::new (lib.rs:159-276): codes, int8 routing trees, released FP32 rows
            L.check(L.lib.rinnd_quantize(self._h, self._encoding))
            if state["quantize_trees"]:
                L.check(L.lib.rinnd_quantize_trees(self._h))
            if not self._retain_fp32:
                L.check(L.lib.rinnd_release_fp32(self._h))
        else:
            self._retain_fp32 = True  # only a quantized index releases its rows

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            L.lib.rinnd_free(h)
            self._h = None

    # ---- queries (lib.rs:775-1010) -------------------------------------------------
    def _check_dim(self, qdim: int) -> None:
        if qdim != self.dim:
            raise ValueError(f"Query dimension {qdim} does not match data dimension {self.dim}")

    def _ensure_rerank_available(self, k: int, candidate_width: int, rerank_width: int) -> None:
        """lib.rs:283-300: exact reranking needs the retained FP32 rows."""
        requested = rerank_width > k if candidate_width == 0 else rerank_width > 0
        if requested and not self._retain_fp32:
            raise ValueError("exact reranking is unavailable because FP32 vector data was released")

    def _run_query(self, q: np.ndarray, k: int, epsilon: float):
        n = q.shape[0]
        idx = np.empty((n, k), np.int32)
        dist = np.empty((n, k), np.float32)
        if self._encoding is not None:
            self._ensure_rerank_available(k, self._candidate_width, self._rerank_width)
            L.check(L.lib.rinnd_query_quantized(self._h, L.ptr(q), n, k, float(epsilon), self._candidate_width,
                                                self._rerank_width, L.ptr(idx), L.ptr(dist)))
        else:
            L.check(L.lib.rinnd_query(self._h, L.ptr(q), n, k, float(epsilon), L.ptr(idx), L.ptr(dist)))
        return idx, dist

    def query(self, query_data, k=10, epsilon=0.1):
        """Approximate k nearest neighbours of each query row (lib.rs:775-821)."""
        q = _as_f32_2d(query_data, "query_data")
        self._check_dim(q.shape[1])
        return self._run_query(q, int(k), epsilon)

    def query_quantized(self, query_data, k=10, epsilon=0.1, candidate_width=0, rerank_width=0):
        """Quantized query with query-time widths (lib.rs:825-874)."""
        _validate_quantized_widths(k, candidate_width, rerank_width)
        if self._encoding is None:
            raise ValueError("query-time quantized widths require a quantized cosine_distance_mode")
        self._ensure_rerank_available(int(k), int(candidate_width), int(rerank_width))
        q = _as_f32_2d(query_data, "query_data")
        self._check_dim(q.shape[1])
        n = q.shape[0]
        idx = np.empty((n, k), np.int32)
        dist = np.empty((n, k), np.float32)
        L.check(L.lib.rinnd_query_quantized(self._h, L.ptr(q), n, int(k), float(epsilon), int(candidate_width),
                                            int(rerank_width), L.ptr(idx), L.ptr(dist)))
        return idx, dist

    def query_one(self, query, k=10, epsilon=0.1):
        """Single-vector query (lib.rs:877-912); same random stream as query row 0."""
        q = np.asarray(query)
        if q.dtype != np.float32:
            raise TypeError(f"query must be a float32 array, got {q.dtype}")
        if q.ndim != 1:
            raise ValueError("query must be 1-dimensional")
        self._check_dim(q.shape[0])
        idx, dist = self._run_query(np.ascontiguousarray(q[None, :]), int(k), epsilon)
        return idx[0], dist[0]

    def query_one_indices(self, query, k=10, epsilon=0.1):
        """Single-vector query returning ids only (lib.rs:918-951)."""
        return self.query_one(query, k, epsilon)[0]

    def query_one_indices_quantized(self, query, k=10, epsilon=0.1, candidate_width=0, rerank_width=0):
        """lib.rs:959-1010."""
        _validate_quantized_widths(k, candidate_width, rerank_width)
        q = np.asarray(query, dtype=np.float32)
        self._check_dim(q.shape[0])
        return self.query_quantized(q[None, :], k, epsilon, candidate_width, rerank_width)[0][0]

    # ---- exports -------------------------------------------------------------------
    @property
    def neighbor_graph(self):
        """(int32[N,k], float32[N,k]) sorted ascending, corrected distances (lib.rs:1087-1103)."""
        idx = np.empty((self.n_points, self.n_neighbors), np.int32)
        dist = np.empty((self.n_points, self.n_neighbors), np.float32)
        L.check(L.lib.rinnd_neighbor_graph(self._h, L.ptr(idx), L.ptr(dist)))
        return idx, dist

    @property
    def search_graph(self):
        """(indptr int32, indices int32, min_distance) in original id order (lib.rs:1013-1025)."""
        nnz = ctypes.c_int64(0)
        L.check(L.lib.rinnd_search_graph_nnz(self._h, ctypes.byref(nnz)))
        indptr = np.empty(self.n_points + 1, np.int32)
        indices = np.empty(max(nnz.value, 1), np.int32)
        md = ctypes.c_float(0)
        L.check(L.lib.rinnd_search_graph(self._h, L.ptr(indptr), L.ptr(indices), ctypes.byref(md)))
        return indptr, indices[: nnz.value], float(md.value)

    @property
    def vertex_order(self):
        out = np.empty(self.n_points, np.int32)
        L.check(L.lib.rinnd_vertex_order(self._h, L.ptr(out)))
        return out

    def export_search_tree(self, with_pivots=False):
        """The first retained RP tree in original id space (lib.rs:1105-1128):
        (hyperplanes float32[n_nodes, dim], offsets float32[n_nodes],
        children int32[n_nodes, 2], leaf_indices int32[N]).  With
        ``with_pivots`` a fifth array int32[n_nodes, 2] holds the two points
        whose split defined each internal node (-1 for leaves)."""
        m = ctypes.c_int64(0)
        L.check(L.lib.rinnd_export_search_tree(self._h, ctypes.byref(m), None, None, None, None, None))
        n = m.value
        hp = np.empty((n, self.dim), np.float32)
        off = np.empty(n, np.float32)
        ch = np.empty((n, 2), np.int32)
        ind = np.empty(self.n_points, np.int32)
        piv = np.empty((n, 2), np.int32) if with_pivots else None
        L.check(L.lib.rinnd_export_search_tree(self._h, None, L.ptr(hp), L.ptr(off), L.ptr(ch), L.ptr(ind),
                                               L.ptr(piv) if with_pivots else None))
        return (hp, off, ch, ind, piv) if with_pivots else (hp, off, ch, ind)

    def save(self, path):
        """Writes the index (every device array, and this object's settings) to
        `path`; `load(path)` restores it.  No counterpart in the reference."""
        meta = json.dumps({**self._state, "retain_fp32": self._retain_fp32}).encode()
        L.check(L.lib.rinnd_save(self._h, os.fsencode(path), meta))

    def search_tree_leaves(self, query_data, tree=0, leaf_budget=None, quantized=False):
        """The leaves FlatTree::search_leaves (flat_tree.rs:239-311) visits in
        retained tree `tree` for each query, as the search seeds them: a list
        per query of (start, end) ranges into the tree's leaf order (the
        `leaf_indices` of export_search_tree for tree 0).  `quantized` routes the
        queries' int8 codes over the int8 routing trees."""
        q = _as_f32_2d(query_data, "query_data")
        self._check_dim(q.shape[1])
        b = int(leaf_budget) if leaf_budget is not None else self._leaf_budget
        n = q.shape[0]
        out = np.empty((n, b, 2), np.int32)
        cnt = np.empty(n, np.int32)
        L.check(L.lib.rinnd_tree_search_leaves(self._h, L.ptr(q), n, int(tree), b, int(bool(quantized)), L.ptr(out),
                                               L.ptr(cnt)))
        return [[(int(s), int(e)) for s, e in out[i, :cnt[i]]] for i in range(n)]

    def search_stats(self, reset=False) -> dict:
        """Distance evaluations, node expansions, visited-table and spill-frontier
        overflows, the queries re-run with the wide and with the exact state, and
        the query runs that used the global-memory visited table or seed store,
        of the searches since the build (or the last reset)."""
        v = (ctypes.c_uint64 * 8)()
        L.check(L.lib.rinnd_search_counters(self._h, v, int(bool(reset))))
        return {"evaluations": v[0], "expansions": v[1], "visited_overflows": v[2], "frontier_overflows": v[3],
                "wide_reruns": v[4], "exact_reruns": v[5], "visited_spills": v[6], "seed_spills": v[7]}

    @property
    def build_info(self) -> dict:
        info = L.BuildInfo()
        L.check(L.lib.rinnd_build_info_get(self._h, ctypes.byref(info)))
        return {f: getattr(info, f) for f, _ in L.BuildInfo._fields_}

    def storage_info(self) -> dict:
        """Storage/encoding metadata (lib.rs:1028-1077) plus device bytes."""
        s = L.StorageInfo()
        L.check(L.lib.rinnd_storage_info_get(self._h, ctypes.byref(s)))
        info = {
            "encoding": s.encoding.decode(), "code_bytes": int(s.code_bytes),
            "metadata_bytes": int(s.metadata_bytes), "retained_fp32_bytes": int(s.retained_fp32_bytes),
            "encode_seconds": float(s.encode_seconds),
            "tree_code_bytes": int(s.tree_code_bytes), "tree_scale_bytes": int(s.tree_scale_bytes),
            "tree_offset_bytes": int(s.tree_offset_bytes), "tree_topology_bytes": int(s.tree_topology_bytes),
            "hypothetical_releasable_fp32_tree_bytes": 0,
            "released_fp32_tree_bytes": int(s.released_fp32_tree_bytes),
            "released_fp32_data_bytes": int(s.released_fp32_data_bytes),
            "retained_fp32_tree_topology_bytes": int(s.retained_fp32_tree_topology_bytes),
            "device_bytes": int(s.device_bytes),
        }
        info["allocated_bytes"] = sum(info[k] for k in (
            "code_bytes", "metadata_bytes", "retained_fp32_bytes", "retained_fp32_tree_topology_bytes",
            "tree_code_bytes", "tree_scale_bytes", "tree_offset_bytes", "tree_topology_bytes"))
        info["bytes_per_vector"] = info["allocated_bytes"] / self.n_points
        return info


def load(path, device=0) -> RINND:
    """An index written by RINND.save, on CUDA device `device`."""
    h = ctypes.c_void_p()
    n = ctypes.c_int64(0)
    buf = ctypes.create_string_buffer(1 << 16)  # the settings string is a few hundred bytes
    L.check(L.lib.rinnd_load(os.fsencode(path), int(device), ctypes.byref(h), buf, 1 << 16, ctypes.byref(n)))
    if n.value >= (1 << 16):
        L.lib.rinnd_free(h)
        raise ValueError(f"{path}: the index settings are unreadable")
    ix = RINND.__new__(RINND)
    ix._h = None
    ix._attach(h, json.loads(buf.value.decode()), encode=False)
    return ix


def build_many(datasets, params=None, n_workers=0, grouped=True, max_group_points=8 << 20, capture_iterations=True,
               **common):
    """Builds many independent indices in one call (the batched form; no
    counterpart in the reference).  `datasets` is a sequence of float32 [N, D]
    arrays of any sizes and dimensions; `params` an optional sequence of per-index
    keyword dicts (metric, n_neighbors, precision, ...) merged over `common`.
    With `grouped`, indices of one NN-Descent shape (dimension, metric, k,
    candidates, leaf size, precision) run their NN-Descent together as one
    group of at most `max_group_points` rows, each index keeping its own
    iteration cap and delta test, and with `capture_iterations` each group
    iteration runs as one CUDA graph; otherwise (and for indices alone in their
    group) each is built as by RINND, concurrently on its own stream
    (rinnd_build_many_ex).  Returns a list of RINND, one per dataset."""
    datasets = list(datasets)
    params = list(params) if params is not None else [{} for _ in datasets]
    if len(params) != len(datasets):
        raise ValueError("params must have one entry per dataset")
    defaults = dict(metric="euclidean", n_neighbors=30, n_trees=None, n_search_trees=1, search_tree_leaf_budget=1,
                    leaf_size=None, max_candidates=None, n_iters=None, delta=0.001, random_state=None,
                    diversify_prob=1.0, pruning_degree_multiplier=1.5, verbose=False, normalize=False,
                    cosine_distance_mode="log", quantized_candidate_width=0, quantized_rerank_width=0,
                    tree_quantization="none", retain_fp32_data=None, device=0, precision="fp32",
                    join_tuning="table")
    prepared = []
    for data, kw in zip(datasets, params):
        args = dict(defaults)
        args.update(common)
        args.update(kw)
        prepared.append(_prepare(data, **args))
    n = len(prepared)
    if n == 0:
        return []
    items = (L.BatchItem * n)()
    for i, (data, p, _) in enumerate(prepared):
        items[i].data = data.ctypes.data
        items[i].n, items[i].d = data.shape
        items[i].data_on_device = 0
        items[i].ld = data.shape[1]
        items[i].params = ctypes.addressof(p)
    handles = (ctypes.c_void_p * n)()
    status = (ctypes.c_int32 * n)()
    opts = L.BatchOptions()
    L.check(L.lib.rinnd_batch_options_default(ctypes.byref(opts)))
    opts.n_workers, opts.grouped, opts.max_group_points = int(n_workers), int(bool(grouped)), int(max_group_points)
    opts.capture_iterations = int(bool(capture_iterations))
    rc = L.lib.rinnd_build_many_ex(items, n, ctypes.byref(opts), handles, status)
    out = []
    for i, (_, _, state) in enumerate(prepared):
        if handles[i]:
            ix = RINND.__new__(RINND)
            ix._h = None
            ix._attach(ctypes.c_void_p(handles[i]), state)
            out.append(ix)
        else:
            out.append(None)
    L.check(rc)
    return out


class Server:
    """Continuous-batching query server over a built index (the serving form;
    rinnd_server_*).  Requests of any size, k and epsilon may be submitted from
    any thread; the server packs them into device batches, keeps several batches
    on the device at once and admits new queries as batch slots free up.  Each
    request's result equals `index.query` (or `index.query_quantized` with the
    index's widths, for a quantized index) run alone.  The index is kept alive
    by the server."""

    def __init__(self, index, max_batch_queries=32768, max_inflight=8, max_k=256, max_pending_queries=1 << 22,
                 quantized=None):
        self._s = None
        self.index = index
        p = L.ServerParams()
        L.check(L.lib.rinnd_server_params_default(ctypes.byref(p)))
        p.max_batch_queries, p.max_inflight, p.max_k = int(max_batch_queries), int(max_inflight), int(max_k)
        p.max_pending_queries = int(max_pending_queries)
        if quantized is None:
            quantized = index._encoding is not None
        p.quantized = int(bool(quantized))
        if quantized:
            index._ensure_rerank_available(1, index._candidate_width, index._rerank_width)
            p.candidate_width, p.rerank_width = index._candidate_width, index._rerank_width
        s = ctypes.c_void_p()
        L.check(L.lib.rinnd_server_create(index._h, ctypes.byref(p), ctypes.byref(s)))
        self._s = s
        self._shapes = {}
        self._lock = threading.Lock()

    def submit(self, queries, k=10, epsilon=0.1) -> int:
        q = _as_f32_2d(queries, "queries")
        self.index._check_dim(q.shape[1])
        rid = ctypes.c_int64(0)
        L.check(L.lib.rinnd_server_submit(self._s, L.ptr(q), q.shape[0], int(k), float(epsilon), ctypes.byref(rid)))
        with self._lock:
            self._shapes[rid.value] = (q.shape[0], int(k))
        return rid.value

    def poll(self, request_id, wait_ms=0):
        """(indices, distances) once the request completed, else None."""
        with self._lock:
            if request_id not in self._shapes:
                raise ValueError("unknown or already collected request id")
            nq, k = self._shapes[request_id]
        idx = np.empty((nq, k), np.int32)
        dist = np.empty((nq, k), np.float32)
        done = ctypes.c_int32(0)
        L.check(L.lib.rinnd_server_poll(self._s, int(request_id), int(wait_ms), L.ptr(idx), L.ptr(dist),
                                        ctypes.byref(done)))
        if not done.value:
            return None
        with self._lock:
            del self._shapes[request_id]
        return idx, dist

    def result(self, request_id, timeout_s=60.0):
        """Blocks until the request completes (TimeoutError after timeout_s)."""
        deadline = time.monotonic() + timeout_s
        while True:
            r = self.poll(request_id, wait_ms=50)
            if r is not None:
                return r
            if time.monotonic() > deadline:
                raise TimeoutError(f"request {request_id} did not complete in {timeout_s} s")

    def stats(self) -> dict:
        st = L.ServerStats()
        L.check(L.lib.rinnd_server_stats_get(self._s, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in L.ServerStats._fields_ if f != "reserved"}

    def close(self):
        if self._s:
            L.check(L.lib.rinnd_server_destroy(self._s))
            self._s = None

    def __del__(self):
        s = getattr(self, "_s", None)
        if s:
            L.lib.rinnd_server_destroy(s)
            self._s = None
