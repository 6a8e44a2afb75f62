"""TEST INFRASTRUCTURE ONLY: ctypes wrapper around the CPU restatement of the
reference's NN-Descent hot path (``oracle/rinnd_oracle.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module.  The product package ``rinnd_b200`` never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liborc_rinnd.so")

# Distance kinds / corrections (same numbering as include/rinnd.h).
SQEUCLIDEAN, MANHATTAN, COSINE, ALT_COSINE, ALT_DOT, DIRECT_COSINE, INNER_PRODUCT, ALT_INNER_PRODUCT = range(8)
CORR_NONE, CORR_SQRT, CORR_ALT_COSINE, CORR_ALT_IP = range(4)

_P = ctypes.c_void_p
_i32, _i64, _u64, _f32 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_float


class Params(ctypes.Structure):
    _fields_ = [
        ("n_neighbors", _i32), ("n_trees", _i32), ("n_search_trees", _i32),
        ("search_tree_leaf_budget", _i32), ("leaf_size", _i32), ("max_candidates", _i32),
        ("n_iters", _i32), ("delta", _f32), ("random_seed", _u64), ("diversify_prob", _f32),
        ("pruning_degree_multiplier", _f32), ("angular", _i32), ("distance_kind", _i32),
        ("correction", _i32), ("n_threads", _i32), ("verbose", _i32),
    ]


def build_library(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, OpenMP, AVX2/FMA)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_library()
        L = ctypes.CDLL(_LIB_PATH)
        sigs = {
            "orc_distance": (_f32, [ctypes.c_int, _P, _P, _i32]),
            "orc_distance_pairs": (None, [ctypes.c_int, _P, _P, _i64, _i32, _P]),
            "orc_correct": (_f32, [ctypes.c_int, _f32]),
            "orc_i8_dot": (_i32, [_P, _P, _i32]),
            "orc_i8_per_dimension_dot": (_f32, [_P, _P, _P, _i32]),
            "orc_rng_u64": (None, [_u64, _i32, _P]),
            "orc_rng_float": (None, [_u64, _i32, _P]),
            "orc_rng_index": (None, [_u64, _u64, _i32, _P]),
            "orc_neighbor_heap_sequence": (None, [_i32, _i32, _P, _P, _P, _P, _P, _P, _P, _P]),
            "orc_neighbor_heap_apply": (None, [_i32, _i32, _i64, _P, _P, _P, _P, _P, _P, _P, _P]),
            "orc_candidate_heap_sequence": (None, [_i32, _i32, _P, _P, _P, _P]),
            "orc_bounded_heap_sequence": (_i32, [_i32, _i32, _P, _P, _P, _P, _P]),
            "orc_build_candidates": (None, [_i32, _i32, _P, _P, _i32, _u64, _i32, _P, _P]),
            "orc_tree_search_leaves": (_i32, [_i32, _i32, _P, _P, _P, _P, _u64, _i32, _P, _P]),
            "orc_search_graph_from_knn": (_i64, [_P, _P, _P, _i32, _i32, _i32, ctypes.c_int, _f32, _f32, _P, _P, _i64, _P]),
            "orc_weighted_union_pruned": (_i64, [_i32, _P, _P, _P, _P, _P, _P, _i32, _P, _P]),
            "orc_params_default": (None, [_P]),
            "orc_build": (_P, [_P, _i64, _i32, _P]),
            "orc_index_from_parts": (_P, [_P, _i64, _i32, ctypes.c_int32, ctypes.c_int32, _P, _P, _f32, _i32, _P,
                                          _P, _P, _P, _P, _i32, _P, _u64, _i32]),
            "orc_free": (None, [_P]),
            "orc_index_k": (_i32, [_P]),
            "orc_neighbor_graph": (None, [_P, _P, _P]),
            "orc_search_graph_nnz": (_i64, [_P]),
            "orc_search_graph": (None, [_P, _P, _P, _P]),
            "orc_vertex_order": (None, [_P, _P]),
            "orc_iterations": (_i32, [_P]),
            "orc_timings": (None, [_P, _P]),
            "orc_query": (None, [_P, _P, _i64, _i32, _f32, _P, _P]),
            "orc_query_one": (None, [_P, _P, _i32, _f32, _P, _P]),
            "orc_quantize_rows": (None, [_P, _i64, _i32, _i32, _P, _P, _P]),
            "orc_query_quantized": (_i32, [_P, _P, _i64, _i32, _f32, _i32, _i32, _i32, _P, _P]),
            "orc_quantize_queries": (None, [_P, _i64, _i32, _i32, _f32, _P, _P]),
            "orc_normalize_rows": (None, [_P, _i64, _i32]),
            "orc_exact_knn_f64": (None, [ctypes.c_int, _P, _i64, _P, _i64, _i32, _i32, _i32, _P, _P]),
            "orc_max_threads": (_i32, []),
            "orc_tree_hyperplane": (_f32, [_P, _P, _i32, _i32, _P]),
            "orc_quantize_per_dimension": (None, [_P, _i64, _i32, _P, _P]),
            "orc_quantize_queries_per_dimension": (None, [_P, _i64, _i32, _P, _P]),
            "orc_tree_route_points": (None, [_i32, _i32, _P, _P, _P, _P, _i64, _P]),
            "orc_quantize_tree_hyperplanes": (None, [_i32, _i32, _P, _P, _P]),
            "orc_tree_search_leaves_quantized": (_i32, [_i32, _i32, _P, _P, _P, _P, _f32, _u64, _i32, _P, _P]),
            "orc_query_quantized_trees": (_i32, [_P, _P, _i64, _i32, _f32, _i32, _i32, _i32, _i32, _P, _P]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def max_threads() -> int:
    return int(lib().orc_max_threads())


def distance(kind: int, a, b) -> float:
    a, b = _f(a), _f(b)
    return float(lib().orc_distance(kind, _p(a), _p(b), a.shape[-1]))


def distance_pairs(kind: int, a, b) -> np.ndarray:
    a, b = _f(a), _f(b)
    out = np.empty(a.shape[0], np.float32)
    lib().orc_distance_pairs(kind, _p(a), _p(b), a.shape[0], a.shape[1], _p(out))
    return out


def correct(corr: int, d: float) -> float:
    return float(lib().orc_correct(corr, d))


def i8_dot(x, y) -> int:
    x = np.ascontiguousarray(x, np.int8)
    y = np.ascontiguousarray(y, np.int8)
    return int(lib().orc_i8_dot(_p(x), _p(y), x.size))


def i8_per_dimension_dot(x, y, scales) -> float:
    x = np.ascontiguousarray(x, np.int8)
    y = np.ascontiguousarray(y, np.int8)
    s = _f(scales)
    return float(lib().orc_i8_per_dimension_dot(_p(x), _p(y), _p(s), x.size))


def rng_u64(seed: int, n: int) -> np.ndarray:
    out = np.empty(n, np.uint64)
    lib().orc_rng_u64(seed, n, _p(out))
    return out


def neighbor_heap_sequence(k, ops, ids, dists, flags=None):
    n = len(ops)
    ops = np.ascontiguousarray(ops, np.int32)
    ids = np.ascontiguousarray(ids, np.int32)
    dists = _f(dists)
    flags = np.ascontiguousarray(flags if flags is not None else np.zeros(n), np.uint8)
    res = np.empty(n, np.int32)
    oi, od, of = np.empty(k, np.int32), np.empty(k, np.float32), np.empty(k, np.uint8)
    lib().orc_neighbor_heap_sequence(k, n, _p(ops), _p(ids), _p(dists), _p(flags), _p(res), _p(oi), _p(od), _p(of))
    return res.astype(bool), oi, od, of


def neighbor_heap_apply(n, k, rows, ids, dists, flags):
    rows = np.ascontiguousarray(rows, np.int32)
    ids = np.ascontiguousarray(ids, np.int32)
    dists = _f(dists)
    flags = np.ascontiguousarray(flags, np.uint8)
    oi = np.empty((n, k), np.int32)
    od = np.empty((n, k), np.float32)
    of = np.empty((n, k), np.uint8)
    acc = ctypes.c_int64(0)
    lib().orc_neighbor_heap_apply(n, k, rows.size, _p(rows), _p(ids), _p(dists), _p(flags),
                                  _p(oi), _p(od), _p(of), ctypes.byref(acc))
    return oi, od, of, acc.value


def candidate_heap_sequence(size, priorities, ids):
    pr = _f(priorities)
    ids = np.ascontiguousarray(ids, np.int32)
    op = np.empty(size, np.float32)
    oi = np.empty(size, np.int32)
    lib().orc_candidate_heap_sequence(size, pr.size, _p(pr), _p(ids), _p(op), _p(oi))
    return op, oi


def bounded_heap_sequence(k, dists, ids):
    d = _f(dists)
    ids = np.ascontiguousarray(ids, np.int32)
    acc = np.empty(d.size, np.int32)
    oi = np.empty(k, np.int32)
    od = np.empty(k, np.float32)
    m = lib().orc_bounded_heap_sequence(k, d.size, _p(d), _p(ids), _p(acc), _p(oi), _p(od))
    return acc.astype(bool), oi[:m], od[:m]


def build_candidates(heap_idx, heap_flags, max_candidates, seed, n_threads=1):
    heap_idx = np.ascontiguousarray(heap_idx, np.int32)
    flags = np.ascontiguousarray(heap_flags, np.uint8).copy()
    n, k = heap_idx.shape
    new = np.empty((n, max_candidates), np.int32)
    old = np.empty((n, max_candidates), np.int32)
    lib().orc_build_candidates(n, k, _p(heap_idx), _p(flags), max_candidates, seed, n_threads, _p(new), _p(old))
    return new, old, flags


def tree_search_leaves(hyperplanes, offsets, children, point, seed, leaf_budget):
    hp = _f(hyperplanes)
    off = _f(offsets)
    ch = np.ascontiguousarray(children, np.int32)
    pt = _f(point)
    n_nodes, dim = hp.shape
    out = np.empty(2 * max(leaf_budget, 1), np.int32)
    nl = ctypes.c_int32(0)
    ev = lib().orc_tree_search_leaves(n_nodes, dim, _p(hp), _p(off), _p(ch), _p(pt), seed, leaf_budget, _p(out), ctypes.byref(nl))
    return int(ev), [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(nl.value)]


def quantize_tree_hyperplanes(hyperplanes):
    """QuantizedFlatTree codes and per-node scales (flat_tree.rs:47-64)."""
    hp = _f(hyperplanes)
    codes = np.empty(hp.shape, np.int8)
    scales = np.empty(hp.shape[0], np.float32)
    lib().orc_quantize_tree_hyperplanes(hp.shape[0], hp.shape[1], _p(hp), _p(codes), _p(scales))
    return codes, scales


def tree_search_leaves_quantized(hyperplanes, offsets, children, qcodes, qscale, seed, leaf_budget):
    """QuantizedFlatTree::search_leaves (flat_tree.rs:106-183) on the int8 form of
    an FP32 tree, for a query's int8 codes and tree_query_scale."""
    hp = _f(hyperplanes)
    off = _f(offsets)
    ch = np.ascontiguousarray(children, np.int32)
    qc = np.ascontiguousarray(qcodes, np.int8)
    n_nodes, dim = hp.shape
    out = np.empty(2 * max(leaf_budget, 1), np.int32)
    nl = ctypes.c_int32(0)
    ev = lib().orc_tree_search_leaves_quantized(n_nodes, dim, _p(hp), _p(off), _p(ch), _p(qc), float(qscale), seed,
                                                leaf_budget, _p(out), ctypes.byref(nl))
    return int(ev), [(int(out[2 * i]), int(out[2 * i + 1])) for i in range(nl.value)]


def tree_hyperplane(p1, p2, angular):
    """(hyperplane, offset) of a split through p1, p2 (builder.rs:249-308)."""
    p1, p2 = _f(p1), _f(p2)
    hp = np.empty(p1.size, np.float32)
    off = lib().orc_tree_hyperplane(_p(p1), _p(p2), p1.size, int(bool(angular)), _p(hp))
    return hp, np.float32(off)


def tree_route_points(hyperplanes, offsets, children, points):
    """Leaf node each point reaches (budget-1 routing, flat_tree.rs:253-273);
    -1 where a margin on its path is a tie (|m| < 1e-8)."""
    hp = _f(hyperplanes)
    off = _f(offsets)
    ch = np.ascontiguousarray(children, np.int32)
    pts = _f(points)
    out = np.empty(pts.shape[0], np.int32)
    lib().orc_tree_route_points(hp.shape[0], hp.shape[1], _p(hp), _p(off), _p(ch), _p(pts), pts.shape[0], _p(out))
    return out


def search_graph_from_knn(knn_idx, knn_dist, data, kind, mult=1.5, diversify_prob=1.0):
    knn_idx = np.ascontiguousarray(knn_idx, np.int32)
    knn_dist = _f(knn_dist)
    data = _f(data)
    n, k = knn_idx.shape
    cap = n * int(round(mult * k)) + 1
    indptr = np.empty(n + 1, np.int32)
    indices = np.empty(cap, np.int32)
    md = ctypes.c_float(0)
    nnz = lib().orc_search_graph_from_knn(_p(knn_idx), _p(knn_dist), _p(data), n, k, data.shape[1], kind,
                                          float(diversify_prob), mult, _p(indptr), _p(indices), cap, ctypes.byref(md))
    return indptr, indices[:nnz].copy(), md.value


def weighted_union_pruned(forward, reverse, max_degree):
    n = len(forward)

    def csr(rows):
        ptr = np.zeros(n + 1, np.int32)
        idx, dist = [], []
        for i, r in enumerate(rows):
            for j, d in r:
                idx.append(j)
                dist.append(d)
            ptr[i + 1] = len(idx)
        return ptr, np.asarray(idx, np.int32).reshape(-1), np.asarray(dist, np.float32).reshape(-1)

    fp, fi, fd = csr(forward)
    rp, ri, rd = csr(reverse)
    fi = np.ascontiguousarray(fi if fi.size else np.zeros(1, np.int32))
    fd = np.ascontiguousarray(fd if fd.size else np.zeros(1, np.float32))
    ri = np.ascontiguousarray(ri if ri.size else np.zeros(1, np.int32))
    rd = np.ascontiguousarray(rd if rd.size else np.zeros(1, np.float32))
    indptr = np.empty(n + 1, np.int32)
    indices = np.empty(max(1, n * max_degree), np.int32)
    nnz = lib().orc_weighted_union_pruned(n, _p(fp), _p(fi), _p(fd), _p(rp), _p(ri), _p(rd), max_degree, _p(indptr), _p(indices))
    return indptr, indices[:nnz].copy()


def quantize_rows(data, encoding):
    data = _f(data)
    n, d = data.shape
    codes = np.empty((n, d), np.int8)
    inv = np.empty(n, np.float32)
    gm = ctypes.c_float(0)
    lib().orc_quantize_rows(_p(data), n, d, encoding, _p(codes), _p(inv), ctypes.byref(gm))
    return codes, inv, gm.value


def quantize_queries(queries, encoding, global_mult):
    queries = _f(queries)
    n, d = queries.shape
    codes = np.empty((n, d), np.int8)
    scales = np.empty(n, np.float32)
    lib().orc_quantize_queries(_p(queries), n, d, encoding, global_mult, _p(codes), _p(scales))
    return codes, scales


def quantize_per_dimension(data):
    """Per-dimension symmetric int8 codes and the per-dimension scales."""
    data = _f(data)
    n, d = data.shape
    codes = np.empty((n, d), np.int8)
    scales = np.empty(d, np.float32)
    lib().orc_quantize_per_dimension(_p(data), n, d, _p(codes), _p(scales))
    return codes, scales


def quantize_queries_per_dimension(queries, dim_scales):
    queries = _f(queries)
    n, d = queries.shape
    codes = np.empty((n, d), np.int8)
    sc = _f(dim_scales)
    lib().orc_quantize_queries_per_dimension(_p(queries), n, d, _p(sc), _p(codes))
    return codes


def normalize_rows(data):
    out = np.array(data, dtype=np.float32, order="C", copy=True)
    lib().orc_normalize_rows(_p(out), out.shape[0], out.shape[1])
    return out


def exact_knn_f64(kind, data, queries, k, exclude_self=False):
    data = _f(data)
    queries = _f(queries)
    idx = np.empty((queries.shape[0], k), np.int32)
    dist = np.empty((queries.shape[0], k), np.float64)
    lib().orc_exact_knn_f64(kind, _p(data), data.shape[0], _p(queries), queries.shape[0], data.shape[1], k,
                            1 if exclude_self else 0, _p(idx), _p(dist))
    return idx, dist


class OracleIndex:
    """CPU restatement of ``NNDescentBuilder::build_with_distance`` + ``NNDescentIndex``
    (core/index.rs:24-733)."""

    def __init__(self, data, *, n_neighbors=30, n_trees=8, n_search_trees=1, search_tree_leaf_budget=1,
                 leaf_size=None, max_candidates=None, n_iters=None, delta=0.001, random_seed=42,
                 pruning_degree_multiplier=1.5, angular=False, distance_kind=SQEUCLIDEAN,
                 correction=CORR_SQRT, n_threads=0, verbose=False):
        self.data = _f(data)
        p = Params()
        lib().orc_params_default(ctypes.byref(p))
        p.n_neighbors, p.n_trees, p.n_search_trees = n_neighbors, n_trees, n_search_trees
        p.search_tree_leaf_budget = search_tree_leaf_budget
        p.leaf_size = leaf_size or 0
        p.max_candidates = max_candidates or 0
        p.n_iters = n_iters or 0
        p.delta, p.random_seed = delta, random_seed
        p.pruning_degree_multiplier = pruning_degree_multiplier
        p.angular, p.distance_kind, p.correction = int(angular), distance_kind, correction
        p.n_threads, p.verbose = n_threads, int(verbose)
        self.params = p
        n, d = self.data.shape
        self.n, self.dim, self.k = n, d, n_neighbors
        self._h = lib().orc_build(_p(self.data), n, d, ctypes.byref(p))

    @classmethod
    def from_parts(cls, data, *, kind, correction, indptr, indices, min_distance, vertex_order, trees=(),
                   leaf_budget=1, seed=42, n_threads=0):
        """A search-only index over another index's graph and trees (internal
        order: `data` rows, CSR `indptr`/`indices` and each tree's leaf order are
        in internal ids; `vertex_order` maps internal to original ids).  `trees`
        is a sequence of (hyperplanes [m, dim], offsets [m], children [m, 2],
        leaf_indices [n]) in FlatTree layout."""
        self = cls.__new__(cls)
        self.data = _f(data)
        n, d = self.data.shape
        self.n, self.dim, self.k = n, d, 0
        self._parts = [np.ascontiguousarray(indptr, np.int32), np.ascontiguousarray(indices, np.int32),
                       np.ascontiguousarray(vertex_order, np.int32)]
        tn = np.array([len(t[1]) for t in trees] or [0], np.int64)
        hp = np.ascontiguousarray(np.concatenate([t[0] for t in trees]) if trees else np.zeros((1, d)), np.float32)
        off = np.ascontiguousarray(np.concatenate([t[1] for t in trees]) if trees else np.zeros(1), np.float32)
        ch = np.ascontiguousarray(np.concatenate([t[2] for t in trees]) if trees else np.zeros((1, 2)), np.int32)
        ti = np.ascontiguousarray(np.concatenate([t[3] for t in trees]) if trees else np.zeros(1), np.int32)
        self._parts += [tn, hp, off, ch, ti]
        self._h = lib().orc_index_from_parts(_p(self.data), n, d, int(kind), int(correction), _p(self._parts[0]),
                                             _p(self._parts[1]), float(min_distance), len(trees), _p(tn), _p(hp),
                                             _p(off), _p(ch), _p(ti), int(leaf_budget), _p(self._parts[2]),
                                             int(seed), int(n_threads))
        return self

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().orc_free(h)
            self._h = None

    @property
    def neighbor_graph(self):
        idx = np.empty((self.n, self.k), np.int32)
        dist = np.empty((self.n, self.k), np.float32)
        lib().orc_neighbor_graph(self._h, _p(idx), _p(dist))
        return idx, dist

    @property
    def search_graph(self):
        nnz = lib().orc_search_graph_nnz(self._h)
        indptr = np.empty(self.n + 1, np.int32)
        indices = np.empty(max(nnz, 1), np.int32)
        md = ctypes.c_float(0)
        lib().orc_search_graph(self._h, _p(indptr), _p(indices), ctypes.byref(md))
        return indptr, indices[:nnz], md.value

    @property
    def vertex_order(self):
        out = np.empty(self.n, np.int32)
        lib().orc_vertex_order(self._h, _p(out))
        return out

    @property
    def iterations(self):
        return int(lib().orc_iterations(self._h))

    @property
    def timings(self):
        out = np.empty(5, np.float64)
        lib().orc_timings(self._h, _p(out))
        return dict(zip(["forest", "leaf_init", "iterations", "graph", "total"], out.tolist()))

    def query(self, queries, k=10, epsilon=0.1):
        q = _f(queries)
        nq = q.shape[0]
        idx = np.empty((nq, k), np.int32)
        dist = np.empty((nq, k), np.float32)
        lib().orc_query(self._h, _p(q), nq, k, epsilon, _p(idx), _p(dist))
        return idx, dist

    def query_one(self, q, k=10, epsilon=0.1):
        q = _f(q)
        idx = np.empty(k, np.int32)
        dist = np.empty(k, np.float32)
        lib().orc_query_one(self._h, _p(q), k, epsilon, _p(idx), _p(dist))
        return idx, dist

    def query_quantized(self, queries, k=10, epsilon=0.1, encoding=0, candidate_width=0, rerank_width=0,
                        quantize_trees=False):
        q = _f(queries)
        nq = q.shape[0]
        idx = np.empty((nq, k), np.int32)
        dist = np.empty((nq, k), np.float32)
        rc = lib().orc_query_quantized_trees(self._h, _p(q), nq, k, epsilon, encoding, candidate_width, rerank_width,
                                             int(bool(quantize_trees)), _p(idx), _p(dist))
        if rc != 0:
            raise ValueError("invalid quantized widths")
        return idx, dist
