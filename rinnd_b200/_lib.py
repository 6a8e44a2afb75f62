"""ctypes binding of librinnd_b200.so (the C ABI declared in include/rinnd.h).

The shared library is built in-tree (``rinnd_b200/librinnd_b200.so``) by
``rinnd_b200.build.build()``.  There is no CPU fallback: importing this module
without the library raises ImportError, and every compute call without a CUDA
device raises RuntimeError from the library.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librinnd_b200.so")

OK = 0
ERR_INVALID, ERR_OOM, ERR_CUDA, ERR_NO_DEVICE, ERR_INTERNAL, ERR_BUSY = -1, -2, -3, -4, -5, -6

DIST_SQEUCLIDEAN, DIST_MANHATTAN, DIST_COSINE, DIST_ALT_COSINE, DIST_ALT_DOT, DIST_DIRECT_COSINE, \
    DIST_INNER_PRODUCT, DIST_ALT_INNER_PRODUCT = range(8)
# the reference's other metrics (core/distance/{minkowski,angular,binary,hellinger}.rs)
DIST_CHEBYSHEV, DIST_CANBERRA, DIST_BRAYCURTIS, DIST_CORRELATION, DIST_TRUE_ANGULAR, DIST_TSSS, DIST_HAMMING, \
    DIST_JACCARD, DIST_DICE, DIST_MATCHING, DIST_KULSINSKI, DIST_ROGERSTANIMOTO, DIST_RUSSELLRAO, \
    DIST_SOKALMICHENER, DIST_SOKALSNEATH, DIST_YULE, DIST_HELLINGER, DIST_JENSEN_SHANNON, \
    DIST_SYMMETRIC_KL = range(8, 27)
CORR_NONE, CORR_SQRT, CORR_ALT_COSINE, CORR_ALT_IP = range(4)
Q8_PER_VECTOR_COSINE, Q8_GLOBAL_SYMMETRIC, Q8_PER_VECTOR_SYMMETRIC, Q8_PER_DIMENSION = range(4)
PRECISION_FP32, PRECISION_BF16 = range(2)
TUNE_TABLE, TUNE_FIXED, TUNE_RETUNE = range(3)
JOIN_CHUNKED_FP32, JOIN_PIPELINED_FP32, JOIN_TENSOR_BF16 = range(3)  # rinnd_build_info.join_form
BRUTE_FP32, BRUTE_BF16, BRUTE_FP64 = 0, 1, 2  # rinnd_brute_force_knn precision

_i32, _i64, _u64, _f32, _f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_float, ctypes.c_double
_P = ctypes.c_void_p


class BuildParams(ctypes.Structure):
    _fields_ = [
        ("n_neighbors", _i32), ("n_trees", _i32), ("n_search_trees", _i32), ("search_tree_leaf_budget", _i32),
        ("leaf_size", _i32), ("max_candidates", _i32), ("n_iters", _i32), ("delta", _f32),
        ("random_seed", _u64), ("diversify_prob", _f32), ("pruning_degree_multiplier", _f32),
        ("angular", _i32), ("distance_kind", _i32), ("correction", _i32), ("normalize", _i32),
        ("verbose", _i32), ("device", _i32), ("precision", _i32), ("join_tuning", _i32), ("reserved", _i32 * 5),
    ]


class BuildInfo(ctypes.Structure):
    _fields_ = [
        ("iterations", _i32), ("forest_levels", _i32), ("n_leaves", _i64),
        ("ms_forest", _f64), ("ms_leaf_init", _f64), ("ms_iterations", _f64), ("ms_candidates", _f64),
        ("ms_join", _f64), ("ms_sort", _f64), ("ms_graph", _f64), ("ms_total", _f64),
        ("pairs_evaluated", _u64), ("pushes_accepted", _u64), ("push_contention", _u64),
        ("search_graph_nnz", _i64), ("min_distance", _f32), ("join_rows_gathered", _u64),
        ("ms_join_kernel", _f64), ("kernel_launches", _u64), ("join_kernel_launches", _u64),
        ("join_updates", _u64), ("join_form", _i32), ("group_items", _i32), ("join_tile_stages", _i32),
        ("join_tile_rows", _i32), ("join_tile_ctas_per_sm", _i32), ("join_tile_tuned", _i32),
    ]


class BatchItem(ctypes.Structure):
    _fields_ = [("data", _P), ("n", _i64), ("d", _i32), ("data_on_device", _i32), ("ld", _i64), ("params", _P)]


class BatchOptions(ctypes.Structure):
    _fields_ = [("n_workers", _i32), ("grouped", _i32), ("max_group_points", _i64), ("capture_iterations", _i32),
                ("reserved", _i32)]


class ServerParams(ctypes.Structure):
    _fields_ = [("max_batch_queries", _i32), ("max_inflight", _i32), ("max_k", _i32), ("quantized", _i32),
                ("candidate_width", _i32), ("rerank_width", _i32), ("max_pending_queries", _i64),
                ("reserved", _i32 * 8)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed_requests", _u64), ("completed_queries", _u64), ("batches", _u64),
                ("pending_queries", _u64), ("mean_batch_queries", _f64), ("p50_ms", _f64), ("p99_ms", _f64),
                ("max_ms", _f64), ("peak_inflight", _i32), ("reserved", _i32 * 7)]


class StorageInfo(ctypes.Structure):
    _fields_ = [
        ("encoding", ctypes.c_char * 32), ("code_bytes", _i64), ("metadata_bytes", _i64),
        ("retained_fp32_bytes", _i64), ("encode_seconds", _f64), ("device_bytes", _i64),
        ("tree_code_bytes", _i64), ("tree_scale_bytes", _i64), ("tree_offset_bytes", _i64),
        ("tree_topology_bytes", _i64), ("released_fp32_tree_bytes", _i64), ("released_fp32_data_bytes", _i64),
        ("retained_fp32_tree_topology_bytes", _i64),
    ]


# name -> (restype, argtypes); every function declared in include/rinnd.h.
SIGNATURES = {
    "rinnd_params_default": (ctypes.c_int, [_P]),
    "rinnd_build": (ctypes.c_int, [_P, _i64, _i32, _P, _P]),
    "rinnd_build_device": (ctypes.c_int, [_P, _i64, _i32, _i64, _P, _P]),
    "rinnd_build_on_stream": (ctypes.c_int, [_P, _i32, _i64, _i32, _i64, _P, _P, _P]),
    "rinnd_free": (ctypes.c_int, [_P]),
    "rinnd_save": (ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_char_p]),
    "rinnd_load": (ctypes.c_int, [ctypes.c_char_p, _i32, _P, _P, _i64, _P]),
    "rinnd_build_many": (ctypes.c_int, [_P, _i32, _i32, _P, _P]),
    "rinnd_batch_options_default": (ctypes.c_int, [_P]),
    "rinnd_build_many_ex": (ctypes.c_int, [_P, _i32, _P, _P, _P]),
    "rinnd_join_tile_table": (ctypes.c_int, [_P, _i32, _P]),
    "rinnd_join_tile_table_clear": (ctypes.c_int, []),
    "rinnd_join_tile_set": (ctypes.c_int, [_P]),
    "rinnd_search_counters": (ctypes.c_int, [_P, _P, _i32]),
    "rinnd_build_info_get": (ctypes.c_int, [_P, _P]),
    "rinnd_index_shape": (ctypes.c_int, [_P, _P, _P, _P]),
    "rinnd_query": (ctypes.c_int, [_P, _P, _i64, _i32, _f32, _P, _P]),
    "rinnd_query_one": (ctypes.c_int, [_P, _P, _i32, _f32, _P, _P]),
    "rinnd_query_device": (ctypes.c_int, [_P, _P, _i64, _i64, _i32, _f32, _u64, _P, _P, _P]),
    "rinnd_neighbor_graph": (ctypes.c_int, [_P, _P, _P]),
    "rinnd_search_graph_nnz": (ctypes.c_int, [_P, _P]),
    "rinnd_search_graph": (ctypes.c_int, [_P, _P, _P, _P]),
    "rinnd_vertex_order": (ctypes.c_int, [_P, _P]),
    "rinnd_export_search_tree": (ctypes.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "rinnd_quantize": (ctypes.c_int, [_P, _i32]),
    "rinnd_query_quantized": (ctypes.c_int, [_P, _P, _i64, _i32, _f32, _i32, _i32, _P, _P]),
    "rinnd_quantize_rows": (ctypes.c_int, [_P, _i64, _i32, _i32, _P, _P, _P]),
    "rinnd_quantize_rows_per_dimension": (ctypes.c_int, [_P, _i64, _i32, _P, _P]),
    "rinnd_quantize_trees": (ctypes.c_int, [_P]),
    "rinnd_release_fp32": (ctypes.c_int, [_P]),
    "rinnd_tree_search_leaves": (ctypes.c_int, [_P, _P, _i64, _i32, _i32, _i32, _P, _P]),
    "rinnd_search_stats_get": (ctypes.c_int, [_P, _P, _P, _P, _i32]),
    "rinnd_server_params_default": (ctypes.c_int, [_P]),
    "rinnd_server_create": (ctypes.c_int, [_P, _P, _P]),
    "rinnd_server_submit": (ctypes.c_int, [_P, _P, _i64, _i32, _f32, _P]),
    "rinnd_server_poll": (ctypes.c_int, [_P, _i64, _i32, _P, _P, _P]),
    "rinnd_server_stats_get": (ctypes.c_int, [_P, _P]),
    "rinnd_server_destroy": (ctypes.c_int, [_P]),
    "rinnd_storage_info_get": (ctypes.c_int, [_P, _P]),
    "rinnd_distance_pairs": (ctypes.c_int, [_i32, _P, _P, _i64, _i32, _P]),
    "rinnd_brute_force_knn": (ctypes.c_int, [_P, _i64, _i64, _P, _i64, _i64, _i32, _i32, _i32, _i32, _P, _i32, _P, _P]),
    "rinnd_search_graph_from_knn": (ctypes.c_int, [_P, _P, _P, _i32, _i32, _i32, _i32, _f32, _P, _P, _P, _P]),
    "rinnd_heap_push_batch": (ctypes.c_int, [_i32, _i32, _i64, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rinnd_nndescent_step": (ctypes.c_int, [_P, _i64, _i32, _i32, _i32, _i32, _i32, _u64, _i32, _P, _P, _P, _P, _P]),
    "rinnd_heap_push_batch_noalloc": (ctypes.c_int, [_i32, _i32, _i64, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rinnd_last_error": (ctypes.c_char_p, []),
    "rinnd_version": (ctypes.c_char_p, []),
    "rinnd_device_count": (ctypes.c_int, [_P]),
    "rinnd_kernel_launches": (ctypes.c_int, [_P]),
    "rinnd_kernel_target": (ctypes.c_int, [_P, _P]),
}

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
        "(the B200 engine has no CPU fallback)")

lib = ctypes.CDLL(LIB_PATH)
for _name, (_res, _args) in SIGNATURES.items():
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def last_error() -> str:
    msg = lib.rinnd_last_error()
    return msg.decode() if msg else ""


def check(rc: int) -> None:
    """Map a C ABI status code to the reference's Python exception types."""
    if rc == OK:
        return
    msg = last_error()
    if rc == ERR_INVALID:
        raise ValueError(msg)
    if rc == ERR_OOM:
        raise MemoryError(msg)
    raise RuntimeError(msg or f"rinnd error {rc}")


def ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def device_count() -> int:
    n = _i32(0)
    check(lib.rinnd_device_count(ctypes.byref(n)))
    return int(n.value)
