"""GPU parity of the hot-path components against the oracle, through the C ABI."""
import ctypes

import numpy as np
import pytest

from tests.helpers import gmm, uniform

pytestmark = pytest.mark.gpu

KIND = {"sqeuclidean": 0, "manhattan": 1, "cosine": 2, "alt_cosine": 3, "alt_dot": 4, "direct_cosine": 5,
        "inner_product": 6, "alt_inner_product": 7}
# Kinds whose value involves log2 (a libm transcendental): compared within
# 2 ulp instead of bit-for-bit.  All others must be bit-identical.
TRANSCENDENTAL = {KIND["alt_cosine"], KIND["alt_dot"]}


def gpu_pairs(kind, a, b):
    from rinnd_b200 import _lib as L

    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    out = np.empty(a.shape[0], np.float32)
    L.check(L.lib.rinnd_distance_pairs(kind, L.ptr(a), L.ptr(b), a.shape[0], a.shape[1], L.ptr(out)))
    return out


def test_kernels_are_sm100a_code(rb):
    """The library's kernels run as sm_100a binaries (cudaFuncGetAttributes
    binaryVersion 100).  ptxVersion is the virtual architecture the code was
    compiled from (compute_100a)."""
    from rinnd_b200 import _lib as L

    b, p = ctypes.c_int32(-1), ctypes.c_int32(-1)
    L.check(L.lib.rinnd_kernel_target(ctypes.byref(b), ctypes.byref(p)))
    assert b.value == 100, b.value
    assert p.value == 100, p.value


def test_distance_kats(rb, kats):
    for c in kats["distances"]:
        d = gpu_pairs(KIND[c["kind"]], np.array([c["a"]]), np.array([c["b"]]))[0]
        assert abs(d - c["expected"]) < c["tol"], (c["source"], d)


@pytest.mark.parametrize("dim", [1, 3, 7, 8, 17, 31, 32, 33, 96, 100, 128, 960])
def test_distance_pairs_match_reference_order(rb, orc, dim):
    rng = np.random.default_rng(dim)
    a = rng.normal(0, 1, (2000, dim)).astype(np.float32)
    b = rng.normal(0, 1, (2000, dim)).astype(np.float32)
    b[:200] = np.abs(b[:200])
    a[:200] = np.abs(a[:200])  # positive dots for the log/reciprocal proxies
    for kind in range(8):
        g = gpu_pairs(kind, a, b)
        r = orc.distance_pairs(kind, a, b)
        if kind in TRANSCENDENTAL:
            finite = np.isfinite(r) & (r != np.float32(3.4028235e38))
            assert np.array_equal(g[~finite], r[~finite])
            ulp = np.spacing(np.abs(r[finite]))
            assert np.all(np.abs(g[finite] - r[finite]) <= 2 * ulp), kind
        else:
            assert np.array_equal(g.view(np.uint32), r.view(np.uint32)), (kind, np.abs(g - r).max())


@pytest.mark.parametrize("k", [12, 20, 30, 32, 48])
def test_heap_push_batch_matches_sequential(rb, orc, k):
    """Concurrent checked_flagged_push == the reference's sequential application
    (final row sets are the k smallest distinct ids offered), for rows of one,
    two and three 16-slot line groups and a full last group (k = 32)."""
    from rinnd_b200 import _lib as L

    rng = np.random.default_rng(3)
    n, n_ops = 200, 60000
    rows = rng.integers(0, n, n_ops).astype(np.int32)
    ids = rng.integers(0, 400, n_ops).astype(np.int32)
    # one distance per (row, id), as in NN-Descent where d(p, q) is a function of
    # the pair, distinct within a row (ids < the prime modulus), so the k smallest
    # leave no tie at a row's boundary for arrival order to decide
    h = (rows.astype(np.uint64) * np.uint64(7919) + ids.astype(np.uint64) * np.uint64(104729)) % np.uint64(1000003)
    dists = (h.astype(np.float32) / np.float32(1000003)) * np.float32(10.0)
    flags = ((h >> np.uint64(7)) & np.uint64(1)).astype(np.uint8)  # also a function of the pair
    oi, od, of, _ = orc.neighbor_heap_apply(n, k, rows, ids, dists, flags)
    gi = np.empty((n, k), np.int32)
    gd = np.empty((n, k), np.float32)
    gf = np.empty((n, k), np.uint8)
    acc = ctypes.c_int64(0)
    L.check(L.lib.rinnd_heap_push_batch(n, k, n_ops, L.ptr(rows), L.ptr(ids), L.ptr(dists), L.ptr(flags),
                                        L.ptr(gi), L.ptr(gd), L.ptr(gf), ctypes.byref(acc)))
    # order within equal distances is unspecified in the reference; compare (d, id) sorted rows
    for r in range(n):
        ko = sorted(zip(od[r].tolist(), oi[r].tolist(), of[r].tolist()))
        kg = sorted(zip(gd[r].tolist(), gi[r].tolist(), gf[r].tolist()))
        assert ko == kg, r
    assert acc.value >= (oi >= 0).sum()


def gpu_search_graph(knn_idx, knn_dist, data, kind, mult=1.5):
    from rinnd_b200 import _lib as L

    knn_idx = np.ascontiguousarray(knn_idx, np.int32)
    knn_dist = np.ascontiguousarray(knn_dist, np.float32)
    data = np.ascontiguousarray(data, np.float32)
    n, k = knn_idx.shape
    indptr = np.empty(n + 1, np.int32)
    indices = np.empty(n * int(round(mult * k)) + 1, np.int32)
    nnz = ctypes.c_int64(0)
    md = ctypes.c_float(0)
    L.check(L.lib.rinnd_search_graph_from_knn(L.ptr(knn_idx), L.ptr(knn_dist), L.ptr(data), n, k, data.shape[1],
                                              kind, mult, L.ptr(indptr), L.ptr(indices), ctypes.byref(nnz),
                                              ctypes.byref(md)))
    return indptr, indices[: nnz.value], md.value


@pytest.mark.parametrize("kind,gen,k,d", [(0, "gmm", 15, 24), (0, "uniform", 15, 24), (3, "gmm", 15, 24),
                                         (7, "uniform", 15, 24), (1, "gmm", 15, 24), (0, "gmm", 30, 128),
                                         (3, "gmm", 30, 300), (0, "gmm", 40, 64), (0, "gmm", 31, 37),
                                         (0, "uniform", 32, 100)])
def test_search_graph_identical_on_shared_input(rb, orc, kind, gen, k, d):
    """from_dense_diversified on the same sorted kNN graph gives the same CSR
    (the staged and the sequential forward-diversify kernels both covered, and
    the staged kernel's 2 x 2 blocked squared-Euclidean pairs with an odd
    candidate count and a dimension that is not a multiple of 8)."""
    data = gmm(3000, d, 30, seed=5) if gen == "gmm" else uniform(3000, d, seed=5)
    if kind == 7:
        data = np.abs(data) + np.float32(0.01)
    ix = orc.OracleIndex(data, n_neighbors=k, n_trees=4, distance_kind=kind, correction=0,
                         angular=kind in (3, 7))
    ki, kd = ix.neighbor_graph
    op, oi, omd = orc.search_graph_from_knn(ki, kd, data, kind)
    gp, gi, gmd = gpu_search_graph(ki, kd, data, kind)
    assert np.array_equal(op, gp)
    assert np.array_equal(oi, gi)
    assert omd == gmd


def test_search_graph_with_missing_neighbors(rb, orc):
    """Rows with -1 padding (k > reachable points) and duplicate points."""
    rng = np.random.default_rng(9)
    base = rng.normal(0, 1, (40, 6)).astype(np.float32)
    data = np.concatenate([base, base[:10]])  # exact duplicates -> zero distances
    ix = orc.OracleIndex(data, n_neighbors=8, n_trees=2, correction=0)
    ki, kd = ix.neighbor_graph
    ki[::7, 5:] = -1
    kd[::7, 5:] = np.inf
    op, oi, omd = orc.search_graph_from_knn(ki, kd, data, 0)
    gp, gi, gmd = gpu_search_graph(ki, kd, data, 0)
    assert np.array_equal(op, gp) and np.array_equal(oi, gi) and omd == gmd


def test_diversify_prob_below_one(rb, orc):
    """diversify_prob (search_graph.rs:457-460, :506-509): at probability 0 no
    qualifying prune is taken, so the search graph is exactly the oracle's from
    the same kNN rows; at 0.5 the GPU's keyed draws and the oracle's stream give
    graphs of the same size within 2 %, between those of probability 0 and 1."""
    X = gmm(6000, 24, 30, seed=41)
    sizes = {}
    for prob in (1.0, 0.5, 0.0):
        ix = rb.RINND(X, metric="sqeuclidean", n_neighbors=12, random_state=2, diversify_prob=prob)
        gi, gd = ix.neighbor_graph
        indptr, indices, _ = ix.search_graph
        oindptr, oindices, _ = orc.search_graph_from_knn(gi, gd, X, 0, mult=1.5, diversify_prob=prob)
        if prob != 0.5:
            np.testing.assert_array_equal(indptr, oindptr)
            np.testing.assert_array_equal(indices, oindices)
        else:
            assert abs(len(indices) - len(oindices)) <= 0.02 * len(oindices), (len(indices), len(oindices))
        sizes[prob] = len(indices)
    assert sizes[1.0] < sizes[0.5] < sizes[0.0], sizes
