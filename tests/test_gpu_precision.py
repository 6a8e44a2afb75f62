"""Precision form: the BF16 tensor-core local join against the FP32 join.

The BF16 Gram tiles (tcgen05, FP32 accumulate) only filter candidate pairs by a
rigorous lower bound of their distance; every pair that may beat its row's
threshold is recomputed in FP32 with the FP32 join's own arithmetic before it
is pushed.  Hence one NN-Descent iteration (candidate sampling + local join +
heap pushes, core/nndescent/mod.rs:101-155, :321-491) from the same rows must
produce bit-identical neighbor rows with either precision -- a filter that
dropped a pair the FP32 join pushes would show up here -- and full builds must
reach the same recall against FP64 exact neighbors.

The comparison starts from rows whose distances all come from the join itself:
a row entry whose distance was computed in another accumulation order (the
pair API's) can be re-offered by the join with a last-bit-different value,
which makes the final row depend on the order of concurrent pushes.
"""
import ctypes

import numpy as np
import pytest

from helpers import gmm, recall

pytestmark = pytest.mark.gpu

SQEUCLIDEAN, ALT_COSINE, DIRECT_COSINE, INNER_PRODUCT = 0, 3, 5, 6


def random_rows(orc, X, k, kind, seed):
    rng = np.random.default_rng(seed)
    n = X.shape[0]
    idx = rng.integers(0, n - 1, (n, k)).astype(np.int32)
    idx += (idx >= np.arange(n, dtype=np.int32)[:, None]).astype(np.int32)  # no self loops; repeats are rejected
    rows = np.repeat(np.arange(n), k)
    dist = orc.distance_pairs(kind, X[rows], X[idx.reshape(-1)]).astype(np.float32).reshape(n, k)
    return idx, dist, np.ones((n, k), np.uint8)


def step(X, heap, k, kind, precision, seed, it):
    """One iteration; the join kernel that ran must be the one the precision asks for."""
    from rinnd_b200 import _lib as L

    idx, dist, flags = (np.ascontiguousarray(a).copy() for a in heap)
    ch = ctypes.c_int64(0)
    form = ctypes.c_int32(-1)
    L.check(L.lib.rinnd_nndescent_step(L.ptr(X), X.shape[0], X.shape[1], k, 0, kind, precision, seed, it,
                                       L.ptr(idx), L.ptr(dist), L.ptr(flags), ctypes.byref(ch), ctypes.byref(form)))
    want = L.JOIN_TENSOR_BF16 if precision == L.PRECISION_BF16 else L.JOIN_PIPELINED_FP32
    assert form.value == want, (precision, form.value)
    return (idx, dist, flags), ch.value


def join_rows(orc, X, k, kind):
    """Rows after one FP32 iteration from random rows, minus the entries carried
    over from the random start (their distances come from the pair API)."""
    from rinnd_b200 import _lib as L

    start = random_rows(orc, X, k, kind, seed=1)
    (idx, dist, flags), _ = step(X, start, k, kind, L.PRECISION_FP32, 77, 0)
    carried = (idx[:, :, None] == start[0][:, None, :]).any(axis=2) & (idx >= 0)
    idx = np.where(carried, -1, idx).astype(np.int32)
    return idx, dist, flags


@pytest.mark.parametrize("kind,d", [(SQEUCLIDEAN, 128), (SQEUCLIDEAN, 72), (SQEUCLIDEAN, 256), (ALT_COSINE, 96),
                                    (DIRECT_COSINE, 64), (INNER_PRODUCT, 64)])
def test_bf16_iteration_matches_fp32_bit_for_bit(rb, orc, kind, d):
    from rinnd_b200 import _lib as L

    X = gmm(12000, d, 40, seed=d + kind)
    if kind != SQEUCLIDEAN:
        X = np.abs(X) + np.float32(0.05)
    if kind == DIRECT_COSINE:
        X = orc.normalize_rows(X)
    k = 30 if kind == SQEUCLIDEAN else 15
    heap = join_rows(orc, X, k, kind)
    for it in (1, 2):
        fp, ch_fp = step(X, heap, k, kind, L.PRECISION_FP32, 77, it)
        bf, ch_bf = step(X, heap, k, kind, L.PRECISION_BF16, 77, it)
        assert ch_fp > 0 and ch_bf > 0
        # identical distances everywhere; identical ids and flags except where a
        # row's last (largest) distance is tied: which of two equally distant
        # candidates keeps the last slot depends on the order of concurrent
        # pushes (the reference rejects d >= max, so arrival order decides)
        np.testing.assert_array_equal(bf[1].view(np.uint32), fp[1].view(np.uint32))
        tied_max = fp[1] == fp[1][:, -1:]
        differ = (bf[0] != fp[0]) | (bf[2] != fp[2])
        assert not np.any(differ & ~tied_max)
        # such ties are rare: at most 0.05 % of the entries
        assert differ.sum() <= 5e-4 * differ.size
        heap = fp


@pytest.mark.parametrize("metric,kind,k,d", [("sqeuclidean", 0, 30, 128), ("cosine", 2, 15, 96)])
def test_bf16_build_recall_equals_fp32(rb, orc, metric, kind, k, d):
    X = gmm(30000, d, 60, seed=11)
    if metric == "cosine":
        X = np.abs(X) + np.float32(0.05)
    truth, _ = orc.exact_knn_f64(kind, X, X[:3000], k + 1)
    truth = truth[:, 1:]
    rec = {}
    for prec in ("fp32", "bf16"):
        ix = rb.RINND(X, metric=metric, n_neighbors=k, random_state=5, precision=prec)
        gi, gd = ix.neighbor_graph
        rec[prec] = recall(gi[:3000], truth)
        want = rb._lib.JOIN_TENSOR_BF16 if prec == "bf16" else rb._lib.JOIN_PIPELINED_FP32
        assert ix.build_info["join_form"] == want, (prec, ix.build_info["join_form"])
        assert np.all(np.diff(gd, axis=1) >= 0)
        assert ix.build_info["push_contention"] == 0
    assert rec["bf16"] >= rec["fp32"] - 0.005, rec


def test_precision_validation(rb):
    X = gmm(500, 16, 5, seed=2)
    with pytest.raises(ValueError, match="Unknown precision"):
        rb.RINND(X, precision="fp8")
    # Manhattan has no Gram form: the BF16 setting falls back to the FP32 tiles
    ix = rb.RINND(X, metric="manhattan", n_neighbors=8, precision="bf16")
    assert ix.neighbor_graph[0].shape == (500, 8)
