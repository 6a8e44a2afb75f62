"""Brute-force exact kNN (rinnd_brute_force_knn) against exact references.

The FP64 form is checked against numpy in float64 on small inputs, and the
FP32 form against the FP64 form at larger ones: "bit-exact ids wherever the
distances are untied" -- a query's ids must match position by position when
the FP64 distances of its first k + 1 neighbors are separated by more than
8 FP32 ulps of the computation's magnitude (the distance itself for sums of
non-negative terms, |x| |q| for the inner product, 1 for the cosine distance
1 - cos, whose FP32 error is of the order of ulp(1) however small it is), and
its FP32 distances must lie within 1e-5 of the FP64 ones on that scale.  The FP32 form computes each distance with the build's join
arithmetic, so its distances also agree with the reference's distance
functions (the oracle) within the build's 1e-5 tolerance.
"""
import numpy as np
import pytest

from helpers import gmm

pytestmark = pytest.mark.gpu

METRICS = ["sqeuclidean", "manhattan", "inner_product", "cosine"]


def numpy_knn(X, Q, k, metric, exclude_self=False):
    X = X.astype(np.float64)
    Q = Q.astype(np.float64)
    if metric == "sqeuclidean":  # the expansion in float64: far below the ties' 1e-12 threshold here
        D = (Q * Q).sum(1)[:, None] + (X * X).sum(1)[None, :] - 2.0 * (Q @ X.T)
    elif metric == "manhattan":
        D = np.abs(Q[:, None, :] - X[None, :, :]).sum(-1)
    elif metric == "inner_product":
        D = -(Q @ X.T)
    else:
        den = np.sqrt((Q * Q).sum(1)[:, None] * (X * X).sum(1)[None, :])
        D = np.where(den < 1e-12, 1.0, 1.0 - np.clip((Q @ X.T) / np.maximum(den, 1e-300), -1.0, 1.0))
    if exclude_self:
        D[np.arange(len(Q)), np.arange(len(Q))] = np.inf
    ids = np.arange(X.shape[0])
    order = np.stack([np.lexsort((ids, row)) for row in D])
    return order[:, :k].astype(np.int32), np.take_along_axis(D, order[:, :k + 1], 1)


def untied(d, rel, scale=None):
    """Rows whose first len(d[0]) distances are each separated by more than
    rel x scale (scale: the distances' magnitudes unless given)."""
    gaps = np.diff(d, axis=1)
    scale = np.maximum(np.abs(d[:, 1:]) if scale is None else scale[:, 1:], 1e-30)
    return np.all(gaps > rel * scale, axis=1)


@pytest.mark.parametrize("metric", METRICS)
def test_fp64_equals_numpy_float64(rb, metric):
    rng = np.random.default_rng(3)
    X = rng.normal(0.0, 1.0, (3000, 37)).astype(np.float32)
    Q = rng.normal(0.0, 1.0, (150, 37)).astype(np.float32)
    gi, gd = rb.brute_force_knn(X, Q, k=10, metric=metric, precision="fp64")
    ni, nd = numpy_knn(X, Q, 10, metric)
    ok = untied(nd, 1e-12)
    assert ok.mean() > 0.99
    np.testing.assert_array_equal(gi[ok], ni[ok])
    np.testing.assert_allclose(gd, nd[:, :10].astype(np.float32), rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("metric", METRICS)
def test_fp32_ids_match_fp64_wherever_untied(rb, orc, metric):
    X = gmm(60000, 128, 50, seed=21)
    Q = gmm(60000 + 1500, 128, 50, seed=21)[60000:]
    fi, fd = rb.brute_force_knn(X, Q, k=15, metric=metric, precision="fp32")
    di, dd = rb.brute_force_knn(X, Q, k=16, metric=metric, precision="fp64")
    # the FP64 distances of the first k + 1 neighbors, as float64 from the checker's ids
    Xd, Qd = X.astype(np.float64), Q.astype(np.float64)
    nb = Xd[di]
    if metric == "sqeuclidean":
        d64 = ((nb - Qd[:, None, :]) ** 2).sum(-1)
        scale = np.abs(d64)
    elif metric == "manhattan":
        d64 = np.abs(nb - Qd[:, None, :]).sum(-1)
        scale = np.abs(d64)
    elif metric == "inner_product":
        d64 = -(nb * Qd[:, None, :]).sum(-1)
        scale = np.sqrt((nb * nb).sum(-1) * (Qd * Qd).sum(-1)[:, None])
    else:
        d64 = 1.0 - (nb * Qd[:, None, :]).sum(-1) / np.sqrt((nb * nb).sum(-1) * (Qd * Qd).sum(-1)[:, None])
        scale = np.maximum(np.abs(d64), 1.0)
    ok = untied(d64, 8 * 2.0 ** -23, scale)
    assert ok.mean() > 0.5, ok.mean()
    np.testing.assert_array_equal(fi[ok], di[ok, :15])
    err = np.abs(fd.astype(np.float64) - d64[:, :15]) / np.maximum(scale[:, :15], 1e-30)
    assert err.max() < 1e-5, err.max()
    # every reported FP32 distance against the reference's distance function (the oracle)
    kinds = {"sqeuclidean": orc.SQEUCLIDEAN, "manhattan": orc.MANHATTAN, "inner_product": orc.INNER_PRODUCT,
             "cosine": orc.COSINE}
    rows = np.repeat(np.arange(len(Q)), 15)
    ref = orc.distance_pairs(kinds[metric], np.ascontiguousarray(Q[rows]), np.ascontiguousarray(X[fi.reshape(-1)]))
    np.testing.assert_allclose(fd.reshape(-1), ref, rtol=1e-5, atol=1e-5)


def test_exclude_self_and_split_rows(rb):
    X = gmm(20000, 64, 20, seed=5)
    # the data's own kNN graph: no row is its own neighbor
    gi, gd = rb.brute_force_knn(X, X[:500], k=12, metric="sqeuclidean", exclude_self=True)
    assert not np.any(gi == np.arange(500)[:, None])
    ni, nd = numpy_knn(X, X[:500], 12, "sqeuclidean", exclude_self=True)
    ok = untied(nd, 8 * 2.0 ** -23)
    np.testing.assert_array_equal(gi[ok], ni[ok])
    # a few queries (their rows split over many CTAs and merged) give the same
    # results as inside a large batch (one CTA per query tile)
    Q = gmm(20000 + 3000, 64, 20, seed=5)[20000:]
    bi, bd = rb.brute_force_knn(X, Q, k=12)
    for sel in (np.arange(3), np.arange(1000, 1037)):
        si, sd = rb.brute_force_knn(X, Q[sel], k=12)
        np.testing.assert_array_equal(si, bi[sel])
        np.testing.assert_array_equal(sd.view(np.uint32), bd[sel].view(np.uint32))


def test_k_above_n_and_errors(rb):
    rng = np.random.default_rng(1)
    X = rng.normal(0.0, 1.0, (5, 8)).astype(np.float32)
    Q = rng.normal(0.0, 1.0, (4, 8)).astype(np.float32)
    gi, gd = rb.brute_force_knn(X, Q, k=8)
    assert np.all(np.sort(gi[:, :5], axis=1) == np.arange(5))
    assert np.all(gi[:, 5:] == -1) and np.all(np.isinf(gd[:, 5:]))
    assert np.all(np.diff(gd[:, :5], axis=1) >= 0)
    with pytest.raises(ValueError):
        rb.brute_force_knn(X, Q, k=129)
    with pytest.raises(ValueError):
        rb.brute_force_knn(X, Q, k=3, metric="hamming")
    with pytest.raises(ValueError):
        rb.brute_force_knn(X, Q[:, :7], k=3)


@pytest.mark.parametrize("metric,d", [("sqeuclidean", 128), ("sqeuclidean", 37), ("inner_product", 96),
                                      ("cosine", 64)])
def test_bf16_tensor_core_form_equals_fp32(rb, metric, d):
    """The tensor-core form filters with BF16 Gram tiles and rechecks in the
    FP32 form's arithmetic: its results are the FP32 form's, bit for bit."""
    X = gmm(40000, d, 40, seed=8)
    Q = gmm(40000 + 700, d, 40, seed=8)[40000:]
    for k, sel in ((10, slice(None)), (32, slice(0, 5))):  # 5 queries: rows split over many CTAs
        fi, fd = rb.brute_force_knn(X, Q[sel], k=k, metric=metric, precision="fp32")
        ti, td = rb.brute_force_knn(X, Q[sel], k=k, metric=metric, precision="bf16")
        np.testing.assert_array_equal(ti, fi)
        np.testing.assert_array_equal(td.view(np.uint32), fd.view(np.uint32))
    # the data's own graph, self excluded
    fi, fd = rb.brute_force_knn(X, X[:300], k=15, metric=metric, precision="fp32", exclude_self=True)
    ti, td = rb.brute_force_knn(X, X[:300], k=15, metric=metric, precision="bf16", exclude_self=True)
    np.testing.assert_array_equal(ti, fi)
    np.testing.assert_array_equal(td.view(np.uint32), fd.view(np.uint32))
    with pytest.raises(ValueError):
        rb.brute_force_knn(X, Q, k=33, metric=metric, precision="bf16")


def test_bf16_tensor_core_form_edge_shapes(rb):
    """One partial row tile, query counts off the 128-query tile, dimensions
    that need padding, k = 1, and all-zero rows under the cosine distance (its
    1.0 for a zero norm): the tensor-core form's results are the FP32 form's."""
    rng = np.random.default_rng(12)
    for n, d, nq, k in ((50, 5, 3, 1), (50, 5, 3, 8), (129, 17, 130, 4), (1000, 128, 257, 32)):
        X = rng.normal(0.0, 1.0, (n, d)).astype(np.float32)
        Q = rng.normal(0.0, 1.0, (nq, d)).astype(np.float32)
        for metric in ("sqeuclidean", "inner_product", "cosine"):
            fi, fd = rb.brute_force_knn(X, Q, k=k, metric=metric, precision="fp32")
            ti, td = rb.brute_force_knn(X, Q, k=k, metric=metric, precision="bf16")
            np.testing.assert_array_equal(ti, fi, err_msg=f"{metric} n={n} d={d} nq={nq} k={k}")
            np.testing.assert_array_equal(td.view(np.uint32), fd.view(np.uint32))
    X = rng.normal(0.0, 1.0, (300, 24)).astype(np.float32)
    X[::7] = 0.0
    Q = np.concatenate([rng.normal(0.0, 1.0, (20, 24)), np.zeros((2, 24))]).astype(np.float32)
    fi, fd = rb.brute_force_knn(X, Q, k=10, metric="cosine", precision="fp32")
    ti, td = rb.brute_force_knn(X, Q, k=10, metric="cosine", precision="bf16")
    np.testing.assert_array_equal(ti, fi)
    np.testing.assert_array_equal(td.view(np.uint32), fd.view(np.uint32))


def test_device_pointers_equal_host_path(rb):
    """rinnd_brute_force_knn with device-resident inputs, outputs and excluded
    ids (on_device = 1) gives the host path's results, in each form."""
    import ctypes

    import torch

    from rinnd_b200 import _lib as L

    X = gmm(30000, 96, 30, seed=4)
    Q = X[:700].copy()
    dev = torch.device("cuda", 0)
    Xd, Qd = torch.from_numpy(X).to(dev), torch.from_numpy(Q).to(dev)
    ex = torch.arange(700, dtype=torch.int32, device=dev)
    for prec in ("fp32", "bf16", "fp64"):
        hi, hd = rb.brute_force_knn(X, Q, k=12, precision=prec, exclude_self=True)
        oi = torch.empty((700, 12), dtype=torch.int32, device=dev)
        od = torch.empty((700, 12), dtype=torch.float32, device=dev)
        code = {"fp32": L.BRUTE_FP32, "bf16": L.BRUTE_BF16, "fp64": L.BRUTE_FP64}[prec]
        L.check(L.lib.rinnd_brute_force_knn(ctypes.c_void_p(Xd.data_ptr()), 30000, 96, ctypes.c_void_p(Qd.data_ptr()),
                                            700, 96, 96, 12, L.DIST_SQEUCLIDEAN, code,
                                            ctypes.c_void_p(ex.data_ptr()), 1, ctypes.c_void_p(oi.data_ptr()),
                                            ctypes.c_void_p(od.data_ptr())))
        np.testing.assert_array_equal(oi.cpu().numpy(), hi)
        np.testing.assert_array_equal(od.cpu().numpy().view(np.uint32), hd.view(np.uint32))
