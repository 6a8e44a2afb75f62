"""GPU build/query parity: recall against FP64 exact neighbours, compared with the
oracle (the CPU restatement of the reference) at the same parameters, plus the
reference's own index/NN-Descent/Python-API invariants."""
import numpy as np
import pytest

from tests.helpers import gmm, recall, sin_fixture, uniform

pytestmark = pytest.mark.gpu

# Recall may not be lower than the oracle's by more than this (0.5 points).
RECALL_TOL = 0.005


@pytest.mark.parametrize("name,metric,kind,corr,angular", [
    ("uniform10k_sqeuclid", "sqeuclidean", 0, 0, False),
    ("gmm20k_euclid", "euclidean", 0, 1, False),
])
def test_build_recall_not_below_oracle(rb, orc, name, metric, kind, corr, angular):
    """Built-graph recall@k and query recall@10 vs FP64 exact, averaged over three
    seeds, no more than 0.5 points below the oracle's at the same parameters."""
    if name.startswith("uniform"):
        X, k, kw = uniform(10000, 128, seed=0), 15, {}
        Q = uniform(1000, 128, seed=11)
    else:
        X, k, kw = gmm(20000, 64, 50, seed=1), 30, {"n_trees": 8, "leaf_size": 30, "n_iters": 10}
        Q = gmm(21000, 64, 50, seed=1)[20000:]
    truth, _ = orc.exact_knn_f64(kind, X, X, k, exclude_self=True)
    qtruth, _ = orc.exact_knn_f64(kind, X, Q, 10)
    g_rec, o_rec, q_g, q_o = [], [], [], []
    for seed in (42, 7, 1234):
        oix = orc.OracleIndex(X, n_neighbors=k, distance_kind=kind, correction=corr, angular=angular,
                              n_trees=kw.get("n_trees", 8), leaf_size=kw.get("leaf_size"),
                              n_iters=kw.get("n_iters"), random_seed=seed)
        gix = rb.RINND(X, metric=metric, n_neighbors=k, random_state=seed, **kw)
        o_rec.append(recall(oix.neighbor_graph[0], truth))
        g_rec.append(recall(gix.neighbor_graph[0], truth))
        q_o.append(recall(oix.query(Q, k=10, epsilon=0.1)[0], qtruth))
        q_g.append(recall(gix.query(Q, k=10, epsilon=0.1)[0], qtruth))
    g, o, qg, qo = map(np.mean, (g_rec, o_rec, q_g, q_o))
    print(f"{name}: graph recall@{k} gpu={g:.4f} oracle={o:.4f}; query recall@10 gpu={qg:.4f} oracle={qo:.4f}")
    assert g >= o - RECALL_TOL
    assert qg >= qo - RECALL_TOL


def test_neighbor_graph_invariants(rb, orc):
    """nndescent/mod.rs:508-568: every point has a finite neighbour, no self
    neighbours; rows ascending; stored distances are the metric within 1e-5 rel."""
    X = gmm(5000, 32, 20, seed=2)
    ix = rb.RINND(X, metric="euclidean", n_neighbors=10, n_trees=4, random_state=3)
    idx, dist = ix.neighbor_graph
    assert idx.dtype == np.int32 and dist.dtype == np.float32 and idx.shape == (5000, 10)
    assert np.all((idx >= 0).sum(1) > 0)
    assert not np.any(idx == np.arange(5000)[:, None])
    assert np.all(np.diff(dist, axis=1) >= 0)
    rows = np.repeat(np.arange(5000), 10)
    ref = np.sqrt(orc.distance_pairs(0, X[rows], X[idx.reshape(-1)]))
    assert np.allclose(dist.reshape(-1), ref, rtol=1e-5, atol=1e-6)
    for r in range(0, 5000, 97):
        assert len(set(idx[r].tolist())) == 10


def test_search_layout_and_point37(rb):
    """index.rs:811-848 and :850-874: vertex_order is a permutation; the query of
    point 37 returns 37 (sin fixture, n=100, dim=10, k=10, 2 trees, 3 iters)."""
    data = sin_fixture(100, 10)
    for n_trees, n_search in ((2, 1), (3, 2)):
        ix = rb.RINND(data, n_neighbors=10, n_trees=n_trees, n_search_trees=n_search, n_iters=3)
        order = ix.vertex_order
        assert sorted(order.tolist()) == list(range(100))
        idx, _ = ix.query_one(data[37], k=10, epsilon=0.1)
        assert 37 in idx.tolist()


def test_search_graph_export(rb, orc):
    X = gmm(3000, 16, 10, seed=4)
    ix = rb.RINND(X, metric="sqeuclidean", n_neighbors=12, n_trees=4, random_state=5)
    indptr, indices, md = ix.search_graph
    assert indptr[0] == 0 and indptr[-1] == len(indices)
    assert np.all(np.diff(indptr) <= round(1.5 * 12))
    for v in range(0, 3000, 37):
        row = indices[indptr[v]:indptr[v + 1]]
        assert np.all(np.diff(row) > 0) and v not in row.tolist()
    # the export equals from_dense_diversified on the index's own kNN graph (oracle)
    ki, kd = ix.neighbor_graph
    op, oi, omd = orc.search_graph_from_knn(ki, kd, X, 0)
    assert np.array_equal(op, indptr) and np.array_equal(oi, indices) and omd == md


# ---- tests/test_rinnd.py of the reference, on the GPU engine --------------------
def make_data(n_points=32, dimension=4):
    return np.arange(n_points * dimension, dtype=np.float32).reshape(n_points, dimension)


def test_builds_neighbor_graph_and_queries(rb):
    data = make_data()
    index = rb.RINND(data, n_neighbors=6, n_trees=2, n_iters=3, random_state=42)
    indices, distances = index.neighbor_graph
    assert indices.shape == (len(data), 6) and distances.shape == (len(data), 6)
    assert indices.dtype == np.int32 and distances.dtype == np.float32
    qi, qd = index.query(data[:3], k=4)
    assert qi.shape == (3, 4) and qd.shape == (3, 4)
    assert np.all(np.isfinite(qd))


def test_single_query_matches_batch_query(rb):
    data = make_data()
    index = rb.RINND(data, n_neighbors=6, n_trees=2, n_iters=3, random_state=42)
    bi, bd = index.query(data[0][None, :], k=4)
    si, sd = index.query_one(data[0], k=4)
    np.testing.assert_array_equal(si, bi[0])
    np.testing.assert_allclose(sd, bd[0])


def test_cosine_direct_mode(rb):
    data = make_data().astype(np.float32)
    index = rb.RINND(data, metric="cosine", normalize=True, cosine_distance_mode="direct", n_neighbors=6,
                     n_trees=2, n_iters=3, random_state=42)
    indices, distances = index.query(data[:2], k=3)
    assert indices.shape == (2, 3)
    assert np.all((distances >= 0.0) & (distances <= 2.0))
    assert isinstance(rb.simd_info(), str)


def test_rejects_unknown_metric_and_query_dimension(rb):
    data = make_data()
    with pytest.raises(ValueError, match="Unknown metric"):
        rb.RINND(data, metric="not-a-metric")
    index = rb.RINND(data, n_neighbors=6, n_trees=2, n_iters=3)
    with pytest.raises(ValueError, match="dimension"):
        index.query(np.zeros((1, data.shape[1] + 1), dtype=np.float32), k=2)


@pytest.mark.parametrize("metric", ["euclidean", "sqeuclidean", "manhattan", "cosine", "dot", "inner_product"])
def test_all_hot_metrics_build_and_query(rb, orc, metric):
    X = np.abs(gmm(4000, 48, 20, seed=6)) + np.float32(0.01)
    kind = {"euclidean": 0, "sqeuclidean": 0, "manhattan": 1, "cosine": 3, "dot": 4, "inner_product": 7}[metric]
    # AlternativeDot / AlternativeInnerProduct rank by inner product on unnormalized rows
    truth_kind = {0: 0, 1: 1, 3: 2, 4: 6, 7: 6}[kind]
    ix = rb.RINND(X, metric=metric, n_neighbors=15, n_trees=4, random_state=1)
    truth, _ = orc.exact_knn_f64(truth_kind, X, X, 15, exclude_self=True)
    rec = recall(ix.neighbor_graph[0], truth)
    print(metric, rec)
    assert rec > (0.5 if metric in ("inner_product", "dot") else 0.9)
    qi, qd = ix.query(X[:100], k=10)
    assert qi.shape == (100, 10)


def test_empty_and_tiny_inputs(rb):
    one = np.ones((1, 5), np.float32)
    ix = rb.RINND(one, n_neighbors=3, n_trees=2)
    idx, dist = ix.neighbor_graph
    assert idx.tolist() == [[-1, -1, -1]] and np.all(np.isinf(dist))
    qi, qd = ix.query(one, k=3)
    assert qi[0, 0] == 0 and qi[0, 1] == -1 and np.isinf(qd[0, 1])
    z = np.zeros((0, 5), np.float32)
    qi, qd = ix.query(z, k=3)
    assert qi.shape == (0, 3)
