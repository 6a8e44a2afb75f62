"""Tree seeding of the search against the oracle: spill search with a leaf
budget (FlatTree::search_leaves, core/tree/flat_tree.rs:239-311) and int8
routing trees (QuantizedFlatTree, flat_tree.rs:35-183; tree_quantization="int8",
crates/rinnd/src/lib.rs:681-704).

The GPU's own routing code (the search kernel's tree_search_leaves) is run
through rinnd_tree_search_leaves on the index's first tree; the oracle runs the
reference's search_leaves on the same tree (exported with export_search_tree),
so the visited leaves must match exactly, in order, for every budget: the
frontier's priorities, tie order (first minimum in insertion order) and near /
far sides are the reference's.  Tied margins (|m| < 1e-8), which take a random
side, do not occur for these continuous queries.
"""
import numpy as np
import pytest

from helpers import gmm, recall

pytestmark = pytest.mark.gpu

DIRECT_COSINE = 5


@pytest.mark.parametrize("metric,d", [("sqeuclidean", 48), ("cosine", 64)])
def test_spill_leaves_match_oracle(rb, orc, metric, d):
    X = gmm(12000, d, 30, seed=31)
    Q = gmm(300, d, 30, seed=32)
    if metric == "cosine":
        X, Q = np.abs(X) + np.float32(0.1), np.abs(Q) + np.float32(0.1)
    ix = rb.RINND(X, metric=metric, n_neighbors=10, n_trees=3, n_search_trees=2, search_tree_leaf_budget=4,
                  leaf_size=30, random_state=4)
    hp, off, ch, ind = ix.export_search_tree()
    for budget in (1, 2, 5, 16):
        got = ix.search_tree_leaves(Q, tree=0, leaf_budget=budget)
        for i in range(len(Q)):
            _, want = orc.tree_search_leaves(hp, off, ch, Q[i], 42, budget)
            assert got[i] == want, (budget, i)
        assert all(len(g) == budget for g in got)


def test_spill_seeding_search_recall(rb, orc):
    """A larger leaf budget seeds more points per tree: recall@10 does not drop,
    and at each budget the GPU build + search is within 0.5 point of the
    oracle's build + search (the reference's default epsilon 0.1) for queries
    from the indexed distribution.  (Queries far from every cluster are routed
    to a cluster by the first tree splits alone, so their recall is a property
    of two random trees rather than of the seeding; the shared-index search
    parity test covers them exactly.)"""
    X = gmm(30000, 32, 80, seed=33)
    Q = gmm(32000, 32, 80, seed=33)[30000:]
    truth = orc.exact_knn_f64(0, X, Q, 10)[0]
    rec, orec = {}, {}
    for budget in (1, 4):
        ix = rb.RINND(X, metric="sqeuclidean", n_neighbors=15, n_trees=4, n_search_trees=2,
                      search_tree_leaf_budget=budget, random_state=6)
        ids, _ = ix.query(Q, k=10, epsilon=0.1)
        rec[budget] = recall(ids, truth)
        oix = orc.OracleIndex(X, n_neighbors=15, n_trees=4, n_search_trees=2, search_tree_leaf_budget=budget,
                              distance_kind=0, correction=orc.CORR_NONE, random_seed=6)
        oids, _ = oix.query(Q, k=10, epsilon=0.1)
        orec[budget] = recall(oids, truth)
    assert rec[4] >= rec[1] - 0.002, rec
    for budget in (1, 4):
        assert rec[budget] >= orec[budget] - 0.005, (rec, orec)


@pytest.mark.parametrize("mode", ["int8", "sq8p"])
def test_int8_routing_leaves_match_oracle(rb, orc, mode):
    enc = {"int8": 0, "sq8p": 2}[mode]
    X = np.abs(gmm(10000, 64, 30, seed=35)) + np.float32(0.05)
    Q = np.abs(gmm(300, 64, 30, seed=36)) + np.float32(0.05)
    ix = rb.RINND(X, metric="cosine", normalize=True, cosine_distance_mode=mode, tree_quantization="int8",
                  n_neighbors=10, n_trees=3, n_search_trees=1, random_state=8, quantized_rerank_width=20)
    hp, off, ch, ind = ix.export_search_tree()
    Xn, Qn = orc.normalize_rows(X), orc.normalize_rows(Q)
    _, _, gm = orc.quantize_rows(Xn, enc)
    qc, _ = orc.quantize_queries(Qn, enc, gm)
    qscale = np.abs(Qn).max(axis=1) / np.float32(127.0)
    for budget in (1, 3, 8):
        got = ix.search_tree_leaves(Q, tree=0, leaf_budget=budget, quantized=True)
        fp = ix.search_tree_leaves(Q, tree=0, leaf_budget=budget, quantized=False)
        same = 0
        for i in range(len(Q)):
            _, want = orc.tree_search_leaves_quantized(hp, off, ch, qc[i], qscale[i], 42, budget)
            assert got[i] == want, (budget, i)
            same += got[i] == fp[i]
        # the int8 margins route most queries like the FP32 hyperplanes
        assert same >= 0.5 * len(Q)


def test_int8_routing_trees_search(rb, orc):
    """Quantized search seeded by int8 routing trees: every distance is the
    exact int8 similarity of the pair, recall@10 within 0.5 point of the
    oracle's search over its own int8 routing trees, and the FP32 rows are
    released by default (no exact rerank, rinnd lib.rs:712-716)."""
    X = gmm(20000, 64, 50, seed=37)
    Q = gmm(22000, 64, 50, seed=37)[20000:]  # the indexed distribution
    ix = rb.RINND(X, metric="cosine", normalize=True, cosine_distance_mode="int8", tree_quantization="int8",
                  n_neighbors=15, random_state=3, search_tree_leaf_budget=2)
    Xn, Qn = orc.normalize_rows(X), orc.normalize_rows(Q)
    ids, dists = ix.query(Q, k=10, epsilon=0.1)
    codes, inv, gm = orc.quantize_rows(Xn, 0)
    qc, qs = orc.quantize_queries(Qn, 0, gm)
    for i in range(0, len(Q), 7):
        v = ids[i][ids[i] >= 0]
        dot = codes[v].astype(np.int32) @ qc[i].astype(np.int32)
        sim = (dot.astype(np.float32) * qs[i]) * inv[v]
        want = np.float32(1.0) - np.clip(sim, np.float32(-1.0), np.float32(1.0))
        np.testing.assert_array_equal(dists[i][: len(v)].view(np.uint32), want.view(np.uint32))
    truth = orc.exact_knn_f64(2, Xn, Qn, 10)[0]
    oix = orc.OracleIndex(Xn, n_neighbors=15, distance_kind=DIRECT_COSINE, angular=True, correction=orc.CORR_NONE,
                          random_seed=3, search_tree_leaf_budget=2)
    oids, _ = oix.query_quantized(Qn, k=10, epsilon=0.1, encoding=0, quantize_trees=True)
    assert recall(ids, truth) >= recall(oids, truth) - 0.005
    with pytest.raises(ValueError, match="FP32 vector data was released"):
        ix.query_quantized(Q, k=10, candidate_width=30, rerank_width=20)
    info = ix.storage_info()
    assert info["released_fp32_data_bytes"] == X.shape[0] * X.shape[1] * 4
    assert info["retained_fp32_bytes"] == X.shape[0] * 15 * 4  # neighbor distances only
    assert info["tree_code_bytes"] > 0 and info["released_fp32_tree_bytes"] > 0
