"""Batched form: many independent indices of uneven size, dimension and metric
built in one call (rinnd_build_many) against one-at-a-time builds.

Criterion (per index): recall@k of the neighbor graph against FP64 exact
neighbors no more than 0.5 point below the one-at-a-time build's.  Queries of
every batch-built index work as for a single build.
"""
import numpy as np
import pytest

from helpers import gmm, recall

pytestmark = pytest.mark.gpu

TRUTH_KIND = {"sqeuclidean": 0, "cosine": 2, "inner_product": 6}


def make_batch(n_items, seed=0):
    rng = np.random.default_rng(seed)
    datasets, params = [], []
    for i in range(n_items):
        n = int(np.exp(rng.uniform(np.log(2000), np.log(30000))))
        d = int(rng.choice([32, 64, 128, 256]))
        metric = ["sqeuclidean", "sqeuclidean", "cosine", "cosine", "inner_product"][i % 5]
        X = gmm(n, d, int(rng.integers(10, 101)), seed=seed * 1000 + i)
        if metric != "sqeuclidean":
            X = np.abs(X) + np.float32(0.05)
        datasets.append(X)
        params.append({"metric": metric, "n_neighbors": 15, "random_state": 100 + i})
    return datasets, params


def graph_recall(orc, X, gi, metric, k, m=400):
    truth, _ = orc.exact_knn_f64(TRUTH_KIND[metric], X, X[:m], k, exclude_self=True)
    return recall(gi[:m], truth)


def test_build_many_matches_one_at_a_time(rb, orc):
    datasets, params = make_batch(10, seed=3)
    many = rb.build_many(datasets, params, n_workers=4)
    assert len(many) == len(datasets)
    for X, kw, ix in zip(datasets, params, many):
        one = rb.RINND(X, **kw)
        gm, dm = ix.neighbor_graph
        go, _ = one.neighbor_graph
        assert gm.shape == (X.shape[0], 15)
        assert np.all(np.diff(dm, axis=1) >= 0)
        r_many = graph_recall(orc, X, gm, kw["metric"], 15)
        r_one = graph_recall(orc, X, go, kw["metric"], 15)
        assert r_many >= r_one - 0.005, (kw, X.shape, r_many, r_one)
        qi, _ = ix.query(X[:20], k=5)
        assert qi.shape == (20, 5)


def test_build_many_reports_the_failing_item(rb):
    datasets, params = make_batch(3, seed=4)
    params[1] = dict(params[1], n_neighbors=0)
    with pytest.raises(ValueError, match="batch item 1"):
        rb.build_many(datasets, params)
    assert rb.build_many([], []) == []


def test_grouped_build_keeps_each_index_own_stop_rule(rb, orc):
    """One group (same d, metric, k) of uneven sizes: every index stops by its
    own iteration cap and delta test, its graph holds only its own points, and
    its recall is no more than 0.5 point below its one-at-a-time build's."""
    sizes = [12000, 2500, 7000, 300, 18]
    data = [gmm(n, 64, 20, seed=70 + i) for i, n in enumerate(sizes)]
    params = [{"metric": "sqeuclidean", "n_neighbors": 15, "random_state": 5 + i} for i in range(len(sizes))]
    params[2]["n_iters"] = 2
    many = rb.build_many(data, params, grouped=True)
    for X, kw, ix in zip(data, params, many):
        n = X.shape[0]
        info = ix.build_info
        assert info["group_items"] == len(sizes)
        cap = kw.get("n_iters") or max(5, int(np.ceil(np.log2(n))))
        assert 1 <= info["iterations"] <= cap
        gi, gd = ix.neighbor_graph
        assert gi.shape == (n, 15)
        valid = gi >= 0
        assert np.all(gi[valid] < n)
        assert not np.any(gi == np.arange(n)[:, None])
        assert np.all(np.diff(gd, axis=1)[np.all(valid, axis=1)] >= 0)
        if n >= 300:
            one = rb.RINND(X, **kw)
            r_many = graph_recall(orc, X, gi, "sqeuclidean", 15, m=min(400, n))
            r_one = graph_recall(orc, X, one.neighbor_graph[0], "sqeuclidean", 15, m=min(400, n))
            assert r_many >= r_one - 0.005, (n, r_many, r_one)
        else:  # the whole index is one leaf: its rows are exact
            assert np.all(valid)
            assert graph_recall(orc, X, gi, "sqeuclidean", 15, m=n) == 1.0
    assert many[2].build_info["iterations"] == 2
    qi, qd = many[0].query(data[0][:50], k=10)
    assert np.all((qi >= 0) & (qi < sizes[0]))


def test_ungrouped_option_builds_each_index_alone(rb):
    datasets, params = make_batch(4, seed=8)
    many = rb.build_many(datasets, params, grouped=False)
    assert all(ix.build_info["group_items"] == 1 for ix in many)
