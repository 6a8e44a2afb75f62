"""Greedy search against the oracle's search on one shared index.

The GPU index's search graph, first search tree, vertex order and rows are
exported and handed to the oracle's restatement of the reference query path
(core/search/greedy.rs:70-241; core/index.rs:157-202) as an index of its own
(OracleIndex.from_parts).  Both then search the same graph from the same tree
leaves with the same per-query random streams, so every query must return the
same neighbors with bit-identical distances -- for queries from the indexed
distribution and for queries far from every point, whose searches expand many
nodes (the GPU's bounded seed set and visited table overflow on those, and the
exact re-run must reproduce the unbounded search).  The random fill of seeds
and the random side of tied tree margins draw from the reference's FastRng
stream (Xoshiro256++ seeded with seed + query id) on both sides.  Exact
distance ties, whose order the reference's BinaryHeap leaves to its internal
layout, do not occur for these continuous inputs.
"""
import numpy as np
import pytest

from helpers import gmm

pytestmark = pytest.mark.gpu

SQEUCLIDEAN, CORR_NONE = 0, 0


def shared_oracle_index(orc, ix, X, kind, corr, leaf_budget, seed):
    indptr, indices, min_d = ix.search_graph
    vo = ix.vertex_order.astype(np.int64)
    inv = np.empty_like(vo)
    inv[vo] = np.arange(len(vo))
    # internal order: row v is original row vo[v]; neighbors mapped by inv
    counts = np.diff(indptr)[vo]
    iptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    iidx = np.concatenate([inv[indices[indptr[o]:indptr[o + 1]]] for o in vo]).astype(np.int32)
    hp, off, ch, leaf_ids = ix.export_search_tree()
    tree = (hp, off, ch, inv[leaf_ids].astype(np.int32))
    return orc.OracleIndex.from_parts(X[vo], kind=kind, correction=corr, indptr=iptr, indices=iidx,
                                      min_distance=min_d, vertex_order=vo, trees=[tree], leaf_budget=leaf_budget,
                                      seed=seed)


@pytest.mark.parametrize("leaf_budget,eps", [(1, 0.1), (4, 0.1), (1, 0.3)])
def test_search_equals_oracle_search_on_the_same_index(rb, orc, leaf_budget, eps):
    X = gmm(30000, 32, 80, seed=33)
    near = gmm(30000 + 800, 32, 80, seed=33)[30000:]  # the indexed mixture
    far = gmm(800, 32, 80, seed=34)                   # other centers: far from every point
    ix = rb.RINND(X, metric="sqeuclidean", n_neighbors=15, n_trees=4, n_search_trees=1,
                  search_tree_leaf_budget=leaf_budget, random_state=6)
    oix = shared_oracle_index(orc, ix, X, SQEUCLIDEAN, CORR_NONE, leaf_budget, 6)
    for Q in (near, far):
        gi, gd = ix.query(Q, k=10, epsilon=eps)
        oi, od = oix.query(Q, k=10, epsilon=eps)
        bad = np.nonzero(~np.all(gi == oi, axis=1))[0]
        assert len(bad) == 0, (len(bad), bad[:5], gi[bad[:2]], oi[bad[:2]])
        np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))


@pytest.mark.parametrize("eps", [0.5, 1.0])
def test_search_equals_oracle_search_on_long_traversals(rb, orc, eps):
    """Tight clusters on the unit sphere: distances within a cluster
    concentrate, so with a wide epsilon a query's bound covers much of its
    cluster and its search expands hundreds to thousands of seeds -- the path
    that refills the sorted seed front from the unsorted back store and spills
    visited ids to the global table.  Results still equal the oracle's on the
    same index."""
    rng = np.random.default_rng(9)
    centers = rng.normal(0.0, 10.0, (10, 64))
    X = centers[rng.integers(0, 10, 20000)] + rng.normal(0.0, 1.0, (20000, 64))
    X = (X / np.linalg.norm(X, axis=1, keepdims=True)).astype(np.float32)
    Q = X[:400] + 0.01 * rng.normal(0.0, 1.0, (400, 64))
    Q = (Q / np.linalg.norm(Q, axis=1, keepdims=True)).astype(np.float32)
    ix = rb.RINND(X, metric="sqeuclidean", n_neighbors=15, n_trees=4, n_search_trees=1, random_state=3)
    oix = shared_oracle_index(orc, ix, X, SQEUCLIDEAN, CORR_NONE, 1, 3)
    ix.search_stats(reset=True)
    gi, gd = ix.query(Q, k=10, epsilon=eps)
    oi, od = oix.query(Q, k=10, epsilon=eps)
    st = ix.search_stats()
    assert st["expansions"] > 200 * len(Q), st  # long traversals did run
    bad = np.nonzero(~np.all(gi == oi, axis=1))[0]
    assert len(bad) == 0, (len(bad), bad[:5], gi[bad[:2]], oi[bad[:2]])
    np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))
