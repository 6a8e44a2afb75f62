"""The GPU RP forest against the oracle's tree construction (tree/builder.rs:172-348).

The forest is exported through export_search_tree (lib.rs:1105-1128) with the
two split points of every internal node.  The random choice of split points is
the engine's own stream (the reference's Xoshiro stream is not pinned by any
reference test), so parity is checked per node given those points:
  * every hyperplane and offset equals the oracle's make_split of the node's two
    split points (builder.rs:249-308) bit for bit, and both points lie in the node;
  * every point lies in the leaf the oracle's routing (margin = dot + offset in
    the reference's dot order, builder.rs:331; flat_tree.rs:253-273) sends it to,
    except for points with a tied margin (|m| < 1e-8), which go to a random side;
  * the tree is the reference's FlatTree: depth-first preorder numbering, leaves
    as (-start, -end) ranges that partition the leaf order, a permutation of the
    points, leaves no larger than leaf_size unless the split degenerated.
"""
import numpy as np
import pytest

from helpers import gmm

pytestmark = pytest.mark.gpu


def subtree_ranges(children):
    """(start, end) leaf-order range covered by every node."""
    n = children.shape[0]
    lo = np.zeros(n, np.int64)
    hi = np.zeros(n, np.int64)
    for v in range(n - 1, -1, -1):  # preorder: children have larger ids than their parent
        a, b = children[v]
        if a <= 0:
            lo[v], hi[v] = -a, -b
        else:
            lo[v], hi[v] = lo[a], hi[b]
    return lo, hi


@pytest.mark.parametrize("metric,d,n,leaf", [("sqeuclidean", 32, 20000, 30), ("sqeuclidean", 100, 6000, 60),
                                             ("cosine", 48, 12000, 40)])
def test_forest_matches_oracle_splits_and_routing(rb, orc, metric, d, n, leaf):
    X = gmm(n, d, 25, seed=d)
    if metric == "cosine":
        X = np.abs(X) + np.float32(0.1)
    ix = rb.RINND(X, metric=metric, n_neighbors=10, n_trees=3, n_search_trees=1, leaf_size=leaf, random_state=9)
    check_exported_tree(orc, X, ix, metric, leaf)


def test_grouped_build_forests_match_oracle(rb, orc):
    """Indices built as one group (rinnd_build_many_ex, grouped) share one
    forest pass; each index's exported tree must still be a complete tree over
    its own points with the oracle's splits and routing, including an index
    small enough to be a single leaf."""
    sizes, trees = [20000, 3000, 25, 9000], [3, 2, 3, 4]
    data = [gmm(n, 32, 25, seed=40 + i) for i, n in enumerate(sizes)]
    params = [dict(metric="sqeuclidean", n_neighbors=10, n_trees=t, n_search_trees=1, leaf_size=30, random_state=9)
              for t in trees]
    many = rb.build_many(data, params, grouped=True)
    for X, ix in zip(data, many):
        assert ix.build_info["group_items"] == len(sizes)
        if X.shape[0] <= 30:
            hp, off, ch, ind = ix.export_search_tree()
            assert ch.shape == (1, 2) and ch[0, 0] == 0 and ch[0, 1] == -X.shape[0]
            assert np.array_equal(np.sort(ind), np.arange(X.shape[0]))
            continue
        check_exported_tree(orc, X, ix, "sqeuclidean", 30)


def check_exported_tree(orc, X, ix, metric, leaf):
    n = X.shape[0]
    hp, off, ch, ind, piv = ix.export_search_tree(with_pivots=True)
    m = hp.shape[0]
    assert off.shape == (m,) and ch.shape == (m, 2) and piv.shape == (m, 2)
    # the leaf order is a permutation of the points
    assert np.array_equal(np.sort(ind), np.arange(n))
    internal = ch[:, 0] > 0
    # preorder numbering: the left child follows its parent, children after parents
    assert np.all(ch[internal, 0] == np.nonzero(internal)[0] + 1)
    assert np.all(ch[internal, 1] > ch[internal, 0])
    lo, hi = subtree_ranges(ch)
    leaves = np.nonzero(~internal)[0]
    starts, ends = -ch[leaves, 0], -ch[leaves, 1]
    order = np.argsort(starts)
    assert starts[order][0] == 0 and ends[order][-1] == n
    assert np.array_equal(starts[order][1:], ends[order][:-1])  # leaves tile [0, n) in DFS order
    assert np.all(ends > starts)
    # leaves hold zero hyperplanes and offsets (builder.rs:183-186)
    assert not hp[leaves].any() and not off[leaves].any()
    assert np.all(piv[leaves] == -1)
    # split hyperplanes: the oracle's make_split of the recorded points, bit for bit
    pos = np.empty(n, np.int64)
    pos[ind] = np.arange(n)
    for v in np.nonzero(internal)[0]:
        a, b = piv[v]
        assert a != b
        assert lo[v] <= pos[a] < hi[v] and lo[v] <= pos[b] < hi[v]
        h, o = orc.tree_hyperplane(X[a], X[b], angular=(metric == "cosine"))
        assert np.array_equal(h.view(np.uint32), hp[v].view(np.uint32)), v
        assert np.float32(o).view(np.uint32) == off[v].view(np.uint32), v
    # routing: each point sits in the leaf the oracle's margins lead to
    leaf_of = orc.tree_route_points(hp, off, ch, X)
    tied = leaf_of < 0
    assert tied.mean() < 0.01
    mine = np.empty(n, np.int64)
    for v in leaves:
        mine[ind[-ch[v, 0]:-ch[v, 1]]] = v
    assert np.array_equal(leaf_of[~tied], mine[~tied])
    # leaf sizes: split until <= leaf_size (builder.rs:182); larger leaves only from degenerate splits
    sizes = ends - starts
    assert np.mean(sizes <= leaf) > 0.99


def test_export_search_tree_requires_a_retained_tree(rb):
    X = gmm(2000, 16, 5, seed=1)
    ix = rb.RINND(X, n_neighbors=8, n_trees=2, n_search_trees=0)
    with pytest.raises(ValueError, match="no retained search tree"):
        ix.export_search_tree()
