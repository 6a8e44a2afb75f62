"""Join tile shapes and their tuner.

The pipelined FP32 join runs one of several tile shapes (row stages in flight
per CTA, candidate rows per work item, CTAs per SM); a shape changes how the
pairs of a vertex are scheduled, never which pairs are evaluated, their
arithmetic or the pushes.  So one NN-Descent iteration (candidate sampling +
local join + heap pushes, core/nndescent/mod.rs:101-155, :321-491) from the
same rows must give the same rows with every shape: bit-identical distances,
and the same ids except where a row's last distance is tied (the push rejects
d >= the row's max as the reference does, so which of two equally distant
candidates keeps the last slot follows arrival order, for any one shape run
twice as well).  The tuner times the shapes on a sample of the first iteration
and restores the heaps it touched: a build that tunes reaches the recall of
one that does not.
"""
import ctypes

import numpy as np
import pytest

from helpers import gmm, recall
from test_gpu_precision import join_rows, step

pytestmark = pytest.mark.gpu

SQEUCLIDEAN, ALT_COSINE = 0, 3
SHAPES = [(ns, jb, per_sm) for ns in (2, 3) for jb in (2, 1) for per_sm in (0, 2)]


def set_tile(d, kind_class, shape, grouped=0):
    from rinnd_b200 import _lib as L

    row = (ctypes.c_int32 * 8)(0, (d + 3) // 4 * 4, 32, kind_class, grouped, *shape)
    L.check(L.lib.rinnd_join_tile_set(row))


def table():
    from rinnd_b200 import _lib as L

    n = ctypes.c_int32(0)
    L.check(L.lib.rinnd_join_tile_table(None, 0, ctypes.byref(n)))
    rows = (ctypes.c_int32 * (8 * max(n.value, 1)))()
    L.check(L.lib.rinnd_join_tile_table(rows, n.value, ctypes.byref(n)))
    return [tuple(rows[8 * i: 8 * i + 8]) for i in range(n.value)]


def assert_same_rows_up_to_last_ties(ref, got, shape):
    (ri, rd, rf), (gi, gd, gf) = ref, got
    np.testing.assert_array_equal(rd.view(np.uint32), gd.view(np.uint32), err_msg=str(shape))
    last = rd[:, -1:]
    free = rd == last  # entries tied with the row's last distance
    assert np.array_equal(np.where(free, 0, ri), np.where(free, 0, gi)), shape
    assert np.array_equal(np.where(free, 0, rf), np.where(free, 0, gf)), shape
    # tied entries differ only where the tie reaches the row's last slot
    tie_rows = np.nonzero(~np.all(ri == gi, axis=1))[0]
    assert np.all(free[tie_rows].sum(axis=1) >= 1)
    assert len(tie_rows) <= 0.01 * len(ri), (shape, len(tie_rows))


@pytest.mark.parametrize("kind,d", [(SQEUCLIDEAN, 64), (SQEUCLIDEAN, 32), (ALT_COSINE, 96)])
def test_every_tile_shape_gives_the_same_iteration(rb, orc, kind, d):
    from rinnd_b200 import _lib as L

    X = gmm(12000, d, 40, seed=d + 7 * kind)
    if kind != SQEUCLIDEAN:
        X = np.abs(X) + np.float32(0.05)
    k = 15
    L.check(L.lib.rinnd_join_tile_table_clear())
    heap = join_rows(orc, X, k, kind)
    kind_class = 0 if kind == SQEUCLIDEAN else 2
    ref = None
    for shape in SHAPES:
        set_tile(d, kind_class, shape)
        got, changes = step(X, heap, k, kind, L.PRECISION_FP32, 77, 1)
        assert changes > 0
        if ref is None:
            ref = got
            continue
        assert_same_rows_up_to_last_ties(ref, got, shape)
    L.check(L.lib.rinnd_join_tile_table_clear())


def test_tuned_build_matches_the_fixed_shape(rb, orc):
    from rinnd_b200 import _lib as L

    X = gmm(30000, 48, 30, seed=5)
    L.check(L.lib.rinnd_join_tile_table_clear())
    truth, _ = orc.exact_knn_f64(0, X, X[:500], 15, exclude_self=True)
    fixed = rb.RINND(X, metric="sqeuclidean", n_neighbors=15, random_state=3, join_tuning="fixed")
    tuned = rb.RINND(X, metric="sqeuclidean", n_neighbors=15, random_state=3)
    info_f, info_t = fixed.build_info, tuned.build_info
    assert info_f["join_tile_tuned"] == 0 and (info_f["join_tile_stages"], info_f["join_tile_rows"]) == (2, 1)
    assert info_t["join_tile_tuned"] == 1
    shape = (info_t["join_tile_stages"], info_t["join_tile_rows"], info_t["join_tile_ctas_per_sm"])
    assert shape in SHAPES
    assert (0, 48, 32, 0, 0) + shape in table()
    r_f = recall(fixed.neighbor_graph[0][:500], truth)
    r_t = recall(tuned.neighbor_graph[0][:500], truth)
    assert r_t >= r_f - 0.005, (r_t, r_f)
    # a later build of the same key reuses the table without trials
    again = rb.RINND(X, metric="sqeuclidean", n_neighbors=15, random_state=4)
    assert again.build_info["join_tile_tuned"] == 0
    assert (again.build_info["join_tile_stages"], again.build_info["join_tile_rows"]) == shape[:2]
    L.check(L.lib.rinnd_join_tile_table_clear())
