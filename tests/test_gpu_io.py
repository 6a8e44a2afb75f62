"""Index files: RINND.save / rinnd_b200.load (rinnd_save / rinnd_load).  The
reference keeps its indices in memory only, so the check is self-consistency: a
loaded index returns exactly what the saved one returned -- neighbor graph,
search graph, exported tree and query results bit for bit -- and a damaged file
is rejected."""
import os

import numpy as np
import pytest

from helpers import gmm

pytestmark = pytest.mark.gpu


def test_fp32_index_round_trip(rb, tmp_path):
    X = gmm(15000, 40, 40, seed=51)
    Q = gmm(500, 40, 40, seed=52)
    ix = rb.RINND(X, metric="euclidean", n_neighbors=12, n_search_trees=2, search_tree_leaf_budget=2,
                  random_state=5)
    path = str(tmp_path / "fp32.rinnd")
    ix.save(path)
    iy = rb.load(path)
    for a, b in zip(ix.neighbor_graph, iy.neighbor_graph):
        np.testing.assert_array_equal(a, b)
    a, b = ix.search_graph, iy.search_graph
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    assert a[2] == b[2]
    for u, v in zip(ix.export_search_tree(), iy.export_search_tree()):
        np.testing.assert_array_equal(u, v)
    qa = ix.query(Q, k=10, epsilon=0.1)
    qb = iy.query(Q, k=10, epsilon=0.1)
    np.testing.assert_array_equal(qa[0], qb[0])
    np.testing.assert_array_equal(qa[1].view(np.uint32), qb[1].view(np.uint32))
    assert iy.build_info["iterations"] == ix.build_info["iterations"]


def test_quantized_index_round_trip(rb, tmp_path):
    X = gmm(12000, 64, 40, seed=53)
    Q = gmm(400, 64, 40, seed=54)
    ix = rb.RINND(X, metric="cosine", normalize=True, cosine_distance_mode="int8", tree_quantization="int8",
                  n_neighbors=15, random_state=3)
    path = str(tmp_path / "q8.rinnd")
    ix.save(path)
    iy = rb.load(path)
    qa = ix.query(Q, k=10)
    qb = iy.query(Q, k=10)
    np.testing.assert_array_equal(qa[0], qb[0])
    np.testing.assert_array_equal(qa[1].view(np.uint32), qb[1].view(np.uint32))
    # settings travel with the file: the FP32 rows were released, reranking stays unavailable
    with pytest.raises(ValueError, match="FP32 vector data was released"):
        iy.query_quantized(Q, k=10, candidate_width=30, rerank_width=20)
    assert iy.storage_info()["encoding"] == ix.storage_info()["encoding"]


def test_damaged_files_are_rejected(rb, tmp_path):
    X = gmm(3000, 16, 10, seed=55)
    ix = rb.RINND(X, n_neighbors=8, random_state=1)
    path = str(tmp_path / "ok.rinnd")
    ix.save(path)
    raw = open(path, "rb").read()
    cut = str(tmp_path / "cut.rinnd")
    with open(cut, "wb") as f:
        f.write(raw[: len(raw) // 2])
    with pytest.raises(ValueError, match="truncated"):
        rb.load(cut)
    bad = str(tmp_path / "bad.rinnd")
    with open(bad, "wb") as f:
        f.write(b"NOTRINND" + raw[8:])
    with pytest.raises(ValueError, match="not a rinnd_b200 index file"):
        rb.load(bad)
    with pytest.raises(ValueError, match="cannot open"):
        rb.load(os.path.join(str(tmp_path), "missing.rinnd"))
