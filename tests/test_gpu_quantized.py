"""int8 serving path on the GPU against the oracle.

Covers QuantizedI8Index (crates/rinnd/src/lib.rs:159-416) and the quantized
query (core/index.rs:283-334, search/greedy.rs:365-413, rerank index.rs:103-126):
  * row encoder: codes, scales and the global multiplier bit-identical to the
    restatement for all three encodings, including round-half-away ties, zero
    rows and saturating values;
  * quantized search: every returned distance equals the exact int8 similarity
    recomputed by the oracle for that (query, id), bit for bit; recall@10 vs
    exact cosine over 2000 queries not below the oracle's quantized search
    minus 0.5 point (200 queries leave about +-0.5 point of sampling noise);
  * exact rerank: returned distances equal the FP32 DirectNormalizedCosine
    distance in the reference's order, sorted by (distance, id);
  * width rules and the released-FP32 error.
"""
import ctypes

import numpy as np
import pytest

from helpers import gmm, recall

pytestmark = pytest.mark.gpu

MODES = {"int8": 0, "sq8u": 1, "sq8p": 2}
DIRECT_COSINE = 5


def edge_rows(d):
    rows = np.zeros((6, d), np.float32)
    rows[1, :6] = [127.0, 2.5, -2.5, 0.5, -0.5, 126.5]  # multiplier 1: ties round away from zero
    rows[2, :] = 1e-30
    rows[3, :3] = [3e38, -3e38, 1.0]
    rows[4, ::2] = -7.25
    rows[5, :] = np.linspace(-1, 1, d, dtype=np.float32)
    return rows


@pytest.mark.parametrize("mode", list(MODES))
def test_quantize_rows_bit_exact(rb, orc, mode):
    from rinnd_b200 import _lib as L

    enc = MODES[mode]
    X = np.concatenate([gmm(3000, 96, 30, seed=21), edge_rows(96)]).astype(np.float32)
    n, d = X.shape
    codes = np.empty((n, d), np.int8)
    scales = np.empty(n, np.float32)
    gm = ctypes.c_float(0)
    L.check(L.lib.rinnd_quantize_rows(L.ptr(X), n, d, enc, L.ptr(codes), L.ptr(scales), ctypes.byref(gm)))
    oc, os_, ogm = orc.quantize_rows(X, enc)
    np.testing.assert_array_equal(codes, oc)
    np.testing.assert_array_equal(scales.view(np.uint32), os_.view(np.uint32))
    assert np.float32(gm.value).view(np.uint32) == np.float32(ogm).view(np.uint32)


def _setup(rb, orc, mode, n=20000, d=64, nq=2000, seed=5, **kw):
    X = gmm(n + nq, d, 50, seed=seed)
    X, Q = X[:n], X[n:]
    ix = rb.RINND(X, metric="cosine", normalize=True, cosine_distance_mode=mode, n_neighbors=15,
                  random_state=3, **kw)
    return X, Q, ix


def _exact_cosine(orc, Xn, Qn, k):
    return orc.exact_knn_f64(2, Xn, Qn, k)[0]  # cosine on normalized rows


@pytest.mark.parametrize("mode", list(MODES))
def test_quantized_search_distances_and_recall(rb, orc, mode):
    enc = MODES[mode]
    X, Q, ix = _setup(rb, orc, mode)
    Xn, Qn = orc.normalize_rows(X), orc.normalize_rows(Q)
    ids, dists = ix.query_quantized(Q, k=10, epsilon=0.1)
    assert ids.shape == (len(Q), 10)
    # the exact int8 similarity of every returned pair (greedy.rs:384-390)
    codes, inv, gm = orc.quantize_rows(Xn, enc)
    qc, qs = orc.quantize_queries(Qn, enc, gm)
    for i in range(len(Q)):
        v = ids[i][ids[i] >= 0]
        dot = codes[v].astype(np.int32) @ qc[i].astype(np.int32)
        sim = (dot.astype(np.float32) * qs[i]) * inv[v]
        want = np.float32(1.0) - np.clip(sim, np.float32(-1.0), np.float32(1.0))
        np.testing.assert_array_equal(dists[i][: len(v)].view(np.uint32), want.view(np.uint32))
        assert np.all(np.diff(dists[i][: len(v)]) >= 0)
    truth = _exact_cosine(orc, Xn, Qn, 10)
    oix = orc.OracleIndex(Xn, n_neighbors=15, distance_kind=DIRECT_COSINE, angular=True,
                          correction=orc.CORR_NONE, random_seed=3)
    oids, _ = oix.query_quantized(Qn, k=10, epsilon=0.1, encoding=enc)
    assert recall(ids, truth) >= recall(oids, truth) - 0.005


@pytest.mark.parametrize("mode", ["int8", "sq8p"])
def test_quantized_rerank_is_exact_fp32(rb, orc, mode):
    enc = MODES[mode]
    X, Q, ix = _setup(rb, orc, mode, seed=9)
    Xn, Qn = orc.normalize_rows(X), orc.normalize_rows(Q)
    ids, dists = ix.query_quantized(Q, k=10, epsilon=0.1, candidate_width=30, rerank_width=20)
    internal = np.argsort(ix.vertex_order)  # original id -> search-layout id
    for i in range(len(Q)):
        v = ids[i][ids[i] >= 0]
        want = orc.distance_pairs(DIRECT_COSINE, np.repeat(Qn[i : i + 1], len(v), 0), Xn[v])
        np.testing.assert_array_equal(dists[i][: len(v)].view(np.uint32), want.astype(np.float32).view(np.uint32))
        # sorted by (distance, id) before ids are mapped back to the original order (index.rs:116-118, :324-328)
        order = np.lexsort((internal[v], dists[i][: len(v)]))
        np.testing.assert_array_equal(order, np.arange(len(v)))
    truth = _exact_cosine(orc, Xn, Qn, 10)
    oix = orc.OracleIndex(Xn, n_neighbors=15, distance_kind=DIRECT_COSINE, angular=True,
                          correction=orc.CORR_NONE, random_seed=3)
    oids, _ = oix.query_quantized(Qn, k=10, epsilon=0.1, encoding=enc, candidate_width=30, rerank_width=20)
    assert recall(ids, truth) >= recall(oids, truth) - 0.005
    # reranking the wider candidate list does not lose recall against the plain quantized search
    pids, _ = ix.query_quantized(Q, k=10, epsilon=0.1)
    assert recall(ids, truth) >= recall(pids, truth) - 0.005


def test_quantized_query_seed_is_shared_and_widths_validated(rb, orc):
    X, Q, ix = _setup(rb, orc, "int8", n=5000, nq=4)
    q2 = np.repeat(Q[:1], 3, 0)
    ids, dists = ix.query_quantized(q2, k=8)
    np.testing.assert_array_equal(ids[0], ids[1])
    np.testing.assert_array_equal(ids[0], ids[2])
    one = ix.query_one_indices_quantized(Q[0], k=8)
    np.testing.assert_array_equal(one, ids[0])
    with pytest.raises(ValueError, match="at least k"):
        ix.query_quantized(Q, k=10, candidate_width=5)
    with pytest.raises(ValueError, match="must not exceed"):
        ix.query_quantized(Q, k=10, candidate_width=12, rerank_width=20)
    with pytest.raises(ValueError, match="zero or at least k"):
        ix.query_quantized(Q, k=10, candidate_width=20, rerank_width=5)
    info = ix.storage_info()
    assert info["encoding"].startswith("int8")
    assert info["code_bytes"] == X.shape[0] * X.shape[1]


def test_released_fp32_rejects_rerank(rb, orc):
    X, Q, ix = _setup(rb, orc, "sq8p", n=5000, nq=4, retain_fp32_data=False)
    ids, _ = ix.query_quantized(Q, k=6, candidate_width=18)
    assert ids.shape == (4, 6)
    with pytest.raises(ValueError, match="FP32 vector data was released"):
        ix.query_quantized(Q, k=6, candidate_width=18, rerank_width=12)


def test_per_dimension_encoder_bit_exact(rb, orc):
    """sq8d codes and per-dimension scales equal the restatement's: zero
    columns, half-away ties (x / scale = k + 0.5) and saturation included."""
    from rinnd_b200 import _lib as L

    X = np.concatenate([gmm(3000, 96, 30, seed=23), edge_rows(96)]).astype(np.float32)
    X[:, 7] = 0.0  # a zero column: scale 0, codes 0
    X[10, 3] = 127.0 * 4.0
    X[11, 3] = 2.5 * 4.0  # scale of column 3 is 4.0: code 2.5 rounds away from zero
    X[12, 3] = -2.5 * 4.0
    n, d = X.shape
    codes = np.empty((n, d), np.int8)
    scales = np.empty(d, np.float32)
    L.check(L.lib.rinnd_quantize_rows_per_dimension(L.ptr(X), n, d, L.ptr(codes), L.ptr(scales)))
    oc, osc = orc.quantize_per_dimension(X)
    np.testing.assert_array_equal(scales.view(np.uint32), osc.view(np.uint32))
    np.testing.assert_array_equal(codes, oc)
    assert codes[11, 3] == 3 and codes[12, 3] == -3 and scales[7] == 0.0


@pytest.mark.parametrize("rerank", [False, True])
def test_per_dimension_search_distances_and_recall(rb, orc, rerank):
    """Every returned distance of an sq8d search is 1 - clamp(per-dimension
    dot) of the returned pair, computed by the oracle's
    quantized_i8_per_dimension_dot (quantized.rs:48-56) bit for bit; with an
    exact rerank the distances are the FP32 direct cosine of the pair.  Recall@10
    vs exact cosine is not below the oracle's sq8d search minus 0.5 point."""
    X, Q, ix = _setup(rb, orc, "sq8d", seed=13)
    Xn, Qn = orc.normalize_rows(X), orc.normalize_rows(Q)
    kw = dict(candidate_width=30, rerank_width=20) if rerank else {}
    ids, dists = ix.query_quantized(Q, k=10, epsilon=0.1, **kw)
    codes, scales = orc.quantize_per_dimension(Xn)
    qc = orc.quantize_queries_per_dimension(Qn, scales)
    for i in range(len(Q)):
        v = ids[i][ids[i] >= 0]
        if rerank:
            want = orc.distance_pairs(DIRECT_COSINE, np.repeat(Qn[i:i + 1], len(v), 0), Xn[v]).astype(np.float32)
        else:
            sims = np.array([orc.i8_per_dimension_dot(qc[i], codes[j], scales) for j in v], np.float32)
            want = np.float32(1.0) - np.clip(sims, np.float32(-1.0), np.float32(1.0))
        np.testing.assert_array_equal(dists[i][: len(v)].view(np.uint32), want.view(np.uint32))
    truth = _exact_cosine(orc, Xn, Qn, 10)
    oix = orc.OracleIndex(Xn, n_neighbors=15, distance_kind=DIRECT_COSINE, angular=True,
                          correction=orc.CORR_NONE, random_seed=3)
    oids, _ = oix.query_quantized(Qn, k=10, epsilon=0.1, encoding=3, **kw)
    assert recall(ids, truth) >= recall(oids, truth) - 0.005
    assert ix.storage_info()["encoding"] == "sq8d_per_dimension_symmetric"


def test_per_dimension_server_results_equal_alone(rb, orc):
    """The continuous-batching server over an sq8d index returns what the index's
    own quantized query returns."""
    X, Q, ix = _setup(rb, orc, "sq8d", n=8000, nq=300, seed=17, quantized_candidate_width=24,
                      quantized_rerank_width=12)
    srv = rb.Server(ix)
    rids = [srv.submit(Q[i:i + 30], k=8) for i in range(0, 300, 30)]
    got = [srv.result(r) for r in rids]
    srv.close()
    alone_i, alone_d = ix.query_quantized(Q, k=8, candidate_width=24, rerank_width=12)
    np.testing.assert_array_equal(np.concatenate([g[0] for g in got]), alone_i)
    np.testing.assert_array_equal(np.concatenate([g[1] for g in got]).view(np.uint32), alone_d.view(np.uint32))
