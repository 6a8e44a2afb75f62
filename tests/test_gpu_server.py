"""Serving form: the continuous-batching server (rinnd_server_*).

Requests of mixed sizes, k and epsilon are submitted from several threads at
once; the server packs them into shared device batches with several batches in
flight.  Every request's result must equal the same request run alone through
the index (query / query_quantized): per-query parameters and random streams
make batching invisible, so the check is exact (ids and distance bits).
"""
import threading

import numpy as np
import pytest

from helpers import gmm

pytestmark = pytest.mark.gpu


def _requests(Q, n_req, ks, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n_req):
        nq = int(np.exp(rng.uniform(0, np.log(300))))
        lo = int(rng.integers(0, len(Q) - nq))
        reqs.append((Q[lo:lo + nq], int(rng.choice(ks)), float(rng.choice([0.1, 0.2]))))
    return reqs


def _serve(server, reqs, n_threads=4):
    results = [None] * len(reqs)
    ids = [None] * len(reqs)

    def client(t):
        for i in range(t, len(reqs), n_threads):
            q, k, eps = reqs[i]
            ids[i] = server.submit(q, k=k, epsilon=eps)
        for i in range(t, len(reqs), n_threads):
            results[i] = server.result(ids[i])

    th = [threading.Thread(target=client, args=(t,)) for t in range(n_threads)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    return results


def test_fp32_server_results_equal_queries_run_alone(rb):
    X = gmm(22000, 64, 40, seed=31)
    X, Q = X[:20000], X[20000:]
    ix = rb.RINND(X, metric="sqeuclidean", n_neighbors=15, random_state=2)
    reqs = _requests(Q, 48, [10, 25, 100], seed=1)
    server = rb.Server(ix, max_batch_queries=512, max_inflight=3)
    got = _serve(server, reqs)
    st = server.stats()
    server.close()
    assert st["completed_requests"] == len(reqs)
    assert st["completed_queries"] == sum(len(q) for q, _, _ in reqs)
    assert st["batches"] >= 2 and st["p99_ms"] >= st["p50_ms"] > 0
    for (q, k, eps), (gi, gd) in zip(reqs, got):
        ai, ad = ix.query(q, k=k, epsilon=eps)
        np.testing.assert_array_equal(gi, ai)
        np.testing.assert_array_equal(gd.view(np.uint32), ad.view(np.uint32))


def test_quantized_server_results_equal_queries_run_alone(rb):
    X = gmm(22000, 96, 60, seed=32)
    X, Q = X[:20000], X[20000:]
    ix = rb.RINND(X, metric="cosine", normalize=True, cosine_distance_mode="int8", n_neighbors=15,
                  quantized_candidate_width=30, quantized_rerank_width=20, random_state=4)
    reqs = _requests(Q, 32, [10, 20], seed=2)
    server = rb.Server(ix, max_batch_queries=256, max_inflight=4)
    got = _serve(server, reqs, n_threads=3)
    server.close()
    for (q, k, eps), (gi, gd) in zip(reqs, got):
        ai, ad = ix.query_quantized(q, k=k, epsilon=eps, candidate_width=30, rerank_width=20)
        np.testing.assert_array_equal(gi, ai)
        np.testing.assert_array_equal(gd.view(np.uint32), ad.view(np.uint32))


def test_server_admission_and_errors(rb):
    from rinnd_b200 import _lib as L

    X = gmm(5000, 32, 10, seed=33)
    ix = rb.RINND(X, n_neighbors=10, random_state=1)
    server = rb.Server(ix, max_batch_queries=64, max_inflight=1, max_pending_queries=64, max_k=50)
    ids, busy = [], 0
    for _ in range(40):  # 64-query requests, one batch slot: the queue fills while a batch runs
        try:
            ids.append(server.submit(X[:64], k=5))
        except RuntimeError as e:
            assert "queue is full" in str(e)
            busy += 1
    assert busy > 0  # the queue holds at most 64 undispatched queries
    for r in ids:
        gi, _ = server.result(r)
        np.testing.assert_array_equal(gi, ix.query(X[:64], k=5)[0])
    with pytest.raises(ValueError):
        server.poll(ids[0])  # already collected
    with pytest.raises(ValueError, match="max_k"):
        server.submit(X[:2], k=51)
    with pytest.raises(ValueError, match="dimension"):
        server.submit(np.zeros((1, 33), np.float32))
    server.close()
    assert L.ERR_BUSY == -6
