"""Pins the oracle (CPU restatement of the reference) to the reference's own
known-answer tests (tests/golden/reference_kats.json)."""
import math

import numpy as np
import pytest

KIND = {"sqeuclidean": 0, "manhattan": 1, "cosine": 2, "alt_cosine": 3, "alt_dot": 4, "direct_cosine": 5,
        "inner_product": 6, "alt_inner_product": 7}
CORR = {"none": 0, "sqrt": 1, "alt_cosine": 2, "alt_ip": 3}


def test_distance_kats(orc, kats):
    for c in kats["distances"]:
        d = orc.distance(KIND[c["kind"]], c["a"], c["b"])
        assert abs(d - c["expected"]) < c["tol"], (c["source"], d, c["expected"])


def test_correction_kats(orc, kats):
    for c in kats["corrections"]:
        assert abs(orc.correct(CORR[c["correction"]], c["d"]) - c["expected"]) < c["tol"], c["source"]


def test_i8_dot_kats(orc, kats):
    for c in kats["i8_dot"]:
        assert orc.i8_dot(c["x"], c["y"]) == c["expected"], c["source"]
    c = kats["i8_per_dimension_dot"]
    assert abs(orc.i8_per_dimension_dot(c["x"], c["y"], c["scales"]) - c["expected"]) < c["tol"]


def test_neighbor_heap_kats(orc, kats):
    for c in kats["neighbor_heap"]:
        acc, idx, dist, flags = orc.neighbor_heap_sequence(c["k"], c["ops"], c["ids"], c["dists"], c["flags"])
        if "accepted" in c:
            assert acc.astype(int).tolist() == c["accepted"], c["name"]
        if "max_after" in c:
            assert abs(dist[0] - c["max_after"]) < 1e-6
        if "count_new" in c:
            assert int(flags.sum()) == c["count_new"]
        if "sorted_ids" in c:
            order = np.argsort(dist, kind="stable")
            assert idx[order].tolist() == c["sorted_ids"]
        if c.get("heap_property"):
            for i in range(c["k"]):
                for ch in (2 * i + 1, 2 * i + 2):
                    if ch < c["k"]:
                        assert dist[i] >= dist[ch]


def test_candidate_heap_kats(orc, kats):
    for c in kats["candidates"]["checked_heap_push_flat"]:
        pri, ids = orc.candidate_heap_sequence(c["size"], c["priorities"], c["ids"])
        for x in c.get("contains", []):
            assert x in ids.tolist(), c["source"]
        for x in c.get("excludes", []):
            assert x not in ids.tolist(), c["source"]
        if "count_of_1" in c:
            assert ids.tolist().count(1) == c["count_of_1"]
    for c in kats["candidates"]["bounded_heap"]:
        acc, ids, dists = orc.bounded_heap_sequence(c["k"], c["dists"], c["ids"])
        if "accepted" in c:
            assert acc.astype(int).tolist() == c["accepted"]
        if "sorted_dists" in c:
            assert np.allclose(dists, c["sorted_dists"], atol=1e-6)
        if "sorted_ids" in c:
            assert ids.tolist() == c["sorted_ids"]


def _heap_from_unchecked(orc, n, k, pushes):
    """Builds heap rows with NeighborHeap::unchecked_flagged_push (neighbor_heap.rs:183-198)."""
    idx = np.full((n, k), -1, np.int32)
    flags = np.zeros((n, k), np.uint8)
    for row in range(n):
        ops = [p for p in pushes if p[0] == row]
        if not ops:
            continue
        _, ri, _, rf = orc.neighbor_heap_sequence(k, [3] * len(ops), [p[1] for p in ops], [p[2] for p in ops], [p[3] for p in ops])
        idx[row], flags[row] = ri, rf
    return idx, flags


def test_build_candidates_kats(orc, kats):
    for c in kats["candidates"]["build_candidates"]:
        idx, flags = _heap_from_unchecked(orc, c["n"], c["k"], c["pushes"])
        for threads in (1, 4):
            new, old, _ = orc.build_candidates(idx, flags, c["max_candidates"], 42, threads)
            for row, members in c.get("new_contains", {}).items():
                for m in members:
                    assert m in new[int(row)].tolist(), c["source"]
            for row, mx in c.get("max_new_count", {}).items():
                assert (new[int(row)] >= 0).sum() <= mx


def test_weighted_union_kats(orc, kats):
    for c in kats["search_graph"]:
        fwd = [[(j, float("inf") if d == "inf" else d) for j, d in row] for row in c["forward"]]
        rev = [[(j, float("inf") if d == "inf" else d) for j, d in row] for row in c["reverse"]]
        indptr, indices = orc.weighted_union_pruned(fwd, rev, c["max_degree"])
        assert indices[indptr[0]:indptr[1]].tolist() == c["row0"], c["source"]
        assert len(indices) == c["nnz"]


def test_flat_tree_kats(orc, kats):
    t = kats["flat_tree"]["tree"]
    for c in kats["flat_tree"]["cases"]:
        ev, leaves = orc.tree_search_leaves(t["hyperplanes"], t["offsets"], t["children"], c["point"], 42, c["budget"])
        assert [list(x) for x in leaves] == c["leaves"], c["source"]
        if "evaluations" in c:
            assert ev == c["evaluations"]


def test_sq8p_error_bound(orc, kats):
    """crates/rinnd/src/lib.rs:1749-1767: |x - code*s| <= 0.501 s (+1e-7)."""
    c = kats["sq8p"]
    n, dim = c["n"], c["dim"]
    i = np.arange(n * dim, dtype=np.float32)
    data = (np.sin((i * 37 + 11) * np.float32(0.071)) + np.cos((i * 13) * np.float32(0.037)) * np.float32(0.3))
    data = data.astype(np.float32).reshape(n, dim)
    data /= np.sqrt((data * data).sum(1, keepdims=True))
    codes, inv, _ = orc.quantize_rows(data, 2)
    assert codes.shape == (n, dim) and inv.shape == (n,)
    err = np.abs(data - codes.astype(np.float32) * inv[:, None])
    assert np.all(err <= inv[:, None] * c["bound_factor"] + c["abs_slack"])


def test_rng_is_xoshiro256pp(orc):
    """FastRng (core/rng.rs:15-86) = Xoshiro256++ seeded via SplitMix64: check the
    published algorithm against an independent restatement."""
    M = (1 << 64) - 1

    def splitmix(x):
        out = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & M
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
            out.append(z ^ (z >> 31))
        return out

    def rotl(v, k):
        return ((v << k) | (v >> (64 - k))) & M

    s = splitmix(42)
    exp = []
    for _ in range(8):
        r = (rotl((s[0] + s[3]) & M, 23) + s[0]) & M
        t = (s[1] << 17) & M
        s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl(s[3], 45)
        exp.append(r)
    assert orc.rng_u64(42, 8).tolist() == exp


def test_query_encoder_matches_row_encoder(orc):
    """lib.rs:325-358 quantize_query uses the row encoder's arithmetic (lib.rs:185-223)."""
    X = np.random.default_rng(3).normal(size=(300, 40)).astype(np.float32)
    X[7] = 0.0
    for enc in range(3):
        codes, scales, gm = orc.quantize_rows(X, enc)
        qc, qs = orc.quantize_queries(X, enc, gm)
        np.testing.assert_array_equal(qc, codes)
        np.testing.assert_array_equal(qs.view(np.uint32), scales.view(np.uint32))


def test_normalize_rows_sequential_sum(orc):
    """lib.rs:1131-1146: sequential f32 sum of squares; tiny rows untouched."""
    X = np.random.default_rng(4).normal(size=(200, 33)).astype(np.float32)
    X[5] = 1e-7
    out = orc.normalize_rows(X)
    nsq = np.add.accumulate(X * X, axis=1, dtype=np.float32)[:, -1]
    inv = np.float32(1.0) / np.sqrt(nsq)
    want = np.where((nsq <= np.float32(1e-12))[:, None], X, X * inv[:, None])
    np.testing.assert_array_equal(out.view(np.uint32), want.astype(np.float32).view(np.uint32))


def test_tree_hyperplane_known_answers(orc):
    """builder.rs:249-308 on hand-checked points: the euclidean split of (0,0)
    and (2,0) is the bisector x = 1 (normal (1,0), offset -1); the angular split
    of (1,0) and (0,1) is normal (-1,1)/sqrt(2) with offset 0; coincident or
    zero points give the zero hyperplane."""
    hp, off = orc.tree_hyperplane([0.0, 0.0], [2.0, 0.0], angular=False)
    assert hp.tolist() == [1.0, 0.0] and off == -1.0
    hp, off = orc.tree_hyperplane([1.0, 0.0], [0.0, 1.0], angular=True)
    r = np.float32(1.0) / np.sqrt(np.float32(2.0))
    assert np.allclose(hp, [-r, r], atol=1e-7) and off == 0.0
    hp, off = orc.tree_hyperplane([3.0, 4.0], [3.0, 4.0], angular=False)
    assert hp.tolist() == [0.0, 0.0] and off == 0.0
    hp, off = orc.tree_hyperplane([0.0, 0.0], [1.0, 1.0], angular=True)
    assert hp.tolist() == [0.0, 0.0] and off == 0.0
    # routing by margin sign: the side of x = 1
    hyperplanes = np.array([[1.0, 0.0], [0.0, 0.0], [0.0, 0.0]], np.float32)
    offsets = np.array([-1.0, 0.0, 0.0], np.float32)
    children = np.array([[1, 2], [0, -1], [-1, -2]], np.int32)
    pts = np.array([[0.0, 5.0], [3.0, -1.0], [1.0, 0.0]], np.float32)
    assert orc.tree_route_points(hyperplanes, offsets, children, pts).tolist() == [1, 2, -1]


def test_oracle_index_from_parts_searches_like_the_built_index(orc):
    """OracleIndex.from_parts over an oracle index's own exported graph and
    vertex order (no search trees) answers queries exactly as that index."""
    import numpy as np

    rng = np.random.default_rng(5)
    X = rng.normal(size=(3000, 16)).astype(np.float32)
    Q = rng.normal(size=(60, 16)).astype(np.float32)
    ix = orc.OracleIndex(X, n_neighbors=10, n_trees=3, n_search_trees=0, distance_kind=0,
                         correction=orc.CORR_NONE, random_seed=9)
    indptr, indices, md = ix.search_graph
    vo = ix.vertex_order.astype(np.int64)
    inv = np.empty_like(vo)
    inv[vo] = np.arange(len(vo))
    counts = np.diff(indptr)[vo]
    iptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    iidx = np.concatenate([inv[indices[indptr[o]:indptr[o + 1]]] for o in vo]).astype(np.int32)
    part = orc.OracleIndex.from_parts(X[vo], kind=0, correction=orc.CORR_NONE, indptr=iptr, indices=iidx,
                                      min_distance=md, vertex_order=vo, seed=9)
    a_i, a_d = ix.query(Q, k=8, epsilon=0.1)
    b_i, b_d = part.query(Q, k=8, epsilon=0.1)
    assert np.array_equal(a_i, b_i)
    assert np.array_equal(a_d.view(np.uint32), b_d.view(np.uint32))
