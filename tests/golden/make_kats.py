"""Writes tests/golden/reference_kats.json: the known-answer tests of the
reference's own unit tests for the hot path (lmcinnes/rinnd, crates/rinnd-core).

Each entry restates one asserted case of a reference test: its inputs, the
expected value(s) the reference asserts, the tolerance the reference uses and
the test it comes from (file:line relative to the reference root).  The
reference is Rust and cannot be run here, so the cases are transcribed from
the test sources; nothing here is computed by this project's code.

Run: python tests/golden/make_kats.py
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))
D = "crates/rinnd-core/src/distance/"


def distance_kats():
    k = []

    def add(kind, a, b, expected, tol, src):
        k.append({"kind": kind, "a": a, "b": b, "expected": expected, "tol": tol, "source": src})

    # euclidean.rs tests
    add("sqeuclidean", [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], 2.0, 1e-6, D + "euclidean.rs:188-195")
    add("sqeuclidean", [0.0, 0.0, 0.0], [3.0, 4.0, 0.0], 25.0, 1e-6, D + "euclidean.rs:213-224")
    a = [i * 0.01 for i in range(1024)]
    add("sqeuclidean", a, [x + 0.5 for x in a], 256.0, 1e-3, D + "euclidean.rs:226-235")
    # cosine.rs tests
    add("cosine", [1.0, 2.0, 3.0], [1.0, 2.0, 3.0], 0.0, 1e-6, D + "cosine.rs:147-152")
    add("cosine", [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], 1.0, 1e-6, D + "cosine.rs:154-160")
    add("cosine", [1.0, 0.0, 0.0], [-1.0, 0.0, 0.0], 2.0, 1e-6, D + "cosine.rs:162-168")
    add("cosine", [1.0, 2.0, 3.0], [2.0, 4.0, 6.0], 0.0, 1e-6, D + "cosine.rs:170-177")
    add("cosine", [1.0, 0.0], [1.0, 1.0], 1.0 - 1.0 / math.sqrt(2.0), 1e-5, D + "cosine.rs:186-197")
    # inner_product.rs tests (InnerProduct = -dot)
    add("inner_product", [1.0, 2.0, 3.0], [4.0, 5.0, 6.0], -32.0, 1e-6, D + "inner_product.rs:151-158")
    add("inner_product", [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], 0.0, 1e-6, D + "inner_product.rs:161-168")
    add("inner_product", [1.0, 0.0, 0.0], [2.0, 0.0, 0.0], -2.0, 1e-6, D + "inner_product.rs:171-178")
    add("inner_product", [1.0, 0.0, 0.0], [-1.0, 0.0, 0.0], 1.0, 1e-6, D + "inner_product.rs:181-188")
    add("inner_product", [3.0, 4.0], [3.0, 4.0], -25.0, 1e-6, D + "inner_product.rs:200-206")
    add("inner_product", [0.0, 0.0, 0.0], [1.0, 2.0, 3.0], 0.0, 1e-6, D + "inner_product.rs:220-226")
    # minkowski.rs Manhattan test
    add("manhattan", [1.0, 2.0, 3.0], [4.0, 0.0, -1.0], 9.0, 1e-6, D + "minkowski.rs:219-226")
    # alternatives.rs tests
    n = 1.0 / math.sqrt(3.0)
    add("alt_dot", [n, n, n], [n, n, n], 0.0, 1e-5, D + "alternatives.rs:302-308")
    add("direct_cosine", [1.0, 0.0, 0.0], [1.0, 0.0, 0.0], 0.0, 1e-6, D + "alternatives.rs:330-339")
    add("direct_cosine", [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], 1.0, 1e-6, D + "alternatives.rs:330-339")
    add("direct_cosine", [1.0, 0.0, 0.0], [-1.0, 0.0, 0.0], 2.0, 1e-6, D + "alternatives.rs:330-339")
    add("alt_inner_product", [1.0, 2.0, 3.0], [1.0, 1.0, 1.0], 1.0 / 6.0, 1e-6, D + "alternatives.rs:341-348")
    return k


def correction_kats():
    return [
        {"correction": "alt_cosine", "d": 0.0, "expected": 0.0, "tol": 1e-6, "source": D + "alternatives.rs:350-356"},
        {"correction": "alt_cosine", "d": 1.0, "expected": 0.5, "tol": 1e-6, "source": D + "alternatives.rs:350-356"},
        {"correction": "alt_ip", "d": 0.5, "expected": -2.0, "tol": 1e-6, "source": D + "alternatives.rs:358-364"},
        {"correction": "alt_ip", "d": 3.4028234663852886e38, "expected": 0.0, "tol": 1e-6,
         "source": D + "alternatives.rs:358-364"},
        {"correction": "sqrt", "d": 25.0, "expected": 5.0, "tol": 1e-6, "source": D + "euclidean.rs:213-224"},
    ]


def i8_kats():
    out = []
    for n in [1, 7, 31, 32, 33, 100, 128, 784]:
        x = [((i * 37) % 255) - 127 for i in range(n)]
        y = [((i * 73 + 11) % 255) - 127 for i in range(n)]
        out.append({"x": x, "y": y, "expected": sum(a * b for a, b in zip(x, y)),
                    "source": D + "quantized.rs:446-463"})
    per_dim = {"x": [2, -3, 4], "y": [-5, -2, -1], "scales": [0.5, 0.25, 2.0],
               "expected": -10.0 * 0.25 + 6.0 * 0.0625 - 4.0 * 4.0, "tol": 1e-6,
               "source": D + "quantized.rs:474-481"}
    return out, per_dim


def heap_kats():
    H = "crates/rinnd-core/src/heap/"
    # ops: 0 simple_push, 1 checked_push, 2 checked_flagged_push
    return [
        {"name": "simple_push", "k": 3, "ops": [0, 0, 0, 0, 0],
         "ids": [5, 3, 7, 9, 11], "dists": [1.0, 0.5, 0.8, 0.3, 2.0], "flags": [0, 0, 0, 0, 0],
         "accepted": [1, 1, 1, 1, 0], "max_after": 0.8, "source": H + "neighbor_heap.rs:354-374"},
        {"name": "checked_push_no_duplicates", "k": 3, "ops": [1, 1, 1, 1],
         "ids": [5, 3, 5, 3], "dists": [1.0, 0.5, 0.1, 0.3], "flags": [0, 0, 0, 0],
         "accepted": [1, 1, 0, 0], "source": H + "neighbor_heap.rs:376-388"},
        {"name": "flagged_push", "k": 3, "ops": [2, 2, 2],
         "ids": [5, 3, 7], "dists": [1.0, 0.5, 0.8], "flags": [1, 0, 1],
         "count_new": 2, "source": H + "neighbor_heap.rs:390-402"},
        {"name": "deheap_sort", "k": 5, "ops": [0, 0, 0, 0, 0],
         "ids": [1, 2, 3, 4, 5], "dists": [0.5, 0.2, 0.8, 0.1, 0.3], "flags": [0, 0, 0, 0, 0],
         "sorted_ids": [4, 2, 5, 1, 3], "source": H + "neighbor_heap.rs:404-420"},
        {"name": "heap_property", "k": 7, "ops": [0] * 7,
         "ids": [5, 2, 8, 1, 9, 3, 7], "dists": [0.5, 0.2, 0.8, 0.1, 0.9, 0.3, 0.7], "flags": [0] * 7,
         "heap_property": True, "source": H + "neighbor_heap.rs:422-452"},
    ]


def candidate_heap_kats():
    C = "crates/rinnd-core/src/nndescent/candidates.rs:"
    B = "crates/rinnd-core/src/heap/candidate_heap.rs:"
    return {
        "checked_heap_push_flat": [
            {"size": 3, "priorities": [0.5, 0.3, 0.7], "ids": [1, 2, 3], "contains": [1, 2, 3], "excludes": [],
             "source": C + "491-504"},
            {"size": 3, "priorities": [0.5, 0.3, 0.7], "ids": [1, 1, 1], "count_of_1": 1, "source": C + "506-517"},
            {"size": 3, "priorities": [0.9, 0.8, 0.7, 0.5], "ids": [1, 2, 3, 4], "contains": [4], "excludes": [1],
             "source": C + "519-534"},
        ],
        "bounded_heap": [
            {"k": 3, "dists": [0.5, 0.2, 0.8, 0.1, 0.9], "ids": [1, 2, 3, 4, 5],
             "accepted": [1, 1, 1, 1, 0], "sorted_dists": [0.1, 0.2, 0.5], "source": B + "198-216"},
            {"k": 5, "dists": [0.5, 0.2, 0.8, 0.1, 0.3], "ids": [5, 2, 8, 1, 3],
             "sorted_ids": [1, 2, 3, 5, 8], "source": B + "218-234"},
            {"k": 3, "dists": [0.5, 0.6, 0.7, 0.1, 0.2, 0.3], "ids": [1, 2, 3, 4, 5, 6],
             "sorted_dists": [0.1, 0.2, 0.3], "source": B + "236-256"},
        ],
        "build_candidates": [
            {"n": 5, "k": 3, "max_candidates": 10,
             "pushes": [[0, 1, 0.1, 1], [0, 2, 0.2, 0], [0, 3, 0.3, 0], [1, 0, 0.1, 1], [1, 2, 0.15, 1]],
             "new_contains": {"0": [1], "1": [0, 2]}, "source": C + "535-556"},
            {"n": 3, "k": 2, "max_candidates": 10, "pushes": [[0, 1, 0.1, 1], [1, 2, 0.2, 1]],
             "new_contains": {"1": [0], "2": [1]}, "source": C + "558-575"},
            {"n": 10, "k": 5, "max_candidates": 3,
             "pushes": [[0, i, i * 0.1, 1] for i in range(1, 10)], "max_new_count": {"0": 3},
             "source": C + "577-592"},
        ],
    }


def search_graph_kats():
    G = "crates/rinnd-core/src/graph/search_graph.rs:"
    return [
        {"forward": [[[4, 0.1], [1, 0.4], [2, 0.3]], [], [], [], []],
         "reverse": [[[3, 0.2], [4, 0.9]], [], [], [], []], "max_degree": 2,
         "row0": [2, 3], "nnz": 2, "source": G + "636-652"},
        {"forward": [[[0, 0.0], [-1, 0.1], [3, 0.2], [2, 0.2]], [], [], []],
         "reverse": [[[1, "inf"]], [], [], []], "max_degree": 1,
         "row0": [2], "nnz": 1, "source": G + "654-668"},
    ]


def tree_kats():
    T = "crates/rinnd-core/src/tree/flat_tree.rs:"
    tree = {"hyperplanes": [[1.0, 0.0], [0.0, 0.0], [0.0, 0.0]], "offsets": [0.0, 0.0, 0.0],
            "children": [[1, 2], [0, -2], [-2, -4]], "indices": [0, 1, 2, 3]}
    return {"tree": tree, "cases": [
        {"point": [-1.0, 0.0], "budget": 1, "leaves": [[0, 2]], "source": T + "409-420"},
        {"point": [1.0, 0.0], "budget": 1, "leaves": [[2, 4]], "source": T + "422-433"},
        {"point": [1.0, 0.0], "budget": 2, "leaves": [[2, 4], [0, 2]], "evaluations": 1, "source": T + "468-479"},
    ]}


def sq8p_kat():
    return {"n": 48, "dim": 5, "bound_factor": 0.501, "abs_slack": 1e-7,
            "fixture": "sin((i*37+11)*0.071) + 0.3*cos((i*13)*0.037), rows L2-normalised",
            "source": "crates/rinnd/src/lib.rs:1718-1767"}


def main():
    i8, per_dim = i8_kats()
    kats = {
        "distances": distance_kats(),
        "corrections": correction_kats(),
        "i8_dot": i8,
        "i8_per_dimension_dot": per_dim,
        "neighbor_heap": heap_kats(),
        "candidates": candidate_heap_kats(),
        "search_graph": search_graph_kats(),
        "flat_tree": tree_kats(),
        "sq8p": sq8p_kat(),
    }
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(kats, f, indent=1)


if __name__ == "__main__":
    main()
