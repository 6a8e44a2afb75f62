"""CPU checks of the drop-in boundary: the C ABI library loads and exports every
symbol include/rinnd.h declares; argument validation mirrors the reference's
Python errors; without a GPU the library fails loudly (no CPU fallback)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "rinnd.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"RINND_EXPORT\s+(?:const\s+)?\w+\s*\*?\s*(rinnd_\w+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["rinnd_build", "rinnd_query", "rinnd_query_one", "rinnd_neighbor_graph", "rinnd_search_graph",
              "rinnd_free", "rinnd_last_error", "rinnd_query_quantized", "rinnd_storage_info_get"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    from rinnd_b200 import _lib as L

    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    for s in declared_symbols():
        assert hasattr(L.lib, s)
        assert s in L.SIGNATURES, f"{s} has no ctypes signature"


def test_kernel_target_query_needs_a_device():
    """rinnd_kernel_target reports the compiled target of the library's kernels
    (cudaFuncGetAttributes); without a device it fails like every other call."""
    from rinnd_b200 import _lib as L

    if L.device_count() > 0:
        pytest.skip("a CUDA device is present (tests/test_gpu_components.py checks the target)")
    b, p = ctypes.c_int32(-1), ctypes.c_int32(-1)
    assert L.lib.rinnd_kernel_target(ctypes.byref(b), ctypes.byref(p)) == L.ERR_NO_DEVICE


def test_params_default_matches_builder_defaults():
    """NNDescentBuilder::new defaults (core/index.rs:475-494)."""
    from rinnd_b200 import _lib as L

    p = L.BuildParams()
    L.check(L.lib.rinnd_params_default(ctypes.byref(p)))
    assert (p.n_neighbors, p.n_trees, p.n_search_trees, p.search_tree_leaf_budget) == (30, 8, 1, 1)
    assert (p.leaf_size, p.max_candidates, p.n_iters) == (0, 0, 0)
    assert abs(p.delta - 0.001) < 1e-9 and p.random_seed == 42
    assert p.diversify_prob == 1.0 and abs(p.pruning_degree_multiplier - 1.5) < 1e-9
    assert p.distance_kind == L.DIST_SQEUCLIDEAN and p.correction == L.CORR_SQRT


def test_invalid_arguments_rejected_before_any_device_work():
    from rinnd_b200 import _lib as L

    p = L.BuildParams()
    L.lib.rinnd_params_default(ctypes.byref(p))
    x = np.zeros((4, 3), np.float32)
    h = ctypes.c_void_p()
    p.n_neighbors = 0
    assert L.lib.rinnd_build(L.ptr(x), 4, 3, ctypes.byref(p), ctypes.byref(h)) == L.ERR_INVALID
    assert "n_neighbors" in L.last_error()
    p.n_neighbors = 5
    assert L.lib.rinnd_build(L.ptr(x), 0, 3, ctypes.byref(p), ctypes.byref(h)) == L.ERR_INVALID
    assert L.lib.rinnd_distance_pairs(99, L.ptr(x), L.ptr(x), 4, 3, L.ptr(x)) == L.ERR_INVALID


def test_no_device_fails_loudly():
    from rinnd_b200 import _lib as L

    if L.device_count() > 0:
        pytest.skip("a CUDA device is present")
    p = L.BuildParams()
    L.lib.rinnd_params_default(ctypes.byref(p))
    x = np.random.default_rng(0).random((64, 8), dtype=np.float32)
    h = ctypes.c_void_p()
    rc = L.lib.rinnd_build(L.ptr(x), 64, 8, ctypes.byref(p), ctypes.byref(h))
    assert rc in (L.ERR_NO_DEVICE, L.ERR_INTERNAL, L.ERR_CUDA)
    assert "no CUDA device" in L.last_error()
    import rinnd_b200

    with pytest.raises(RuntimeError, match="no CUDA device"):
        rinnd_b200.RINND(x, n_neighbors=5)


def test_python_validation_messages():
    """ValueError texts of crates/rinnd/src/lib.rs:643-709 (raised before building)."""
    import rinnd_b200

    x = np.arange(32 * 4, dtype=np.float32).reshape(32, 4)
    with pytest.raises(ValueError, match="Unknown metric: not-a-metric"):
        rinnd_b200.RINND(x, metric="not-a-metric")
    with pytest.raises(ValueError, match="Unknown cosine_distance_mode: zz"):
        rinnd_b200.RINND(x, metric="cosine", normalize=True, cosine_distance_mode="zz")
    with pytest.raises(ValueError, match="require metric='cosine' and normalize=True"):
        rinnd_b200.RINND(x, metric="cosine", cosine_distance_mode="direct")
    with pytest.raises(ValueError, match="Unknown tree_quantization"):
        rinnd_b200.RINND(x, tree_quantization="int4")
    with pytest.raises(ValueError, match="available only with a quantized cosine_distance_mode"):
        rinnd_b200.RINND(x, tree_quantization="int8")
    with pytest.raises(ValueError, match="incompatible with cosine_distance_mode='sq8u'"):
        rinnd_b200.RINND(x, metric="cosine", normalize=True, cosine_distance_mode="sq8u", tree_quantization="int8")
    with pytest.raises(ValueError, match="must not exceed quantized_candidate_width"):
        rinnd_b200.RINND(x, quantized_candidate_width=5, quantized_rerank_width=6)
    with pytest.raises(TypeError):
        rinnd_b200.RINND(x.astype(np.float64))


def test_quantized_width_validation():
    """crates/rinnd/src/lib.rs:1898-1905."""
    from rinnd_b200 import _validate_quantized_widths as v

    v(10, 0, 5)
    for args in [(10, 9, 0), (10, 20, 21), (10, 20, 5)]:
        with pytest.raises(ValueError):
            v(*args)
    v(10, 20, 10)


STRUCTS = {"rinnd_build_params": "BuildParams", "rinnd_build_info": "BuildInfo", "rinnd_batch_item": "BatchItem",
           "rinnd_batch_options": "BatchOptions", "rinnd_server_params": "ServerParams", "rinnd_server_stats": "ServerStats",
           "rinnd_storage_info": "StorageInfo"}


def test_ctypes_mirrors_match_the_header_layout(tmp_path):
    """Every ctypes structure in rinnd_b200/_lib.py has the size and field
    offsets the C compiler gives the struct in include/rinnd.h (a field added on
    one side only would shift every later field)."""
    import shutil

    from rinnd_b200 import _lib as L

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "rinnd.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in getattr(L, pyname)._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    for cname, pyname in STRUCTS.items():
        cls = getattr(L, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert got[(cname, field)] == getattr(cls, field).offset, (cname, field)


def test_join_tile_table_rejects_shapes_that_do_not_exist():
    """rinnd_join_tile_set validates a row on the host (no device needed)."""
    from rinnd_b200 import _lib as L

    for row in [(0, 64, 32, 0, 0, 4, 2, 0), (0, 64, 32, 0, 0, 2, 3, 0), (0, 64, 64, 0, 0, 3, 1, 0),
                (0, 64, 48, 0, 0, 2, 2, 0), (0, 64, 32, 5, 0, 2, 2, 0), (0, 4000, 32, 0, 0, 3, 2, 0)]:
        with pytest.raises(ValueError):
            L.check(L.lib.rinnd_join_tile_set((ctypes.c_int32 * 8)(*row)))
    L.check(L.lib.rinnd_join_tile_set((ctypes.c_int32 * 8)(0, 64, 32, 0, 0, 3, 1, 2)))
    n = ctypes.c_int32(0)
    rows = (ctypes.c_int32 * 8)()
    L.check(L.lib.rinnd_join_tile_table(rows, 1, ctypes.byref(n)))
    assert n.value == 1 and tuple(rows) == (0, 64, 32, 0, 0, 3, 1, 2)
    L.check(L.lib.rinnd_join_tile_table_clear())
    L.check(L.lib.rinnd_join_tile_table(None, 0, ctypes.byref(n)))
    assert n.value == 0


def test_brute_force_arguments_rejected_before_any_device_work():
    """rinnd_brute_force_knn validates shapes, k, precision and the metric
    before touching a device; the Python wrapper raises ValueError for the same."""
    from rinnd_b200 import _lib as L
    import rinnd_b200

    x = np.zeros((4, 3), np.float32)
    oi = np.empty((4, 2), np.int32)
    od = np.empty((4, 2), np.float32)

    def call(k=2, kind=L.DIST_SQEUCLIDEAN, prec=L.BRUTE_FP32, n=4, d=3):
        return L.lib.rinnd_brute_force_knn(L.ptr(x), n, d, L.ptr(x), 4, d, d, k, kind, prec, None, 0, L.ptr(oi),
                                           L.ptr(od))

    assert call(k=0) == L.ERR_INVALID and "k must be" in L.last_error()
    assert call(k=129) == L.ERR_INVALID
    assert call(prec=7) == L.ERR_INVALID and "precision" in L.last_error()
    assert call(kind=L.DIST_HAMMING) == L.ERR_INVALID and "brute force supports" in L.last_error()
    assert call(n=0) == L.ERR_INVALID
    with pytest.raises(ValueError, match="Unknown metric"):
        rinnd_b200.brute_force_knn(x, x, k=2, metric="hamming")
    with pytest.raises(ValueError, match="does not match"):
        rinnd_b200.brute_force_knn(x, x[:, :2], k=2)
    with pytest.raises(ValueError, match="precision"):
        rinnd_b200.brute_force_knn(x, x, k=2, precision="fp16")
