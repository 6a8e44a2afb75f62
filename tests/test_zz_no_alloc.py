"""The allocation-free push batch (rinnd_heap_push_batch_noalloc) against the
allocating entry point (rinnd_heap_push_batch).

This entry point exists for callers that cannot allocate device memory, e.g. a
host engine that owns the whole device budget or code that must not call
cudaMalloc/cudaFree: they pass their own device buffers and the heap rows live
in the library's static scratch.  The test drives it through the C ABI with
device buffers owned by the test, twice in a row with different inputs (the
scratch keeps the previous call's contents, so the second call proves it is
cleared), and requires outputs identical to the allocating entry point's.
It sits in its own file, collected last, and works alone or after the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_pushes(seed, n, k, n_ops, n_ids):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, n, n_ops).astype(np.int32)
    ids = rng.integers(0, n_ids, n_ops).astype(np.int32)
    # one distance and flag per (row, id), as in NN-Descent where both are functions of the pair
    h = (rows.astype(np.uint64) * np.uint64(2654435761) + ids.astype(np.uint64) * np.uint64(40503)) % np.uint64(1 << 20)
    dists = (h.astype(np.float32) / np.float32(1 << 20)) * np.float32(10.0)
    flags = ((h >> np.uint64(7)) & np.uint64(1)).astype(np.uint8)
    return rows, ids, dists, flags


def allocating(L, n, k, rows, ids, dists, flags):
    oi = np.empty((n, k), np.int32)
    od = np.empty((n, k), np.float32)
    of = np.empty((n, k), np.uint8)
    acc = ctypes.c_int64(0)
    L.check(L.lib.rinnd_heap_push_batch(n, k, rows.size, L.ptr(rows), L.ptr(ids), L.ptr(dists), L.ptr(flags),
                                        L.ptr(oi), L.ptr(od), L.ptr(of), ctypes.byref(acc)))
    return oi, od, of, acc.value


def noalloc(L, torch, n, k, rows, ids, dists, flags):
    dev = torch.device("cuda", 0)
    t_rows, t_ids = torch.from_numpy(rows).to(dev), torch.from_numpy(ids).to(dev)
    t_d, t_f = torch.from_numpy(dists).to(dev), torch.from_numpy(flags).to(dev)
    oi = torch.empty((n, k), dtype=torch.int32, device=dev)
    od = torch.empty((n, k), dtype=torch.float32, device=dev)
    of = torch.empty((n, k), dtype=torch.uint8, device=dev)
    acc = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream(dev)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    L.check(L.lib.rinnd_heap_push_batch_noalloc(n, k, rows.size, p(t_rows), p(t_ids), p(t_d), p(t_f), p(oi),
                                                p(od), p(of), ctypes.byref(acc), ctypes.c_void_p(stream.cuda_stream)))
    return oi.cpu().numpy(), od.cpu().numpy(), of.cpu().numpy(), acc.value


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    from rinnd_b200 import _lib as L

    assert L.device_count() > 0
    for seed, (n, k, n_ops, n_ids) in [(11, (300, 12, 80000, 600)), (12, (1000, 30, 120000, 3000))]:
        rows, ids, dists, flags = make_pushes(seed, n, k, n_ops, n_ids)
        ai, ad, af, _ = allocating(L, n, k, rows, ids, dists, flags)
        ni, nd, nf, nacc = noalloc(L, torch, n, k, rows, ids, dists, flags)
        # both sort rows by (distance, id): outputs are bit-identical
        np.testing.assert_array_equal(ni, ai)
        np.testing.assert_array_equal(nd.view(np.uint32), ad.view(np.uint32))
        np.testing.assert_array_equal(nf, af)
        assert nacc >= int((ai >= 0).sum())


def test_noalloc_rejects_oversized_requests():
    from rinnd_b200 import _lib as L

    # 70000 rows > 65536; 40000 x round_up(30, 16) = 1.28M slots > 1,048,576
    for n, k in [(70000, 4), (40000, 30)]:
        rc = L.lib.rinnd_heap_push_batch_noalloc(n, k, 0, None, None, None, None, ctypes.c_void_p(8),
                                                 ctypes.c_void_p(8), None, None, None)
        assert rc == L.ERR_INVALID
        assert "allocation-free" in L.last_error()


def test_noalloc_invalid_pushes_fail_like_the_allocating_entry_point():
    """Row n and id -1 are out of range for both entry points; id 2^31 - 3 is the
    largest id both accept and 2^31 - 2 the smallest both reject.  The allocation-
    free call checks on the device, so it reports the failure after writing the
    rows built from the valid pushes."""
    torch = pytest.importorskip("torch")
    from rinnd_b200 import _lib as L

    n, k = 64, 8
    rows, ids, dists, flags = make_pushes(21, n, k, 2000, 200)
    ok_ids = ids.copy()
    ok_ids[5] = 0x7FFFFFFD
    ai, ad, af, _ = allocating(L, n, k, rows, ok_ids, dists, flags)
    ni, nd, nf, _ = noalloc(L, torch, n, k, rows, ok_ids, dists, flags)
    np.testing.assert_array_equal(ni, ai)
    np.testing.assert_array_equal(nd.view(np.uint32), ad.view(np.uint32))
    cases = []
    r1, i1 = rows.copy(), ids.copy()
    r1[3] = n
    cases.append((r1, i1))
    r2, i2 = rows.copy(), ids.copy()
    i2[7] = -1
    cases.append((r2, i2))
    r3, i3 = rows.copy(), ids.copy()
    i3[9] = 0x7FFFFFFE
    cases.append((r3, i3))
    dev = torch.device("cuda", 0)
    for br, bi in cases:
        oi = np.empty((n, k), np.int32)
        od = np.empty((n, k), np.float32)
        rc = L.lib.rinnd_heap_push_batch(n, k, br.size, L.ptr(br), L.ptr(bi), L.ptr(dists), L.ptr(flags), L.ptr(oi),
                                         L.ptr(od), None, None)
        assert rc == L.ERR_INVALID and "out of range" in L.last_error()
        t = [torch.from_numpy(a).to(dev) for a in (br, bi, dists, flags)]
        toi = torch.empty((n, k), dtype=torch.int32, device=dev)
        tod = torch.empty((n, k), dtype=torch.float32, device=dev)
        p = lambda x: ctypes.c_void_p(x.data_ptr())
        rc = L.lib.rinnd_heap_push_batch_noalloc(n, k, br.size, *(p(x) for x in t), p(toi), p(tod), None, None,
                                                 ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
        assert rc == L.ERR_INVALID and "out of range" in L.last_error()
    # the scratch is usable again after a failed call
    ni2, nd2, _, _ = noalloc(L, torch, n, k, rows, ok_ids, dists, flags)
    np.testing.assert_array_equal(ni2, ai)
    np.testing.assert_array_equal(nd2.view(np.uint32), ad.view(np.uint32))


def test_noalloc_takes_no_device_memory():
    """Every device allocation of the library is a cudaMallocAsync from the
    device's default memory pool; the pool's high-water mark of memory in use,
    reset before the calls, shows that the allocation-free entry point takes
    none (not even transiently), while the allocating entry point, measured
    the same way, does."""
    torch = pytest.importorskip("torch")
    cudart = pytest.importorskip("cuda.bindings.runtime")
    cudrv = pytest.importorskip("cuda.bindings.driver")
    from rinnd_b200 import _lib as L

    ok = cudart.cudaError_t.cudaSuccess
    high_attr = cudart.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
    cur_attr = cudart.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent
    err, pool = cudart.cudaDeviceGetDefaultMemPool(0)
    assert err == ok

    def attr(a):
        err, v = cudart.cudaMemPoolGetAttribute(pool, a)
        assert err == ok
        return int(v)

    def reset_high():
        (err,) = cudart.cudaMemPoolSetAttribute(pool, high_attr, cudrv.cuuint64_t(0))
        assert err == ok

    n, k = 1000, 30
    rows, ids, dists, flags = make_pushes(31, n, k, 120000, 3000)
    ref = noalloc(L, torch, n, k, rows, ids, dists, flags)  # first call on the device: resolves the scratch
    dev = torch.device("cuda", 0)
    t_rows, t_ids = torch.from_numpy(rows).to(dev), torch.from_numpy(ids).to(dev)
    t_d, t_f = torch.from_numpy(dists).to(dev), torch.from_numpy(flags).to(dev)
    oi = torch.empty((n, k), dtype=torch.int32, device=dev)
    od = torch.empty((n, k), dtype=torch.float32, device=dev)
    of = torch.empty((n, k), dtype=torch.uint8, device=dev)
    stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    torch.cuda.synchronize(dev)
    base = attr(cur_attr)
    reset_high()
    for _ in range(2):
        L.check(L.lib.rinnd_heap_push_batch_noalloc(n, k, rows.size, p(t_rows), p(t_ids), p(t_d), p(t_f), p(oi),
                                                    p(od), p(of), None, stream))
    torch.cuda.synchronize(dev)
    assert attr(high_attr) <= base and attr(cur_attr) == base, (attr(high_attr), base)
    np.testing.assert_array_equal(oi.cpu().numpy(), ref[0])
    # the measurement sees allocations: the allocating entry point's buffers raise the mark
    reset_high()
    allocating(L, n, k, rows, ids, dists, flags)
    assert attr(high_attr) > base
