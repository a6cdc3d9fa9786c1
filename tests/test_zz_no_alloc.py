"""The batched query that allocates nothing (rts_query_batched_noalloc).

Some callers cannot allocate device memory once they serve requests: they
reserve HBM for the index and its buffers up front and forbid cudaMalloc on
the request path, or only hand the library buffers from their own memory
manager.  For them the library offers a batched query whose scratch (work
counter and descriptor copy) is a fixed array inside the library.  These
tests call it through the C-ABI and check that two calls in a row give
exactly the pairs and counts of the regular rts_query_batched, on a float and
on a double index; that neither call moves the library's caching allocator
(where its own allocations come from) or the device's default pool nor,
once the first call has looked up the fixed array, the device's free memory; that it rejects what
rts_query_batched rejects; and that it refuses more non-empty batches than
its fixed scratch holds.  Each test builds its own index, so the file runs the
same alone in a fresh process or after the other tests.
"""
import numpy as np
import pytest
import torch
from cuda.bindings import runtime as cudart

import rtspatial_b200 as rb
from rtspatial_b200 import _lib as L
from rtspatial_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _canon(qu: rb.Queue) -> np.ndarray:
    p = qu.result().cpu().numpy().astype(np.uint64)
    return p[np.lexsort((p[:, 0], p[:, 1]))]


def _batches(specs, queues):
    arr = (L.rts_batch * len(specs))()
    for i, ((kind, pred, q), qu) in enumerate(zip(specs, queues)):
        arr[i].query_kind = kind
        arr[i].predicate = pred
        arr[i].queries = q.data_ptr()
        arr[i].n = q.shape[0]
        arr[i].handler = L.RTS_HANDLER_COLLECT
        arr[i].arg = qu.DeviceObject()
    return arr


def _pool_bytes() -> tuple:
    """(used, reserved) bytes of the current device's default memory pool and
    of the library's caching allocator (where every library allocation comes
    from)."""
    err, dev = cudart.cudaGetDevice()
    assert err == cudart.cudaError_t.cudaSuccess
    err, pool = cudart.cudaDeviceGetDefaultMemPool(dev)
    assert err == cudart.cudaError_t.cudaSuccess
    out = []
    for attr in (cudart.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent,
                 cudart.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent):
        err, v = cudart.cudaMemPoolGetAttribute(pool, attr)
        assert err == cudart.cudaError_t.cudaSuccess
        out.append(int(v))
    reserved, used = rb.memory_pool_stats(dev)
    assert reserved >= used > 0  # the index's buffers live there
    return tuple(out) + (used, reserved)


def _free_bytes() -> int:
    err, free, _total = cudart.cudaMemGetInfo()
    assert err == cudart.cudaError_t.cudaSuccess
    return int(free)


def _check_against_regular(ix, specs):
    """Regular batched call once, then the no-allocation call twice in a row:
    identical pairs per batch, and no device memory taken by either call."""
    lib = L.lib()
    want_q = [rb.Queue(400_000) for _ in specs]
    L.check(lib.rts_query_batched(ix._h, _batches(specs, want_q), len(specs), None))
    torch.cuda.synchronize()
    want = [_canon(q) for q in want_q]
    assert all(q.size() <= q.capacity() for q in want_q)
    assert sum(w.shape[0] for w in want) > 0

    # every output buffer exists before the first measurement
    got_qs = [[rb.Queue(400_000) for _ in specs] for _ in range(2)]
    arrs = [_batches(specs, g) for g in got_qs]
    torch.cuda.synchronize()
    pool0 = _pool_bytes()
    free1 = None
    for call in range(2):  # two calls in a row share the fixed scratch
        L.check(lib.rts_query_batched_noalloc(ix._h, arrs[call], len(specs), None))
        torch.cuda.synchronize()
        if call == 0:
            free1 = _free_bytes()  # after the first call's one-time lookup
    pool2, free2 = _pool_bytes(), _free_bytes()
    # (results are read only now: reading them allocates through torch)
    for call in range(2):
        for i, (g, w) in enumerate(zip(got_qs[call], want)):
            assert g.size() <= g.capacity()
            assert np.array_equal(_canon(g), w), f"call {call}, batch {i}"
    assert pool2 == pool0, "the no-allocation call took memory from a device pool"
    assert free2 == free1, "the second no-allocation call changed the free device memory"


def test_noalloc_batched_matches_regular_batched(cuda):
    rng = np.random.default_rng(2024)
    boxes = wl.clustered_boxes(rng, 200_000, 1e-2)
    pts = torch.from_numpy(wl.uniform_points(rng, 6_000)).cuda()
    qs = torch.from_numpy(wl.uniform_boxes(rng, 6_000, 2e-2)).cuda()
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(torch.from_numpy(boxes).cuda())
    _check_against_regular(ix, [
        (L.RTS_QUERY_POINTS, L.RTS_PREDICATE_CONTAINS, pts[:2500]),
        (L.RTS_QUERY_ENVELOPES, L.RTS_PREDICATE_CONTAINS, qs[:4000]),
        (L.RTS_QUERY_ENVELOPES, L.RTS_PREDICATE_INTERSECTS, qs[1000:]),
        (L.RTS_QUERY_POINTS, L.RTS_PREDICATE_CONTAINS, pts[3000:3001])])
    # all range-intersects: the packet scheme rts_query_batched picks for it
    _check_against_regular(ix, [
        (L.RTS_QUERY_ENVELOPES, L.RTS_PREDICATE_INTERSECTS, qs[:3000]),
        (L.RTS_QUERY_ENVELOPES, L.RTS_PREDICATE_INTERSECTS, qs[3000:])])

    # counting handler, one batch (no descriptor copy), also twice
    lib = L.lib()
    for call in range(2):
        c_ref, c_new = rb.Counter(), rb.Counter()
        one = (L.rts_batch * 1)()
        one[0].query_kind = L.RTS_QUERY_ENVELOPES
        one[0].predicate = L.RTS_PREDICATE_INTERSECTS
        one[0].queries = qs.data_ptr()
        one[0].n = qs.shape[0]
        one[0].handler = L.RTS_HANDLER_COUNT
        one[0].arg = c_ref.data()
        L.check(lib.rts_query_batched(ix._h, one, 1, None))
        one[0].arg = c_new.data()
        L.check(lib.rts_query_batched_noalloc(ix._h, one, 1, None))
        torch.cuda.synchronize()
        assert c_new.get() == c_ref.get() > 0


def test_noalloc_double_index(cuda):
    """SpatialIndex<double, 2>: the _F64 kinds give the regular call's pairs
    (double slab test for range-intersects); float kinds are refused, as
    rts_query_batched refuses them."""
    rng = np.random.default_rng(77)
    boxes = wl.uniform_boxes(rng, 100_000, 2e-2).astype(np.float64) + 1e-9
    pts = torch.from_numpy(wl.uniform_points(rng, 3_000).astype(np.float64)).cuda()
    qs = torch.from_numpy(wl.uniform_boxes(rng, 3_000, 2e-2).astype(np.float64) + 3e-9).cuda()
    ix = rb.SpatialIndex(rb.Config(coord_bits=64))
    ix.Insert(torch.from_numpy(boxes).cuda())
    _check_against_regular(ix, [
        (L.RTS_QUERY_POINTS_F64, L.RTS_PREDICATE_CONTAINS, pts),
        (L.RTS_QUERY_ENVELOPES_F64, L.RTS_PREDICATE_CONTAINS, qs[:1500]),
        (L.RTS_QUERY_ENVELOPES_F64, L.RTS_PREDICATE_INTERSECTS, qs)])

    q32 = qs.float().contiguous()
    c = rb.Counter()
    one = (L.rts_batch * 1)()
    one[0].query_kind = L.RTS_QUERY_ENVELOPES
    one[0].predicate = L.RTS_PREDICATE_INTERSECTS
    one[0].queries = q32.data_ptr()
    one[0].n = q32.shape[0]
    one[0].handler = L.RTS_HANDLER_COUNT
    one[0].arg = c.data()
    lib = L.lib()
    assert lib.rts_query_batched(ix._h, one, 1, None) == L.RTS_ERR_INVALID_ARGUMENT
    assert lib.rts_query_batched_noalloc(ix._h, one, 1, None) == L.RTS_ERR_INVALID_ARGUMENT
    assert b"float queries on a double index" in lib.rts_last_error()


def test_noalloc_rejects_more_batches_than_its_scratch_holds(cuda):
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(torch.tensor([[0, 0, 1, 1]], dtype=torch.float32, device="cuda"))
    c = rb.Counter()
    q = torch.tensor([[0.5, 0.5]], dtype=torch.float32, device="cuda")
    n = L.RTS_NOALLOC_MAX_BATCHES + 1
    arr = (L.rts_batch * (n + 8))()
    for i in range(n + 8):
        arr[i].query_kind = L.RTS_QUERY_POINTS
        arr[i].predicate = L.RTS_PREDICATE_CONTAINS
        arr[i].queries = q.data_ptr()
        arr[i].n = 1
        arr[i].handler = L.RTS_HANDLER_COUNT
        arr[i].arg = c.data()
    lib = L.lib()
    rc = lib.rts_query_batched_noalloc(ix._h, arr, n, None)
    assert rc == L.RTS_ERR_CAPACITY
    assert b"at most 1024 non-empty batches" in lib.rts_last_error()
    # the maximum itself is accepted
    L.check(lib.rts_query_batched_noalloc(ix._h, arr, n - 1, None))
    torch.cuda.synchronize()
    assert c.get() == n - 1
    # empty batches do not count toward the maximum
    for i in range(9):
        arr[i].n = 0
    c.set(0)
    L.check(lib.rts_query_batched_noalloc(ix._h, arr, n + 8, None))
    torch.cuda.synchronize()
    assert c.get() == n - 1
