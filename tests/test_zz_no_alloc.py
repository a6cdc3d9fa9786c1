"""The batched query that allocates nothing (rts_query_batched_noalloc).

Some callers cannot allocate device memory once they serve requests: they
reserve HBM for the index and its buffers up front and forbid cudaMalloc on
the request path, or only hand the library buffers from their own memory
manager.  For them the library offers a batched query whose scratch (work
counter and descriptor copy) is a fixed array inside the library.  This test
calls it through the C-ABI and checks that two calls in a row give exactly the
pairs and counts of the regular rts_query_batched, and that it refuses more
batches than its fixed scratch holds.  It builds its own index, so it runs
the same alone in a fresh process or after the other tests.
"""
import ctypes

import numpy as np
import pytest
import torch

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


def test_noalloc_batched_matches_regular_batched(cuda):
    rng = np.random.default_rng(2024)
    boxes = wl.clustered_boxes(rng, 200_000, 1e-2)
    pts = torch.from_numpy(wl.uniform_points(rng, 6_000)).cuda()
    qs = torch.from_numpy(wl.uniform_boxes(rng, 6_000, 2e-2)).cuda()
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(torch.from_numpy(boxes).cuda())
    specs = [(L.RTS_QUERY_POINTS, L.RTS_PREDICATE_CONTAINS, pts[:2500]),
             (L.RTS_QUERY_ENVELOPES, L.RTS_PREDICATE_CONTAINS, qs[:4000]),
             (L.RTS_QUERY_ENVELOPES, L.RTS_PREDICATE_INTERSECTS, qs[1000:]),
             (L.RTS_QUERY_POINTS, L.RTS_PREDICATE_CONTAINS, pts[3000:3001])]
    lib = L.lib()

    want_q = [rb.Queue(400_000) for _ in specs]
    L.check(lib.rts_query_batched(ix._h, _batches(specs, want_q), len(specs), None))
    torch.cuda.synchronize()
    want = [_canon(q) for q in want_q]
    assert all(q.size() <= q.capacity() for q in want_q)
    assert sum(w.shape[0] for w in want) > 0

    for call in range(2):  # two calls in a row share the fixed scratch
        got_q = [rb.Queue(400_000) for _ in specs]
        L.check(lib.rts_query_batched_noalloc(ix._h, _batches(specs, got_q), len(specs), None))
        torch.cuda.synchronize()
        for i, (g, w) in enumerate(zip(got_q, want)):
            assert np.array_equal(_canon(g), w), f"call {call}, batch {i}"

    # counting handler, one batch (no descriptor copy), also twice
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


def test_noalloc_rejects_more_batches_than_its_scratch_holds(cuda):
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(torch.tensor([[0, 0, 1, 1]], dtype=torch.float32, device="cuda"))
    c = rb.Counter()
    q = torch.tensor([[0.5, 0.5]], dtype=torch.float32, device="cuda")
    n = L.RTS_NOALLOC_MAX_BATCHES + 1
    arr = (L.rts_batch * n)()
    for i in range(n):
        arr[i].query_kind = L.RTS_QUERY_POINTS
        arr[i].predicate = L.RTS_PREDICATE_CONTAINS
        arr[i].queries = q.data_ptr()
        arr[i].n = 1
        arr[i].handler = L.RTS_HANDLER_COUNT
        arr[i].arg = c.data()
    rc = L.lib().rts_query_batched_noalloc(ix._h, arr, n, None)
    assert rc == L.RTS_ERR_CAPACITY
    assert b"at most 1024 batches" in L.lib().rts_last_error()
    # the maximum itself is accepted
    L.check(L.lib().rts_query_batched_noalloc(ix._h, arr, n - 1, None))
    torch.cuda.synchronize()
    assert c.get() == n - 1
