"""Serving engine: continuous batching keeps every request's result equal to
the same query run alone; updates apply in submission order; overflowed
parts are re-run exactly; statistics are reported."""
import threading

import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from rtspatial_b200 import workloads as wl
from tests._gpu_util import assert_same_pairs, canon, dev, gpu_pairs

pytestmark = pytest.mark.gpu
P = rb.Predicate
KIND = {0: (KIND_POINT, P.kContains), 1: (KIND_CONTAINS, P.kContains),
        2: (KIND_INTERSECTS, P.kIntersects)}


def make_requests(rng, n_req, max_n=20000):
    reqs = []
    for i in range(n_req):
        k = int(rng.choice([0, 0, 1, 2]))
        n = int(np.exp(rng.uniform(0, np.log(max_n))))
        q = wl.uniform_points(rng, n) if k == 0 else wl.uniform_boxes(rng, n, 2e-2)
        reqs.append((k, q))
    return reqs


def test_server_mix_equals_alone(cuda, oracle):
    rng = np.random.default_rng(31)
    boxes = np.concatenate([wl.uniform_boxes(rng, 100_000, 1e-2),
                            wl.clustered_boxes(rng, 50_000, 1e-2)])
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(boxes))
    torch.cuda.synchronize()
    reqs = make_requests(rng, 48)
    sv = rb.Server(ix, slots=3, max_queries_per_launch=64 * 1024, pairs_per_launch=4 << 20)
    tickets = [None] * len(reqs)

    def submit(idx):
        for i in idx:
            tickets[i] = sv.submit(KIND[reqs[i][0]][1], reqs[i][1])

    threads = [threading.Thread(target=submit, args=(range(j, len(reqs), 2),)) for j in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    got = [canon(sv.take(t)) for t in tickets]
    st = sv.stats()
    sv.close()
    assert st["requests_done"] == len(reqs)
    assert st["queries_done"] == sum(q.shape[0] for _, q in reqs)
    assert st["latency_p99_s"] >= st["latency_p50_s"] > 0
    for (k, q), g in zip(reqs, got):
        alone = gpu_pairs(ix, KIND[k][1], q)
        assert_same_pairs(g, alone, f"request kind {k} n {q.shape[0]} vs alone")
        assert_same_pairs(g, oracle.run(KIND[k][0], boxes, q)[2], "vs oracle")


def test_server_updates_in_submission_order(cuda, oracle):
    rng = np.random.default_rng(32)
    boxes = wl.uniform_boxes(rng, 80_000, 1e-2)
    ix = rb.SpatialIndex(rb.Config(max_trees=4))
    ix.Insert(dev(boxes))
    torch.cuda.synchronize()
    sv = rb.Server(ix, slots=2, max_queries_per_launch=32 * 1024, pairs_per_launch=2 << 20)
    state = boxes.copy()
    expect = []
    for step in range(12):
        for k, q in make_requests(rng, 3, 8000):
            expect.append((sv.submit(KIND[k][1], q), k, q, state.copy()))
        dele = rng.choice(state.shape[0], 300, replace=False)
        upd = rng.choice(state.shape[0], 300, replace=False)
        upd = upd[~np.isin(upd, dele)]
        newb = wl.uniform_boxes(rng, upd.shape[0], 1e-2)
        ins = wl.uniform_boxes(rng, 500, 1e-2)
        t = sv.submit_update(delete_ids=dele, update_ids=upd, update_boxes=newb, inserts=ins)
        state[dele, 2] = state[dele, 0]
        state[dele, 3] = state[dele, 1]
        state[upd] = newb
        first = state.shape[0]
        state = np.concatenate([state, ins])
        assert sv.take(t) == first
    for t, k, q, st in expect:
        assert_same_pairs(canon(sv.take(t)), oracle.run(KIND[k][0], st, q)[2], "ordered update")
    sv.close()
    assert ix.size() == state.shape[0]


def test_server_overflow_reruns_exactly(cuda, oracle):
    rng = np.random.default_rng(33)
    boxes = wl.uniform_boxes(rng, 50_000, 5e-2)   # dense: many pairs per query
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(boxes))
    torch.cuda.synchronize()
    sv = rb.Server(ix, slots=2, max_queries_per_launch=4096, pairs_per_launch=20_000,
                   max_parts_per_launch=8)
    reqs = [(k, q) for k, q in make_requests(rng, 10, 6000)]
    tickets = [sv.submit(KIND[k][1], q) for k, q in reqs]
    got = [canon(sv.take(t)) for t in tickets]
    st = sv.stats()
    sv.close()
    assert st["retried_parts"] > 0
    for (k, q), g in zip(reqs, got):
        assert_same_pairs(g, oracle.run(KIND[k][0], boxes, q)[2], "after re-runs")


def test_server_zero_copy_views_and_stage_times(cuda, oracle):
    """rts_server_view hands out the pinned segments of a request's pairs
    without a copy; after release the memory serves later requests; the
    per-stage times of the statistics add up to something positive."""
    rng = np.random.default_rng(33)
    boxes = wl.uniform_boxes(rng, 80_000, 1e-2)
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(boxes))
    torch.cuda.synchronize()
    # a small result arena: released views must make room for later requests
    sv = rb.Server(ix, slots=2, max_queries_per_launch=16 * 1024, pairs_per_launch=1 << 20,
                   host_result_bytes=8 << 20)
    for rnd in range(3):
        reqs = make_requests(rng, 12, max_n=8000)
        tickets = [sv.submit(KIND[k][1], q) for k, q in reqs]
        for (k, q), t in zip(reqs, tickets):
            segs = sv.view(t)
            got = np.concatenate(segs) if segs else np.zeros((0, 2), np.uint32)
            assert_same_pairs(canon(got), oracle.run(KIND[k][0], boxes, q)[2], f"round {rnd}")
            sv.release(t)
    st = sv.stats()
    sv.close()
    assert st["parts"] >= st["launches"] > 0
    assert st["launch_s"] > 0 and st["copy_s"] > 0 and st["pack_s"] > 0


def test_server_graph_replay_equals_direct_launches(cuda, oracle):
    """Launches replayed through each slot's CUDA graph (updated in place per
    launch) give the pairs of direct launches, for small and sorted launches."""
    rng = np.random.default_rng(35)
    boxes = wl.uniform_boxes(rng, 60_000, 1e-2)
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(boxes))
    torch.cuda.synchronize()
    reqs = make_requests(rng, 24, max_n=30000)
    got = {}
    for graphs in (True, False):
        sv = rb.Server(ix, slots=2, max_queries_per_launch=64 * 1024, pairs_per_launch=4 << 20,
                       use_graphs=graphs)
        tickets = [sv.submit(KIND[k][1], q) for k, q in reqs]
        got[graphs] = [canon(sv.take(t)) for t in tickets]
        st = sv.stats()
        sv.close()
        assert (st["graph_launches"] == st["launches"]) if graphs else st["graph_launches"] == 0
    for (k, q), a, b in zip(reqs, got[True], got[False]):
        assert np.array_equal(a, b)
        assert_same_pairs(a, oracle.run(KIND[k][0], boxes, q)[2], "graph replay vs oracle")
