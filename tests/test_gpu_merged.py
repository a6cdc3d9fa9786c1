"""Merged launches: when every batch of a sorted launch shares one predicate
and handler, the queries of all batches are sorted together and results are
routed back per query.  Each batch must still see exactly its own pairs (with
its own 0-based query ids), its own count, and its own overflow behaviour."""
import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from rtspatial_b200 import workloads as wl
from tests._gpu_util import (SOME_COMBOS, assert_same_pairs, canon, combo_id, dev, make_index)

pytestmark = pytest.mark.gpu
P = rb.Predicate
KINDS = {"point": (KIND_POINT, P.kContains), "contains": (KIND_CONTAINS, P.kContains),
         "intersects": (KIND_INTERSECTS, P.kIntersects)}


def split_sizes(rng, n, parts):
    """Ragged batch sizes summing to n, including a 1-query batch."""
    cuts = np.sort(rng.choice(np.arange(2, n - 1), parts - 2, replace=False))
    sizes = np.diff(np.concatenate([[0], [1], cuts, [n]]))
    assert sizes.sum() == n and (sizes > 0).all()
    return sizes


@pytest.fixture(scope="module")
def scene():
    rng = np.random.default_rng(31)
    boxes = np.concatenate([wl.clustered_boxes(rng, 40_000, 2e-2),
                            wl.uniform_boxes(rng, 20_000, 1e-2)])
    pts = wl.uniform_points(rng, 6000)
    qs = wl.uniform_boxes(rng, 6000, 1e-2)
    return rng, boxes, pts, qs


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
@pytest.mark.parametrize("kind", ["point", "contains", "intersects"])
def test_merged_collect_and_count_per_batch(cuda, oracle, scene, combo, kind):
    rng, boxes, pts, qs = scene
    src = pts if kind == "point" else qs
    ix = make_index(combo, sort_queries=1, max_trees=4, rebuild_fraction=1e9)
    for part in np.array_split(boxes, 2):   # two sub-trees
        ix.Insert(dev(part))
    sizes = split_sizes(np.random.default_rng(5), src.shape[0], 9)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    parts = [src[offs[i]:offs[i + 1]] for i in range(len(sizes))]
    wants = [oracle.run(KINDS[kind][0], boxes, a)[2] for a in parts]
    pred = KINDS[kind][1]
    queues = [rb.Queue(max(16, w.shape[0] + 16)) for w in wants]
    ix.query_batched([(pred, dev(a), rb.Handler.COLLECT, qu.DeviceObject())
                      for a, qu in zip(parts, queues)])
    counters = [rb.Counter() for _ in parts]
    ix.query_batched([(pred, dev(a), rb.Handler.COUNT, c.data()) for a, c in zip(parts, counters)])
    torch.cuda.synchronize()
    for i, (qu, c, w) in enumerate(zip(queues, counters, wants)):
        assert qu.size() == w.shape[0], f"batch {i}"
        assert_same_pairs(canon(qu.result()), w, f"{kind} batch {i}")
        assert c.get() == w.shape[0], f"count batch {i}"


def test_merged_overflow_is_per_batch(cuda, oracle, scene):
    rng, boxes, pts, qs = scene
    ix = rb.SpatialIndex(rb.Config(sort_queries=1))
    ix.Insert(dev(boxes))
    parts = np.array_split(pts, 3)
    wants = [oracle.run(KIND_POINT, boxes, a)[2] for a in parts]
    assert wants[1].shape[0] > 10
    caps = [wants[0].shape[0], wants[1].shape[0] // 3, wants[2].shape[0]]
    queues = []
    for cap in caps:
        qu = rb.Queue(cap + 64)   # 64 guard entries beyond the advertised capacity
        qu.pairs.fill_(-7)
        qu.obj.copy_(torch.tensor([qu.pairs.data_ptr(), cap, qu.counter.data_ptr()],
                                  dtype=torch.int64))
        queues.append(qu)
    ix.query_batched([(P.kContains, dev(a), rb.Handler.COLLECT, qu.DeviceObject())
                      for a, qu in zip(parts, queues)])
    torch.cuda.synchronize()
    for i, (qu, cap, w) in enumerate(zip(queues, caps, wants)):
        assert qu.size() == w.shape[0], f"batch {i} reports what it needs"
        assert bool((qu.pairs[cap:] == -7).all()), f"batch {i} wrote past its capacity"
        kept = canon(qu.pairs[:cap].to(torch.int64) & 0xFFFFFFFF)
        if cap == w.shape[0]:
            assert_same_pairs(kept, w, f"batch {i}")
        else:
            assert set(map(tuple, kept.tolist())) <= set(map(tuple, w.tolist()))


@pytest.mark.parametrize("w", [4, 8, 16, 32])
@pytest.mark.parametrize("traversal", [rb._lib.RTS_TRAVERSAL_THREAD, rb._lib.RTS_TRAVERSAL_TEAM,
                                       rb._lib.RTS_TRAVERSAL_PACKET, rb._lib.RTS_TRAVERSAL_STAGED],
                         ids=["thread", "team", "packet", "staged"])
def test_dense_hits_bypass_the_warp_buffer(cuda, oracle, w, traversal):
    # Every query lies in every box: a warp step finds more pairs than its
    # staging buffer holds and writes them straight to each batch's queue;
    # per-lane packet counts pass 255 (3000 / 4 hits per entry lane at W=4).
    rng = np.random.default_rng(8)
    n = 3000
    lo = rng.uniform(0.0, 0.1, (n, 2)).astype(np.float32)
    hi = rng.uniform(0.9, 1.0, (n, 2)).astype(np.float32)
    boxes = np.concatenate([lo, hi], axis=1)
    pts = rng.uniform(0.4, 0.6, (96, 2)).astype(np.float32)
    parts = [pts[:40], pts[40:41], pts[41:]]
    ix = rb.SpatialIndex(rb.Config(node_width=w, traversal=traversal, sort_queries=1))
    ix.Insert(dev(boxes))
    queues = [rb.Queue(a.shape[0] * n + 16) for a in parts]
    ix.query_batched([(P.kContains, dev(a), rb.Handler.COLLECT, qu.DeviceObject())
                      for a, qu in zip(parts, queues)])
    torch.cuda.synchronize()
    for a, qu in zip(parts, queues):
        assert qu.size() == a.shape[0] * n
        assert_same_pairs(canon(qu.result()), oracle.run(KIND_POINT, boxes, a)[2], "dense")
    counters = [rb.Counter() for _ in parts]
    ix.query_batched([(P.kContains, dev(a), rb.Handler.COUNT, c.data())
                      for a, c in zip(parts, counters)])
    torch.cuda.synchronize()
    assert [c.get() for c in counters] == [a.shape[0] * n for a in parts]
    single = rb.Counter()
    ix.Query(P.kContains, dev(pts), single.data(), handler=rb.Handler.COUNT)
    torch.cuda.synchronize()
    assert single.get() == pts.shape[0] * n


def test_merged_plan_graph_replay(cuda, oracle, scene):
    rng, boxes, pts, qs = scene
    ix = rb.SpatialIndex(rb.Config(sort_queries=1, max_trees=8, rebuild_fraction=1e9))
    ix.Insert(dev(boxes[:40_000]))
    parts = np.array_split(qs, 5)
    queues = [rb.Queue(200_000) for _ in parts]
    plan = ix.plan([(P.kIntersects, dev(a), rb.Handler.COLLECT, qu.DeviceObject())
                    for a, qu in zip(parts, queues)])

    def check(bx):
        for qu in queues:
            qu.Clear()
        plan.launch(graph=True)
        torch.cuda.synchronize()
        for a, qu in zip(parts, queues):
            assert_same_pairs(canon(qu.result()), oracle.run(KIND_INTERSECTS, bx, a)[2], "plan")

    check(boxes[:40_000])
    check(boxes[:40_000])            # replay
    ix.Insert(dev(boxes[40_000:]))   # re-capture with a second sub-tree
    check(boxes)
    plan.close()


@pytest.mark.parametrize("traversal", [rb._lib.RTS_TRAVERSAL_THREAD, rb._lib.RTS_TRAVERSAL_PACKET,
                                       rb._lib.RTS_TRAVERSAL_STAGED],
                         ids=["thread", "packet", "staged"])
def test_merged_many_batches_fill_the_route_table(cuda, oracle, scene, traversal):
    # 300 batches of 20 queries, interleaved by the launch-wide sort: a flush
    # holds pairs of more batches than its table has slots.
    rng, boxes, pts, qs = scene
    ix = rb.SpatialIndex(rb.Config(node_width=16, traversal=traversal, sort_queries=1))
    ix.Insert(dev(boxes))
    big = np.tile(np.array([[0.2, 0.2, 0.8, 0.8]], np.float32), (20, 1))
    boxes2 = np.concatenate([boxes, big])   # every batch gets pairs from these boxes
    ix.Insert(dev(big))
    parts = np.array_split(pts, 300)
    wants = [oracle.run(KIND_POINT, boxes2, a)[2] for a in parts]
    queues = [rb.Queue(w.shape[0] + 8) for w in wants]
    ix.query_batched([(P.kContains, dev(a), rb.Handler.COLLECT, qu.DeviceObject())
                      for a, qu in zip(parts, queues)])
    torch.cuda.synchronize()
    for i, (qu, w) in enumerate(zip(queues, wants)):
        assert qu.size() == w.shape[0], f"batch {i}"
        assert_same_pairs(canon(qu.result()), w, f"batch {i}")
