"""Prepared launches (rts_plan_*): direct and CUDA-graph launches give the
same pairs as rts_query_batched and as the oracle; after an Insert the next
graph launch re-captures and sees the new boxes."""
import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from rtspatial_b200 import workloads as wl
from tests._gpu_util import SOME_COMBOS, assert_same_pairs, canon, combo_id, dev, make_index

pytestmark = pytest.mark.gpu
P = rb.Predicate


@pytest.mark.parametrize("combo", SOME_COMBOS[:4], ids=combo_id)
@pytest.mark.parametrize("order", [0, 1], ids=["as-given", "curve-sorted"])
def test_plan_graph_replay(cuda, oracle, combo, order):
    rng = np.random.default_rng(77)
    b1 = wl.clustered_boxes(rng, 60_000, 1e-2)
    b2 = wl.uniform_boxes(rng, 30_000, 1e-2)
    pts = wl.uniform_points(rng, 5000)
    qs = wl.uniform_boxes(rng, 5000, 2e-2)
    ix = make_index(combo, sort_queries=order, max_trees=8, rebuild_fraction=1e9)
    ix.Insert(dev(b1))
    specs = [(P.kContains, dev(pts), KIND_POINT, pts), (P.kContains, dev(qs), KIND_CONTAINS, qs),
             (P.kIntersects, dev(qs), KIND_INTERSECTS, qs)]
    queues = [rb.Queue(300_000) for _ in specs]
    plan = ix.plan([(pr, q, rb.Handler.COLLECT, qu.DeviceObject())
                    for (pr, q, _, _), qu in zip(specs, queues)])

    def check(boxes, graph):
        for qu in queues:
            qu.Clear()
        plan.launch(graph=graph)
        torch.cuda.synchronize()
        for (_, _, kind, q), qu in zip(specs, queues):
            assert qu.size() <= qu.capacity()
            assert_same_pairs(canon(qu.result()), oracle.run(kind, boxes, q)[2], f"graph={graph}")

    check(b1, False)
    check(b1, True)
    check(b1, True)   # replay
    ix.Insert(dev(b2))  # new sub-tree: the next graph launch re-captures
    both = np.concatenate([b1, b2])
    check(both, True)
    check(both, False)
    ix.Delete(dev(np.arange(0, 60_000, 7, dtype=np.int64)))  # in place: replay stays valid
    cut = both.copy()
    cut[0:60_000:7, 2] = cut[0:60_000:7, 0]
    cut[0:60_000:7, 3] = cut[0:60_000:7, 1]
    check(cut, True)
    plan.close()


def test_autotune_keeps_results_and_leaves_outputs_alone(cuda, oracle):
    rng = np.random.default_rng(78)
    boxes = wl.clustered_boxes(rng, 80_000, 1e-2)
    pts = wl.uniform_points(rng, 6000)
    qs = wl.uniform_boxes(rng, 6000, 2e-2)
    ix = rb.SpatialIndex(rb.Config(max_trees=4, rebuild_fraction=1e9))
    for part in np.array_split(boxes, 3):
        ix.Insert(dev(part))
    queues = [rb.Queue(200_000) for _ in range(3)]
    specs = [(P.kContains, dev(pts)), (P.kContains, dev(qs)), (P.kIntersects, dev(qs))]
    batches = [(pr, q, rb.Handler.COLLECT, qu.DeviceObject()) for (pr, q), qu in zip(specs, queues)]
    res = ix.autotune(batches, tune_width=True)
    torch.cuda.synchronize()
    assert all(qu.size() == 0 for qu in queues)       # the tuner used its own outputs
    assert res["candidates"] >= 30 and res["collecting"] == 1
    assert res["node_width"] in (4, 8, 16, 32) and res["best_ms"] <= res["first_ms"]
    assert ix.num_trees() == 1 and ix.size() == boxes.shape[0]
    ix.query_batched(batches)
    torch.cuda.synchronize()
    for (kind, q), qu in zip([(KIND_POINT, pts), (KIND_CONTAINS, qs), (KIND_INTERSECTS, qs)], queues):
        assert_same_pairs(canon(qu.result()), oracle.run(kind, boxes, q)[2], "after autotune")
