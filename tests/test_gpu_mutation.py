"""Insert / Delete / Update sequences against the oracle: after every step the
GPU's pair sets equal the oracle's over the same (mutated) box array.  Covers
sub-tree inserts, merge rebuilds, refits and update-triggered re-sorts."""
import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from rtspatial_b200 import workloads as wl
from tests._gpu_util import SOME_COMBOS, assert_same_pairs, combo_id, dev, gpu_pairs, make_index

pytestmark = pytest.mark.gpu
P = rb.Predicate


def check_all(ix, oracle, boxes, pts, qs, tag):
    assert_same_pairs(gpu_pairs(ix, P.kContains, pts), oracle.run(KIND_POINT, boxes, pts)[2],
                      f"{tag} point")
    assert_same_pairs(gpu_pairs(ix, P.kContains, qs), oracle.run(KIND_CONTAINS, boxes, qs)[2],
                      f"{tag} contains")
    assert_same_pairs(gpu_pairs(ix, P.kIntersects, qs),
                      oracle.run(KIND_INTERSECTS, boxes, qs)[2], f"{tag} intersects")


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_mutation_sequence(cuda, oracle, combo):
    rng = np.random.default_rng(sum(combo))
    ix = make_index(combo, max_trees=4, rebuild_fraction=0.5, rebuild_update_fraction=0.1)
    boxes = np.zeros((0, 4), np.float32)
    pts = wl.uniform_points(rng, 4000)
    qs = wl.uniform_boxes(rng, 3000, 3e-2)
    for step in range(10):
        op = ["insert", "insert", "delete", "update"][step % 4] if step > 0 else "insert"
        if op == "insert":
            new = wl.uniform_boxes(rng, int(rng.integers(1, 20000)), 2e-2)
            ix.Insert(dev(new))
            boxes = np.concatenate([boxes, new])
        elif op == "delete":
            ids = rng.choice(boxes.shape[0], max(1, boxes.shape[0] // 50), replace=False)
            ids = np.concatenate([ids, [boxes.shape[0] + 5]])  # out of range: ignored
            ix.Delete(dev(ids.astype(np.int64)))
            keep = ids[ids < boxes.shape[0]]
            boxes[keep, 2] = boxes[keep, 0]
            boxes[keep, 3] = boxes[keep, 1]
        else:
            ids = rng.choice(boxes.shape[0], max(1, boxes.shape[0] // 20), replace=False)
            moved = boxes[ids].copy()
            d = rng.uniform(-5e-3, 5e-3, (ids.shape[0], 2)).astype(np.float32)
            moved[:, [0, 2]] += d[:, [0]]
            moved[:, [1, 3]] += d[:, [1]]
            ix.Update(dev(ids.astype(np.int64)), dev(moved))
            boxes[ids] = moved
        assert ix.size() == boxes.shape[0]
        assert 1 <= ix.num_trees() <= 4
        check_all(ix, oracle, boxes, pts, qs, f"step {step} {op}")


def test_clear_restarts_ids(cuda, oracle):
    rng = np.random.default_rng(4)
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(wl.uniform_boxes(rng, 1000, 0.1)))
    ix.Clear()
    assert ix.size() == 0
    b = wl.uniform_boxes(rng, 500, 0.1)
    ix.Insert(dev(b))
    pts = wl.uniform_points(rng, 300)
    assert_same_pairs(gpu_pairs(ix, P.kContains, pts), oracle.run(KIND_POINT, b, pts)[2], "clear")


def test_deleted_box_semantics(cuda, oracle):
    # A deleted box collapses to its min corner and stays indexed
    # (spatial_index.cuh:216-224): a point on that corner still hits it; an
    # intersects query strictly containing it no longer reports it.
    b = np.array([[0.2, 0.2, 0.4, 0.4], [0.6, 0.6, 0.8, 0.8]], np.float32)
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(b))
    ix.Delete(torch.tensor([0], dtype=torch.int64, device="cuda"))
    b[0, 2:] = b[0, :2]
    pts = np.array([[0.2, 0.2], [0.3, 0.3]], np.float32)
    qs = np.array([[0.1, 0.1, 0.5, 0.5], [0.2, 0.2, 0.2, 0.2]], np.float32)
    got_p = gpu_pairs(ix, P.kContains, pts)
    assert got_p.tolist() == [[0, 0]]
    assert_same_pairs(got_p, oracle.run(KIND_POINT, b, pts)[2], "point")
    assert_same_pairs(gpu_pairs(ix, P.kIntersects, qs), oracle.run(KIND_INTERSECTS, b, qs)[2],
                      "intersects")
    assert_same_pairs(gpu_pairs(ix, P.kContains, qs), oracle.run(KIND_CONTAINS, b, qs)[2],
                      "contains")
