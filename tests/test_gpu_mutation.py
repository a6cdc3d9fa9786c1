"""Insert / Delete / Update sequences against the oracle: after every step the
GPU's pair sets equal the oracle's over the same (mutated) box array.  Covers
sub-tree inserts, merge rebuilds, in-place updates, updates moved to a new
sub-tree, ids updated twice in one call and update-triggered re-sorts."""
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


@pytest.mark.parametrize("w,t", [(16, rb._lib.RTS_TRAVERSAL_THREAD), (32, rb._lib.RTS_TRAVERSAL_PACKET),
                                 (8, rb._lib.RTS_TRAVERSAL_TEAM), (16, rb._lib.RTS_TRAVERSAL_STAGED)],
                         ids=["w16-thread", "w32-packet", "w8-team", "w16-staged"])
def test_update_moves_far_envelopes_to_a_new_subtree(cuda, oracle, w, t):
    # Updates to random far positions leave their leaf group: their slots are
    # emptied and they move (same ids) into a new sub-tree; small moves stay.
    rng = np.random.default_rng(5 + w)
    boxes = wl.uniform_boxes(rng, 40_000, 5e-3)
    pts = wl.uniform_points(rng, 3000)
    qs = wl.uniform_boxes(rng, 3000, 2e-2)
    ix = rb.SpatialIndex(rb.Config(node_width=w, traversal=t, max_trees=8,
                                   rebuild_update_fraction=0.9))
    ix.Insert(dev(boxes))
    far = rng.choice(boxes.shape[0], 3000, replace=False)
    near = np.setdiff1d(rng.choice(boxes.shape[0], 3000, replace=False), far)
    ups = np.concatenate([far, near])
    nb = np.concatenate([wl.uniform_boxes(rng, far.shape[0], 5e-3),
                         boxes[near] + np.float32(1e-7)])
    ix.Update(torch.from_numpy(ups.astype(np.int64)).cuda(), dev(nb))
    cur = boxes.copy()
    cur[ups] = nb
    assert ix.num_trees() == 2     # the moved envelopes form one new sub-tree
    check_all(ix, oracle, cur, pts, qs, "after far updates")
    # deletes reach moved ids through their new slots
    dels = far[:500]
    ix.Delete(torch.from_numpy(dels.astype(np.int64)).cuda())
    oracle.invalidate(cur, dels)
    check_all(ix, oracle, cur, pts, qs, "after deleting moved ids")
    # a re-sort keeps every id once (emptied slots drop out)
    ix2 = rb.SpatialIndex(rb.Config(node_width=w, traversal=t, rebuild_update_fraction=0.0))
    ix2.Insert(dev(boxes))
    ix2.Update(torch.from_numpy(ups.astype(np.int64)).cuda(), dev(nb))
    assert ix2.num_trees() == 1
    cur2 = boxes.copy()
    cur2[ups] = nb
    check_all(ix2, oracle, cur2, pts, qs, "after re-sort")


@pytest.mark.parametrize("w,t", [(16, rb._lib.RTS_TRAVERSAL_THREAD), (32, rb._lib.RTS_TRAVERSAL_PACKET),
                                 (8, rb._lib.RTS_TRAVERSAL_TEAM),
                                 (8, rb._lib.RTS_TRAVERSAL_FRONTIER), (8, rb._lib.RTS_TRAVERSAL_STAGED)],
                         ids=["w16-thread", "w32-packet", "w8-team", "w8-frontier", "w8-staged"])
def test_emptied_slots_match_no_query(cuda, oracle, w, t):
    # A slot emptied by a move keeps its id; it must not answer any query, not
    # even the inverted infinite envelope that every stored box contains
    # (closed-interval compares), nor infinite points and windows.
    rng = np.random.default_rng(90 + w)
    boxes = wl.uniform_boxes(rng, 5000, 5e-3)
    ix = rb.SpatialIndex(rb.Config(node_width=w, traversal=t, max_trees=8,
                                   rebuild_update_fraction=0.9))
    ix.Insert(dev(boxes))
    far = rng.choice(boxes.shape[0], 300, replace=False)
    nb = wl.uniform_boxes(rng, far.shape[0], 5e-3)
    ix.Update(torch.from_numpy(far.astype(np.int64)).cuda(), dev(nb))
    assert ix.num_trees() == 2
    cur = boxes.copy()
    cur[far] = nb
    inf = np.float32(np.inf)
    qs = np.array([[inf, inf, -inf, -inf], [-inf, -inf, inf, inf], [inf, inf, inf, inf],
                   [-inf, -inf, -inf, -inf], [0.2, 0.2, 0.21, 0.21], [inf, -inf, -inf, inf]],
                  np.float32)
    pts = np.array([[inf, inf], [-inf, -inf], [inf, -inf], [0.5, 0.5]], np.float32)
    check_all(ix, oracle, cur, pts, qs, "extreme queries after moves")
    for pred, kind, src in ((P.kContains, KIND_CONTAINS, qs), (P.kIntersects, KIND_INTERSECTS, qs),
                            (P.kContains, KIND_POINT, pts)):
        assert ix.query_count(pred, dev(src)) == oracle.run(kind, cur, src)[2].shape[0]
    # stored envelopes with infinite coordinates (node hulls and the
    # intersects margin become infinite)
    wild = np.array([[-inf, 0.2, 0.3, 0.4], [0.1, 0.1, inf, inf], [-inf, -inf, inf, inf],
                     [0.5, -inf, 0.5, inf]], np.float32)
    ix.Insert(dev(wild))
    cur = np.concatenate([cur, wild])
    normal_qs = wl.uniform_boxes(rng, 500, 2e-2)
    check_all(ix, oracle, cur, np.concatenate([pts, wl.uniform_points(rng, 500)]),
              np.concatenate([qs, normal_qs]), "infinite stored envelopes")


@pytest.mark.parametrize("w,t", [(16, rb._lib.RTS_TRAVERSAL_THREAD), (32, rb._lib.RTS_TRAVERSAL_PACKET),
                                 (8, rb._lib.RTS_TRAVERSAL_TEAM)], ids=["w16-thread", "w32-packet",
                                                                        "w8-team"])
def test_small_subtrees_merge_beside_the_base(cuda, oracle, w, t):
    # At the sub-tree limit, sub-trees that are small beside the largest merge
    # into one new sub-tree and the largest keeps its slots (no full re-sort:
    # at least two sub-trees remain).  Slots emptied by moved updates come
    # along into the merge; their ids must keep pointing at the live copies.
    rng = np.random.default_rng(77 + w)
    base = wl.uniform_boxes(rng, 120_000, 5e-3)
    pts = wl.uniform_points(rng, 2000)
    qs = wl.uniform_boxes(rng, 2000, 2e-2)
    ix = rb.SpatialIndex(rb.Config(node_width=w, traversal=t, max_trees=4, rebuild_fraction=0.5,
                                   rebuild_update_fraction=0.9))
    ix.Insert(dev(base))
    cur = base.copy()
    merged_seen = False
    for step in range(14):
        before = ix.num_trees()
        if step % 3 == 2:   # far moves: emptied slots plus a moved sub-tree
            ids = rng.choice(cur.shape[0], 400, replace=False)
            nb = wl.uniform_boxes(rng, ids.shape[0], 5e-3)
            ix.Update(torch.from_numpy(ids.astype(np.int64)).cuda(), dev(nb))
            cur[ids] = nb
        else:
            new = wl.uniform_boxes(rng, int(rng.integers(300, 1500)), 5e-3)
            ix.Insert(dev(new))
            cur = np.concatenate([cur, new])
        if step % 4 == 3:   # deletes reach ids wherever they now live
            dels = rng.choice(cur.shape[0], 300, replace=False)
            ix.Delete(torch.from_numpy(dels.astype(np.int64)).cuda())
            oracle.invalidate(cur, dels)
        merged_seen |= ix.num_trees() < before
        assert 2 <= ix.num_trees() <= 4, f"step {step}: {ix.num_trees()} sub-trees"
        assert ix.size() == cur.shape[0]
        check_all(ix, oracle, cur, pts, qs, f"step {step}")
    assert merged_seen
    # a full re-sort afterwards still finds every id once
    ix2 = rb.SpatialIndex(rb.Config(node_width=w, traversal=t))
    ix2.Insert(dev(cur))
    for pred, src in ((P.kContains, pts), (P.kContains, qs), (P.kIntersects, qs)):
        assert ix.query_count(pred, dev(src)) == ix2.query_count(pred, dev(src))


def test_update_listing_an_id_twice_keeps_one_envelope(cuda, oracle):
    rng = np.random.default_rng(17)
    boxes = wl.uniform_boxes(rng, 20_000, 5e-3)
    qs = wl.uniform_boxes(rng, 4000, 5e-2)
    ix = rb.SpatialIndex(rb.Config(rebuild_update_fraction=0.9))
    ix.Insert(dev(boxes))
    a = np.array([[0.1, 0.1, 0.3, 0.3]], np.float32)
    b = np.array([[0.6, 0.6, 0.9, 0.9]], np.float32)
    ix.Update(torch.tensor([7, 7], dtype=torch.int64).cuda(), dev(np.concatenate([a, b])))
    got = gpu_pairs(ix, P.kIntersects, qs)
    wants = []
    for v in (a, b):
        cur = boxes.copy()
        cur[7] = v[0]
        wants.append(oracle.run(KIND_INTERSECTS, cur, qs)[2])
    assert any(got.shape == w_.shape and np.array_equal(got, w_) for w_ in wants)
