"""The reference's own unit tests, re-run on the B200 library through its
C-ABI: the same inputs (std::mt19937 fixtures), the same calls, the same
expected counts (test/test_point_queries.h, test/test_envelope_queries.h) —
plus pair-level equality with the oracle, which the reference never checked."""
import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from tests._gpu_util import (ALL_COMBOS, SOME_COMBOS, assert_same_pairs, combo_id, dev,
                             gpu_pairs, make_index)

pytestmark = pytest.mark.gpu

P = rb.Predicate


@pytest.fixture(scope="module")
def kat(oracle):
    b = oracle.uniform_boxes(100000, 0.5, 0.5)
    p = oracle.uniform_points(1000)
    q = oracle.uniform_boxes(1000, 0.1, 0.1)
    return b, p, q


@pytest.fixture(scope="module")
def kat_pairs(oracle, kat):
    b, p, q = kat
    return {
        "point": oracle.run(KIND_POINT, b, p, grid=False)[2],
        "intersects": oracle.run(KIND_INTERSECTS, b, q, grid=False)[2],
        "contains": oracle.run(KIND_CONTAINS, b, q, grid=False)[2],
    }


def insert_batches(ix, boxes, n_batches):
    avg = (boxes.shape[0] + n_batches - 1) // n_batches
    d = dev(boxes)
    for i in range(n_batches):
        ix.Insert(d[i * avg:min((i + 1) * avg, boxes.shape[0])])


@pytest.mark.parametrize("combo", ALL_COMBOS, ids=combo_id)
def test_fp32_contains_point_large(cuda, kat, kat_pairs, combo):
    # test/test_point_queries.h:9-28
    b, p, _ = kat
    ix = make_index(combo)
    ix.Insert(dev(b))
    assert ix.query_count(P.kContains, dev(p)) == 4224111
    assert_same_pairs(gpu_pairs(ix, P.kContains, p), kat_pairs["point"], "point pairs")


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_fp32_contains_point_large_batch(cuda, kat, kat_pairs, combo):
    # test/test_point_queries.h:30-60 (10 insert batches)
    b, p, _ = kat
    ix = make_index(combo)
    insert_batches(ix, b, 10)
    assert ix.size() == 100000
    assert ix.query_count(P.kContains, dev(p)) == 4224111
    assert_same_pairs(gpu_pairs(ix, P.kContains, p), kat_pairs["point"], "point pairs")


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_fp32_contains_point_large_batch_subtrees(cuda, kat, kat_pairs, combo):
    # same, keeping every batch as its own sub-tree (no merge rebuild)
    b, p, _ = kat
    ix = make_index(combo, max_trees=16, rebuild_fraction=1e9)
    insert_batches(ix, b, 10)
    assert ix.num_trees() == 10
    assert ix.query_count(P.kContains, dev(p)) == 4224111
    assert_same_pairs(gpu_pairs(ix, P.kContains, p), kat_pairs["point"], "point pairs")


def _hand_point_case(ix, pinned):
    boxes = torch.tensor([[0, 0, 1, 1], [0.2, 0.2, 0.8, 0.8]], dtype=torch.float32)
    pts = torch.tensor([[0.1, 0.1], [0.5, 0.5], [0.5, 0.6], [1.0, 1.1], [2.0, 2.0]],
                       dtype=torch.float32)
    if pinned:
        boxes, pts = boxes.pin_memory(), pts.pin_memory()
        return boxes, pts
    return boxes.cuda(), pts.cuda()


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_fp32_contains_point(cuda, combo):
    # test/test_point_queries.h:62-90 -> 5
    ix = make_index(combo)
    boxes, pts = _hand_point_case(ix, False)
    ix.Insert(boxes)
    assert ix.query_count(P.kContains, pts) == 5
    got = gpu_pairs(ix, P.kContains, pts.cpu().numpy())
    assert got.tolist() == [[0, 0], [0, 1], [1, 1], [0, 2], [1, 2]]


def test_fp32_contains_point_pinned_host_inputs(cuda):
    # The reference's test passes pinned host vectors; the kernels address them
    # through unified virtual addressing.
    from rtspatial_b200 import _lib as L
    import ctypes
    ix = rb.SpatialIndex(rb.Config())
    boxes, pts = _hand_point_case(ix, True)
    L.check(L.lib().rts_insert(ix._h, boxes.data_ptr(), 2, None))
    c = rb.Counter()
    L.check(L.lib().rts_query_points(ix._h, 1, pts.data_ptr(), 5, 0, c.data(), None))
    torch.cuda.synchronize()
    assert c.get() == 5


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_fp32_intersects_envelope(cuda, combo):
    # test/test_envelope_queries.h:11-36 -> 2
    ix = make_index(combo)
    ix.Insert(dev(np.array([[0, 0, 1, 1], [0.5, -0.5, 1.5, 0.5]], np.float32)))
    q = np.array([[0.75, 0.25, 1.25, 0.75]], np.float32)
    assert ix.query_count(P.kIntersects, dev(q)) == 2


@pytest.mark.parametrize("combo", ALL_COMBOS, ids=combo_id)
def test_fp32_intersects_envelope_big(cuda, kat, kat_pairs, combo):
    # test/test_envelope_queries.h:38-58 -> 6549771
    b, _, q = kat
    ix = make_index(combo)
    ix.Insert(dev(b))
    assert ix.query_count(P.kIntersects, dev(q)) == 6549771
    assert_same_pairs(gpu_pairs(ix, P.kIntersects, q), kat_pairs["intersects"], "intersects")


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_fp32_intersects_envelope_batch(cuda, kat, kat_pairs, combo):
    # test/test_envelope_queries.h:60-91
    b, _, q = kat
    ix = make_index(combo)
    insert_batches(ix, b, 10)
    assert ix.query_count(P.kIntersects, dev(q)) == 6549771
    assert_same_pairs(gpu_pairs(ix, P.kIntersects, q), kat_pairs["intersects"], "intersects")


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_range_contains_kat_data(cuda, kat, kat_pairs, combo):
    b, _, q = kat
    ix = make_index(combo)
    ix.Insert(dev(b))
    assert_same_pairs(gpu_pairs(ix, P.kContains, q), kat_pairs["contains"], "contains")


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
@pytest.mark.parametrize("refit", [True, False], ids=["refit", "rebuild"])
def test_fp32_intersects_envelope_batch_update(cuda, oracle, kat, combo, refit):
    # test/test_envelope_queries.h:93-164: 5% of ids updated; the answer is a
    # fresh index over the updated boxes (and here also the oracle's pairs).
    b, _, q = kat
    n1, n_upd = 100000, 5000
    ix = make_index(combo, rebuild_update_fraction=1.0 if refit else 0.0)
    insert_batches(ix, b, 10)
    ids = oracle.update_ids(n1, n_upd)
    new_boxes = oracle.uniform_boxes(n_upd, 0.5, 0.5)
    tmp = b.copy()
    tmp[ids.astype(np.int64)] = new_boxes
    fresh = make_index(combo)
    fresh.Insert(dev(tmp))
    answer = fresh.query_count(P.kIntersects, dev(q))
    ix.Update(dev(ids.astype(np.int64)), dev(new_boxes))
    assert ix.query_count(P.kIntersects, dev(q)) == answer
    want = oracle.run(KIND_INTERSECTS, tmp, q, grid=False)[2]
    assert want.shape[0] == answer
    assert_same_pairs(gpu_pairs(ix, P.kIntersects, q), want, "after update")


@pytest.mark.parametrize("compact", [False, True], ids=["plain", "compact"])
@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
def test_fp32_test_delete(cuda, combo, compact):
    # test/test_envelope_queries.h:166-245: 2 -> 1 after deleting id 1
    ix = make_index(combo, compact=compact)
    ix.Insert(dev(np.array([[0, 0, 1, 1], [0.5, -0.5, 1.5, 0.5]], np.float32)))
    q = dev(np.array([[0.75, 0.25, 1.25, 0.75]], np.float32))
    assert ix.query_count(P.kIntersects, q) == 2
    ix.Delete(torch.tensor([1], dtype=torch.int64, device="cuda"))
    assert ix.query_count(P.kIntersects, q) == 1
