"""Pair-level parity of the CUDA library with the oracle: golden edge cases
(reference-computed), seeded random workloads of each configuration's shape at
oracle-friendly sizes, empty inputs, queue overflow, batched = plain."""
import os

import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from rtspatial_b200 import workloads as wl
from tests._gpu_util import (ALL_COMBOS, SOME_COMBOS, assert_same_pairs, canon, combo_id, dev,
                             gpu_pairs, make_index)

pytestmark = pytest.mark.gpu
P = rb.Predicate
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KINDS = {"point": (KIND_POINT, P.kContains), "contains": (KIND_CONTAINS, P.kContains),
         "intersects": (KIND_INTERSECTS, P.kIntersects)}


@pytest.fixture(scope="module")
def edge():
    return np.load(os.path.join(GOLDEN, "edge_cases.npz"))


@pytest.mark.parametrize("combo", ALL_COMBOS, ids=combo_id)
@pytest.mark.parametrize("kind", ["point", "contains", "intersects"])
def test_golden_edge_cases(cuda, edge, combo, kind):
    ix = make_index(combo)
    ix.Insert(dev(edge["boxes"]))
    qs = edge["points"] if kind == "point" else edge["queries"]
    assert_same_pairs(gpu_pairs(ix, KINDS[kind][1], qs), edge[kind], kind)


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
@pytest.mark.parametrize("kind", ["point", "contains", "intersects"])
def test_golden_edge_cases_subtrees(cuda, edge, combo, kind):
    # the same boxes spread over several sub-trees
    ix = make_index(combo, max_trees=16, rebuild_fraction=1e9)
    b = edge["boxes"]
    for part in np.array_split(np.arange(b.shape[0]), 5):
        ix.Insert(dev(b[part]))
    assert ix.num_trees() == 5
    qs = edge["points"] if kind == "point" else edge["queries"]
    assert_same_pairs(gpu_pairs(ix, KINDS[kind][1], qs), edge[kind], kind)


def _workload(name, rng):
    if name == "uniform":
        return wl.uniform_boxes(rng, 200_000, 1e-2), wl.uniform_points(rng, 20_000), \
            wl.uniform_boxes(rng, 20_000, 2e-2)
    if name == "clustered":
        return wl.clustered_boxes(rng, 200_000, 5e-3), wl.uniform_points(rng, 20_000), \
            wl.uniform_boxes(rng, 20_000, 1e-3)
    if name == "lognormal":
        return wl.lognormal_boxes(rng, 200_000, np.log(1e-3), 1.5), wl.uniform_points(rng, 20_000), \
            wl.lognormal_boxes(rng, 20_000, np.log(5e-3), 1.0)
    raise ValueError(name)


@pytest.fixture(scope="module")
def workloads(oracle):
    out = {}
    for i, name in enumerate(["uniform", "clustered", "lognormal"]):
        rng = np.random.default_rng(100 + i)
        b, p, q = _workload(name, rng)
        out[name] = (b, p, q, {
            "point": oracle.run(KIND_POINT, b, p)[2],
            "contains": oracle.run(KIND_CONTAINS, b, q)[2],
            "intersects": oracle.run(KIND_INTERSECTS, b, q)[2],
        })
    return out


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
@pytest.mark.parametrize("name", ["uniform", "clustered", "lognormal"])
@pytest.mark.parametrize("order", [0, 1], ids=["as-given", "curve-sorted"])
def test_random_parity(cuda, workloads, combo, name, order):
    b, p, q, want = workloads[name]
    ix = make_index(combo, sort_queries=order)
    ix.Insert(dev(b))
    assert_same_pairs(gpu_pairs(ix, P.kContains, p), want["point"], f"{name} point")
    assert_same_pairs(gpu_pairs(ix, P.kContains, q), want["contains"], f"{name} contains")
    assert_same_pairs(gpu_pairs(ix, P.kIntersects, q), want["intersects"], f"{name} intersects")
    # counting handler agrees with the collecting one
    assert ix.query_count(P.kIntersects, dev(q)) == want["intersects"].shape[0]


def test_large_magnitude_and_negative_coordinates(cuda, oracle):
    rng = np.random.default_rng(5)
    b = wl.uniform_boxes(rng, 50_000, 1e-2) * np.float32(1000) - np.float32(3.0e5)
    q = wl.uniform_boxes(rng, 5_000, 2e-2) * np.float32(1000) - np.float32(3.0e5)
    for combo in SOME_COMBOS[:4]:
        ix = make_index(combo)
        ix.Insert(dev(b))
        for k in ("contains", "intersects"):
            kind, pred = KINDS[k]
            assert_same_pairs(gpu_pairs(ix, pred, q), oracle.run(kind, b, q)[2], k)


def test_empty_inputs(cuda):
    ix = rb.SpatialIndex(rb.Config())
    c = rb.Counter()
    q = dev(np.zeros((10, 4), np.float32))
    ix.Query(P.kIntersects, q, c.data(), handler=rb.Handler.COUNT)  # empty index
    ix.Insert(dev(np.array([[0, 0, 1, 1]], np.float32)))
    ix.Query(P.kIntersects, q[:0], c.data(), handler=rb.Handler.COUNT)  # no queries
    torch.cuda.synchronize()
    assert c.get() == 0
    assert ix.query_count(P.kIntersects, q) == 10


def test_queue_overflow_reports_needed_size(cuda, oracle):
    rng = np.random.default_rng(9)
    b = wl.uniform_boxes(rng, 20_000, 5e-2)
    p = wl.uniform_points(rng, 2_000)
    want = oracle.run(KIND_POINT, b, p)[2]
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(b))
    cap = want.shape[0] // 3
    qu = rb.Queue(cap + 64)  # 64 guard entries beyond the advertised capacity
    qu.pairs.fill_(-7)
    host = torch.tensor([qu.pairs.data_ptr(), cap, qu.counter.data_ptr()], dtype=torch.int64)
    qu.obj.copy_(host)
    ix.Query(P.kContains, dev(p), qu.DeviceObject(), handler=rb.Handler.COLLECT)
    torch.cuda.synchronize()
    assert qu.size() == want.shape[0]
    assert bool((qu.pairs[cap:] == -7).all())
    kept = canon(qu.pairs[:cap].to(torch.int64) & 0xFFFFFFFF)
    assert set(map(tuple, kept.tolist())) <= set(map(tuple, want.tolist()))


@pytest.mark.parametrize("combo", SOME_COMBOS, ids=combo_id)
@pytest.mark.parametrize("order", [0, 1], ids=["as-given", "curve-sorted"])
@pytest.mark.parametrize("occ", [0, 3, 4], ids=["occ-default", "occ-3", "occ-4"])
def test_batched_equals_plain(cuda, workloads, combo, order, occ):
    b, p, q, want = workloads["clustered"]
    ix = make_index(combo, sort_queries=order, query_occupancy=occ)
    ix.Insert(dev(b))
    rng = np.random.default_rng(1)
    specs = []
    for i in range(12):
        kind = ["point", "contains", "intersects"][i % 3]
        src = p if kind == "point" else q
        lo = int(rng.integers(0, src.shape[0] - 10))
        n = int(rng.integers(1, min(3000, src.shape[0] - lo)))
        specs.append((kind, src[lo:lo + n]))
    queues = [rb.Queue(max(64, 8 * s[1].shape[0])) for s in specs]
    ix.query_batched([(KINDS[k][1], dev(a), rb.Handler.COLLECT, qu.DeviceObject())
                      for (k, a), qu in zip(specs, queues)])
    torch.cuda.synchronize()
    for (k, a), qu in zip(specs, queues):
        assert qu.size() <= qu.capacity()
        alone = gpu_pairs(ix, KINDS[k][1], a)
        assert_same_pairs(canon(qu.result()), alone, f"batched {k}")
        assert_same_pairs(alone, oracle_pairs(k, b, a), f"plain {k}")


def oracle_pairs(kind, b, a):
    from oracle.oracle import Oracle
    return Oracle("port").run(KINDS[kind][0], b, a)[2]


def test_batched_count_handlers(cuda, workloads):
    b, p, q, want = workloads["uniform"]
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(b))
    cs = [rb.Counter() for _ in range(3)]
    ix.query_batched([(P.kContains, dev(p), rb.Handler.COUNT, cs[0].data()),
                      (P.kContains, dev(q), rb.Handler.COUNT, cs[1].data()),
                      (P.kIntersects, dev(q), rb.Handler.COUNT, cs[2].data())])
    torch.cuda.synchronize()
    assert [c.get() for c in cs] == [want["point"].shape[0], want["contains"].shape[0],
                                     want["intersects"].shape[0]]


@pytest.mark.parametrize("w", [4, 8, 16, 32])
@pytest.mark.parametrize("factor", [0.05, 0.5, 2.0, 64.0],
                         ids=["spill-most", "spill-many", "spill-some", "fits"])
def test_frontier_spill_falls_back_exactly(cuda, workloads, w, factor):
    # A frontier too small for the launch flags the overflowing queries; the
    # depth-first pass answers exactly those, so no pair is lost or doubled.
    b, p, q, want = workloads["clustered"]
    ix = rb.SpatialIndex(rb.Config(node_width=w, traversal=rb._lib.RTS_TRAVERSAL_FRONTIER,
                                   frontier_factor=factor, max_trees=4, rebuild_fraction=1e9))
    for part in np.array_split(b, 3):
        ix.Insert(dev(part))
    assert ix.num_trees() == 3
    assert_same_pairs(gpu_pairs(ix, P.kContains, p), want["point"], "point")
    assert_same_pairs(gpu_pairs(ix, P.kContains, q), want["contains"], "contains")
    assert_same_pairs(gpu_pairs(ix, P.kIntersects, q), want["intersects"], "intersects")
    # batched, several batches of one predicate
    queues = [rb.Queue(400_000) for _ in range(4)]
    parts = np.array_split(q, 4)
    ix.query_batched([(P.kIntersects, dev(a), rb.Handler.COLLECT, qu.DeviceObject())
                      for a, qu in zip(parts, queues)])
    torch.cuda.synchronize()
    for a, qu in zip(parts, queues):
        assert_same_pairs(canon(qu.result()), oracle_pairs("intersects", b, a), "batched")
