"""Double indexes (SpatialIndex<double, 2>, coord_bits = 64) against the
double oracle: point- and range-contains compare float-rounded coordinates,
range-intersects runs the ray-slab test in double.  Covers every traversal
scheme, several sub-trees, Delete and Update, batched / merged / planned
launches and serving."""
import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from tests._gpu_util import assert_same_pairs, canon

pytestmark = pytest.mark.gpu
P = rb.Predicate
L = rb._lib
KINDS = {"point": (KIND_POINT, P.kContains), "contains": (KIND_CONTAINS, P.kContains),
         "intersects": (KIND_INTERSECTS, P.kIntersects)}


def ddev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def rounding_sensitive(rng, a, frac=0.3):
    """Moves a fraction of coordinates halfway between two floats (give or
    take one double ulp), where rounding to float decides contains."""
    a = a.copy()
    sel = rng.random(a.shape) < frac
    f = a.astype(np.float32)
    up = np.nextafter(f, np.float32(np.inf)).astype(np.float64)
    mid = (f.astype(np.float64) + up) / 2
    j = rng.integers(-1, 2, a.shape)
    mid = np.where(j < 0, np.nextafter(mid, -np.inf), np.where(j > 0, np.nextafter(mid, np.inf), mid))
    return np.where(sel, mid, a)


@pytest.fixture(scope="module")
def scene():
    rng = np.random.default_rng(64)
    n, nq = 30000, 3000
    c = rng.random((n, 2))
    s = rng.random((n, 2)) * 0.02
    boxes = np.concatenate([c - s / 2, c + s / 2], axis=1)
    boxes[:200, 2:] = boxes[:200, :2]          # degenerate (point) boxes
    boxes[200:300, 2] = boxes[200:300, 0]      # zero width
    boxes = rounding_sensitive(rng, boxes)
    # boxes that differ from a neighbour by one double ulp
    boxes[300:600] = np.nextafter(boxes[600:900], np.inf)
    pts = rounding_sensitive(rng, rng.random((nq, 2)))
    pts[:300] = boxes[1000:1300, :2]           # on corners
    qc = rng.random((nq, 2))
    qs_ = rng.random((nq, 2)) * 0.03
    qs = rounding_sensitive(rng, np.concatenate([qc - qs_ / 2, qc + qs_ / 2], axis=1))
    qs[:300] = boxes[2000:2300]                # identical to stored boxes
    return boxes, pts, qs


SCHEMES = [(16, L.RTS_TRAVERSAL_THREAD), (8, L.RTS_TRAVERSAL_THREAD), (32, L.RTS_TRAVERSAL_PACKET),
           (16, L.RTS_TRAVERSAL_PACKET), (4, L.RTS_TRAVERSAL_AUTO), (16, L.RTS_TRAVERSAL_TEAM),
           (8, L.RTS_TRAVERSAL_FRONTIER), (16, L.RTS_TRAVERSAL_STAGED), (4, L.RTS_TRAVERSAL_STAGED)]


def make(w, t, **kw):
    return rb.SpatialIndex(rb.Config(node_width=w, traversal=t, coord_bits=64, **kw))


@pytest.mark.parametrize("w,t", SCHEMES, ids=[f"w{w}-t{t}" for w, t in SCHEMES])
def test_double_queries_match_oracle(cuda, oracle, scene, w, t):
    boxes, pts, qs = scene
    ix = make(w, t, max_trees=4, rebuild_fraction=1e9)
    for part in np.array_split(boxes, 3):   # three sub-trees
        ix.Insert(ddev(part))
    assert ix.num_trees() == 3
    for kind, src in (("point", pts), ("contains", qs), ("intersects", qs)):
        want = oracle.run64(KINDS[kind][0], boxes, src)[2]
        got = canon(ix.query_pairs(KINDS[kind][1], ddev(src)))
        assert_same_pairs(got, want, kind)
        assert ix.query_count(KINDS[kind][1], ddev(src)) == want.shape[0]


@pytest.mark.parametrize("t", [L.RTS_TRAVERSAL_THREAD, L.RTS_TRAVERSAL_PACKET,
                               L.RTS_TRAVERSAL_STAGED])
def test_double_delete_and_update(cuda, oracle, scene, t):
    boxes, pts, qs = scene
    rng = np.random.default_rng(65)
    ix = make(16, t, rebuild_update_fraction=0.5)
    ix.Insert(ddev(boxes))
    cur = boxes.copy()
    dels = rng.choice(boxes.shape[0], 2000, replace=False)
    ix.Delete(torch.from_numpy(dels.astype(np.int64)).cuda())
    oracle.invalidate64(cur, dels)
    ups = rng.choice(boxes.shape[0], 3000, replace=False)
    nb = cur[ups] + rng.uniform(-1e-3, 1e-3, (ups.shape[0], 1))
    nb = rounding_sensitive(rng, nb)
    ix.Update(torch.from_numpy(ups.astype(np.int64)).cuda(), ddev(nb))   # refit
    cur[ups] = nb
    for kind, src in (("point", pts), ("contains", qs), ("intersects", qs)):
        assert_same_pairs(canon(ix.query_pairs(KINDS[kind][1], ddev(src))),
                          oracle.run64(KINDS[kind][0], cur, src)[2], f"after refit {kind}")
    ups2 = rng.choice(boxes.shape[0], 20000, replace=False)             # re-sort
    nb2 = cur[ups2][:, [0, 1, 0, 1]] + np.abs(rng.normal(0, 5e-3, (ups2.shape[0], 4))) * [0, 0, 1, 1]
    ix.Update(torch.from_numpy(ups2.astype(np.int64)).cuda(), ddev(nb2))
    cur[ups2] = nb2
    ix.Insert(ddev(boxes[:500]))                                          # new ids after
    cur = np.concatenate([cur, boxes[:500]])
    for kind, src in (("point", pts), ("contains", qs), ("intersects", qs)):
        assert_same_pairs(canon(ix.query_pairs(KINDS[kind][1], ddev(src))),
                          oracle.run64(KINDS[kind][0], cur, src)[2], f"after re-sort {kind}")


@pytest.mark.parametrize("t", [L.RTS_TRAVERSAL_THREAD, L.RTS_TRAVERSAL_PACKET,
                               L.RTS_TRAVERSAL_STAGED])
def test_double_batched_merged_and_planned(cuda, oracle, scene, t):
    boxes, pts, qs = scene
    ix = make(16, t, sort_queries=1)
    ix.Insert(ddev(boxes))
    parts = np.array_split(qs, 7)
    wants = [oracle.run64(KIND_INTERSECTS, boxes, a)[2] for a in parts]
    queues = [rb.Queue(w.shape[0] + 16) for w in wants]
    ix.query_batched([(P.kIntersects, ddev(a), rb.Handler.COLLECT, qu.DeviceObject())
                      for a, qu in zip(parts, queues)])
    counters = [rb.Counter() for _ in parts]
    ix.query_batched([(P.kIntersects, ddev(a), rb.Handler.COUNT, c.data())
                      for a, c in zip(parts, counters)])
    torch.cuda.synchronize()
    for qu, c, w in zip(queues, counters, wants):
        assert_same_pairs(canon(qu.result()), w, "batched")
        assert c.get() == w.shape[0]
    # mixed predicates in one prepared, graph-replayed launch
    pparts = np.array_split(pts, 2)
    specs = [(P.kContains, pparts[0], KIND_POINT), (P.kContains, parts[0], KIND_CONTAINS),
             (P.kIntersects, parts[1], KIND_INTERSECTS), (P.kContains, pparts[1], KIND_POINT)]
    tensors = [ddev(a) for _, a, _ in specs]
    queues = [rb.Queue(200_000) for _ in specs]
    plan = ix.plan([(pr, q, rb.Handler.COLLECT, qu.DeviceObject())
                    for (pr, _, _), q, qu in zip(specs, tensors, queues)])
    for _ in range(2):
        for qu in queues:
            qu.Clear()
        plan.launch(graph=True)
        torch.cuda.synchronize()
        for (_, a, kind), qu in zip(specs, queues):
            assert_same_pairs(canon(qu.result()), oracle.run64(kind, boxes, a)[2], "plan")
    plan.close()


def test_double_server(cuda, oracle, scene):
    boxes, pts, qs = scene
    ix = make(16, L.RTS_TRAVERSAL_AUTO)
    ix.Insert(ddev(boxes))
    sv = rb.Server(ix)
    t1 = sv.submit(P.kIntersects, qs[:1000])
    t2 = sv.submit(P.kContains, pts[:1000])
    t3 = sv.submit_update(delete_ids=np.arange(0, 30000, 3))
    t4 = sv.submit(P.kIntersects, qs[:1000])
    for t in (t1, t2, t3, t4):
        sv.wait(t)
    cut = boxes.copy()
    oracle.invalidate64(cut, np.arange(0, 30000, 3))
    assert_same_pairs(canon(sv.take(t1)), oracle.run64(KIND_INTERSECTS, boxes, qs[:1000])[2], "t1")
    assert_same_pairs(canon(sv.take(t2)), oracle.run64(KIND_POINT, boxes, pts[:1000])[2], "t2")
    assert_same_pairs(canon(sv.take(t4)), oracle.run64(KIND_INTERSECTS, cut, qs[:1000])[2], "t4")
    sv.close()


@pytest.mark.parametrize("t", [L.RTS_TRAVERSAL_THREAD, L.RTS_TRAVERSAL_PACKET,
                               L.RTS_TRAVERSAL_STAGED])
def test_double_emptied_slots_match_no_query(cuda, oracle, scene, t):
    # Slots emptied by updates that move envelopes to a new sub-tree answer
    # nothing, including queries with infinite coordinates.
    boxes, pts, qs = scene
    rng = np.random.default_rng(66)
    ix = make(16, t, max_trees=8, rebuild_update_fraction=0.9)
    ix.Insert(ddev(boxes))
    far = rng.choice(boxes.shape[0], 1000, replace=False)
    c = rng.random((far.shape[0], 2))
    nb = np.concatenate([c, c + 0.01], axis=1)
    ix.Update(torch.from_numpy(far.astype(np.int64)).cuda(), ddev(nb))
    assert ix.num_trees() == 2
    cur = boxes.copy()
    cur[far] = nb
    inf = np.inf
    xq = np.concatenate([[[inf, inf, -inf, -inf], [-inf, -inf, inf, inf], [inf, inf, inf, inf],
                          [inf, -inf, -inf, inf]], qs[:500]])
    xp = np.concatenate([[[inf, inf], [-inf, -inf]], pts[:500]])
    for kind, src in (("point", xp), ("contains", xq), ("intersects", xq)):
        want = oracle.run64(KINDS[kind][0], cur, src)[2]
        assert_same_pairs(canon(ix.query_pairs(KINDS[kind][1], ddev(src))), want, kind)
        assert ix.query_count(KINDS[kind][1], ddev(src)) == want.shape[0]


def test_double_small_subtrees_merge(cuda, oracle, scene):
    # Sub-tree merges carry the double envelopes with their slots.
    boxes, pts, qs = scene
    rng = np.random.default_rng(67)
    ix = make(16, L.RTS_TRAVERSAL_THREAD, max_trees=3, rebuild_fraction=0.5,
              rebuild_update_fraction=0.9)
    ix.Insert(ddev(boxes))
    cur = boxes.copy()
    for step in range(6):
        if step % 2:
            ids = rng.choice(cur.shape[0], 200, replace=False)
            c = rng.random((ids.shape[0], 2))
            nb = np.concatenate([c, c + 0.01], axis=1)
            ix.Update(torch.from_numpy(ids.astype(np.int64)).cuda(), ddev(nb))
            cur[ids] = nb
        else:
            new = boxes[rng.choice(boxes.shape[0], 500, replace=False)] + 1e-9
            ix.Insert(ddev(new))
            cur = np.concatenate([cur, new])
        assert 2 <= ix.num_trees() <= 3
    for kind, src in (("point", pts), ("contains", qs), ("intersects", qs)):
        assert_same_pairs(canon(ix.query_pairs(KINDS[kind][1], ddev(src))),
                          oracle.run64(KINDS[kind][0], cur, src)[2], kind)


def test_double_and_float_calls_do_not_mix(cuda):
    ix = make(16, L.RTS_TRAVERSAL_AUTO)
    with pytest.raises(Exception):
        ix.Insert(torch.zeros((4, 4), dtype=torch.float32, device="cuda"))
    ix.Insert(torch.rand((64, 4), dtype=torch.float64, device="cuda"))
    with pytest.raises(Exception):
        ix.query_count(P.kContains, torch.zeros((4, 2), dtype=torch.float32, device="cuda"))
    fx = rb.SpatialIndex(rb.Config())
    with pytest.raises(Exception):
        fx.Insert(torch.zeros((4, 4), dtype=torch.float64, device="cuda"))
