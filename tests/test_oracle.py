"""CPU checks of the oracle: the reference's known answers, agreement of the
restated predicates with the reference's own predicate code, and soundness of
the oracle's grid filter."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def kat():
    with open(os.path.join(GOLDEN, "kat.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def kat_data(oracle):
    return (oracle.uniform_boxes(100000, 0.5, 0.5), oracle.uniform_points(1000),
            oracle.uniform_boxes(1000, 0.1, 0.1))


def test_slab_constant_bits(oracle):
    # 1 + 2*FLT_GAMMA(3) in float = 1 + 6*2^-23 (details/ray_params.h:40,158)
    assert np.float32(oracle.slab_k()).view(np.uint32) == 0x3F800006


def test_fixture_generators_match_reference_streams(oracle, kat, kat_data):
    b, p, q = kat_data
    assert sha(b) == kat["boxes_100000_0.5"]
    assert sha(p) == kat["points_1000"]
    assert sha(q) == kat["boxes_1000_0.1"]
    assert sha(oracle.update_ids(100000, 5000)) == kat["update_ids_100000_5000"]
    assert sha(oracle.uniform_boxes(5000, 0.5, 0.5)) == kat["update_boxes_5000_0.5"]


def test_kat_point_contains(oracle, kat_data):
    # PointQueries.fp32_contains_point_large (test/test_point_queries.h:9-28)
    b, p, _ = kat_data
    assert oracle.run(KIND_POINT, b, p, collect=False, grid=False)[0] == 4224111


def test_kat_intersects(oracle, kat_data):
    # EnvelopeQueries.fp32_intersects_envelope_big (test/test_envelope_queries.h:38-58)
    b, _, q = kat_data
    assert oracle.run(KIND_INTERSECTS, b, q, collect=False, grid=False)[0] == 6549771


def test_kat_range_contains_golden(oracle, kat, kat_data):
    b, _, q = kat_data
    assert oracle.run(KIND_CONTAINS, b, q, collect=False, grid=False)[0] == kat[
        "range_contains_100000x1000"]


def test_small_hand_kats(oracle):
    # PointQueries.fp32_contains_point (test/test_point_queries.h:62-90)
    boxes = np.array([[0, 0, 1, 1], [0.2, 0.2, 0.8, 0.8]], np.float32)
    pts = np.array([[0.1, 0.1], [0.5, 0.5], [0.5, 0.6], [1.0, 1.1], [2.0, 2.0]], np.float32)
    assert oracle.run(KIND_POINT, boxes, pts, collect=False, grid=False)[0] == 5
    # EnvelopeQueries.fp32_intersects_envelope (test/test_envelope_queries.h:11-36)
    boxes = np.array([[0, 0, 1, 1], [0.5, -0.5, 1.5, 0.5]], np.float32)
    q = np.array([[0.75, 0.25, 1.25, 0.75]], np.float32)
    assert oracle.run(KIND_INTERSECTS, boxes, q, collect=False, grid=False)[0] == 2
    # EnvelopeQueries.fp32_test_delete: delete id 1 -> 1 (:166-204)
    oracle.invalidate(boxes, [1])
    assert oracle.run(KIND_INTERSECTS, boxes, q, collect=False, grid=False)[0] == 1


def test_plain_box_intersects_differs_by_one_pair(oracle, kat_data):
    # The ray-slab formulation (not Envelope::Intersects) is the contract: the
    # closed box test misses geom 76881 x query 362 (query min.y is 1 ulp
    # above the geom's max.y, inside the slab tolerance).
    b, _, q = kat_data
    g, qq = b[76881], q[362]
    assert not (qq[1] <= g[3])
    got = oracle.eval_pairs(KIND_INTERSECTS, g[None], qq[None])
    assert got[0] == 1


def _adversarial_pairs(rng, n):
    a = rng.random((n, 4)).astype(np.float32)
    b = a.copy()
    # move b's coordinates by a few ulps / swap roles, zero extents, inversions
    for c in range(4):
        k = rng.integers(-3, 4, n)
        b[:, c] = np.nextafter(b[:, c], np.where(k > 0, np.inf, -np.inf).astype(np.float32))
    sel = rng.random(n) < 0.2
    b[sel, 2] = b[sel, 0]
    sel = rng.random(n) < 0.2
    b[sel, 3] = b[sel, 1]
    sel = rng.random(n) < 0.1
    b[sel] = b[sel][:, [2, 1, 0, 3]]
    scale = np.where(rng.random(n) < 0.2, np.float32(1e5), np.float32(1)).astype(np.float32)
    return (a * scale[:, None]).astype(np.float32), (b * scale[:, None]).astype(np.float32)


def test_port_matches_reference_predicates(oracle, ref_oracle):
    rng = np.random.default_rng(3)
    g, q = _adversarial_pairs(rng, 200000)
    for kind in (KIND_CONTAINS, KIND_INTERSECTS):
        assert np.array_equal(oracle.eval_pairs(kind, g, q), ref_oracle.eval_pairs(kind, g, q))
        assert np.array_equal(oracle.eval_pairs(kind, q, g), ref_oracle.eval_pairs(kind, q, g))
    pts = np.concatenate([q[:, :2], q[:, 2:]]).astype(np.float32)
    gg = np.concatenate([g, g])
    assert np.array_equal(oracle.eval_pairs(KIND_POINT, gg, pts),
                          ref_oracle.eval_pairs(KIND_POINT, gg, pts))


def test_port_matches_golden_edge_cases(oracle):
    z = np.load(os.path.join(GOLDEN, "edge_cases.npz"))
    for name, kind, qs in (("point", KIND_POINT, z["points"]), ("contains", KIND_CONTAINS, z["queries"]),
                           ("intersects", KIND_INTERSECTS, z["queries"])):
        _, _, pairs = oracle.run(kind, z["boxes"], qs, collect=True, grid=False)
        assert np.array_equal(pairs, z[name]), name


@pytest.mark.parametrize("kind", [KIND_POINT, KIND_CONTAINS, KIND_INTERSECTS])
def test_grid_filter_is_sound(oracle, kind):
    rng = np.random.default_rng(11 + kind)
    from rtspatial_b200 import workloads as wl
    boxes = np.concatenate([wl.uniform_boxes(rng, 20000, 0.01),
                            wl.lognormal_boxes(rng, 20000, np.log(1e-3), 1.5, 0.2)])
    if kind == KIND_POINT:
        qs = wl.uniform_points(rng, 3000)
    else:
        qs = np.concatenate([wl.uniform_boxes(rng, 1500, 0.02), boxes[:1500]])
    t0, c0, p0 = oracle.run(kind, boxes, qs, grid=False)
    t1, c1, p1 = oracle.run(kind, boxes, qs, grid=True)
    assert t0 == t1 and np.array_equal(c0, c1) and np.array_equal(p0, p1)


# ---- double indexes (SpatialIndex<double, 2>) --------------------------------
def _adversarial_pairs64(rng, n):
    """Double pairs around the places the double predicates are decided:
    coordinates a few double ulps apart, halfway between two floats (the
    contains predicates compare float-rounded values), zero extents,
    inversions, deleted boxes (max = min) and large magnitudes."""
    a = rng.random((n, 4))
    a[:, 2:] = a[:, :2] + rng.random((n, 2)) * 0.1
    b = a.copy()
    for c in range(4):
        k = rng.integers(-3, 4, n)
        step = np.where(k > 0, np.inf, -np.inf)
        for _ in range(3):
            sel = rng.random(n) < 0.5
            b[sel, c] = np.nextafter(b[sel, c], step[sel])
    # halfway between neighbouring floats: rounding to float decides contains
    for arr in (a, b):
        sel = rng.random(n) < 0.3
        f = arr[sel].astype(np.float32)
        up = np.nextafter(f, np.float32(np.inf))
        mid = (f.astype(np.float64) + up.astype(np.float64)) / 2
        jitter = rng.integers(-1, 2, mid.shape)
        arr[sel] = np.where(jitter < 0, np.nextafter(mid, -np.inf),
                            np.where(jitter > 0, np.nextafter(mid, np.inf), mid))
    sel = rng.random(n) < 0.15
    b[sel, 2] = b[sel, 0]
    sel = rng.random(n) < 0.15
    b[sel, 3] = b[sel, 1]
    sel = rng.random(n) < 0.1
    b[sel] = b[sel][:, [2, 1, 0, 3]]
    sel = rng.random(n) < 0.1
    a[sel, 2:] = a[sel, :2]     # deleted geometry
    scale = np.where(rng.random(n) < 0.2, 1e5, 1.0)
    return a * scale[:, None], b * scale[:, None]


def test_double_slab_constant(oracle):
    assert oracle.slab_k64() == 1.0 + 6.0 * 2.0 ** -52


def test_double_port_matches_reference_predicates(oracle, ref_oracle):
    rng = np.random.default_rng(21)
    g, q = _adversarial_pairs64(rng, 200000)
    for kind in (KIND_CONTAINS, KIND_INTERSECTS):
        assert np.array_equal(oracle.eval_pairs64(kind, g, q), ref_oracle.eval_pairs64(kind, g, q))
        assert np.array_equal(oracle.eval_pairs64(kind, q, g), ref_oracle.eval_pairs64(kind, q, g))
    pts = np.concatenate([q[:, :2], q[:, 2:]])
    gg = np.concatenate([g, g])
    assert np.array_equal(oracle.eval_pairs64(KIND_POINT, gg, pts),
                          ref_oracle.eval_pairs64(KIND_POINT, gg, pts))


def test_double_contains_compares_float_rounded_coordinates(oracle):
    # A point between a box's double max and the next float above it is
    # contained: both round to the same float (geom/point.cuh:68-71).
    f = np.float32(0.5)
    up = float(np.nextafter(f, np.float32(1)))
    box = np.array([[0.25, 0.25, float(f) + 1e-12, 0.75]])
    inside_as_float = np.array([[float(f) + (up - float(f)) * 0.25, 0.5]])
    assert oracle.eval_pairs64(KIND_POINT, box, inside_as_float)[0] == 1
    outside = np.array([[up, 0.5]])
    assert oracle.eval_pairs64(KIND_POINT, box, outside)[0] == 0
    # ... while validity (used by intersects) compares the doubles
    thin = np.array([[0.5, 0.5, 0.5 + 1e-12, 0.6]])   # float-rounded: zero width
    q = np.array([[0.4, 0.55, 0.6, 0.56]])
    assert oracle.eval_pairs64(KIND_INTERSECTS, thin, q)[0] == 1


def test_double_bulk_matches_pairwise(oracle, ref_oracle):
    rng = np.random.default_rng(22)
    g, q = _adversarial_pairs64(rng, 3000)
    for kind, qs in ((KIND_POINT, q[:400, :2]), (KIND_CONTAINS, q[:400]), (KIND_INTERSECTS, q[:400])):
        total, counts, pairs = oracle.run64(kind, g, qs)
        want = []
        for j in range(qs.shape[0]):
            hits = np.nonzero(oracle.eval_pairs64(kind, g, np.repeat(qs[j:j + 1], g.shape[0], 0)))[0]
            want.extend((int(h), j) for h in hits)
        assert total == len(want)
        assert pairs.tolist() == [list(p) for p in want]
        assert ref_oracle.run64(kind, g, qs)[0] == total
