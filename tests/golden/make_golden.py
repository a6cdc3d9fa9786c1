"""Generates the committed golden fixtures of the parity tests.

Run where the reference-header oracle exists (``oracle/_ref``, built from the
reference's own predicate headers):

    python tests/golden/make_golden.py

Outputs (this folder):
  kat.json        sha256 of the known-answer-test inputs (the reference tests'
                  std::mt19937 generators) and the expected counts: the
                  reference's own KATs (test/test_point_queries.h:26,
                  test/test_envelope_queries.h:56) plus range-contains on the
                  same data computed by the reference-header oracle.
  edge_cases.npz  adversarial boxes, points and query boxes (shared edges,
                  ulp-adjacent edges, zero-extent and collapsed boxes, inverted
                  boxes, large and negative coordinates, subnormal extents)
                  with the pairs the reference's predicate code reports.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT, Oracle  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def nudge(x: np.ndarray, ulps: np.ndarray) -> np.ndarray:
    """Moves float32 values by an integer number of ulps."""
    x = x.astype(np.float32).copy()
    for i in range(x.shape[0]):
        k = int(ulps[i])
        d = np.float32(np.inf) if k > 0 else np.float32(-np.inf)
        for _ in range(abs(k)):
            x[i] = np.nextafter(x[i], d)
    return x


def edge_case_sets(seed: int = 7):
    rng = np.random.default_rng(seed)
    boxes = []
    # 1. an 8x8 grid of cells sharing edges exactly
    g = np.arange(8, dtype=np.float32) / 8
    gx, gy = np.meshgrid(g, g)
    cells = np.stack([gx.ravel(), gy.ravel(), gx.ravel() + 0.125, gy.ravel() + 0.125], 1)
    boxes.append(cells.astype(np.float32))
    # 2. random small boxes, then copies with edges moved by -3..3 ulps
    base = rng.random((150, 2)).astype(np.float32)
    side = (rng.random((150, 2)) * 0.05).astype(np.float32)
    b = np.concatenate([base, base + side], 1).astype(np.float32)
    boxes.append(b)
    nb = b.copy()
    for c in range(4):
        nb[:, c] = nudge(nb[:, c], rng.integers(-3, 4, nb.shape[0]))
    boxes.append(nb)
    # 3. zero-width, zero-height and collapsed (deleted) boxes
    z = b[:60].copy()
    z[:20, 2] = z[:20, 0]
    z[20:40, 3] = z[20:40, 1]
    z[40:, 2] = z[40:, 0]
    z[40:, 3] = z[40:, 1]
    boxes.append(z)
    # 4. inverted boxes (min > max on one or both axes)
    inv = b[60:90].copy()
    inv[:15, [0, 2]] = inv[:15, [2, 0]]
    inv[15:, [1, 3]] = inv[15:, [3, 1]]
    inv[25:, [0, 2]] = inv[25:, [2, 0]]
    boxes.append(inv)
    # 5. large and negative coordinates
    big = b[90:130].copy() * np.float32(8.0) + np.float32(1.0e6)
    neg = b[90:130].copy() - np.float32(1.0)
    boxes.append(big.astype(np.float32))
    boxes.append(neg.astype(np.float32))
    # 6. subnormal extents at the origin, and huge boxes
    tiny = np.array([[0, 0, 1e-40, 1e-40], [0, 0, 1e-45, 1e-38], [-1e-40, -1e-40, 0, 0],
                     [1e-39, 0, 1e-39, 1e-39]], dtype=np.float32)
    huge = np.array([[-1e6, -1e6, 1e6, 1e6], [0, 0, 1, 1], [-0.5, 0.25, 1.5, 0.75]],
                    dtype=np.float32)
    boxes.append(tiny)
    boxes.append(huge)
    boxes = np.concatenate(boxes).astype(np.float32)

    # query boxes: the same families, perturbed differently, plus exact copies
    q = []
    q.append(cells[::3].astype(np.float32))
    q.append(boxes[64:214:2].copy())
    qq = boxes[64:214:3].copy()
    for c in range(4):
        qq[:, c] = nudge(qq[:, c], rng.integers(-2, 3, qq.shape[0]))
    q.append(qq)
    zq = boxes[64:124].copy()
    zq[:20, 2] = zq[:20, 0]
    zq[20:40, 3] = zq[20:40, 1]
    zq[40:, 2] = zq[40:, 0]
    zq[40:, 3] = zq[40:, 1]
    q.append(zq)
    iq = boxes[130:150].copy()
    iq[:10, [0, 2]] = iq[:10, [2, 0]]
    iq[10:, [1, 3]] = iq[10:, [3, 1]]
    q.append(iq)
    q.append(big[::4].copy())
    q.append(neg[::4].copy())
    q.append(tiny.copy())
    q.append(np.array([[0.1, 0.1, 0.9, 0.9], [0.5, 0.5, 0.5, 0.5], [-2, -2, -1.5, -1.5]],
                      dtype=np.float32))
    queries = np.concatenate(q).astype(np.float32)

    # points: box corners and edge midpoints, ulp-nudged copies, random
    corners = np.concatenate([boxes[:, [0, 1]], boxes[:, [2, 3]], boxes[:, [0, 3]],
                              boxes[:, [2, 1]]])[::5]
    mids = np.stack([(boxes[:, 0] + boxes[:, 2]) * 0.5, boxes[:, 1]], 1)[::7]
    pn = corners[::3].copy()
    pn[:, 0] = nudge(pn[:, 0], rng.integers(-1, 2, pn.shape[0]))
    pn[:, 1] = nudge(pn[:, 1], rng.integers(-1, 2, pn.shape[0]))
    pts = np.concatenate([corners, mids, pn, rng.random((50, 2))]).astype(np.float32)
    return boxes, queries, pts


def main() -> None:
    ref = Oracle("ref")
    port = Oracle("port")
    b100k = port.uniform_boxes(100000, 0.5, 0.5)
    p1k = port.uniform_points(1000)
    q1k = port.uniform_boxes(1000, 0.1, 0.1)
    n_pt = ref.run(KIND_POINT, b100k, p1k, collect=False, grid=False)[0]
    n_is = ref.run(KIND_INTERSECTS, b100k, q1k, collect=False, grid=False)[0]
    n_ct = ref.run(KIND_CONTAINS, b100k, q1k, collect=False, grid=False)[0]
    assert n_pt == 4224111 and n_is == 6549771, (n_pt, n_is)
    upd_ids = port.update_ids(100000, 5000)
    kat = {
        "boxes_100000_0.5": sha(b100k),
        "points_1000": sha(p1k),
        "boxes_1000_0.1": sha(q1k),
        "update_ids_100000_5000": sha(upd_ids),
        "update_boxes_5000_0.5": sha(port.uniform_boxes(5000, 0.5, 0.5)),
        "point_contains_100000x1000": n_pt,
        "intersects_100000x1000": n_is,
        "range_contains_100000x1000": n_ct,
    }
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1, sort_keys=True)

    boxes, queries, pts = edge_case_sets()
    out = {"boxes": boxes, "queries": queries, "points": pts}
    for name, kind, qs in (("point", KIND_POINT, pts), ("contains", KIND_CONTAINS, queries),
                           ("intersects", KIND_INTERSECTS, queries)):
        tot, _, pairs = ref.run(kind, boxes, qs, collect=True, grid=False)
        out[name] = pairs.astype(np.uint32)
        print(name, tot)
    np.savez_compressed(os.path.join(HERE, "edge_cases.npz"), **out)
    print("boxes", boxes.shape, "queries", queries.shape, "points", pts.shape)


if __name__ == "__main__":
    main()
