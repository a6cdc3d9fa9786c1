"""Helpers of the GPU parity tests: run the CUDA library through its C-ABI
(via the Python mirror) and bring results into the oracle's canonical order."""
from __future__ import annotations

import itertools

import numpy as np
import torch

import rtspatial_b200 as rb
from rtspatial_b200 import _lib as L

WIDTHS = (4, 8, 16, 32)
TRAVERSALS = (L.RTS_TRAVERSAL_THREAD, L.RTS_TRAVERSAL_TEAM, L.RTS_TRAVERSAL_FRONTIER,
              L.RTS_TRAVERSAL_PACKET, L.RTS_TRAVERSAL_STAGED)
CURVES = (L.RTS_CURVE_MORTON, L.RTS_CURVE_HILBERT)

# every (width, traversal, curve) combination
ALL_COMBOS = list(itertools.product(WIDTHS, TRAVERSALS, CURVES))
# a cheaper cover: each width with both traversals, curves alternating
SOME_COMBOS = [(w, t, CURVES[i % 2]) for i, (w, t) in
               enumerate(itertools.product(WIDTHS, TRAVERSALS))]


def combo_id(c):
    w, t, cu = c
    tn = {L.RTS_TRAVERSAL_THREAD: "thread", L.RTS_TRAVERSAL_TEAM: "team",
          L.RTS_TRAVERSAL_FRONTIER: "frontier", L.RTS_TRAVERSAL_PACKET: "packet",
          L.RTS_TRAVERSAL_STAGED: "staged"}[t]
    return f"w{w}-{tn}-" \
           f"{'morton' if cu == L.RTS_CURVE_MORTON else 'hilbert'}"


def make_index(combo, **kw) -> rb.SpatialIndex:
    w, t, cu = combo
    cfg = rb.Config(node_width=w, traversal=t, curve=cu, **kw)
    return rb.SpatialIndex(cfg)


def dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def canon(p: torch.Tensor | np.ndarray) -> np.ndarray:
    """(R, 2) (geom_id, query_id) sorted by (query_id, geom_id), uint32."""
    if isinstance(p, torch.Tensor):
        p = p.cpu().numpy()
    p = np.asarray(p).reshape(-1, 2).astype(np.uint64)
    order = np.lexsort((p[:, 0], p[:, 1]))
    return p[order].astype(np.uint32)


def gpu_pairs(ix: rb.SpatialIndex, pred, queries: np.ndarray, capacity=None) -> np.ndarray:
    q = dev(queries)
    out = ix.query_pairs(pred, q, capacity=capacity)
    torch.cuda.synchronize()
    return canon(out)


def gpu_count(ix: rb.SpatialIndex, pred, queries: np.ndarray) -> int:
    return ix.query_count(pred, dev(queries))


def assert_same_pairs(got: np.ndarray, want: np.ndarray, what: str = "") -> None:
    if got.shape == want.shape and np.array_equal(got, want):
        return
    gs = set(map(tuple, got.tolist()))
    ws = set(map(tuple, want.tolist()))
    extra = sorted(gs - ws)[:10]
    missing = sorted(ws - gs)[:10]
    raise AssertionError(f"{what}: got {len(got)} pairs, want {len(want)}; "
                         f"dups={len(got) - len(gs)} extra={extra} missing={missing}")
