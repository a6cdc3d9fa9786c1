"""TEST INFRASTRUCTURE ONLY — ctypes wrapper of the CPU oracle.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline
leg (and its reference arm) use this module, as the checker.  The product
path (``rtspatial_b200``) never imports it.

Two back ends with one interface:
  * ``port``: the plain-C restatement of the reference predicates
    (``rts_predicates.h``), built into ``oracle/librts_oracle.so``;
  * ``ref``: the reference's own predicate headers compiled for the host
    (``oracle/_ref/libref_oracle.so``), present only where the reference
    source tree was available at build time.

Kinds follow the reference's three query shaders: 0 = point-contains
(``shaders_contains_point_query_2d.cu:14-25``), 1 = range-contains
(``shaders_contains_envelope_query_2d.cu:14-25``), 2 = range-intersects
(``shaders_intersects_envelope_query_2d.cu:14-129``).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(_HERE, "librts_oracle.so")
REF_LIB = os.path.join(_HERE, "_ref", "libref_oracle.so")

KIND_POINT, KIND_CONTAINS, KIND_INTERSECTS = 0, 1, 2

_u64 = ctypes.c_uint64
_vp = ctypes.c_void_p


def build(ref_root: str | None = None) -> None:
    """Builds the restated oracle and, when ``ref_root`` holds the reference
    source tree, the reference-header build under ``oracle/_ref``."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "librts_oracle.so"])
    if ref_root and os.path.isdir(os.path.join(ref_root, "include", "rtspatial")):
        subprocess.check_call(["make", "-s", "-C", _HERE, "ref", f"REF_ROOT={ref_root}"])


def _bind(lib: ctypes.CDLL, pfx: str) -> None:
    f = getattr(lib, pfx + "grid_build")
    f.restype = _vp
    f.argtypes = [_vp, _u64, ctypes.c_double]
    f = getattr(lib, pfx + "grid_free")
    f.restype = None
    f.argtypes = [_vp]
    f = getattr(lib, pfx + "run")
    f.restype = _u64
    f.argtypes = [_vp, _vp, _u64, ctypes.c_int, _vp, _u64, _vp, _vp, _u64, ctypes.c_int]
    f = getattr(lib, pfx + "run_digest")
    f.restype = _u64
    f.argtypes = [_vp, _vp, _u64, ctypes.c_int, _vp, _u64, _vp, _vp, _vp, ctypes.c_int]
    f = getattr(lib, pfx + "eval_pairs")
    f.restype = None
    f.argtypes = [ctypes.c_int, _vp, _vp, _u64, _vp]
    f = getattr(lib, pfx + "invalidate")
    f.restype = None
    f.argtypes = [_vp, _vp, _u64]


def pair_mix(geom_ids: np.ndarray, query_ids: np.ndarray) -> np.ndarray:
    """Digest term of each (geom_id, query_id) pair, as ``ob_pair_mix`` in
    grid_driver.h computes it (splitmix64's finaliser of geom << 32 | query),
    in uint64 arithmetic modulo 2^64."""
    x = (np.asarray(geom_ids).astype(np.uint64) << np.uint64(32)) | \
        np.asarray(query_ids).astype(np.uint64)
    x ^= x >> np.uint64(30)
    x *= np.uint64(0xbf58476d1ce4e5b9)
    x ^= x >> np.uint64(27)
    x *= np.uint64(0x94d049bb133111eb)
    x ^= x >> np.uint64(31)
    return x


def pair_digest(pairs: np.ndarray) -> int:
    """Order-independent digest of an (R, 2) array of (geom_id, query_id):
    the sum modulo 2^64 of ``pair_mix`` over its rows."""
    pairs = np.asarray(pairs).reshape(-1, 2)
    if pairs.shape[0] == 0:
        return 0
    total = np.uint64(0)
    step = 1 << 24  # bounded temporaries for large result sets
    for i in range(0, pairs.shape[0], step):
        part = pairs[i:i + step]
        total += pair_mix(part[:, 0], part[:, 1]).sum(dtype=np.uint64)
    return int(total)


def _bind64(lib: ctypes.CDLL, pfx: str) -> None:
    f = getattr(lib, pfx + "run")
    f.restype = _u64
    f.argtypes = [_vp, _u64, ctypes.c_int, _vp, _u64, _vp, _vp, _u64, ctypes.c_int]
    f = getattr(lib, pfx + "eval_pairs")
    f.restype = None
    f.argtypes = [ctypes.c_int, _vp, _vp, _u64, _vp]
    f = getattr(lib, pfx + "invalidate")
    f.restype = None
    f.argtypes = [_vp, _vp, _u64]


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


class Oracle:
    """Counts or collects (geom_id, query_id) pairs on the CPU."""

    def __init__(self, backend: str = "port"):
        if backend == "port":
            path, pfx = PORT_LIB, "ob_port_"
        elif backend == "ref":
            path, pfx = REF_LIB, "ob_ref_"
        else:
            raise ValueError(backend)
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path} (run oracle.build())")
        self.backend = backend
        self.lib = ctypes.CDLL(path)
        self.pfx = pfx
        self.pfx64 = pfx.replace("ob_", "ob64_")
        _bind(self.lib, pfx)
        _bind64(self.lib, self.pfx64)
        if backend == "port":
            self.lib.ob_port_slab_k.restype = ctypes.c_float
            self.lib.ob64_port_slab_k.restype = ctypes.c_double
            for name, args in (
                ("ob_fix_uniform_boxes", [_u64, ctypes.c_float, ctypes.c_float, _vp]),
                ("ob_fix_uniform_points", [_u64, _vp]),
                ("ob_fix_update_ids", [_u64, _u64, _vp]),
            ):
                fn = getattr(self.lib, name)
                fn.restype = None
                fn.argtypes = args

    def _f(self, name):
        return getattr(self.lib, self.pfx + name)

    # -- bulk ----------------------------------------------------------------
    def run(self, kind: int, boxes: np.ndarray, queries: np.ndarray, *,
            collect: bool = True, grid: bool | str = "auto", threads: int | None = None,
            boxes_per_cell: float = 2.0):
        """Returns (total, per_query_counts, pairs or None).

        ``pairs`` is an (R, 2) uint32 array of (geom_id, query_id), sorted by
        (query_id, geom_id)."""
        boxes = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 4)
        width = 2 if kind == KIND_POINT else 4
        queries = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, width)
        nb, nq = boxes.shape[0], queries.shape[0]
        if grid == "auto":
            grid = nb * max(nq, 1) > 2_000_000
        threads = threads or os.cpu_count() or 1
        g = None
        if grid:
            g = self._f("grid_build")(_ptr(boxes), nb, boxes_per_cell)
        try:
            counts = np.zeros(max(nq, 1), dtype=np.uint64)
            total = int(self._f("run")(g, _ptr(boxes), nb, kind, _ptr(queries), nq,
                                       _ptr(counts), None, 0, threads))
            pairs = None
            if collect:
                pairs = np.zeros((max(total, 1), 2), dtype=np.uint32)
                got = int(self._f("run")(g, _ptr(boxes), nb, kind, _ptr(queries), nq,
                                         _ptr(counts), _ptr(pairs), total, threads))
                assert got == total
                pairs = pairs[:total]
            return total, counts[:nq], pairs
        finally:
            if g:
                self._f("grid_free")(g)

    def grid_build(self, boxes: np.ndarray, boxes_per_cell: float = 2.0) -> int:
        return self._f("grid_build")(_ptr(boxes), boxes.shape[0], boxes_per_cell)

    def grid_free(self, g: int) -> None:
        self._f("grid_free")(g)

    def digest(self, kind: int, boxes: np.ndarray, queries: np.ndarray, *,
               rid: np.ndarray | None = None, grid=None, threads: int | None = None,
               boxes_per_cell: float = 2.0):
        """Returns (total, per-query counts, per-query digests): query q's
        digest is the sum modulo 2^64 of pair_mix(geom_id, rid[q]) over its
        matches (rid None: rid[q] = q).  ``grid``: a prebuilt grid handle,
        True (build one here), or False (brute force)."""
        boxes = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 4)
        width = 2 if kind == KIND_POINT else 4
        queries = np.ascontiguousarray(queries, dtype=np.float32).reshape(-1, width)
        nb, nq = boxes.shape[0], queries.shape[0]
        if rid is not None:
            rid = np.ascontiguousarray(rid, dtype=np.uint32)
            assert rid.shape[0] == nq
        threads = threads or os.cpu_count() or 1
        own = grid is None or grid is True
        g = self._f("grid_build")(_ptr(boxes), nb, boxes_per_cell) if own else (grid or None)
        try:
            counts = np.zeros(max(nq, 1), dtype=np.uint64)
            digests = np.zeros(max(nq, 1), dtype=np.uint64)
            total = int(self._f("run_digest")(g, _ptr(boxes), nb, kind, _ptr(queries), nq,
                                              _ptr(rid), _ptr(counts), _ptr(digests), threads))
            return total, counts[:nq], digests[:nq]
        finally:
            if own and g:
                self._f("grid_free")(g)

    def run_on_grid(self, g: int, kind: int, boxes: np.ndarray, queries: np.ndarray,
                    threads: int) -> int:
        """Count-only run over a prebuilt grid (used for timing)."""
        return int(self._f("run")(g, _ptr(boxes), boxes.shape[0], kind, _ptr(queries),
                                  queries.shape[0], None, None, 0, threads))

    # -- per pair --------------------------------------------------------------
    def eval_pairs(self, kind: int, g: np.ndarray, q: np.ndarray) -> np.ndarray:
        g = np.ascontiguousarray(g, dtype=np.float32).reshape(-1, 4)
        width = 2 if kind == KIND_POINT else 4
        q = np.ascontiguousarray(q, dtype=np.float32).reshape(-1, width)
        assert g.shape[0] == q.shape[0]
        out = np.zeros(g.shape[0], dtype=np.uint8)
        self._f("eval_pairs")(kind, _ptr(g), _ptr(q), g.shape[0], _ptr(out))
        return out

    def invalidate(self, boxes: np.ndarray, ids) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.uint64)
        assert boxes.dtype == np.float32 and boxes.flags.c_contiguous
        self._f("invalidate")(_ptr(boxes), _ptr(ids), ids.shape[0])

    # -- double indexes (SpatialIndex<double, 2>), brute force --------------------
    def run64(self, kind: int, boxes: np.ndarray, queries: np.ndarray, *,
              collect: bool = True, threads: int | None = None):
        """Same as ``run`` for float64 boxes and queries."""
        boxes = np.ascontiguousarray(boxes, dtype=np.float64).reshape(-1, 4)
        width = 2 if kind == KIND_POINT else 4
        queries = np.ascontiguousarray(queries, dtype=np.float64).reshape(-1, width)
        nb, nq = boxes.shape[0], queries.shape[0]
        threads = threads or os.cpu_count() or 1
        f = getattr(self.lib, self.pfx64 + "run")
        counts = np.zeros(max(nq, 1), dtype=np.uint64)
        total = int(f(_ptr(boxes), nb, kind, _ptr(queries), nq, _ptr(counts), None, 0, threads))
        pairs = None
        if collect:
            pairs = np.zeros((max(total, 1), 2), dtype=np.uint32)
            got = int(f(_ptr(boxes), nb, kind, _ptr(queries), nq, _ptr(counts), _ptr(pairs),
                        total, threads))
            assert got == total
            pairs = pairs[:total]
        return total, counts[:nq], pairs

    def eval_pairs64(self, kind: int, g: np.ndarray, q: np.ndarray) -> np.ndarray:
        g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1, 4)
        width = 2 if kind == KIND_POINT else 4
        q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1, width)
        assert g.shape[0] == q.shape[0]
        out = np.zeros(g.shape[0], dtype=np.uint8)
        getattr(self.lib, self.pfx64 + "eval_pairs")(kind, _ptr(g), _ptr(q), g.shape[0], _ptr(out))
        return out

    def invalidate64(self, boxes: np.ndarray, ids) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.uint64)
        assert boxes.dtype == np.float64 and boxes.flags.c_contiguous
        getattr(self.lib, self.pfx64 + "invalidate")(_ptr(boxes), _ptr(ids), ids.shape[0])

    def slab_k64(self) -> float:
        return float(self.lib.ob64_port_slab_k())

    # -- fixtures (restated generator of the reference tests) ------------------
    def uniform_boxes(self, n: int, max_w: float, max_h: float) -> np.ndarray:
        out = np.zeros((n, 4), dtype=np.float32)
        self.lib.ob_fix_uniform_boxes(n, max_w, max_h, _ptr(out))
        return out

    def uniform_points(self, n: int) -> np.ndarray:
        out = np.zeros((n, 2), dtype=np.float32)
        self.lib.ob_fix_uniform_points(n, _ptr(out))
        return out

    def update_ids(self, n1: int, n_updates: int) -> np.ndarray:
        out = np.zeros(n_updates, dtype=np.uint64)
        self.lib.ob_fix_update_ids(n1, n_updates, _ptr(out))
        return out

    def slab_k(self) -> float:
        return float(self.lib.ob_port_slab_k())


def available(backend: str) -> bool:
    return os.path.exists(PORT_LIB if backend == "port" else REF_LIB)
