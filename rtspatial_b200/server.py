"""Python mirror of the serving engine (``rts_server_*`` in
``include/rtspatial_b200.h``): submit query requests and update batches from
any thread; results come back per request with their own query ids."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L
from ._lib import check, lib


class Server:
    def __init__(self, index, slots: int = 3, max_queries_per_launch: int = 1 << 20,
                 pairs_per_launch: int = 32 << 20, max_parts_per_launch: int = 1024,
                 hbm_budget_bytes: int = 0, host_result_bytes: int = 1 << 30,
                 use_graphs: bool = True):
        c = L.rts_server_config()
        check(lib().rts_server_config_default(ctypes.byref(c)))
        c.slots = slots
        c.max_queries_per_launch = max_queries_per_launch
        c.pairs_per_launch = pairs_per_launch
        c.max_parts_per_launch = max_parts_per_launch
        c.hbm_budget_bytes = hbm_budget_bytes
        c.host_result_bytes = host_result_bytes
        c.use_graphs = 1 if use_graphs else 0
        self.index = index
        self._h = ctypes.c_void_p()
        check(lib().rts_server_create(index._handle(), ctypes.byref(c), ctypes.byref(self._h)))

    def submit(self, predicate, queries: np.ndarray) -> int:
        """Queues a query request; float64 arrays go to a double index."""
        f64 = np.asarray(queries).dtype == np.float64
        q = np.ascontiguousarray(queries, dtype=np.float64 if f64 else np.float32)
        pts = q.ndim == 2 and q.shape[1] == 2
        if f64:
            kind = L.RTS_QUERY_POINTS_F64 if pts else L.RTS_QUERY_ENVELOPES_F64
        else:
            kind = L.RTS_QUERY_POINTS if pts else L.RTS_QUERY_ENVELOPES
        n = q.shape[0] if q.ndim == 2 else q.size // (2 if pts else 4)
        t = ctypes.c_uint64()
        check(lib().rts_server_submit_query(self._h, kind, int(predicate), q.ctypes.data, n,
                                            ctypes.byref(t)))
        return t.value

    def submit_update(self, delete_ids=None, inserts=None, update_ids=None,
                      update_boxes=None) -> int:
        d = np.ascontiguousarray(delete_ids if delete_ids is not None else [], dtype=np.uint64)
        ins = np.ascontiguousarray(inserts if inserts is not None else np.zeros((0, 4)),
                                   dtype=np.float32).reshape(-1, 4)
        if update_ids is not None and len(update_ids):
            rec = np.zeros(len(update_ids), dtype=[("id", "<u8"), ("b", "<f4", 4)])
            rec["id"] = np.asarray(update_ids, dtype=np.uint64)
            rec["b"] = np.asarray(update_boxes, dtype=np.float32).reshape(-1, 4)
        else:
            rec = np.zeros(0, dtype=[("id", "<u8"), ("b", "<f4", 4)])
        t = ctypes.c_uint64()
        check(lib().rts_server_submit_update(self._h, d.ctypes.data if d.size else None, d.size,
                                             ins.ctypes.data if ins.size else None, ins.shape[0],
                                             rec.ctypes.data if rec.size else None, rec.size,
                                             ctypes.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0) -> None:
        check(lib().rts_server_wait(self._h, ticket, timeout))

    def take(self, ticket: int, out: np.ndarray | None = None) -> np.ndarray:
        """(R, 2) uint32 (geom_id, query_id) of a query request (waits for it);
        for an update request, the first id its inserts received.  `out`, when
        given and large enough, receives the pairs (a view of it is returned)."""
        self.wait(ticket)
        n = ctypes.c_uint64()
        rc = lib().rts_server_take(self._h, ticket, None, 0, ctypes.byref(n))
        if rc == L.RTS_OK:
            return np.zeros((0, 2), dtype=np.uint32) if n.value == 0 else n.value
        if rc != L.RTS_ERR_QUEUE_FULL:
            check(rc)
        if out is None or out.shape[0] < n.value:
            out = np.empty((n.value, 2), dtype=np.uint32)
        check(lib().rts_server_take(self._h, ticket, out.ctypes.data, n.value, ctypes.byref(n)))
        return out[:n.value]

    def view(self, ticket: int) -> list:
        """Zero-copy: the request's pairs as (k, 2) uint32 numpy arrays over the
        server's pinned result memory, one per part in query order (waits for
        the request).  Valid until ``release(ticket)``."""
        self.wait(ticket)
        n_seg = ctypes.c_uint32()
        n = ctypes.c_uint64()
        cap = 64
        while True:
            segs = (ctypes.c_void_p * cap)()
            cnts = (ctypes.c_uint64 * cap)()
            rc = lib().rts_server_view(self._h, ticket, segs, cnts, cap, ctypes.byref(n_seg),
                                       ctypes.byref(n))
            if rc == L.RTS_ERR_QUEUE_FULL and n_seg.value > cap:
                cap = n_seg.value
                continue
            check(rc)
            break
        out = []
        for i in range(n_seg.value):
            k = int(cnts[i])
            buf = (ctypes.c_uint32 * (2 * k)).from_address(segs[i])
            out.append(np.frombuffer(buf, dtype=np.uint32).reshape(k, 2))
        return out

    def release(self, ticket: int) -> None:
        """Ends a ``view``: the pinned memory returns to the server."""
        check(lib().rts_server_release(self._h, ticket))

    def stats(self) -> dict:
        st = L.rts_server_stats()
        check(lib().rts_server_get_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in L.rts_server_stats._fields_}

    def reset_stats(self) -> None:
        check(lib().rts_server_reset_stats(self._h))

    def close(self) -> None:
        if self._h:
            lib().rts_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
