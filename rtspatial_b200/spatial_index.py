"""Python mirror of ``rtspatial::SpatialIndex<float, 2>`` over the C-ABI.

Method names, argument meaning and error behaviour follow the reference's
public class (``include/rtspatial/spatial_index.cuh:62-931``):

=========================  ====================================================
reference                  here
=========================  ====================================================
``Init(const Config&)``    ``Init(config)``
``Clear()``                ``Clear(stream=None)``
``Insert(ArrayView<envelope_t>, stream)``  ``Insert(envelopes, stream=None)``
``Delete(ArrayView<size_t>, stream)``      ``Delete(ids, stream=None)``
``Update(ArrayView<pair<size_t, envelope_t>>, stream)``
                           ``Update(ids, envelopes, stream=None)``
``Query(Predicate, ArrayView<point_t|envelope_t>, void* arg, stream)``
                           ``Query(predicate, queries, arg, stream=None,
                           handler=...)``
=========================  ====================================================

Inputs are CUDA tensors (float32 ``(n, 4)`` envelopes as min.x, min.y, max.x,
max.y; ``(n, 2)`` points; int64 ids).  ``arg`` is a device pointer exactly as
in the reference: an ``unsigned long long`` counter for the counting handler,
or a device ``Queue`` object for the collecting handler.  ``Counter`` and
``Queue`` below mirror ``SharedValue<unsigned long long>`` and
``rtspatial::Queue<thrust::pair<uint32_t, uint32_t>>`` (``utils/queue.h``).
Torch provides device memory and streams only; all index work runs in the
CUDA library.
"""
from __future__ import annotations

import ctypes
import enum
import os
from dataclasses import dataclass, fields
from typing import Iterable, Sequence

import torch

from . import _lib as L
from ._lib import check, lib


class Predicate(enum.IntEnum):
    """``rtspatial::Predicate`` (geom/predicates.h:7-10)."""

    kIntersects = L.RTS_PREDICATE_INTERSECTS
    kContains = L.RTS_PREDICATE_CONTAINS


class Handler(enum.IntEnum):
    """The two shipped handler headers (default_handlers/*.h), and the
    caller's own rtspatial_handle_* functions from a loaded handler module."""

    COUNT = L.RTS_HANDLER_COUNT
    COLLECT = L.RTS_HANDLER_COLLECT
    MODULE = L.RTS_HANDLER_MODULE


@dataclass
class Config:
    """``rtspatial::Config`` (spatial_index.cuh:22-37) plus structure knobs."""

    ptx_root: str = ""
    max_geometries: int = 1000 * 1000 * 10
    max_queries: int = 1000 * 1000
    preallocate: bool = False
    prefer_fast_build_geom: bool = False
    prefer_fast_build_query: bool = False
    compact: bool = False
    geom_sample_rate: float = 0.2
    query_sample_rate: float = 0.2
    intersect_cost_weight: float = 0.95
    max_geom_samples: int = 10000
    max_query_samples: int = 1000
    max_parallelism: int = 512
    # structure / traversal
    node_width: int = 16
    traversal: int = L.RTS_TRAVERSAL_AUTO
    curve: int = L.RTS_CURVE_HILBERT
    max_trees: int = 4
    rebuild_fraction: float = 0.25
    sort_queries: int = 2
    rebuild_update_fraction: float = 0.25
    chunk: int = 0
    query_occupancy: int = 0
    frontier_factor: float = 0.0
    coord_bits: int = 32    # 64: SpatialIndex<double, 2> (float64 tensors throughout)
    group_loads: int = L.RTS_LOADS_AUTO  # L1 use of the thread scheme's group loads

    def to_c(self) -> L.rts_config:
        c = L.rts_config()
        check(lib().rts_config_default(ctypes.byref(c)))
        for f in fields(self):
            if f.name == "ptx_root":
                continue
            setattr(c, f.name, int(getattr(self, f.name)) if isinstance(getattr(self, f.name), bool)
                    else getattr(self, f.name))
        return c


def _stream_handle(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _f32(t: torch.Tensor, width: int, name: str, dtype=torch.float32) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {str(dtype).replace('torch.', '')}")
    t = t.reshape(-1, width)
    if not t.is_contiguous():
        t = t.contiguous()
    return t


class Counter:
    """Device ``unsigned long long`` for the counting handler (the
    reference's ``SharedValue<unsigned long long>``, utils/shared_value.h)."""

    def __init__(self, device=None):
        self.buf = torch.zeros(1, dtype=torch.int64, device=device or "cuda")

    def data(self) -> int:
        return self.buf.data_ptr()

    def set(self, value: int = 0, stream=None) -> None:
        with torch.cuda.stream(stream) if stream is not None else _nullctx():
            self.buf.fill_(value)

    def get(self, stream=None) -> int:
        if stream is not None:
            stream.synchronize()
        return int(self.buf.item())


class Queue:
    """Host wrapper of a collecting queue (``rtspatial::Queue<T>``,
    utils/queue.h:65-113) whose ``DeviceObject()`` is the ``arg`` a collecting
    query takes: a device struct {pairs*, capacity, uint32* size}."""

    def __init__(self, capacity: int = 0, device=None):
        self.device = torch.device(device or "cuda")
        self.pairs = torch.empty((0, 2), dtype=torch.int32, device=self.device)
        self.counter = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.obj = torch.zeros(3, dtype=torch.int64, device=self.device)
        if capacity:
            self.Init(capacity)

    def Init(self, capacity: int) -> None:
        self.pairs = torch.empty((max(int(capacity), 1), 2), dtype=torch.int32, device=self.device)
        host = torch.tensor([self.pairs.data_ptr(), int(capacity), self.counter.data_ptr()],
                            dtype=torch.int64)
        self.obj.copy_(host)
        self.counter.zero_()

    def Clear(self, stream=None) -> None:
        with torch.cuda.stream(stream) if stream is not None else _nullctx():
            self.counter.zero_()

    def capacity(self) -> int:
        return int(self.obj[1].item())

    def size(self, stream=None) -> int:
        """Pairs reported (may exceed capacity: then only capacity were kept)."""
        if stream is not None:
            stream.synchronize()
        return int(self.counter.item()) & 0xFFFFFFFF

    def DeviceObject(self) -> int:
        return self.obj.data_ptr()

    def result(self, stream=None) -> torch.Tensor:
        """(R, 2) int64 tensor of (geom_id, query_id) as stored (unsorted)."""
        n = min(self.size(stream), self.pairs.shape[0])
        return self.pairs[:n].to(torch.int64) & 0xFFFFFFFF


class _nullctx:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False


class SpatialIndex:
    """``rtspatial::SpatialIndex<float, 2>`` on the B200 library."""

    def __init__(self, config: Config | None = None):
        self._h = ctypes.c_void_p()
        self.config = None
        if config is not None:
            self.Init(config)

    # -- lifecycle ------------------------------------------------------------
    def Init(self, config: Config | None = None) -> None:
        self._destroy()
        self.config = config or Config()
        c = self.config.to_c()
        check(lib().rts_create(ctypes.byref(c), ctypes.byref(self._h)))

    def _destroy(self) -> None:
        if self._h:
            lib().rts_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    def _handle(self):
        if not self._h:
            raise RuntimeError("SpatialIndex used before Init()")
        return self._h

    def Clear(self, stream=None) -> None:
        check(lib().rts_clear(self._handle(), _stream_handle(stream)))

    # -- mutation ---------------------------------------------------------------
    @property
    def _f64(self) -> bool:
        return self.config.coord_bits == 64

    @property
    def _dtype(self):
        return torch.float64 if self._f64 else torch.float32

    def Insert(self, envelopes: torch.Tensor, stream=None) -> None:
        e = _f32(envelopes, 4, "envelopes", self._dtype)
        fn = lib().rts_insert_f64 if self._f64 else lib().rts_insert
        check(fn(self._handle(), e.data_ptr(), e.shape[0], _stream_handle(stream)))
        self._keep = e  # the copy is asynchronous

    def Delete(self, ids: torch.Tensor, stream=None) -> None:
        if not ids.is_cuda:
            raise TypeError("ids must be a CUDA tensor")
        ids = ids.to(torch.int64).contiguous()
        check(lib().rts_delete(self._handle(), ids.data_ptr(), ids.numel(), _stream_handle(stream)))
        self._keep = ids

    def Update(self, ids: torch.Tensor, envelopes: torch.Tensor, stream=None) -> None:
        """Overwrites envelopes[i] at id ids[i] (the reference takes
        ``thrust::pair<size_t, envelope_t>``; this packs the same 24-byte
        records)."""
        e = _f32(envelopes, 4, "envelopes", self._dtype)
        ids = ids.to(device=e.device, dtype=torch.int64).reshape(-1, 1)
        if ids.shape[0] != e.shape[0]:
            raise ValueError("ids and envelopes differ in length")
        rec = torch.cat([ids, e.view(torch.int64)], dim=1).contiguous()   # 24 or 40 bytes
        fn = lib().rts_update_f64 if self._f64 else lib().rts_update
        check(fn(self._handle(), rec.data_ptr(), rec.shape[0], _stream_handle(stream)))
        self._keep = rec

    # -- queries ------------------------------------------------------------------
    def Query(self, predicate: Predicate, queries: torch.Tensor, arg: int, stream=None,
              handler: Handler = Handler.COLLECT) -> None:
        """Reference-shaped query: results go to the handler's ``arg``."""
        f64 = self._f64
        if queries.dim() == 2 and queries.shape[1] == 2:
            q = _f32(queries, 2, "queries", self._dtype)
            fn = lib().rts_query_points_f64 if f64 else lib().rts_query_points
        else:
            q = _f32(queries, 4, "queries", self._dtype)
            fn = lib().rts_query_envelopes_f64 if f64 else lib().rts_query_envelopes
        check(fn(self._handle(), int(predicate), q.data_ptr(), q.shape[0], int(handler), arg,
                 _stream_handle(stream)))

    def query_count(self, predicate: Predicate, queries: torch.Tensor, stream=None) -> int:
        c = Counter(queries.device)
        self.Query(predicate, queries, c.data(), stream, Handler.COUNT)
        torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
        return c.get()

    def query_pairs(self, predicate: Predicate, queries: torch.Tensor, capacity: int | None = None,
                    stream=None) -> torch.Tensor:
        """(R, 2) int64 tensor of (geom_id, query_id), in device order.  Grows
        the queue and re-runs once if the first capacity was too small."""
        cap = capacity or max(1024, 4 * queries.shape[0])
        for _ in range(2):
            qu = Queue(cap, queries.device)
            self.Query(predicate, queries, qu.DeviceObject(), stream, Handler.COLLECT)
            n = qu.size(stream if stream is not None else torch.cuda.current_stream())
            if n <= cap:
                return qu.result()
            cap = n
        raise RuntimeError("queue overflow after resize")

    def query_batched(self, batches: Sequence[tuple], stream=None) -> None:
        """Runs several Query calls in one persistent launch.  Each batch is
        ``(predicate, queries, handler, arg)``; points are (n, 2) tensors."""
        arr, keep = _batch_array(batches)
        check(lib().rts_query_batched(self._handle(), arr, len(batches), _stream_handle(stream)))
        self._keep = keep

    def autotune(self, batches: Sequence[tuple], tune_width: bool = True, stream=None) -> dict:
        """Times candidate launch settings on `batches` (run through internal
        counters and queues) and keeps the fastest; see ``rts_autotune``."""
        arr, keep = _batch_array(batches)
        r = L.rts_tune_result()
        check(lib().rts_autotune(self._handle(), arr, len(batches), 1 if tune_width else 0,
                                 _stream_handle(stream), ctypes.byref(r)))
        res = {f: getattr(r, f) for f, _ in L.rts_tune_result._fields_}
        for k in ("node_width", "traversal", "query_occupancy", "sort_queries", "chunk",
                  "group_loads"):
            setattr(self.config, k, res[k])
        return res

    def plan(self, batches: Sequence[tuple]) -> "Plan":
        """A prepared launch of fixed batches, replayable through a CUDA graph
        (``rts_plan_*``).  Query tensors and outputs must stay allocated."""
        return Plan(self, batches)

    def load_handler_module(self, path: str) -> None:
        """Loads a handler module (``rtspatial_b200.handlers.compile_module``):
        queries with ``Handler.MODULE`` then call its rtspatial_handle_*
        functions once per pair."""
        check(lib().rts_load_handler_module(self._handle(), os.fsencode(path)))

    def handler_module_builtin(self) -> int:
        """RTS_HANDLER_COUNT / RTS_HANDLER_COLLECT when the loaded module was
        built from a shipped handler header, else -1."""
        return int(lib().rts_handler_module_builtin(self._handle()))

    def device_status(self, stream=None) -> int:
        """The index's device status bits (RTS_STATUS_*); 0 when every launch
        completed normally."""
        st = ctypes.c_uint32()
        check(lib().rts_device_status(self._handle(), ctypes.byref(st), _stream_handle(stream)))
        return int(st.value)

    def report_query_time(self, ms: float) -> float:
        """Feeds the refit-vs-rebuild tuner; returns the new re-sort threshold."""
        f = ctypes.c_float()
        check(lib().rts_report_query_time(self._handle(), float(ms), ctypes.byref(f)))
        self.config.rebuild_update_fraction = f.value
        return f.value

    # -- introspection ------------------------------------------------------------
    def size(self) -> int:
        return int(lib().rts_size(self._handle()))

    def num_trees(self) -> int:
        return int(lib().rts_num_trees(self._handle()))

    def memory_usage(self) -> int:
        return int(lib().rts_memory_usage(self._handle()))

    def PrintMemoryUsage(self) -> None:
        print(f"Index {self.memory_usage() / 2**20:.1f} MB")


def _batch_array(batches):
    arr = (L.rts_batch * len(batches))()
    keep = []
    for i, (pred, q, handler, arg) in enumerate(batches):
        is_pt = q.dim() == 2 and q.shape[1] == 2
        f64 = q.dtype == torch.float64
        q = _f32(q, 2 if is_pt else 4, "queries", torch.float64 if f64 else torch.float32)
        keep.append(q)
        if f64:
            arr[i].query_kind = L.RTS_QUERY_POINTS_F64 if is_pt else L.RTS_QUERY_ENVELOPES_F64
        else:
            arr[i].query_kind = L.RTS_QUERY_POINTS if is_pt else L.RTS_QUERY_ENVELOPES
        arr[i].predicate = int(pred)
        arr[i].queries = q.data_ptr()
        arr[i].n = q.shape[0]
        arr[i].handler = int(handler)
        arr[i].arg = arg
    return arr, keep


class Plan:
    """Prepared batched launch (``rts_plan_create/launch/destroy``)."""

    def __init__(self, index: "SpatialIndex", batches: Sequence[tuple]):
        self.index = index
        arr, self._keep = _batch_array(batches)
        self._h = ctypes.c_void_p()
        check(lib().rts_plan_create(index._handle(), arr, len(batches), ctypes.byref(self._h)))

    def launch(self, stream=None, graph: bool = True) -> None:
        check(lib().rts_plan_launch(self._h, _stream_handle(stream), 1 if graph else 0))

    def close(self) -> None:
        if self._h:
            lib().rts_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sort_pairs(p: torch.Tensor) -> torch.Tensor:
    """Canonical order of a (R, 2) (geom_id, query_id) tensor: by query, then
    geom (the order the CPU oracle emits)."""
    if p.numel() == 0:
        return p.reshape(0, 2)
    key = p[:, 1] * (1 << 32) + p[:, 0]
    return p[torch.argsort(key)]


def memory_pool_stats(device: int | None = None) -> tuple:
    """(reserved, used) bytes of the library's device-memory pool on `device`
    (default: the current CUDA device)."""
    dev = torch.cuda.current_device() if device is None else int(device)
    r, u = ctypes.c_uint64(), ctypes.c_uint64()
    check(lib().rts_memory_pool_stats(dev, ctypes.byref(r), ctypes.byref(u)))
    return int(r.value), int(u.value)


def trim_memory(device: int | None = None) -> None:
    """Returns the unused part of the library's pool on `device` to the driver."""
    dev = torch.cuda.current_device() if device is None else int(device)
    check(lib().rts_trim_memory(dev))
