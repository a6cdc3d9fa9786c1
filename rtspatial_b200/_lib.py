"""Loads ``librtspatial_b200.so`` and declares the C-ABI of
``include/rtspatial_b200.h`` for ctypes.

The library must exist: there is no fallback implementation.  Build it with
``python -m rtspatial_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librtspatial_b200.so")

RTS_OK = 0
RTS_ERR_INVALID_ARGUMENT = 1
RTS_ERR_CUDA = 2
RTS_ERR_OUT_OF_MEMORY = 3
RTS_ERR_QUEUE_FULL = 4
RTS_ERR_CAPACITY = 5
RTS_ERR_UNSUPPORTED = 6
RTS_ERR_TIMEOUT = 7

RTS_PREDICATE_INTERSECTS = 0
RTS_PREDICATE_CONTAINS = 1
RTS_HANDLER_COUNT = 0
RTS_HANDLER_COLLECT = 1
RTS_HANDLER_MODULE = 2
RTS_TRAVERSAL_AUTO = 0
RTS_TRAVERSAL_THREAD = 1
RTS_TRAVERSAL_TEAM = 2
RTS_TRAVERSAL_FRONTIER = 3
RTS_TRAVERSAL_PACKET = 4
RTS_TRAVERSAL_STAGED = 5
RTS_LOADS_AUTO = 0
RTS_LOADS_CACHED = 1
RTS_LOADS_STREAMING = 2
RTS_STATUS_WAIT_TIMEOUT = 1
RTS_CURVE_MORTON = 0
RTS_CURVE_HILBERT = 1
RTS_QUERY_POINTS = 0
RTS_QUERY_ENVELOPES = 1
RTS_QUERY_POINTS_F64 = 2
RTS_QUERY_ENVELOPES_F64 = 3
RTS_NOALLOC_MAX_BATCHES = 1024


class rts_config(ctypes.Structure):
    _fields_ = [
        ("max_geometries", ctypes.c_uint64),
        ("max_queries", ctypes.c_uint64),
        ("preallocate", ctypes.c_int32),
        ("prefer_fast_build_geom", ctypes.c_int32),
        ("prefer_fast_build_query", ctypes.c_int32),
        ("compact", ctypes.c_int32),
        ("geom_sample_rate", ctypes.c_float),
        ("query_sample_rate", ctypes.c_float),
        ("intersect_cost_weight", ctypes.c_float),
        ("max_geom_samples", ctypes.c_uint32),
        ("max_query_samples", ctypes.c_uint32),
        ("max_parallelism", ctypes.c_uint32),
        ("node_width", ctypes.c_int32),
        ("traversal", ctypes.c_int32),
        ("curve", ctypes.c_int32),
        ("max_trees", ctypes.c_int32),
        ("rebuild_fraction", ctypes.c_float),
        ("sort_queries", ctypes.c_int32),
        ("rebuild_update_fraction", ctypes.c_float),
        ("chunk", ctypes.c_uint32),
        ("query_occupancy", ctypes.c_int32),
        ("frontier_factor", ctypes.c_float),
        ("coord_bits", ctypes.c_int32),
        ("group_loads", ctypes.c_int32),
    ]


class rts_queue(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("capacity", ctypes.c_uint64), ("size", ctypes.c_void_p)]


class rts_update_entry(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("min_x", ctypes.c_float), ("min_y", ctypes.c_float),
                ("max_x", ctypes.c_float), ("max_y", ctypes.c_float)]


class rts_update_entry_f64(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("min_x", ctypes.c_double), ("min_y", ctypes.c_double),
                ("max_x", ctypes.c_double), ("max_y", ctypes.c_double)]


class rts_batch(ctypes.Structure):
    _fields_ = [
        ("query_kind", ctypes.c_int32),
        ("predicate", ctypes.c_int32),
        ("queries", ctypes.c_void_p),
        ("n", ctypes.c_uint64),
        ("handler", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("arg", ctypes.c_void_p),
    ]


class rts_server_config(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_uint32), ("max_parts_per_launch", ctypes.c_uint32),
                ("max_queries_per_launch", ctypes.c_uint64), ("pairs_per_launch", ctypes.c_uint64),
                ("hbm_budget_bytes", ctypes.c_uint64), ("host_result_bytes", ctypes.c_uint64),
                ("use_graphs", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class rts_server_stats(ctypes.Structure):
    _fields_ = [("requests_done", ctypes.c_uint64), ("queries_done", ctypes.c_uint64),
                ("pairs_done", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("retried_parts", ctypes.c_uint64), ("updates_done", ctypes.c_uint64),
                ("latency_p50_s", ctypes.c_double), ("latency_p99_s", ctypes.c_double),
                ("latency_max_s", ctypes.c_double), ("elapsed_s", ctypes.c_double),
                ("pack_s", ctypes.c_double), ("launch_s", ctypes.c_double),
                ("copy_s", ctypes.c_double), ("take_s", ctypes.c_double),
                ("update_s", ctypes.c_double), ("parts", ctypes.c_uint64),
                ("graph_launches", ctypes.c_uint64), ("issue_s", ctypes.c_double)]


class rts_tune_result(ctypes.Structure):
    _fields_ = [("node_width", ctypes.c_int32), ("traversal", ctypes.c_int32),
                ("query_occupancy", ctypes.c_int32), ("sort_queries", ctypes.c_int32),
                ("chunk", ctypes.c_uint32), ("candidates", ctypes.c_uint32),
                ("collecting", ctypes.c_int32), ("group_loads", ctypes.c_int32),
                ("best_ms", ctypes.c_double), ("first_ms", ctypes.c_double)]


# name -> (restype, argtypes); every symbol the header declares.
_P = ctypes.c_void_p
_I = ctypes.c_int
_U64 = ctypes.c_uint64
SIGNATURES = {
    "rts_config_default": (_I, [ctypes.POINTER(rts_config)]),
    "rts_create": (_I, [ctypes.POINTER(rts_config), ctypes.POINTER(_P)]),
    "rts_destroy": (_I, [_P]),
    "rts_clear": (_I, [_P, _P]),
    "rts_insert": (_I, [_P, _P, _U64, _P]),
    "rts_delete": (_I, [_P, _P, _U64, _P]),
    "rts_update": (_I, [_P, _P, _U64, _P]),
    "rts_query_points": (_I, [_P, _I, _P, _U64, _I, _P, _P]),
    "rts_query_envelopes": (_I, [_P, _I, _P, _U64, _I, _P, _P]),
    "rts_insert_f64": (_I, [_P, _P, _U64, _P]),
    "rts_update_f64": (_I, [_P, _P, _U64, _P]),
    "rts_query_points_f64": (_I, [_P, _I, _P, _U64, _I, _P, _P]),
    "rts_query_envelopes_f64": (_I, [_P, _I, _P, _U64, _I, _P, _P]),
    "rts_query_batched": (_I, [_P, ctypes.POINTER(rts_batch), ctypes.c_uint32, _P]),
    "rts_query_batched_noalloc": (_I, [_P, ctypes.POINTER(rts_batch), ctypes.c_uint32, _P]),
    "rts_device_status": (_I, [_P, ctypes.POINTER(ctypes.c_uint32), _P]),
    "rts_load_handler_module": (_I, [_P, ctypes.c_char_p]),
    "rts_handler_module_builtin": (_I, [_P]),
    "rts_plan_create": (_I, [_P, ctypes.POINTER(rts_batch), ctypes.c_uint32, ctypes.POINTER(_P)]),
    "rts_plan_launch": (_I, [_P, _P, _I]),
    "rts_plan_destroy": (_I, [_P]),
    "rts_server_config_default": (_I, [ctypes.POINTER(rts_server_config)]),
    "rts_server_create": (_I, [_P, ctypes.POINTER(rts_server_config), ctypes.POINTER(_P)]),
    "rts_server_destroy": (_I, [_P]),
    "rts_server_submit_query": (_I, [_P, _I, _I, _P, _U64, ctypes.POINTER(_U64)]),
    "rts_server_submit_update": (_I, [_P, _P, _U64, _P, _U64, _P, _U64, ctypes.POINTER(_U64)]),
    "rts_server_wait": (_I, [_P, _U64, ctypes.c_double]),
    "rts_server_take": (_I, [_P, _U64, _P, _U64, ctypes.POINTER(_U64)]),
    "rts_server_view": (_I, [_P, _U64, ctypes.POINTER(_P), ctypes.POINTER(_U64), ctypes.c_uint32,
                             ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(_U64)]),
    "rts_server_release": (_I, [_P, _U64]),
    "rts_server_get_stats": (_I, [_P, ctypes.POINTER(rts_server_stats)]),
    "rts_server_reset_stats": (_I, [_P]),
    "rts_autotune": (_I, [_P, ctypes.POINTER(rts_batch), ctypes.c_uint32, _I, _P,
                          ctypes.POINTER(rts_tune_result)]),
    "rts_report_query_time": (_I, [_P, ctypes.c_double, ctypes.POINTER(ctypes.c_float)]),
    "rts_size": (_U64, [_P]),
    "rts_num_trees": (ctypes.c_uint32, [_P]),
    "rts_memory_usage": (_U64, [_P]),
    "rts_memory_pool_stats": (_I, [_I, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]),
    "rts_trim_memory": (_I, [_I]),
    "rts_last_error": (ctypes.c_char_p, []),
    "rts_version": (ctypes.c_char_p, []),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"rtspatial_b200: CUDA library not built ({LIB_PATH}); "
                "run `python -m rtspatial_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class RtsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"rtspatial_b200 error {code}: {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != RTS_OK:
        raise RtsError(rc, lib().rts_last_error().decode(errors="replace"))
