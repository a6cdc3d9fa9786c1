"""rtspatial_b200 — B200-native spatial index with the interface of
``rtspatial::SpatialIndex<float, 2>``.

The index, its build/refit kernels and its query kernels live in the CUDA
library ``librtspatial_b200.so`` (C-ABI in ``include/rtspatial_b200.h``);
this package is the host-side mirror used from Python.  Importing it does not
require a GPU; using an index does, and fails loudly if the library is
missing.
"""
from ._lib import LIB_PATH, RtsError, lib  # noqa: F401
from .spatial_index import (  # noqa: F401
    Config,
    Counter,
    Handler,
    Plan,
    Predicate,
    Queue,
    SpatialIndex,
    memory_pool_stats,
    sort_pairs,
    trim_memory,
)
from .server import Server  # noqa: F401

__all__ = ["Config", "Counter", "Handler", "Plan", "Predicate", "Queue", "SpatialIndex", "sort_pairs",
           "memory_pool_stats", "trim_memory", "RtsError", "lib", "LIB_PATH", "Server"]
