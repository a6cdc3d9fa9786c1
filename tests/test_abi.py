"""CPU checks of the C-ABI surface: the library loads, exports every symbol
the header declares, its structs have the layout the header defines (and the
reference's types imply), and argument validation needs no GPU."""
import ctypes
import os
import re
import subprocess

import pytest

import rtspatial_b200
from rtspatial_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rtspatial_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rts_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(L.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.SIGNATURES), set(names) ^ set(L.SIGNATURES)


def test_struct_layout_matches_header(tmp_path):
    prog = tmp_path / "layout.c"
    prog.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "rtspatial_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(rts_config), sizeof(rts_queue), sizeof(rts_pair),
         sizeof(rts_update_entry), sizeof(rts_batch));
  printf("%zu %zu %zu %zu\n", offsetof(rts_update_entry, min_x), offsetof(rts_queue, size),
         offsetof(rts_batch, arg), offsetof(rts_config, chunk));
  printf("%zu %zu %zu\n", sizeof(rts_update_entry_f64), offsetof(rts_update_entry_f64, min_x),
         offsetof(rts_config, coord_bits));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(prog),
                           "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split()
    sizes = list(map(int, out))
    assert sizes[:5] == [ctypes.sizeof(L.rts_config), ctypes.sizeof(L.rts_queue), 8,
                         ctypes.sizeof(L.rts_update_entry), ctypes.sizeof(L.rts_batch)]
    # thrust::pair<size_t, Envelope<Point<float,2>>>: 8-byte id then 16 bytes
    assert sizes[3] == 24 and sizes[5] == 8
    # dev::Queue<pair<uint32,uint32>>: {T* data; size_t size;} then uint32_t* last_pos
    assert sizes[1] == 24 and sizes[6] == 16
    assert sizes[7] == L.rts_batch.arg.offset
    assert sizes[8] == L.rts_config.chunk.offset
    # thrust::pair<size_t, Envelope<Point<double,2>>>: 8-byte id then 32 bytes
    assert sizes[9] == 40 == ctypes.sizeof(L.rts_update_entry_f64) and sizes[10] == 8
    assert sizes[11] == L.rts_config.coord_bits.offset


def test_config_defaults_follow_reference():
    c = L.rts_config()
    assert L.lib().rts_config_default(ctypes.byref(c)) == 0
    # rtspatial::Config (spatial_index.cuh:22-37)
    assert c.max_geometries == 10_000_000 and c.max_queries == 1_000_000
    assert c.preallocate == 0 and c.compact == 0
    assert abs(c.geom_sample_rate - 0.2) < 1e-7 and abs(c.intersect_cost_weight - 0.95) < 1e-7
    assert c.max_geom_samples == 10000 and c.max_query_samples == 1000
    assert c.max_parallelism == 512
    assert c.node_width in (4, 8, 16, 32)


def test_argument_validation_without_gpu():
    lib = L.lib()
    c = L.rts_config()
    lib.rts_config_default(ctypes.byref(c))
    h = ctypes.c_void_p()
    c.node_width = 5
    assert lib.rts_create(ctypes.byref(c), ctypes.byref(h)) == L.RTS_ERR_INVALID_ARGUMENT
    assert b"node_width" in lib.rts_last_error()
    c.node_width = 8
    c.max_trees = 0
    assert lib.rts_create(ctypes.byref(c), ctypes.byref(h)) == L.RTS_ERR_INVALID_ARGUMENT
    c.max_trees = 8
    # every traversal scheme the header defines is accepted at creation
    for t in (L.RTS_TRAVERSAL_AUTO, L.RTS_TRAVERSAL_THREAD, L.RTS_TRAVERSAL_TEAM,
              L.RTS_TRAVERSAL_FRONTIER, L.RTS_TRAVERSAL_PACKET, L.RTS_TRAVERSAL_STAGED):
        c.traversal = t
        h2 = ctypes.c_void_p()
        assert lib.rts_create(ctypes.byref(c), ctypes.byref(h2)) == L.RTS_OK, t
        lib.rts_destroy(h2)
    c.traversal = 9
    assert lib.rts_create(ctypes.byref(c), ctypes.byref(h)) == L.RTS_ERR_INVALID_ARGUMENT
    c.traversal = L.RTS_TRAVERSAL_AUTO
    # the L1 policy of the group loads: auto, cached, streaming
    for gl in (L.RTS_LOADS_AUTO, L.RTS_LOADS_CACHED, L.RTS_LOADS_STREAMING):
        c.group_loads = gl
        h2 = ctypes.c_void_p()
        assert lib.rts_create(ctypes.byref(c), ctypes.byref(h2)) == L.RTS_OK, gl
        lib.rts_destroy(h2)
    c.group_loads = 3
    assert lib.rts_create(ctypes.byref(c), ctypes.byref(h)) == L.RTS_ERR_INVALID_ARGUMENT
    assert b"group_loads" in lib.rts_last_error()
    c.group_loads = L.RTS_LOADS_AUTO
    assert lib.rts_create(ctypes.byref(c), ctypes.byref(h)) == L.RTS_OK
    try:
        assert lib.rts_size(h) == 0 and lib.rts_num_trees(h) == 0
        dummy = ctypes.c_uint64(0)
        # points only support kContains (spatial_index.cuh:387-389 aborts; we return)
        assert lib.rts_query_points(h, L.RTS_PREDICATE_INTERSECTS, None, 0, L.RTS_HANDLER_COUNT,
                                    ctypes.addressof(dummy), None) == L.RTS_ERR_INVALID_ARGUMENT
        assert lib.rts_query_envelopes(h, 7, None, 0, L.RTS_HANDLER_COUNT,
                                       ctypes.addressof(dummy), None) == L.RTS_ERR_INVALID_ARGUMENT
        assert lib.rts_query_envelopes(h, L.RTS_PREDICATE_CONTAINS, None, 0, 9,
                                       ctypes.addressof(dummy), None) == L.RTS_ERR_INVALID_ARGUMENT
        assert lib.rts_query_envelopes(h, L.RTS_PREDICATE_CONTAINS, None, 0, L.RTS_HANDLER_COUNT,
                                       None, None) == L.RTS_ERR_INVALID_ARGUMENT
        # empty inputs are no-ops (spatial_index.cuh:144-146, :354-356)
        assert lib.rts_insert(h, None, 0, None) == L.RTS_OK
        assert lib.rts_query_envelopes(h, L.RTS_PREDICATE_CONTAINS, None, 0, L.RTS_HANDLER_COUNT,
                                       ctypes.addressof(dummy), None) == L.RTS_OK
        assert lib.rts_delete(h, None, 0, None) == L.RTS_OK
        assert lib.rts_update(h, None, 0, None) == L.RTS_OK
        assert lib.rts_query_batched(h, None, 0, None) == L.RTS_OK
    finally:
        assert lib.rts_destroy(h) == L.RTS_OK
    assert lib.rts_insert(None, None, 0, None) == L.RTS_ERR_INVALID_ARGUMENT


def test_memory_calls_without_gpu():
    # the library's device memory: without a GPU nothing was allocated in this
    # process, so the stats read zero and a trim has nothing to return; bad
    # arguments are refused
    import torch
    lib = L.lib()
    r, u = ctypes.c_uint64(7), ctypes.c_uint64(7)
    assert lib.rts_memory_pool_stats(0, ctypes.byref(r), ctypes.byref(u)) == L.RTS_OK
    assert r.value >= u.value
    if not torch.cuda.is_available():
        assert r.value == 0 and u.value == 0
        assert lib.rts_trim_memory(0) == L.RTS_OK
    assert lib.rts_memory_pool_stats(-1, ctypes.byref(r), ctypes.byref(u)) == \
        L.RTS_ERR_INVALID_ARGUMENT
    assert lib.rts_memory_pool_stats(0, None, ctypes.byref(u)) == L.RTS_ERR_INVALID_ARGUMENT
    assert lib.rts_trim_memory(64) == L.RTS_ERR_INVALID_ARGUMENT


def test_python_mirror_surface():
    # names of rtspatial::SpatialIndex's public methods
    for m in ("Init", "Clear", "Insert", "Delete", "Update", "Query", "PrintMemoryUsage"):
        assert hasattr(rtspatial_b200.SpatialIndex, m)
    assert int(rtspatial_b200.Predicate.kIntersects) == 0
    assert int(rtspatial_b200.Predicate.kContains) == 1
