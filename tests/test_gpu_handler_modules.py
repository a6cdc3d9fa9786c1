"""User device handlers: the reference's plugin boundary.

The reference compiles its query shaders with the user's handler header
force-included (CMakeLists.txt:73-104) and calls rtspatial_handle_{point_contains,
envelope_contains, envelope_intersects}(geom_id, query_id, arg) once per pair.
Here a handler module is compiled from the same kind of header (the compile of
RTSPATIAL_COMPILE_SHADERS, run by tests/cpp/Makefile) and loaded into an
index.  These tests check, against the oracle, that every pair reaches the
right handler exactly once, for every node width, predicate, launch form
(single, batched, prepared graph) and a double index; that the C++ drop-in
loads the module from Config::ptx_root and runs a custom (histogram) handler;
that the shipped counting and collecting headers select the library's own
handlers; and that misuse is refused with a clear error.
"""
import os
import subprocess

import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT
from rtspatial_b200 import _lib as L
from rtspatial_b200 import workloads as wl

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
CPP = os.path.join(HERE, "cpp")
MODULES = os.path.join(CPP, "_build", "modules")
P = rb.Predicate


@pytest.fixture(scope="module")
def built():
    subprocess.check_call(["make", "-s", "-C", CPP])
    return MODULES


def module(built, name):
    return os.path.join(built, name, "rtspatial_handlers.cubin")


class PairSink:
    """Device struct of handlers/pair_append_handlers.h: {uint32* pairs;
    u64 capacity; u64* size; u64* calls[4]}."""

    def __init__(self, capacity):
        self.pairs = torch.zeros((max(capacity, 1), 2), dtype=torch.int32, device="cuda")
        self.size = torch.zeros(1, dtype=torch.int64, device="cuda")
        self.calls = torch.zeros(4, dtype=torch.int64, device="cuda")
        self.obj = torch.tensor([self.pairs.data_ptr(), capacity, self.size.data_ptr(),
                                 self.calls.data_ptr()], dtype=torch.int64, device="cuda")

    def arg(self) -> int:
        return self.obj.data_ptr()

    def canon(self) -> np.ndarray:
        torch.cuda.synchronize()
        n = int(self.size.item())
        assert n <= self.pairs.shape[0]
        p = self.pairs[:n].cpu().numpy().view(np.uint32).astype(np.uint64)
        return p[np.lexsort((p[:, 0], p[:, 1]))].astype(np.uint32)


def _scene(seed=11):
    rng = np.random.default_rng(seed)
    boxes = wl.uniform_boxes(rng, 60_000, 2e-2)
    pts = wl.uniform_points(rng, 3000)
    qs = wl.uniform_boxes(rng, 3000, 2e-2)
    qs[:200] = boxes[100:300]  # identical to stored boxes
    return boxes, pts, qs


CASES = [(KIND_POINT, P.kContains, "pts", 0), (KIND_CONTAINS, P.kContains, "qs", 1),
         (KIND_INTERSECTS, P.kIntersects, "qs", 2)]


@pytest.mark.parametrize("w", [4, 8, 16, 32])
def test_every_pair_reaches_its_handler_once(cuda, oracle, built, w):
    boxes, pts, qs = _scene()
    ix = rb.SpatialIndex(rb.Config(node_width=w))
    ix.Insert(torch.from_numpy(boxes).cuda())
    ix.load_handler_module(module(built, "pairs"))
    assert ix.handler_module_builtin() == -1
    q = {"pts": pts, "qs": qs}
    for kind, pred, qn, which in CASES:
        want = oracle.run(kind, boxes, q[qn])[2]
        sink = PairSink(want.shape[0] + 16)
        ix.Query(pred, torch.from_numpy(q[qn]).cuda(), sink.arg(), handler=rb.Handler.MODULE)
        got = sink.canon()
        assert np.array_equal(got, want), (w, kind, got.shape, want.shape)
        calls = sink.calls.cpu().numpy()
        assert calls[which] == want.shape[0] and calls.sum() == want.shape[0], calls
    assert ix.device_status() == 0


def test_batched_and_prepared_launches_with_a_module(cuda, oracle, built):
    boxes, pts, qs = _scene(12)
    ix = rb.SpatialIndex(rb.Config(node_width=16, sort_queries=1))
    ix.Insert(torch.from_numpy(boxes).cuda())
    ix.load_handler_module(module(built, "pairs"))
    dq, dp = torch.from_numpy(qs).cuda(), torch.from_numpy(pts).cuda()
    specs = [(P.kIntersects, dq[:1500], KIND_INTERSECTS, qs[:1500]),
             (P.kContains, dp, KIND_POINT, pts),
             (P.kContains, dq[1500:], KIND_CONTAINS, qs[1500:])]
    wants = [oracle.run(k, boxes, h)[2] for _, _, k, h in specs]
    for form in ("batched", "plan-graph", "plan"):
        sinks = [PairSink(w.shape[0] + 16) for w in wants]
        batches = [(p, d, rb.Handler.MODULE, s.arg()) for (p, d, _, _), s in zip(specs, sinks)]
        if form == "batched":
            ix.query_batched(batches)
        else:
            plan = ix.plan(batches)
            plan.launch(graph=(form == "plan-graph"))
            torch.cuda.synchronize()
            plan.close()
        for i, (s, w) in enumerate(zip(sinks, wants)):
            assert np.array_equal(s.canon(), w), (form, i)


@pytest.mark.parametrize("t", [L.RTS_TRAVERSAL_THREAD, L.RTS_TRAVERSAL_PACKET])
def test_double_index_calls_the_module_with_double_results(cuda, oracle, built, t):
    boxes, pts, qs = _scene(13)
    b64, p64, q64 = (a.astype(np.float64) + 1e-9 for a in (boxes, pts, qs))
    ix = rb.SpatialIndex(rb.Config(node_width=16, traversal=t, coord_bits=64))
    ix.Insert(torch.from_numpy(b64).cuda())
    ix.load_handler_module(module(built, "pairs"))
    for kind, pred, q in ((KIND_POINT, P.kContains, p64), (KIND_CONTAINS, P.kContains, q64),
                          (KIND_INTERSECTS, P.kIntersects, q64)):
        want = oracle.run64(kind, b64, q)[2]
        sink = PairSink(want.shape[0] + 16)
        ix.Query(pred, torch.from_numpy(q).cuda(), sink.arg(), handler=rb.Handler.MODULE)
        assert np.array_equal(sink.canon(), want), kind


def test_cpp_dropin_loads_the_module_from_ptx_root(cuda, oracle, built, tmp_path):
    """tests/cpp/test_user_handlers.cu: Config::ptx_root -> Init loads the
    histogram module; per-query counts and geom-id sums equal the oracle's,
    on SpatialIndex<float, 2> and <double, 2>."""
    out = tmp_path / "hist.bin"
    exe = os.path.join(CPP, "_build", "test_user_handlers")
    r = subprocess.run([exe, os.path.join(built, "hist"), str(out)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = out.read_bytes()
    boxes = oracle.uniform_boxes(100000, 0.01, 0.01)
    pts = oracle.uniform_points(2000)
    qs = oracle.uniform_boxes(2000, 0.02, 0.02)
    off = 0
    for f64 in (False, True):
        for kind, q in ((KIND_POINT, pts), (KIND_CONTAINS, qs), (KIND_INTERSECTS, qs)):
            n = int(np.frombuffer(raw, np.uint64, 1, off)[0])
            off += 8
            cnt = np.frombuffer(raw, np.uint32, n, off)
            off += 4 * n
            ids = np.frombuffer(raw, np.uint64, n, off)
            off += 8 * n
            if f64:
                _t, want_c, pairs = oracle.run64(kind, boxes.astype(np.float64), q.astype(np.float64))
            else:
                _t, want_c, pairs = oracle.run(kind, boxes, q)
            want_s = np.zeros(n, np.uint64)
            np.add.at(want_s, pairs[:, 1].astype(np.int64), pairs[:, 0].astype(np.uint64))
            assert n == q.shape[0] and want_c.sum() > 0
            assert np.array_equal(cnt, want_c.astype(np.uint32)), (f64, kind)
            assert np.array_equal(ids, want_s), (f64, kind)
    assert off == len(raw)


def test_shipped_headers_run_the_builtin_handlers(cuda, oracle, built):
    boxes, pts, qs = _scene(14)
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(torch.from_numpy(boxes).cuda())
    ix.load_handler_module(module(built, "collect"))
    assert ix.handler_module_builtin() == L.RTS_HANDLER_COLLECT
    want = oracle.run(KIND_INTERSECTS, boxes, qs)[2]
    qu = rb.Queue(want.shape[0] + 16)
    ix.Query(P.kIntersects, torch.from_numpy(qs).cuda(), qu.DeviceObject(),
             handler=rb.Handler.MODULE)
    got = rb.sort_pairs(qu.result()).cpu().numpy().astype(np.uint32)
    assert np.array_equal(got, want)
    ix.load_handler_module(module(built, "count"))  # replaces the collecting module
    assert ix.handler_module_builtin() == L.RTS_HANDLER_COUNT
    c = rb.Counter()
    ix.Query(P.kContains, torch.from_numpy(pts).cuda(), c.data(), handler=rb.Handler.MODULE)
    assert c.get() == oracle.run(KIND_POINT, boxes, pts)[0]


def test_module_misuse_is_refused(cuda, built, tmp_path):
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(torch.from_numpy(wl.uniform_boxes(np.random.default_rng(1), 1000, 0.1)).cuda())
    lib = L.lib()
    pts = torch.rand((10, 2), device="cuda")
    sink = PairSink(64)
    # MODULE handler before any module is loaded
    with pytest.raises(RuntimeError, match="without a loaded handler module"):
        ix.Query(P.kContains, pts, sink.arg(), handler=rb.Handler.MODULE)
    # files that are not handler modules
    junk = tmp_path / "junk.cubin"
    junk.write_bytes(b"not a cubin")
    assert lib.rts_load_handler_module(ix._h, str(junk).encode()) == L.RTS_ERR_INVALID_ARGUMENT
    assert lib.rts_load_handler_module(ix._h, os.path.join(built, "foreign.cubin").encode()) == \
        L.RTS_ERR_INVALID_ARGUMENT
    assert b"rts_module_abi_version" in lib.rts_last_error()
    # a module and a built-in handler in one launch
    ix.load_handler_module(module(built, "pairs"))
    c = rb.Counter()
    with pytest.raises(RuntimeError, match="in one launch"):
        ix.query_batched([(P.kContains, pts, rb.Handler.MODULE, sink.arg()),
                          (P.kContains, pts, rb.Handler.COUNT, c.data())])
    # still usable afterwards
    ix.Query(P.kContains, pts, sink.arg(), handler=rb.Handler.MODULE)
    torch.cuda.synchronize()
    assert ix.device_status() == 0
