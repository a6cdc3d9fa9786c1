"""Benchmark of the hot path: SpatialIndex::Query on the B200 library.

Default workload (the headline: the configuration quoted as batched vs plain
one-launch-per-batch): range-contains, float32 2-D, 10M boxes from 64
Gaussian clusters, 1M query boxes split into 256 log-uniform batches
(1K-16K) run in ONE persistent launch (rts_query_batched), collecting handler
(pairs written to per-batch device queues).  One step = all 256 batches once.

Printed on rank 0 as one JSON line:
  value        queries/s of the batched launch, inputs resident in HBM, L2
               flushed before every timed step (CUDA events per step)
  forms.plain  the same batches as 256 separate launches (one per batch)
  e2e          queries/s through the same C-ABI call with host buffers:
               pinned H2D of the queries and D2H of every result pair inside
               the timed region
  roofline     algorithmic bytes per launch / launch time vs measured HBM peak
  cpu_baseline CPU oracle (grid filter + the reference's predicates) on the
               host cores over a bounded sample of the same queries
  parity       after timing: per-batch pair counts and order-independent pair
               digests of the last timed launch against the oracle over the
               same inputs, at full size (a mismatch exits non-zero)
  clocks       nvidia-smi samples taken during warm-up + timed steps
  other_configs  (default run, one GPU) reduced runs of configurations 1, 3,
               4 and 5 with the same keys, each checked against the oracle

Queue capacities are sized exactly by a counting pass before timing (the
reference's contract: the caller sizes the queue); `sizing_pass` reports
that pass's own time, which a caller with unknown output sizes pays on top.

--impl reference times the reference's CPU implementation of the path (the
reference's own predicate code compiled for the host, under the same grid
filter; the restated oracle when that build is absent) with all host threads.

Multi-GPU (torchrun): every rank holds a replica of the index and runs its own
query set (weak scaling, no data-path collective); times are the max over
ranks.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "queries/s & result pairs/s (batched/served vs plain, bit-exact); p50/p99 latency"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--scale", type=float, default=1.0, help="scales boxes and queries (profiling)")
    ap.add_argument("--node-width", type=int, default=0)
    ap.add_argument("--traversal", type=int, default=-1)
    ap.add_argument("--curve", type=int, default=-1)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--max-trees", type=int, default=0, help="sub-trees before a merge (0: library default)")
    ap.add_argument("--sort", type=int, default=-1, help="sort_queries: 0 never, 1 always, 2 auto")
    ap.add_argument("--occupancy", type=int, default=-1)
    ap.add_argument("--group-loads", type=int, default=-1,
                    help="L1 use of the group loads: 0 auto, 1 cached, 2 streaming")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-others", action="store_true",
                    help="default run only: skip the reduced runs of configs 1, 3, 4, 5")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the full-size comparison with the oracle after timing")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch settings")
    ap.add_argument("--rounds", type=int, default=0,
                    help="config 4: mutation rounds (default 50, the configuration's)")
    ap.add_argument("--rounds-out", default="",
                    help="config 4: write each timed round's times and sub-tree count to this "
                         "JSON file")
    ap.add_argument("--requests", type=int, default=600, help="config 5: requests per run")
    ap.add_argument("--no-graphs", action="store_true",
                    help="config 5: the server issues its launches directly (no graph replay)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def make_workload(cfg: int, scale: float, rank: int):
    from rtspatial_b200 import workloads as wl
    if cfg == 2:
        nb, nq = int(10_000_000 * scale), int(1_000_000 * scale)
        boxes, queries, sizes = wl.config2(seed=42, n_boxes=nb, n_queries=nq)
        if rank:
            rng = np.random.default_rng(1000 + rank)
            queries = wl.uniform_boxes(rng, nq, 1e-3)
            sizes = wl.log_uniform_sizes(rng, 256, 1024, 16384, nq)
        desc = (f"range-contains: {nb} boxes (64 Gaussian clusters, sigma 0.02, sides U[0,5e-3]) x "
                f"{nq} query boxes (uniform, sides U[0,1e-3]) in 256 log-uniform batches "
                f"[1K,16K], one persistent launch, collecting handler")
        return dict(kind="contains", pred=1, boxes=boxes, queries=queries, sizes=sizes, desc=desc,
                    qwidth=4)
    if cfg == 1:
        nb, nq = int(1_000_000 * scale), int(100_000 * scale)
        boxes, pts = wl.config1(seed=42, n_boxes=nb, n_points=nq)
        if rank:
            pts = wl.uniform_points(np.random.default_rng(1000 + rank), nq)
        desc = (f"point-contains: {nb} boxes (uniform, sides U[0,1e-3]) x {nq} points, "
                f"one launch, collecting handler")
        return dict(kind="point", pred=1, boxes=boxes, queries=pts,
                    sizes=np.array([nq], dtype=np.int64), desc=desc, qwidth=2)
    if cfg == 4:
        nb, nq = int(20_000_000 * scale), int(1_000_000 * scale)
        boxes = wl.config4_base(seed=42, n_boxes=nb)
        pts = wl.uniform_points(np.random.default_rng(1000 + rank), nq)
        desc = f"mutable-index round queries: {nb} boxes (sides U[0,1e-3]) x {nq} points"
        return dict(kind="point", pred=1, boxes=boxes, queries=pts,
                    sizes=np.array([nq], dtype=np.int64), desc=desc, qwidth=2)
    if cfg == 5:
        nb, nq = int(50_000_000 * scale), int(1_000_000 * scale)
        boxes = wl.config5_boxes(seed=42, n_boxes=nb)
        queries = wl.uniform_boxes(np.random.default_rng(1000 + rank), nq, 1e-3)
        desc = f"serving mix proxy: {nb} resident boxes x {nq} range-contains queries"
        return dict(kind="contains", pred=1, boxes=boxes, queries=queries,
                    sizes=np.array([nq], dtype=np.int64), desc=desc, qwidth=4)
    nb, nq = int(10_000_000 * scale), int(1_000_000 * scale)
    boxes, queries = wl.config3(seed=42, n_boxes=nb, n_queries=nq)
    if rank:
        queries = wl.lognormal_boxes(np.random.default_rng(1000 + rank), nq, np.log(5e-4), 1.0)
    desc = (f"range-intersects: {nb} boxes (sides lognormal(ln 1e-4, 1.5) cap 0.05) x {nq} "
            f"queries (lognormal(ln 5e-4, 1.0)), one launch, collecting handler")
    return dict(kind="intersects", pred=0, boxes=boxes, queries=queries,
                sizes=np.array([nq], dtype=np.int64), desc=desc, qwidth=4)


def algorithmic_bytes(w, pairs: int) -> int:
    """Compulsory bytes of one query launch: every indexed box read once
    (16 B), every query read once (8 or 16 B), every pair written (8 B)."""
    return 16 * w["boxes"].shape[0] + 4 * w["qwidth"] * w["queries"].shape[0] + 8 * pairs


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        # the raw samples go to RTS_CLOCKS_DIR (default: the system temp dir);
        # the JSON line carries their summary
        out_dir = os.environ.get("RTS_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"clocks_rank{gpu_index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# CPU legs
# ---------------------------------------------------------------------------
def cpu_query_rate(w, seconds: float, backend: str):
    """Queries/s of the CPU oracle over a bounded prefix of the query set,
    grid prebuilt (index build is not part of the query metric)."""
    from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT, Oracle, available
    if backend == "ref" and not available("ref"):
        backend = "port"
    ora = Oracle(backend)
    kind = {"point": KIND_POINT, "contains": KIND_CONTAINS, "intersects": KIND_INTERSECTS}[w["kind"]]
    boxes = np.ascontiguousarray(w["boxes"])
    qs = np.ascontiguousarray(w["queries"])
    threads = os.cpu_count() or 1
    g = ora.grid_build(boxes, 2.0)
    try:
        n = min(qs.shape[0], 2000)
        while True:
            t0 = time.perf_counter()
            ora.run_on_grid(g, kind, boxes, qs[:n], threads)
            dt = time.perf_counter() - t0
            if dt > seconds / 4 or n >= qs.shape[0]:
                break
            n = min(qs.shape[0], int(n * max(2.0, (seconds / 4) / max(dt, 1e-4))))
        # best of up to 3 repeats of the sized sample
        best = dt
        for _ in range(2):
            t0 = time.perf_counter()
            ora.run_on_grid(g, kind, boxes, qs[:n], threads)
            best = min(best, time.perf_counter() - t0)
    finally:
        ora.grid_free(g)
    kindname = "reference" if backend == "ref" else "port"
    return n / best, n, threads, kindname


def oracle_backend():
    """The checker: the reference's own predicate code compiled for the host
    (oracle/_ref) when that build exists, else the restated oracle."""
    from oracle.oracle import available
    return "ref" if available("ref") else "port"


KINDS = {"point": 0, "contains": 1, "intersects": 2}


def gpu_batch_digests(pairs_h: np.ndarray, counts: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    """Per-batch order-independent digests of GPU results: batch b's pairs
    are rows [offsets[b], offsets[b] + counts[b]) of pairs_h."""
    from oracle.oracle import pair_digest
    return np.array([pair_digest(pairs_h[int(o):int(o) + int(c)]) if c else 0
                     for o, c in zip(offsets, counts)], dtype=np.uint64)


def oracle_batch_check(w, sizes, gpu_counts: np.ndarray, gpu_digests: np.ndarray,
                       boxes=None, queries=None) -> dict:
    """Runs the oracle over the same boxes and queries and compares, batch by
    batch, the pair count and the order-independent digest of the
    (geom_id, query_id) pairs, query ids 0-based within each batch as a
    reference Query call reports them."""
    from oracle.oracle import Oracle
    backend = oracle_backend()
    ora = Oracle(backend)
    boxes = w["boxes"] if boxes is None else boxes
    queries = w["queries"] if queries is None else queries
    sizes = np.asarray(sizes, dtype=np.int64)
    offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    rid = (np.arange(offs[-1], dtype=np.int64) - np.repeat(offs[:-1], sizes)).astype(np.uint32)
    t0 = time.perf_counter()
    total, counts, digests = ora.digest(KINDS[w["kind"]], boxes, queries, rid=rid, grid=True)
    nz = sizes > 0
    want_c = np.zeros(len(sizes), dtype=np.uint64)
    want_d = np.zeros(len(sizes), dtype=np.uint64)
    if nz.any():
        want_c[nz] = np.add.reduceat(counts, offs[:-1][nz])
        want_d[nz] = np.add.reduceat(digests, offs[:-1][nz])
    bad = np.nonzero((want_c != gpu_counts.astype(np.uint64)) |
                     (want_d != gpu_digests.astype(np.uint64)))[0]
    return {"checked": True, "oracle": "reference" if backend == "ref" else "port",
            "pairs": int(total), "gpu_pairs": int(gpu_counts.sum()), "batches": len(sizes),
            "equal": bool(bad.size == 0 and int(gpu_counts.sum()) == total),
            "mismatched_batches": [int(b) for b in bad[:8]],
            "oracle_seconds": time.perf_counter() - t0,
            "what": "per-batch pair counts and order-independent (geom_id, query_id) digests "
                    "vs the oracle on the same inputs"}


def run_reference_arm(args, rank: int, world: int):
    if rank != 0:
        return
    w = make_workload(args.config, args.scale, 0)
    from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT, Oracle, available
    backend = "ref" if available("ref") else "port"
    ora = Oracle(backend)
    kind = {"point": KIND_POINT, "contains": KIND_CONTAINS, "intersects": KIND_INTERSECTS}[w["kind"]]
    boxes, qs = w["boxes"], w["queries"]
    threads = os.cpu_count() or 1
    g = ora.grid_build(boxes, 2.0)
    # size one step to about 1/(steps+warmup) of a few-minute budget
    budget = 90.0 / max(1, args.steps + args.warmup)
    n = min(qs.shape[0], 2000)
    t0 = time.perf_counter()
    ora.run_on_grid(g, kind, boxes, qs[:n], threads)
    dt = time.perf_counter() - t0
    n = int(min(qs.shape[0], max(1000, n * budget / max(dt, 1e-4))))
    for _ in range(args.warmup):
        ora.run_on_grid(g, kind, boxes, qs[:n], threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ora.run_on_grid(g, kind, boxes, qs[:n], threads)
        times.append(time.perf_counter() - t0)
    ora.grid_free(g)
    tot = sum(times)
    rate = n * args.steps / tot
    cores = threads
    kindname = "reference" if backend == "ref" else "port"
    sample = (f"first {n} of {qs.shape[0]} queries per step against all {boxes.shape[0]} boxes; "
              f"{'reference predicate headers compiled for the host' if backend == 'ref' else 'restated predicates'}"
              f" under a uniform-grid filter, OpenMP {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * tot / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": w["desc"]},
        "cpu_baseline": {"value": rate, "unit": "queries/s", "cores": cores, "kind": kindname,
                         "sample": sample},
        "e2e": {"value": rate, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


# ---------------------------------------------------------------------------
# GPU leg
# ---------------------------------------------------------------------------
class Ctx:
    """Rank, device and the timing collectives of one bench process."""

    def __init__(self):
        import torch
        import torch.distributed as dist
        from rtspatial_b200 import replicas
        self.torch, self.dist, self.replicas = torch, dist, replicas
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(self.local)
        self.dev = torch.device("cuda", self.local)
        if self.world > 1:
            from datetime import timedelta
            dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=self.dev)

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, x: float) -> float:
        return self.replicas.max_over_ranks(x, self.dist, self.dev)

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


def make_index(args, rb):
    cfg = rb.Config()
    for k, v in (("node_width", args.node_width), ("chunk", args.chunk),
                 ("max_trees", args.max_trees)):
        if v:
            setattr(cfg, k, v)
    for k, v in (("traversal", args.traversal), ("curve", args.curve), ("sort_queries", args.sort),
                 ("query_occupancy", args.occupancy), ("group_loads", args.group_loads)):
        if v >= 0:
            setattr(cfg, k, v)
    return rb.SpatialIndex(cfg)


def peak_hbm():
    if os.path.exists(PEAKS_FILE):
        with open(PEAKS_FILE) as f:
            peaks = json.load(f)
        if peaks.get("hbm_gbs"):
            return float(peaks["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def run_query_bench(args, ctx):
    """Configs 1-3: batches of one predicate over a static index."""
    torch = ctx.torch
    import rtspatial_b200 as rb
    dev = ctx.dev
    w = make_workload(args.config, args.scale, ctx.rank)
    ix = make_index(args, rb)
    boxes_d = torch.from_numpy(w["boxes"]).to(dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ix.Insert(boxes_d)
    torch.cuda.synchronize()
    build_ms = 1000 * (time.perf_counter() - t0)
    del boxes_d

    queries_d = torch.from_numpy(w["queries"]).to(dev)
    sizes = [int(x) for x in w["sizes"]]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    nbatch, nq = len(sizes), int(offs[-1])
    qslices = [queries_d[offs[i]:offs[i + 1]] for i in range(nbatch)]
    pred = rb.Predicate(w["pred"])

    # size every batch's queue exactly with a counting pass
    counters = torch.zeros(nbatch, dtype=torch.int64, device=dev)
    ix.query_batched([(pred, qslices[i], rb.Handler.COUNT, counters[i:i + 1].data_ptr())
                      for i in range(nbatch)])
    torch.cuda.synchronize()
    per_batch = counters.cpu().numpy().astype(np.int64)
    total_pairs = int(per_batch.sum())
    poffs = np.concatenate([[0], np.cumsum(np.maximum(per_batch, 1))])
    pairs = torch.empty((int(poffs[-1]), 2), dtype=torch.int32, device=dev)
    qsize = torch.zeros(nbatch, dtype=torch.int32, device=dev)
    qobj_host = torch.zeros((nbatch, 3), dtype=torch.int64)
    for i in range(nbatch):
        qobj_host[i, 0] = pairs.data_ptr() + 8 * int(poffs[i])
        qobj_host[i, 1] = max(int(per_batch[i]), 1)
        qobj_host[i, 2] = qsize.data_ptr() + 4 * i
    qobj = qobj_host.to(dev)
    batch_args = [(pred, qslices[i], rb.Handler.COLLECT, qobj[i].data_ptr()) for i in range(nbatch)]

    tune = None
    if not args.no_tune:
        t0 = time.perf_counter()
        tune = ix.autotune(batch_args, tune_width=True)
        tune["seconds"] = time.perf_counter() - t0
    plan = ix.plan(batch_args)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()

    def step_graph():
        qsize.zero_()
        plan.launch(graph=True)

    def step_nograph():
        qsize.zero_()
        plan.launch(graph=False)

    def step_plain():
        qsize.zero_()
        for i in range(nbatch):
            ix.Query(pred, qslices[i], qobj[i].data_ptr(), handler=rb.Handler.COLLECT)

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        ctx.barrier()
        torch.cuda.synchronize()
        for a, b in evs:
            flush.fill_(1.0)
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        ctx.barrier()
        return [a.elapsed_time(b) for a, b in evs]

    def checksum():
        torch.cuda.synchronize()
        p = pairs.to(torch.int64) & 0xFFFFFFFF
        h = (p[:, 0] * 0x9E3779B1 + p[:, 1] * 0x85EBCA77) & 0xFFFFFFFFFFFF
        return int(qsize.sum().item()), int(h.sum().item())

    clocks = ClockSampler(ctx.local)
    clocks.start()
    for _ in range(args.warmup):
        flush.fill_(1.0)
        step_graph()
    cs = checksum()
    if cs[0] != total_pairs:
        raise SystemExit(f"batched launch reported {cs[0]} pairs, counting pass {total_pairs}")
    t_main = timed(step_graph, args.steps)
    clocks_info = clocks.stop()

    # Parity at full size, outside every timed region: the last timed launch's
    # per-batch counts and pair digests against the oracle (rank 0's queries).
    parity = None
    if ctx.rank == 0 and not args.no_parity:
        torch.cuda.synchronize()
        got_c = qsize.cpu().numpy().astype(np.int64) & 0xFFFFFFFF
        pairs_h = pairs.cpu().numpy().view(np.uint32)
        got_d = gpu_batch_digests(pairs_h, np.minimum(got_c, np.maximum(per_batch, 1)),
                                  poffs[:-1])
        parity = oracle_batch_check(w, sizes, got_c, got_d)
        del pairs_h

    forms = {}
    if not args.no_plain:
        # The counting pass that sized the queues, as a prepared launch: what a
        # caller that does not know its output sizes pays before each step.
        count_batches = [(pred, qslices[i], rb.Handler.COUNT, counters[i:i + 1].data_ptr())
                         for i in range(nbatch)]
        count_plan = ix.plan(count_batches)

        def step_count():
            counters.zero_()
            count_plan.launch(graph=True)

        step_count()
        torch.cuda.synchronize()
        if not np.array_equal(counters.cpu().numpy().astype(np.int64), per_batch):
            raise SystemExit("counting launch differs from the sizing pass")
        t = timed(step_count, max(3, args.steps // 2))
        ms = ctx.max(sum(t) / len(t))
        forms["sizing_pass"] = {
            "ms_per_step": ms, "launches_per_step": 1,
            "two_pass_value": nq * ctx.world / ((ms + ctx.max(sum(t_main) / len(t_main))) / 1000),
            "unit": "queries/s",
            "what": "counting launch of the same batches (prepared, graph); two_pass_value = "
                    "queries/s of count-then-collect for callers that size queues per step"}
        count_plan.close()
        form_list = [("batched_no_graph", step_nograph, max(3, args.steps // 2))]
        if nbatch > 1:  # one batch: the plain form is the launch without a graph
            form_list.append(("plain", step_plain, max(3, args.steps // 4)))
        for name, fn, k in form_list:
            fn()
            if checksum() != cs:
                raise SystemExit(f"{name} results differ from the graph launch")
            t = timed(fn, k)
            ms = ctx.max(sum(t) / len(t))
            forms[name] = {"value": nq * ctx.world / (ms / 1000), "unit": "queries/s",
                           "ms_per_step": ms,
                           "launches_per_step": nbatch if name == "plain" else 1}

    e2e = None
    if not args.no_e2e:
        # Steady state through the public API with host buffers: every step
        # copies its queries from pinned host memory and all of its pairs
        # (and counts) back.  Two prepared launches write alternate output
        # buffers, so step k's pairs travel to the host while step k+1 runs;
        # K steps are timed end to end (to the last step's pairs on the host).
        q_host = torch.from_numpy(w["queries"]).pin_memory()
        sides = []
        for side in range(2):
            if side == 0:
                p_d, s_d, pl = pairs, qsize, plan
            else:
                p_d = torch.empty_like(pairs)
                s_d = torch.zeros_like(qsize)
                ho = torch.zeros((nbatch, 3), dtype=torch.int64)
                for i in range(nbatch):
                    ho[i, 0] = p_d.data_ptr() + 8 * int(poffs[i])
                    ho[i, 1] = max(int(per_batch[i]), 1)
                    ho[i, 2] = s_d.data_ptr() + 4 * i
                ob = ho.to(dev)
                pl = ix.plan([(pred, qslices[i], rb.Handler.COLLECT, ob[i].data_ptr())
                              for i in range(nbatch)])
            sides.append(dict(pairs=p_d, qsize=s_d, plan=pl, keep=None if side == 0 else ob,
                              out=torch.empty((pairs.shape[0], 2), dtype=torch.int32).pin_memory(),
                              cnt=torch.empty(nbatch, dtype=torch.int32).pin_memory(),
                              ready=torch.cuda.Event(), copied=torch.cuda.Event()))
        comp, copy = torch.cuda.Stream(), torch.cuda.Stream()

        def run_e2e(k):
            comp.wait_stream(stream)
            copy.wait_stream(stream)
            for i in range(k):
                x = sides[i % 2]
                if i >= 2:
                    comp.wait_event(x["copied"])   # its buffers' last copy is done
                with torch.cuda.stream(comp):
                    queries_d.copy_(q_host, non_blocking=True)
                    x["qsize"].zero_()
                    x["plan"].launch(stream=comp)
                    x["ready"].record(comp)
                copy.wait_event(x["ready"])
                with torch.cuda.stream(copy):
                    x["cnt"].copy_(x["qsize"], non_blocking=True)
                    x["out"].copy_(x["pairs"], non_blocking=True)
                    x["copied"].record(copy)
            stream.wait_stream(copy)

        run_e2e(2)
        torch.cuda.synchronize()
        for x in sides:
            if int(x["cnt"].to(torch.int64).sum()) != total_pairs:
                raise SystemExit("end-to-end launches reported a different pair count")
        k = max(4, args.steps // 2)
        per = []
        for _ in range(2):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ctx.barrier()
            torch.cuda.synchronize()
            flush.fill_(1.0)
            a.record(stream)
            run_e2e(k)
            b.record(stream)
            torch.cuda.synchronize()
            per.append(a.elapsed_time(b) / k)
        ms = ctx.max(min(per))
        e2e = {"value": nq * ctx.world / (ms / 1000), "unit": "queries/s",
               "h2d_bytes_per_step": int(q_host.numel() * 4),
               "d2h_bytes_per_step": int(sides[0]["out"].numel() * 4 + sides[0]["cnt"].numel() * 4),
               "ms_per_step": ms, "steps_timed": k,
               "path": "per step: pinned H2D of the queries + rts_plan_launch (graph) on a compute "
                       "stream, D2H of counts and all pairs on a copy stream; two plans with "
                       "alternate output buffers so a step's D2H overlaps the next step"}
        sides[1]["plan"].close()

    mean_ms = sum(t_main) / len(t_main)
    step_ms = ctx.max(mean_ms)
    lat = sorted(t_main)
    peak, peak_src = peak_hbm()
    alg = algorithmic_bytes(w, total_pairs)
    achieved = alg / (mean_ms / 1000) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", f"traffic_config{args.config}.json")
    if os.path.exists(tfile) and args.scale == 1.0:
        with open(tfile) as f:
            traffic = json.load(f).get("bytes_per_launch")

    cpu = None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu:
        rate, n, cores, kind = cpu_query_rate(w, args.cpu_seconds, "ref")
        cpu = {"value": rate, "unit": "queries/s", "cores": cores, "kind": kind,
               "sample": f"first {n} of {nq} queries against all {w['boxes'].shape[0]} boxes, "
                         f"uniform-grid filter, OpenMP, counting only, best of 3"}

    line = None
    if ctx.rank == 0:
        line = {
            "metric": METRIC,
            "value": nq * ctx.world / (step_ms / 1000),
            "unit": "queries/s",
            "n_gpus": ctx.world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": step_ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded numpy generators with the configuration's shapes)",
            "config": {
                "workload": w["desc"],
                "boxes": int(w["boxes"].shape[0]), "queries": nq, "batches": nbatch,
                "form": "rts_plan_launch replaying a captured CUDA graph (1 persistent kernel)",
                "node_width": ix.config.node_width, "traversal": ix.config.traversal,
                "curve": ix.config.curve, "sort_queries": ix.config.sort_queries,
                "query_occupancy": ix.config.query_occupancy, "chunk": ix.config.chunk,
                "group_loads": ix.config.group_loads,
                "l2": "index > L2 and L2 flushed before every timed step (256 MiB write "
                      "outside the events)",
            },
            "pairs_per_s": total_pairs * ctx.world / (step_ms / 1000),
            "pairs_per_step": total_pairs,
            "latency_ms": {"p50": lat[len(lat) // 2],
                           "p99": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))],
                           "what": "one step (all batches), rank 0"},
            "forms": forms,
            "batched_over_plain": (forms["plain"]["ms_per_step"] / step_ms) if "plain" in forms else None,
            "autotune": tune,
            "build_ms": build_ms,
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                         "algorithmic_bytes_per_launch": alg,
                         "kernel": "rts::k_query (+ order sort when enabled)"},
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clocks_info,
            "gpu_launches": args.steps * kernels_per_step(ix.config, nq, nbatch, int(pred)),
        }
    plan.close()
    if parity is not None and not parity["equal"]:
        raise SystemExit(f"parity check failed: {parity}")
    return line if ctx.rank == 0 else None


def kernels_per_step(cfg, nq: int, nbatch: int, pred: int = 1, handler: int = 1) -> int:
    """Kernels of this library one batched launch runs: the query kernel, plus
    the order-key kernel and the radix sort's histogram, scan and one
    onesweep pass per 8 key bits when queries are curve-sorted, plus the
    query gather of a merged launch (several batches of one predicate that
    count or use the packet scheme, sorted together on 32-bit keys), or, for
    an unmerged launch of several batches, the chunk-order key kernel and its
    32-bit sort (histogram, scan, 4 passes)."""
    sorted_ = cfg.sort_queries == 1 or (cfg.sort_queries == 2 and nq >= 8192)
    if not sorted_:
        return 1
    packet = cfg.traversal == 4 or (cfg.traversal == 0 and pred == 0)   # 0 = kIntersects
    merged = nbatch > 1 and cfg.traversal not in (2, 3) and (handler == 0 or packet)
    lg = 0
    while lg < 40 and (1 << lg) < nq:
        lg += 1
    curve_bits = 2 * min(16, (lg + 1) // 2 + 2)      # order_curve_bits in rts_build.cu
    bbits = 0
    while not merged and (1 << bbits) < nbatch:
        bbits += 1
    if bbits > 0 and curve_bits + bbits > 24:
        curve_bits = max(16, min(curve_bits, (24 - bbits) & ~1))
    passes = (curve_bits + bbits + 7) // 8
    chunk_order = nbatch > 1 and not merged and cfg.traversal != 3
    chunk_kernels = 1 + 2 + (curve_bits + 7) // 8 if chunk_order else 0
    return 1 + 1 + 2 + passes + (1 if merged else 0) + chunk_kernels


def run_mutable_bench(args, ctx):
    """Config 4: 20M boxes; each round deletes 1%, inserts 1%, updates 2%
    (moved by U[-1e-3, 1e-3]) and answers 1M point queries (counting
    handler).  One step = one round, mutations included; the refit-vs-rebuild
    threshold is tuned online from the measured round query times.

    Every round (warm-up rounds included) is checked against the oracle,
    outside the timed region: the same points run once more with the
    collecting handler, and the pair count and order-independent pair digest
    are compared with the oracle's over a host copy of the box set that
    applies the reference's semantics (Delete = Envelope::Invalid, Update =
    overwrite, Insert = append).

    e2e: the same round through the public API with host buffers: pinned H2D
    of the round's deletes, inserts, updates and points, the round, and D2H of
    the count, timed on the device per round."""
    torch = ctx.torch
    import rtspatial_b200 as rb
    from rtspatial_b200 import workloads as wl
    dev = ctx.dev
    n0 = int(20_000_000 * args.scale)
    nq = int(1_000_000 * args.scale)
    rng = np.random.default_rng(42 + ctx.rank)
    state = wl.config4_base(seed=42, n_boxes=n0)
    ix = make_index(args, rb)
    ix.Insert(torch.from_numpy(state).to(dev))
    torch.cuda.synchronize()
    rounds = args.rounds or 50
    stream = torch.cuda.current_stream()
    counter = torch.zeros(1, dtype=torch.int64, device=dev)
    count_h = torch.zeros(1, dtype=torch.int64).pin_memory()
    rows, checks = [], []
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    n_live = n0
    clocks = ClockSampler(ctx.local)
    clocks.start()
    total_ms = e2e_ms = 0.0
    h2d_bytes = 0
    check = ctx.rank == 0 and not args.no_parity
    w_chk = {"kind": "point"}
    for r in range(args.warmup + rounds):
        del_ids, ins, upd_ids, upd, pts = wl.config4_round(rng, n_live, state.shape[0], nq,
                                                            current=state)
        host = [torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
                for a in (del_ids, ins, upd_ids, upd, pts)]
        flush.fill_(1.0)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        ctx.barrier()
        torch.cuda.synchronize()
        e[0].record(stream)
        d_del, d_ins, d_uid, d_upd, d_pts = (h.to(dev, non_blocking=True) for h in host)
        e[1].record(stream)
        ix.Delete(d_del)
        ix.Update(d_uid, d_upd)
        ix.Insert(d_ins)
        e[2].record(stream)
        counter.zero_()
        ix.Query(rb.Predicate.kContains, d_pts, counter.data_ptr(), handler=rb.Handler.COUNT)
        e[3].record(stream)
        count_h.copy_(counter, non_blocking=True)
        e[4].record(stream)
        torch.cuda.synchronize()
        maint_ms, query_ms = e[1].elapsed_time(e[2]), e[2].elapsed_time(e[3])
        round_e2e_ms = e[0].elapsed_time(e[4])
        thr = ix.report_query_time(query_ms)
        state[del_ids, 2] = state[del_ids, 0]
        state[del_ids, 3] = state[del_ids, 1]
        state[upd_ids] = upd
        state = np.concatenate([state, ins])
        n_live += ins.shape[0] - del_ids.shape[0]
        got = int(count_h.item())
        if r >= args.warmup:
            total_ms += maint_ms + query_ms
            e2e_ms += round_e2e_ms
            h2d_bytes = sum(int(h.numel() * h.element_size()) for h in host)
            rows.append({"round": r - args.warmup, "maintenance_ms": maint_ms,
                         "query_ms": query_ms, "e2e_ms": round_e2e_ms, "pairs": got,
                         "trees": ix.num_trees(), "rebuild_update_fraction": thr})
        if check:
            qu = rb.Queue(max(got, 1), dev)
            ix.Query(rb.Predicate.kContains, d_pts, qu.DeviceObject(), handler=rb.Handler.COLLECT)
            torch.cuda.synchronize()
            n_col = qu.size()
            pairs_h = qu.pairs[:min(n_col, max(got, 1))].cpu().numpy().view(np.uint32)
            got_d = gpu_batch_digests(pairs_h, np.array([min(n_col, max(got, 1))]),
                                      np.array([0]))
            res = oracle_batch_check(w_chk, [nq], np.array([n_col], dtype=np.int64), got_d,
                                     boxes=state, queries=pts)
            res["count_handler_equal"] = got == res["pairs"]
            checks.append(res)
            if not (res["equal"] and res["count_handler_equal"]):
                raise SystemExit(f"round {r}: mutated index differs from the oracle: {res}")
            del qu, pairs_h
    clocks_info = clocks.stop()
    if args.rounds_out and ctx.rank == 0:
        with open(args.rounds_out, "w") as f:
            json.dump(rows, f, indent=0)
    step_ms = ctx.max(total_ms / rounds)
    e2e_step_ms = ctx.max(e2e_ms / rounds)
    if ctx.rank != 0:
        return None
    q = np.array([x["query_ms"] for x in rows])
    m = np.array([x["maintenance_ms"] for x in rows])
    pairs_med = int(np.median([x["pairs"] for x in rows]))
    n_final = int(state.shape[0])
    alg = 16 * n_final + 8 * nq + 8 * pairs_med
    achieved = alg / (float(np.median(q)) / 1000) / 1e9
    peak, peak_src = peak_hbm()
    cpu = None
    if ctx.world == 1 and not args.no_cpu:
        rate, n, cores, kind = cpu_query_rate({"kind": "point", "boxes": state, "queries": pts},
                                              args.cpu_seconds, "ref")
        cpu = {"value": rate, "unit": "queries/s", "cores": cores, "kind": kind,
               "sample": f"first {n} of the last round's {nq} points against its {n_final} boxes, "
                         f"uniform-grid filter (built outside the timing), OpenMP, counting only, "
                         f"best of 3; queries only, no index maintenance"}
    return {
        "metric": METRIC, "value": nq * ctx.world / (step_ms / 1000), "unit": "queries/s",
        "n_gpus": ctx.world, "steps": rounds, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded numpy generators with the configuration's shapes)",
        "config": {"workload": f"mutable index: {n0} boxes (sides U[0,1e-3]); per round 1% "
                               f"deletes, 1% inserts, 2% updates (moved U[-1e-3,1e-3]), "
                               f"{nq} uniform point queries (counting handler); step = one "
                               f"round, mutations included",
                   "node_width": ix.config.node_width, "rounds": rounds,
                   "l2": "index > L2 and L2 flushed before every round (256 MiB write "
                         "outside the events)"},
        "rounds": {"query_ms_p50": float(np.median(q)), "query_ms_max": float(q.max()),
                   "maintenance_ms_p50": float(np.median(m)),
                   "maintenance_ms_max": float(m.max()),
                   "final_rebuild_update_fraction": rows[-1]["rebuild_update_fraction"],
                   "trees_max": max(x["trees"] for x in rows)},
        "latency_ms": {"p50": float(np.percentile(q + m, 50)),
                       "p99": float(np.percentile(q + m, 99)),
                       "what": "one round (maintenance + query), device time"},
        "e2e": {"value": nq * ctx.world / (e2e_step_ms / 1000), "unit": "queries/s",
                "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": 8,
                "ms_per_step": e2e_step_ms,
                "path": "per round: pinned H2D of deletes, inserts, updates and points, "
                        "Delete/Update/Insert/Query(count) through the public API, D2H of the "
                        "count; device events around all of it"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                     "algorithmic_bytes_per_launch": alg,
                     "kernel": "rts::k_query point-contains (median round query time)"},
        "cpu_baseline": cpu,
        "parity": {"checked": bool(checks), "oracle": checks[-1]["oracle"] if checks else None,
                   "rounds_checked": len(checks),
                   "equal": all(c["equal"] and c["count_handler_equal"] for c in checks),
                   "pairs_last_round": checks[-1]["pairs"] if checks else None,
                   "what": "every round (warm-up included): count-handler total, and the "
                           "collected pairs' count and order-independent digest, vs the oracle "
                           "over the host mirror of the mutated box set"},
        "clocks": clocks_info,
    }


def serving_check(sv, reqs, boxes, grid=None) -> dict:
    """Submits `reqs` (closed loop), takes every request's pairs and compares
    each request's count and order-independent pair digest with the oracle
    over `boxes` (query ids 0-based per request)."""
    from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT, Oracle, pair_digest
    import rtspatial_b200 as rb
    backend = oracle_backend()
    ora = Oracle(backend)
    tickets = [sv.submit(p, q) for p, q in reqs]
    got = []
    for t in tickets:
        segs = sv.view(t)
        got.append((sum(s.shape[0] for s in segs), sum(pair_digest(s) for s in segs) % (1 << 64)))
        sv.release(t)
    t0 = time.perf_counter()
    own = grid is None
    g = ora.grid_build(boxes, 2.0) if own else grid
    bad, total = [], 0
    try:
        for i, ((p, q), (n, d)) in enumerate(zip(reqs, got)):
            if q.shape[1] == 2:
                kind = KIND_POINT
            else:
                kind = KIND_INTERSECTS if p == rb.Predicate.kIntersects else KIND_CONTAINS
            tot, _c, dig = ora.digest(kind, boxes, q, grid=g)
            total += tot
            if tot != n or int(dig.sum(dtype=np.uint64)) != d:
                bad.append(i)
    finally:
        if own:
            ora.grid_free(g)
    return {"requests": len(reqs), "pairs": total, "equal": not bad,
            "mismatched_requests": bad[:8], "oracle": "reference" if backend == "ref" else "port",
            "oracle_seconds": time.perf_counter() - t0}


def serving_plain_form(ix, reqs, ctx) -> dict:
    """The plain form of the served mix: each request as one synchronous Query
    launch through the public API with host buffers (pinned H2D of its
    queries, the collecting handler into a preallocated queue, D2H of its
    count and pairs; a request whose pairs overflow the queue runs again with
    the exact capacity).  Requests run back to back on one stream."""
    torch = ctx.torch
    import rtspatial_b200 as rb
    dev = ctx.dev
    max_q = max(q.shape[0] for _, q in reqs)
    q_host = torch.empty(max_q * 4, dtype=torch.float32).pin_memory()
    q_dev = torch.empty(max_q * 4, dtype=torch.float32, device=dev)
    cap = 16 << 20
    qu = rb.Queue(cap, dev)
    out_host = torch.empty((cap, 2), dtype=torch.int32).pin_memory()
    stream = torch.cuda.current_stream()
    lat = []
    outs = [out_host]

    def one(p, q):
        n, w = q.shape
        q_host[:n * w].numpy()[:] = q.reshape(-1)
        q_dev[:n * w].copy_(q_host[:n * w], non_blocking=True)
        qd = q_dev[:n * w].view(n, w)
        for _ in range(2):
            qu.Clear()
            ix.Query(p, qd, qu.DeviceObject(), handler=rb.Handler.COLLECT)
            k = qu.size(stream)
            if k <= qu.capacity():
                break
            qu.Init(k)
        if k > outs[0].shape[0]:
            outs[0] = torch.empty((k, 2), dtype=torch.int32).pin_memory()
        if k:
            outs[0][:k].copy_(qu.pairs[:k], non_blocking=True)
        stream.synchronize()
        return k

    for p, q in reqs[:5]:  # warm-up
        one(p, q)
    qu.Init(cap)
    t_all = time.perf_counter()
    pairs = 0
    for p, q in reqs:
        t0 = time.perf_counter()
        pairs += one(p, q)
        lat.append(time.perf_counter() - t0)
    wall = time.perf_counter() - t_all
    nq = sum(q.shape[0] for _, q in reqs)
    lat.sort()
    return {"value": nq * ctx.world / wall, "unit": "queries/s", "requests": len(reqs),
            "pairs": pairs, "latency_ms": {"p50": 1000 * lat[len(lat) // 2],
                                           "p99": 1000 * lat[min(len(lat) - 1,
                                                                 int(0.99 * (len(lat) - 1)))]},
            "launches_per_request": 1,
            "what": "one synchronous Query launch per request, host buffers, requests in "
                    "sequence (no updates)"}


def serving_cpu_rate(boxes, reqs, seconds: float) -> dict:
    """The CPU reference on the served mix: the oracle's grid (built outside
    the timing) counts the requests' pairs with every host thread, over as
    many requests as fit in about `seconds`."""
    from oracle.oracle import KIND_CONTAINS, KIND_INTERSECTS, KIND_POINT, Oracle
    import rtspatial_b200 as rb
    backend = oracle_backend()
    ora = Oracle(backend)
    threads = os.cpu_count() or 1
    g = ora.grid_build(boxes, 2.0)
    try:
        n_q, t_used, used = 0, 0.0, 0
        for p, q in reqs:
            kind = KIND_POINT if q.shape[1] == 2 else (
                KIND_INTERSECTS if p == rb.Predicate.kIntersects else KIND_CONTAINS)
            t0 = time.perf_counter()
            ora.run_on_grid(g, kind, boxes, np.ascontiguousarray(q), threads)
            t_used += time.perf_counter() - t0
            n_q += q.shape[0]
            used += 1
            if t_used > seconds:
                break
    finally:
        ora.grid_free(g)
    return {"value": n_q / t_used, "unit": "queries/s", "cores": threads,
            "kind": "reference" if backend == "ref" else "port",
            "sample": f"the first {used} of {len(reqs)} open-loop requests ({n_q} queries) against "
                      f"the initial {boxes.shape[0]} boxes, uniform-grid filter built outside the "
                      f"timing, OpenMP, counting only"}


def run_serving_bench(args, ctx):
    """Config 5: 50M resident boxes (half uniform, half clustered); requests of
    log-uniform size in [1, 100K] (50% point, 25% contains, 25% intersects)
    arrive as a Poisson stream at 70% of the closed-loop capacity measured
    first, with update batches of 0.1% of the boxes interleaved (one per ten
    requests).  Reports p50/p99 request latency (submit -> pairs on the host)
    and the served queries/s.

    Parity (rank 0, untimed): every closed-loop request is compared with the
    oracle on the initial box set (the closed loop runs before any update),
    and a closed tail of requests submitted after the open loop is compared
    with the oracle on the final box set, mirrored on the host with the
    reference's semantics (deletes, then updates, then inserts per batch)."""
    torch = ctx.torch
    import rtspatial_b200 as rb
    from rtspatial_b200 import workloads as wl
    dev = ctx.dev
    nb = int(50_000_000 * args.scale)
    boxes = wl.config5_boxes(seed=42, n_boxes=nb)
    ix = make_index(args, rb)
    ix.Insert(torch.from_numpy(boxes).to(dev))
    torch.cuda.synchronize()
    rng = np.random.default_rng(7 + ctx.rank)
    n_req = args.requests
    check = ctx.rank == 0 and not args.no_parity

    def make_requests(k):
        out = []
        for _ in range(k):
            u = rng.random()
            n = int(np.exp(rng.uniform(0, np.log(100_000))))
            if u < 0.5:
                out.append((rb.Predicate.kContains, wl.uniform_points(rng, n)))
            elif u < 0.75:
                out.append((rb.Predicate.kContains, wl.uniform_boxes(rng, n, 1e-3)))
            else:
                out.append((rb.Predicate.kIntersects, wl.uniform_boxes(rng, n, 1e-3)))
        return out

    n_ids = [nb]

    def make_update():
        k = max(1, int(nb * 0.001) // 3)
        ids = rng.choice(n_ids[0], 2 * k, replace=False)
        u = dict(delete_ids=ids[:k], update_ids=ids[k:],
                 update_boxes=wl.uniform_boxes(rng, k, 1e-3),
                 inserts=wl.uniform_boxes(rng, k, 1e-3))
        n_ids[0] += k
        return u

    sv = rb.Server(ix, slots=3, max_queries_per_launch=1 << 19, pairs_per_launch=16 << 20,
                   host_result_bytes=4 << 30, use_graphs=not args.no_graphs)
    def take(t):
        # zero-copy: the pairs are on the host in the server's pinned memory
        sv.view(t)
        sv.release(t)

    # closed loop: everything submitted at once -> capacity
    warm = make_requests(20)
    for t in [sv.submit(p, q) for p, q in warm]:
        take(t)
    reqs = make_requests(n_req)
    sv.reset_stats()
    t0 = time.perf_counter()
    tickets = [sv.submit(p, q) for p, q in reqs]
    for t in tickets:
        take(t)
    closed_s = time.perf_counter() - t0
    closed = sv.stats()
    total_q = sum(q.shape[0] for _, q in reqs)
    capacity_qps = total_q / closed_s
    parity = {}
    if check:  # every 4th request of the closed loop, run again and checked
        parity["initial"] = serving_check(sv, reqs[::4], boxes)
    # open loop: Poisson arrivals at 70% of capacity, updates interleaved
    mean_q = total_q / n_req
    lam = 0.7 * capacity_qps / mean_q
    reqs = make_requests(n_req)
    gaps = rng.exponential(1.0 / lam, n_req)
    ups = [make_update() for _ in range(n_req // 10)]
    applied = []
    sv.reset_stats()
    clocks = ClockSampler(ctx.local)
    clocks.start()
    t0 = time.perf_counter()
    next_t = t0
    tickets, up_tickets = [], []
    for i, ((p, q), g) in enumerate(zip(reqs, gaps)):
        next_t += g
        while True:
            d = next_t - time.perf_counter()
            if d <= 0:
                break
            time.sleep(min(d, 0.002))
        tickets.append(sv.submit(p, q))
        if i % 10 == 9 and ups:
            u = ups.pop(0)
            applied.append(u)
            up_tickets.append(sv.submit_update(**u))
    for t in tickets:
        take(t)
    for t in up_tickets:
        sv.take(t)
    open_s = time.perf_counter() - t0
    clocks_info = clocks.stop()
    st = sv.stats()
    plain = serving_plain_form(ix, reqs, ctx) if not args.no_plain else None
    cpu = None
    if ctx.rank == 0 and ctx.world == 1 and not args.no_cpu:
        cpu = serving_cpu_rate(boxes, reqs, args.cpu_seconds)
    if check:
        # the host mirror of the box set after every applied update batch
        final = boxes
        for u in applied:
            final[u["delete_ids"], 2] = final[u["delete_ids"], 0]
            final[u["delete_ids"], 3] = final[u["delete_ids"], 1]
            final[u["update_ids"]] = u["update_boxes"]
            final = np.concatenate([final, u["inserts"]])
        parity["final"] = serving_check(sv, make_requests(max(10, n_req // 20)), final)
    sv.close()
    served_q = sum(q.shape[0] for _, q in reqs)
    if parity and not all(v["equal"] for v in parity.values()):
        raise SystemExit(f"served results differ from the oracle: {parity}")
    if ctx.rank != 0:
        return None
    return {
        "metric": METRIC, "value": served_q * ctx.world / open_s, "unit": "queries/s",
        "n_gpus": ctx.world, "steps": n_req, "warmup": 20, "ms_per_step": 1000 * open_s / n_req,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded numpy generators with the configuration's shapes)",
        "config": {"workload": f"serving: {nb} resident boxes (half uniform, half 64-cluster); "
                               f"{n_req} requests, sizes log-uniform [1,100K], 50% point / "
                               f"25% contains / 25% intersects, Poisson arrivals at 70% of "
                               f"closed-loop capacity, update batches of 0.1% every 10 requests",
                   "slots": 3,
                   "launches": "CUDA-graph replay per slot" if not args.no_graphs else "direct"},
        "latency_ms": {"p50": 1000 * st["latency_p50_s"], "p99": 1000 * st["latency_p99_s"],
                       "max": 1000 * st["latency_max_s"],
                       "what": "request submit -> its pairs on the host"},
        "closed_loop": {"queries_per_s": capacity_qps,
                        "p50_ms": 1000 * closed["latency_p50_s"],
                        "p99_ms": 1000 * closed["latency_p99_s"],
                        "launches": closed["launches"]},
        "open_loop": {"offered_requests_per_s": lam, "launches": st["launches"],
                      "parts": st["parts"], "pairs": st["pairs_done"],
                      "retried_parts": st["retried_parts"], "updates": st["updates_done"]},
        "stages_s": {"what": "open loop, summed over launches: worker packing, device time of a "
                             "launch (query copy, sort, kernel, count copy), device copies of "
                             "pairs to pinned host memory, client take copies, worker applying "
                             "updates; wall time of the open loop for scale",
                     "wall": open_s, "pack": st["pack_s"], "issue": st["issue_s"],
                     "launch": st["launch_s"], "copy_pairs": st["copy_s"], "take": st["take_s"],
                     "update": st["update_s"]},
        "graph_launches": st["graph_launches"],
        "forms": {"plain": plain},
        "served_over_plain": (served_q / open_s) / plain["value"] if plain else None,
        "cpu_baseline": cpu,
        "parity": {"checked": bool(parity), "equal": all(v["equal"] for v in parity.values()),
                   **parity,
                   "what": "every 4th closed-loop request, run again, vs the oracle on the "
                           "initial boxes; a closed tail after the open loop vs the oracle on "
                           "the final boxes (per request: pair count and order-independent "
                           "digest)"},
        "clocks": clocks_info,
    }


def main():
    args = parse()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference_arm(args, rank, int(os.environ.get("WORLD_SIZE", "1")))
        return
    ctx = Ctx()
    try:
        line = run_config(args, ctx)
        if args.config == 2 and ctx.world == 1 and not args.no_others:
            line["other_configs"] = run_other_configs(args, ctx)
        if ctx.rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        ctx.close()


def run_config(args, ctx):
    if args.config in (1, 2, 3):
        return run_query_bench(args, ctx)
    if args.config == 4:
        return run_mutable_bench(args, ctx)
    return run_serving_bench(args, ctx)


# Reduced runs of the other configurations that the default (config 2) run
# nests in its line: full-size inputs, fewer steps.
OTHER_CONFIGS = {1: dict(steps=10), 3: dict(steps=10), 4: dict(rounds=5, warmup=3),
                 5: dict(requests=200)}


def run_other_configs(args, ctx) -> dict:
    import copy
    out = {}
    for cfg, over in OTHER_CONFIGS.items():
        a = copy.copy(args)
        a.config = cfg
        a.warmup = min(args.warmup, 3)
        a.cpu_seconds = min(args.cpu_seconds, 6.0)
        for k, v in over.items():
            setattr(a, k, v)
        t0 = time.perf_counter()
        # Indexes of the previous configuration are destroyed here, not during
        # this one's timed steps (a destroy synchronises the device and returns
        # the library's kept memory).
        gc.collect()
        line = run_config(a, ctx)
        gc.collect()
        ctx.torch.cuda.empty_cache()
        keep = ("value", "unit", "ms_per_step", "steps", "warmup", "config", "latency_ms",
                "pairs_per_s", "pairs_per_step", "forms", "e2e", "roofline", "cpu_baseline",
                "parity", "rounds", "closed_loop", "open_loop", "autotune", "clocks")
        out[f"config{cfg}"] = {k: line[k] for k in keep if k in line}
        out[f"config{cfg}"]["wall_s"] = time.perf_counter() - t0
    return out


if __name__ == "__main__":
    main()
