"""Benchmark of the hot path: SpatialIndex::Query on the B200 library.

Default workload (the BASELINE metric's configuration that fits one GPU):
range-contains, float32 2-D, 10M boxes from 64 Gaussian clusters, 1M query
boxes split into 256 log-uniform batches (1K-16K) run in ONE persistent
launch (rts_query_batched), collecting handler (pairs written to per-batch
device queues).  One step = all 256 batches once.

Printed on rank 0 as one JSON line:
  value        queries/s of the batched launch, inputs resident in HBM, L2
               flushed before every timed step (CUDA events per step)
  plain        the same batches as 256 separate launches (one per batch)
  e2e          queries/s through the same C-ABI call with host buffers:
               pinned H2D of the queries and D2H of every result pair inside
               the timed region
  roofline     algorithmic bytes per launch / launch time vs measured HBM peak
  cpu_baseline CPU oracle (grid filter + the reference's predicates) on the
               host cores over a bounded sample of the same queries
  clocks       nvidia-smi samples taken during warm-up + timed steps

--impl reference times the reference's CPU implementation of the path (the
reference's own predicate code compiled for the host, under the same grid
filter; the restated oracle when that build is absent) with all host threads.

Multi-GPU (torchrun): every rank holds a replica of the index and runs its own
query set (weak scaling, no data-path collective); times are the max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
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
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3])
    ap.add_argument("--scale", type=float, default=1.0, help="scales boxes and queries (profiling)")
    ap.add_argument("--node-width", type=int, default=0)
    ap.add_argument("--traversal", type=int, default=-1)
    ap.add_argument("--curve", type=int, default=-1)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--sort", type=int, default=-1, help="sort_queries: 0 never, 1 always, 2 auto")
    ap.add_argument("--occupancy", type=int, default=-1)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
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
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{gpu_index}.csv")

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
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    import torch.distributed as dist

    import rtspatial_b200 as rb
    from rtspatial_b200 import _lib as L

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    w = make_workload(args.config, args.scale, rank)
    cfg = rb.Config()
    if args.node_width:
        cfg.node_width = args.node_width
    if args.traversal >= 0:
        cfg.traversal = args.traversal
    if args.curve >= 0:
        cfg.curve = args.curve
    if args.chunk:
        cfg.chunk = args.chunk
    if args.sort >= 0:
        cfg.sort_queries = args.sort
    if args.occupancy >= 0:
        cfg.query_occupancy = args.occupancy
    ix = rb.SpatialIndex(cfg)
    boxes_d = torch.from_numpy(w["boxes"]).to(dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ix.Insert(boxes_d)
    torch.cuda.synchronize()
    build_ms = 1000 * (time.perf_counter() - t0)
    del boxes_d

    queries_d = torch.from_numpy(w["queries"]).to(dev)
    sizes = [int(s) for s in w["sizes"]]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    nbatch = len(sizes)
    nq = int(offs[-1])
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

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def l2_flush():
        flush.fill_(1.0)

    def step_batched():
        qsize.zero_()
        ix.query_batched(batch_args)

    def step_plain():
        qsize.zero_()
        for i in range(nbatch):
            ix.Query(pred, qslices[i], qobj[i].data_ptr(), handler=rb.Handler.COLLECT)

    stream = torch.cuda.current_stream()

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        barrier()
        torch.cuda.synchronize()
        for a, b in evs:
            l2_flush()
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        barrier()
        return [a.elapsed_time(b) for a, b in evs]

    # parity property: batched pair multiset == plain pair multiset per batch
    def checksum():
        torch.cuda.synchronize()
        p = pairs.to(torch.int64) & 0xFFFFFFFF
        h = (p[:, 0] * 0x9E3779B1 + p[:, 1] * 0x85EBCA77) & 0xFFFFFFFFFFFF
        return int(qsize.sum().item()), int(h.sum().item())

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        l2_flush()
        step_batched()
    torch.cuda.synchronize()
    cs_batched = checksum()
    t_batched = timed(step_batched, args.steps)
    clocks_info = clocks.stop()
    assert cs_batched[0] == total_pairs, (cs_batched, total_pairs)

    plain = None
    if not args.no_plain:
        for _ in range(max(1, args.warmup // 2)):
            l2_flush()
            step_plain()
        torch.cuda.synchronize()
        cs_plain = checksum()
        if cs_plain != cs_batched:
            raise SystemExit(f"batched and plain results differ: {cs_batched} vs {cs_plain}")
        t_plain = timed(step_plain, max(3, args.steps // 2))
        plain_ms = max_over_ranks(sum(t_plain) / len(t_plain))
        plain = {"value": nq * world / (plain_ms / 1000), "unit": "queries/s",
                 "ms_per_step": plain_ms, "launches_per_step": nbatch}

    # end to end through the C-ABI with host buffers
    e2e = None
    if not args.no_e2e:
        q_host = torch.from_numpy(w["queries"]).pin_memory()
        out_host = torch.empty((pairs.shape[0], 2), dtype=torch.int32).pin_memory()
        cnt_host = torch.empty(nbatch, dtype=torch.int32).pin_memory()

        def step_e2e():
            queries_d.copy_(q_host, non_blocking=True)
            step_batched()
            cnt_host.copy_(qsize, non_blocking=True)
            out_host.copy_(pairs, non_blocking=True)

        for _ in range(2):
            step_e2e()
        t_e2e = timed(step_e2e, max(3, args.steps // 2))
        e2e_ms = max_over_ranks(sum(t_e2e) / len(t_e2e))
        e2e = {"value": nq * world / (e2e_ms / 1000), "unit": "queries/s",
               "h2d_bytes_per_step": int(q_host.numel() * 4),
               "d2h_bytes_per_step": int(out_host.numel() * 4 + cnt_host.numel() * 4),
               "ms_per_step": e2e_ms}

    mean_ms = sum(t_batched) / len(t_batched)
    step_ms = max_over_ranks(mean_ms)
    lat = sorted(t_batched)
    p50 = lat[len(lat) // 2]
    p99 = lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))]

    peaks = {}
    if os.path.exists(PEAKS_FILE):
        with open(PEAKS_FILE) as f:
            peaks = json.load(f)
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or FALLBACK_HBM_GBS
    alg = algorithmic_bytes(w, total_pairs)
    achieved = alg / (mean_ms / 1000) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", f"traffic_config{args.config}.json")
    if os.path.exists(tfile) and args.scale == 1.0:
        with open(tfile) as f:
            traffic = json.load(f).get("bytes_per_launch")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, n, cores, kind = cpu_query_rate(w, args.cpu_seconds, "ref")
        cpu = {"value": rate, "unit": "queries/s", "cores": cores, "kind": kind,
               "sample": f"first {n} of {nq} queries against all {w['boxes'].shape[0]} boxes, "
                         f"uniform-grid filter, OpenMP, best of 3"}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": nq * world / (step_ms / 1000),
            "unit": "queries/s",
            "n_gpus": world,
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
                "node_width": ix.config.node_width, "traversal": ix.config.traversal,
                "curve": ix.config.curve, "sort_queries": ix.config.sort_queries,
                "query_occupancy": ix.config.query_occupancy, "chunk": ix.config.chunk,
                "l2": "flushed before every timed step (256 MiB write outside the events)",
            },
            "pairs_per_s": total_pairs * world / (step_ms / 1000),
            "pairs_per_step": total_pairs,
            "latency_ms": {"p50": p50, "p99": p99, "what": "batched step (all batches), rank 0"},
            "plain": plain,
            "batched_over_plain": (plain["ms_per_step"] / step_ms) if plain else None,
            "build_ms": build_ms,
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_src,
                         "algorithmic_bytes_per_launch": alg},
            "cpu_baseline": cpu,
            "clocks": clocks_info,
            "gpu_launches": args.steps,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
