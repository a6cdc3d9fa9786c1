"""Multi-process check of the replica/shard host logic with the gloo backend
on CPU (world size 2): shards cover every batch exactly once, per-rank
oracle counts of the shards add up to the single-process count, and the
timing reduction returns the slowest rank's time on every rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from rtspatial_b200 import replicas


def test_shard_partitions():
    for total in (0, 1, 7, 256, 1000):
        for world in (1, 2, 3, 8):
            got = [list(replicas.shard(total, r, world)) for r in range(world)]
            flat = [i for g in got for i in g]
            assert flat == list(range(total))
            assert max(map(len, got)) - min(map(len, got)) <= 1
    with pytest.raises(ValueError):
        replicas.shard(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from oracle.oracle import KIND_CONTAINS, Oracle
    from rtspatial_b200 import workloads as wl
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        boxes = wl.clustered_boxes(rng, 20000, 2e-2)
        sizes = wl.log_uniform_sizes(np.random.default_rng(6), 16, 10, 200)
        ora = Oracle("port")
        idx, _, _ = replicas.shard_queries(sizes, rank, world)
        local = 0
        for b in idx:
            q = wl.uniform_boxes(np.random.default_rng(replicas.batch_seed(1, int(b))),
                                 int(sizes[b]), 2e-2)
            local += ora.run(KIND_CONTAINS, boxes, q, collect=False, grid=False, threads=1)[0]
        total = replicas.sum_over_ranks(local, dist)
        slowest = replicas.max_over_ranks(float(rank + 1), dist)
        out.put((rank, total, slowest))
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_add_up(oracle):
    from oracle.oracle import KIND_CONTAINS
    from rtspatial_b200 import workloads as wl
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    rng = np.random.default_rng(5)
    boxes = wl.clustered_boxes(rng, 20000, 2e-2)
    sizes = wl.log_uniform_sizes(np.random.default_rng(6), 16, 10, 200)
    want = 0
    for b in range(len(sizes)):
        qq = wl.uniform_boxes(np.random.default_rng(replicas.batch_seed(1, b)), int(sizes[b]), 2e-2)
        want += oracle.run(KIND_CONTAINS, boxes, qq, collect=False, grid=False)[0]
    assert [r[1] for r in res] == [want, want]
    assert [r[2] for r in res] == [2.0, 2.0]
