"""Accounting of bench.py, checked on the CPU: how many of this library's
kernels one batched launch runs (the bench's `gpu_launches` claim, which must
follow the order-key sizing of rts_build.cu) and the compulsory bytes its
roofline divides by the launch time."""
import importlib.util
import os
import types

import numpy as np

_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_spec = importlib.util.spec_from_file_location("bench_module", os.path.join(_ROOT, "bench.py"))
bench = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(bench)

THREAD, TEAM, FRONTIER, PACKET = 1, 2, 3, 4
INTERSECTS, CONTAINS = 0, 1
COUNT, COLLECT = 0, 1


def cfg(traversal=THREAD, sort=1):
    return types.SimpleNamespace(traversal=traversal, sort_queries=sort)


def test_unmerged_batches_sort_24_bit_keys_and_their_chunks():
    # 256 collecting thread-scheme batches of 1M queries in all: order keys,
    # radix sort of (8 batch + 16 curve) bits = histogram, scan, 3 passes;
    # chunk keys and their 16-bit sort = histogram, scan, 2 passes; the query
    # kernel.
    assert bench.kernels_per_step(cfg(), 1_000_000, 256, CONTAINS, COLLECT) == \
        (1 + 2 + 3) + (1 + 2 + 2) + 1


def test_single_batch_sorts_its_curve_keys_only():
    # 1M queries: 24 curve bits (about 16 cells per query), 3 passes, no
    # chunk order
    assert bench.kernels_per_step(cfg(PACKET), 1_000_000, 1, INTERSECTS, COLLECT) == 1 + 1 + 2 + 3
    # unsorted: the query kernel alone
    assert bench.kernels_per_step(cfg(sort=0), 100_000, 1, CONTAINS, COUNT) == 1


def test_merged_counting_launch_adds_the_query_gather():
    # counting batches sort together on curve bits alone, then gather the
    # queries into launch order
    assert bench.kernels_per_step(cfg(), 1_000_000, 256, CONTAINS, COUNT) == 1 + 1 + 2 + 3 + 1


def test_many_batches_keep_8_bits_per_axis():
    # 1024 batches (10 bits) leave 14 bits, below 8 per axis: the curve keeps
    # 16 bits and the key takes 26 bits, 4 passes
    assert bench.kernels_per_step(cfg(), 4_000_000, 1024, CONTAINS, COLLECT) == \
        (1 + 2 + 4) + (1 + 2 + 2) + 1


def test_algorithmic_bytes_per_launch():
    w = {"boxes": np.zeros((10, 4), np.float32), "queries": np.zeros((3, 4), np.float32),
         "qwidth": 4}
    assert bench.algorithmic_bytes(w, 5) == 16 * 10 + 16 * 3 + 8 * 5
    w["queries"], w["qwidth"] = np.zeros((3, 2), np.float32), 2
    assert bench.algorithmic_bytes(w, 0) == 16 * 10 + 8 * 3


def _bench_layout(ora, kind, boxes, queries, sizes, rng):
    """Per-batch results laid out as the bench's queues hold them: batch b's
    pairs (query ids 0-based in the batch, in a shuffled order) at rows
    [poffs[b], poffs[b] + count_b), one spare row for an empty batch."""
    offs = np.concatenate([[0], np.cumsum(sizes)])
    per = []
    for b in range(len(sizes)):
        _t, _c, p = ora.run(kind, boxes, queries[offs[b]:offs[b + 1]], grid=False)
        per.append(p[rng.permutation(p.shape[0])])
    counts = np.array([p.shape[0] for p in per], dtype=np.int64)
    poffs = np.concatenate([[0], np.cumsum(np.maximum(counts, 1))])
    pairs = np.full((int(poffs[-1]), 2), 0xDEADBEEF, dtype=np.uint32)
    for b, p in enumerate(per):
        pairs[poffs[b]:poffs[b] + p.shape[0]] = p
    return pairs, counts, poffs


def test_parity_check_accepts_the_oracles_pairs_and_catches_a_planted_mistake(oracle):
    from rtspatial_b200 import workloads as wl
    rng = np.random.default_rng(5)
    boxes = wl.uniform_boxes(rng, 20_000, 3e-2)
    queries = wl.uniform_boxes(rng, 900, 3e-2)
    sizes = np.array([300, 0, 250, 350], dtype=np.int64)
    for kind, name in ((1, "contains"), (2, "intersects")):
        w = {"kind": name, "boxes": boxes, "queries": queries}
        pairs, counts, poffs = _bench_layout(oracle, kind, boxes, queries, sizes, rng)
        assert counts.sum() > 0
        dig = bench.gpu_batch_digests(pairs, counts, poffs[:-1])
        res = bench.oracle_batch_check(w, sizes, counts, dig)
        assert res["equal"] and res["pairs"] == counts.sum(), res
        # a missing pair (count and digest both change)
        b = int(np.argmax(counts))
        c2 = counts.copy()
        c2[b] -= 1
        dig2 = bench.gpu_batch_digests(pairs, c2, poffs[:-1])
        res = bench.oracle_batch_check(w, sizes, c2, dig2)
        assert not res["equal"] and res["mismatched_batches"] == [b]
        # a wrong geom id at the right count (digest alone catches it)
        p3 = pairs.copy()
        p3[poffs[b], 0] ^= 1
        dig3 = bench.gpu_batch_digests(p3, counts, poffs[:-1])
        res = bench.oracle_batch_check(w, sizes, counts, dig3)
        assert not res["equal"] and res["mismatched_batches"] == [b]
