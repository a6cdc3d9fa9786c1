"""The library's caching allocator: every index buffer comes from it,
destroying an index gives the memory back, and rounds of updates that merge
sub-trees and re-sort the index (swapping its slot arrays) run from kept
blocks once warm, with results still equal to the oracle's."""
import numpy as np
import pytest
import torch

import rtspatial_b200 as rb
from oracle.oracle import KIND_POINT
from rtspatial_b200 import workloads as wl
from tests._gpu_util import assert_same_pairs, dev, gpu_pairs

pytestmark = pytest.mark.gpu


def test_index_buffers_come_from_the_allocator_and_go_back(cuda):
    d = torch.cuda.current_device()
    torch.cuda.synchronize()
    rb.trim_memory(d)
    r0, u0 = rb.memory_pool_stats(d)
    rng = np.random.default_rng(5)
    ix = rb.SpatialIndex(rb.Config())
    ix.Insert(dev(wl.uniform_boxes(rng, 1_000_000, 1e-3)))
    torch.cuda.synchronize()
    r1, u1 = rb.memory_pool_stats(d)
    assert u1 - u0 >= 16 * 1_000_000  # the leaf slots at least
    assert r1 >= u1
    ix._destroy()
    torch.cuda.synchronize()
    r2, u2 = rb.memory_pool_stats(d)
    assert u2 == u0
    assert r2 <= r0, "destroy did not return the index's memory"


def test_update_rounds_reuse_kept_blocks(cuda, oracle):
    d = torch.cuda.current_device()
    rng = np.random.default_rng(6)
    n = 300_000
    boxes = wl.uniform_boxes(rng, n, 1e-3)
    ix = rb.SpatialIndex(rb.Config(max_trees=4, rebuild_update_fraction=0.05))
    ix.Insert(dev(boxes))
    reserved = []
    for r in range(30):  # moved updates add sub-trees; merges and re-sorts follow
        ids = rng.choice(n, 6000, replace=False)
        new = wl.uniform_boxes(rng, ids.size, 1e-3)
        ix.Update(torch.from_numpy(ids.astype(np.int64)).cuda(), dev(new))
        boxes[ids] = new
        torch.cuda.synchronize()
        reserved.append(rb.memory_pool_stats(d)[0])
    assert reserved[-1] <= 1.25 * reserved[9], f"kept memory kept growing: {reserved}"
    pts = wl.uniform_points(rng, 20_000)
    assert_same_pairs(gpu_pairs(ix, rb.Predicate.kContains, pts),
                      oracle.run(KIND_POINT, boxes, pts)[2], "after update rounds")
