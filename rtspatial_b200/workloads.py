"""Seeded synthetic workloads with the shapes, sizes and distributions of the
five benchmark configurations (float32 2-D boxes as min.x, min.y, max.x,
max.y).  Host numpy arrays; deterministic for a given seed.

1. point-contains: 1M boxes (centres U[0,1]^2, sides U[0,1e-3]) x 100K points
   U[0,1]^2, seed 42.
2. range-contains: 10M boxes from 64 Gaussian clusters (means U[0,1]^2,
   sigma 0.02, centres clipped to [0,1]), sides U[0,5e-3]; 1M query boxes with
   uniform centres and sides U[0,1e-3], split into 256 batches whose sizes are
   log-uniform in [1K, 16K] and rescaled to sum to the query count.
3. range-intersects with skew: 10M boxes, uniform centres, sides
   lognormal(ln 1e-4, 1.5) capped at 0.05; 1M queries, sides
   lognormal(ln 5e-4, 1.0) capped at 0.05.
4. mutable index: 20M boxes (centres U[0,1]^2, sides U[0,1e-3]); rounds of 1%
   deletes, 1% inserts, 2% updates moving boxes by U[-1e-3,1e-3], then 1M
   uniform point queries.
5. serving: 50M resident boxes (half config-4 uniform, half config-2
   clustered); requests of log-uniform size in [1, 100K], 50% point / 25%
   contains / 25% intersects.
"""
from __future__ import annotations

import numpy as np


def _boxes_from(cx, cy, w, h) -> np.ndarray:
    out = np.empty((cx.shape[0], 4), dtype=np.float32)
    out[:, 0] = cx - 0.5 * w
    out[:, 1] = cy - 0.5 * h
    out[:, 2] = cx + 0.5 * w
    out[:, 3] = cy + 0.5 * h
    return out


def uniform_boxes(rng: np.random.Generator, n: int, max_side: float) -> np.ndarray:
    c = rng.random((n, 2))
    s = rng.random((n, 2)) * max_side
    return _boxes_from(c[:, 0], c[:, 1], s[:, 0], s[:, 1])


def clustered_boxes(rng: np.random.Generator, n: int, max_side: float, n_clusters: int = 64,
                    sigma: float = 0.02) -> np.ndarray:
    means = rng.random((n_clusters, 2))
    k = rng.integers(0, n_clusters, n)
    c = np.clip(means[k] + rng.normal(0.0, sigma, (n, 2)), 0.0, 1.0)
    s = rng.random((n, 2)) * max_side
    return _boxes_from(c[:, 0], c[:, 1], s[:, 0], s[:, 1])


def lognormal_boxes(rng: np.random.Generator, n: int, mu: float, sigma: float,
                    cap: float = 0.05) -> np.ndarray:
    c = rng.random((n, 2))
    s = np.minimum(rng.lognormal(mu, sigma, (n, 2)), cap)
    return _boxes_from(c[:, 0], c[:, 1], s[:, 0], s[:, 1])


def uniform_points(rng: np.random.Generator, n: int) -> np.ndarray:
    return rng.random((n, 2)).astype(np.float32)


def log_uniform_sizes(rng: np.random.Generator, n_batches: int, lo: int, hi: int,
                      total: int | None = None) -> np.ndarray:
    """Batch sizes log-uniform in [lo, hi]; rescaled to sum to `total`."""
    s = np.exp(rng.uniform(np.log(lo), np.log(hi), n_batches))
    if total is None:
        return np.maximum(np.round(s).astype(np.int64), 1)
    assert total >= n_batches
    s = s * (total / s.sum())
    out = np.maximum(np.floor(s).astype(np.int64), 1)
    # hand out the remainder by largest fractional part (largest remainder)
    rest = total - int(out.sum())
    frac = s - np.floor(s)
    order = np.argsort(-frac, kind="stable")
    i = 0
    while rest > 0:
        out[order[i % n_batches]] += 1
        rest -= 1
        i += 1
    while rest < 0:
        j = int(np.argmax(out))
        out[j] -= 1
        rest += 1
    assert out.sum() == total and out.min() >= 1
    return out


# ---- the five configurations --------------------------------------------
def config1(seed: int = 42, n_boxes: int = 1_000_000, n_points: int = 100_000):
    rng = np.random.default_rng(seed)
    return uniform_boxes(rng, n_boxes, 1e-3), uniform_points(rng, n_points)


def config2(seed: int = 42, n_boxes: int = 10_000_000, n_queries: int = 1_000_000,
            n_batches: int = 256):
    rng = np.random.default_rng(seed)
    boxes = clustered_boxes(rng, n_boxes, 5e-3)
    queries = uniform_boxes(rng, n_queries, 1e-3)
    sizes = log_uniform_sizes(rng, n_batches, 1024, 16384, n_queries)
    return boxes, queries, sizes


def config3(seed: int = 42, n_boxes: int = 10_000_000, n_queries: int = 1_000_000):
    rng = np.random.default_rng(seed)
    boxes = lognormal_boxes(rng, n_boxes, np.log(1e-4), 1.5)
    queries = lognormal_boxes(rng, n_queries, np.log(5e-4), 1.0)
    return boxes, queries


def config4_base(seed: int = 42, n_boxes: int = 20_000_000):
    rng = np.random.default_rng(seed)
    return uniform_boxes(rng, n_boxes, 1e-3)


def config4_round(rng: np.random.Generator, n_live: int, n_total: int, n_points: int = 1_000_000,
                  frac_delete: float = 0.01, frac_insert: float = 0.01,
                  frac_update: float = 0.02, current: np.ndarray | None = None):
    """One mutation round: (delete ids, insert boxes, update ids, update boxes,
    query points).  Ids are drawn from [0, n_total); updates move the current
    box (when given) by U[-1e-3, 1e-3] per axis."""
    nd = int(round(n_live * frac_delete))
    ni = int(round(n_live * frac_insert))
    nu = int(round(n_live * frac_update))
    perm = rng.choice(n_total, nd + nu, replace=False)
    del_ids = perm[:nd].astype(np.int64)
    upd_ids = perm[nd:].astype(np.int64)
    ins = uniform_boxes(rng, ni, 1e-3)
    if current is not None:
        delta = rng.uniform(-1e-3, 1e-3, (nu, 2)).astype(np.float32)
        upd = current[upd_ids].copy()
        upd[:, 0] += delta[:, 0]
        upd[:, 2] += delta[:, 0]
        upd[:, 1] += delta[:, 1]
        upd[:, 3] += delta[:, 1]
    else:
        upd = uniform_boxes(rng, nu, 1e-3)
    pts = uniform_points(rng, n_points)
    return del_ids, ins, upd_ids, upd, pts


def config5_boxes(seed: int = 42, n_boxes: int = 50_000_000):
    rng = np.random.default_rng(seed)
    half = n_boxes // 2
    return np.concatenate([uniform_boxes(rng, half, 1e-3),
                           clustered_boxes(rng, n_boxes - half, 5e-3)])
