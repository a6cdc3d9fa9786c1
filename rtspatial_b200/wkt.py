"""WKT input for the index: geometries reduced to the float32 envelopes the
index stores (the reference's example loads WKT polygons and points with
Boost.Geometry and indexes each geometry's envelope, examples/wkt_loader.h).

Supported: POINT, MULTIPOINT, LINESTRING, MULTILINESTRING, POLYGON,
MULTIPOLYGON (2-D coordinates; Z/M values are ignored).  One geometry per
line; blank lines and lines starting with '#' are skipped.  EMPTY geometries
are skipped.
"""
from __future__ import annotations

import re

import numpy as np

_NUM = re.compile(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?|nan|inf", re.IGNORECASE)
_KINDS = ("MULTIPOLYGON", "MULTILINESTRING", "MULTIPOINT", "POLYGON", "LINESTRING", "POINT")


def _coords(body: str, dims: int) -> np.ndarray:
    vals = np.array([float(v) for v in _NUM.findall(body)], dtype=np.float64)
    if vals.size % dims:
        raise ValueError(f"odd coordinate count in {body[:60]!r}")
    return vals.reshape(-1, dims)[:, :2]


def _parse(line: str):
    s = line.strip()
    up = s.upper()
    for k in _KINDS:
        if up.startswith(k):
            rest = s[len(k):].strip()
            dims = 2
            tag = rest.split("(", 1)[0].strip().upper()
            if tag in ("Z", "M"):
                dims = 3
            elif tag == "ZM":
                dims = 4
            if rest.upper().endswith("EMPTY"):
                return k, None
            xy = _coords(rest[rest.index("("):], dims)
            return k, xy
    raise ValueError(f"not a supported WKT geometry: {s[:60]!r}")


def load_envelopes(lines) -> np.ndarray:
    """(n, 4) float32 envelopes (min.x, min.y, max.x, max.y) of the geometries."""
    out = []
    for line in lines:
        if not line.strip() or line.lstrip().startswith("#"):
            continue
        _, xy = _parse(line)
        if xy is None or xy.shape[0] == 0:
            continue
        lo, hi = xy.min(axis=0), xy.max(axis=0)
        out.append((lo[0], lo[1], hi[0], hi[1]))
    return np.asarray(out, dtype=np.float64).astype(np.float32).reshape(-1, 4)


def load_points(lines) -> np.ndarray:
    """(n, 2) float32 points (POINT lines; MULTIPOINT lines give every point)."""
    out = []
    for line in lines:
        if not line.strip() or line.lstrip().startswith("#"):
            continue
        kind, xy = _parse(line)
        if xy is None:
            continue
        if kind not in ("POINT", "MULTIPOINT"):
            raise ValueError(f"{kind} is not a point geometry")
        out.extend(map(tuple, xy))
    return np.asarray(out, dtype=np.float64).astype(np.float32).reshape(-1, 2)


def read_envelopes(path: str) -> np.ndarray:
    with open(path) as f:
        return load_envelopes(f)


def read_points(path: str) -> np.ndarray:
    with open(path) as f:
        return load_points(f)
