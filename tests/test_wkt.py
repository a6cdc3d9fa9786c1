"""WKT loader (CPU): envelopes and points from hand-written geometries."""
import numpy as np
import pytest

from rtspatial_b200 import wkt

TEXT = """
# boxes
POLYGON ((0 0, 1 0, 1 1, 0 1, 0 0))
POLYGON((0.25 -0.5,1.5 -0.5,1.5 0.5,0.25 0.5,0.25 -0.5))
MULTIPOLYGON (((0 0, 2 0, 2 1, 0 0)), ((5 5, 6 5, 6 7, 5 5)))
LINESTRING (3 4, -1 2, 0.5 8)
POINT (0.5 0.25)
POLYGON Z ((1 1 9, 2 1 9, 2 3 9, 1 1 9))
POLYGON EMPTY
MULTIPOINT ((1 2), (3 -4))
"""


def test_envelopes():
    e = wkt.load_envelopes(TEXT.splitlines())
    want = np.array([[0, 0, 1, 1], [0.25, -0.5, 1.5, 0.5], [0, 0, 6, 7], [-1, 2, 3, 8],
                     [0.5, 0.25, 0.5, 0.25], [1, 1, 2, 3], [1, -4, 3, 2]], np.float32)
    assert e.dtype == np.float32 and np.array_equal(e, want)


def test_points():
    p = wkt.load_points(["POINT (1.5 -2)", "POINT(3e-1 4)", "MULTIPOINT (0 0, 1 1)"])
    assert np.array_equal(p, np.array([[1.5, -2], [0.3, 4], [0, 0], [1, 1]], np.float32))
    with pytest.raises(ValueError):
        wkt.load_points(["POLYGON ((0 0, 1 0, 1 1, 0 0))"])
    with pytest.raises(ValueError):
        wkt.load_envelopes(["CIRCLE (0 0, 1)"])
