"""Runs the C++ drop-in API test (tests/cpp/test_spatial_index.cu): the
reference's unit tests written against include/rtspatial/* and linked to the
B200 library."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "cpp", "_build", "test_spatial_index")


def test_cpp_dropin_api(cuda):
    # always re-make: a binary built against an older header must not run
    subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "cpp")])
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert re.search(r"\b(\d+) tests, 0 failed", r.stdout), r.stdout
    assert int(re.search(r"\b(\d+) tests, 0 failed", r.stdout).group(1)) >= 12
