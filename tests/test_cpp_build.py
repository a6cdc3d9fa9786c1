"""The C++ drop-in headers (include/rtspatial/*) compile and link against the
library without a GPU: the reference's unit tests written against them
(tests/cpp/test_spatial_index.cu) build here; running them is the GPU test
test_gpu_cpp_api.py."""
import os
import subprocess

import pytest

from rtspatial_b200 import build as rbuild

HERE = os.path.dirname(os.path.abspath(__file__))
CPP = os.path.join(HERE, "cpp")


def test_cpp_dropin_headers_build():
    if not os.path.exists(rbuild.LIB):
        pytest.skip("library not built (python -m rtspatial_b200.build)")
    subprocess.check_call(["make", "-s", "-B", "-C", CPP, f"NVCC={rbuild.nvcc()}"], timeout=900)
    assert os.path.exists(os.path.join(CPP, "_build", "test_spatial_index"))
