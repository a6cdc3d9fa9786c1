"""Test configuration: the `gpu` marker, import paths and the oracle build.

CPU tests (-m "not gpu") check the oracle against the reference's known
answers, the C-ABI surface and host logic.  GPU tests (-m gpu) are the parity
tests proper: they call the CUDA library through its C-ABI and compare with
the oracle on the same inputs.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as om
    if not om.available("port"):
        om.build(None)
    return om.Oracle("port")


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import oracle as om
    if not om.available("ref"):
        pytest.skip("reference-header oracle not built (reference tree absent)")
    return om.Oracle("ref")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    import rtspatial_b200
    rtspatial_b200.lib()  # fails loudly when the library is missing
    return torch.device("cuda:0")
