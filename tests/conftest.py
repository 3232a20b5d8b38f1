import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels through the C ABI)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def cuda():
    """Torch with a CUDA device and the in-tree libpff loaded (no fallback)."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyfastflow_b200 import _lib

    _lib.load()  # raises if libpff.so is missing
    return torch
