"""Test configuration: the `gpu` marker and the repository on sys.path.

Tests marked `gpu` need a CUDA device and exercise the sm_100a library
through its C-ABI; the rest run on the CPU (the oracle against the
reference's golden vectors, host logic, and the library's exported symbols).
"""

import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def cuda_device():
    """Fails (never skips) when a gpu test runs without a usable device."""
    import torch

    if not torch.cuda.is_available():
        pytest.fail("a gpu-marked test ran without a CUDA device")
    return torch.cuda.get_device_name(0)
