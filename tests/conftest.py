"""Shared test configuration.

Tests marked `gpu` need a CUDA device (a B200); everything else runs on the
CPU: the oracle against its known answers and the golden vectors, host-side
logic, the C ABI library's exports, and multi-process paths on `gloo`.
"""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
