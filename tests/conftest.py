"""Shared test configuration.

Markers: ``gpu`` -- needs a CUDA device and the built library (run with ``-m gpu``); everything else runs on
the CPU (``-m "not gpu"``): the oracle against the reference's golden vectors, host-side logic, and that the
C-ABI library loads and exports its symbols.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: long-running (large sizes)")


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
