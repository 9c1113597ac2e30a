"""Shared test configuration.

Tests marked `gpu` need a CUDA device and call the product through the C ABI;
everything else runs on CPU (oracle vs golden fixtures, oracle vs the
reference build, host logic, library exports, multi-process gloo paths).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the CUDA path through the C ABI")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return True


def golden(name):
    import numpy as np
    return np.load(os.path.join(GOLDEN, name))
