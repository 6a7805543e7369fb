"""Test configuration: the `gpu` marker and shared fixtures.

Tests marked `gpu` need a CUDA device and the built libbia_b200.so; the rest run on
the CPU (oracle pins, host logic, library symbol table).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_0001332.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libbia_b200.so")


@pytest.fixture(scope="session")
def golden():
    g = np.load(GOLDEN)
    return {k: g[k] for k in g.files}


@pytest.fixture(scope="session")
def golden_ic(golden):
    return np.ascontiguousarray(golden["ic_aos"].reshape(-1, 6).T)


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    return torch


def rel_err(a, b):
    """Global relative error ||a - b|| / ||b|| (2-norm over every particle and component)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def max_rel_err(a, b):
    """max |a - b| / max |b| over every particle and component."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / np.abs(b).max())
