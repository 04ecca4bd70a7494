"""Shared fixtures: build the oracle (checker) and the CUDA library once."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import eddy_oracle
    eddy_oracle.build()
    return eddy_oracle


@pytest.fixture(scope="session")
def product():
    import eddy_hybrid_b200
    from eddy_hybrid_b200 import build
    build.build()
    return eddy_hybrid_b200


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max|a-b| / max|b| (normwise relative error)."""
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(a - b))) / (den if den > 0 else 1.0)
