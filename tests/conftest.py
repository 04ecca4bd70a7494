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


def p_err(p_test: np.ndarray, p_ref: np.ndarray, scale: float) -> float:
    """Pressure disagreement, gauge-free (the mean difference over the interior
    removed) and normwise against the run's pressure scale (the largest |p|
    it reached).  The singular mode of the Neumann solve (x-mode 0, J = 0: a
    profile along z) is determined to about 5e-11 absolute per solve by two
    exact FP64 solvers whatever the right-hand side's size, while the
    velocities it projects agree to 1e-15; against the final |p| of a run
    whose first projection is a thousand times larger that is a 1e-10
    relative difference, against the run's pressure scale it is 1e-12."""
    d = (p_test - p_ref)[1:-1, 1:-1, 1:-1]
    return float(np.max(np.abs(d - d.mean())) / scale)


def run_with_scale(solver, steps: int) -> float:
    """Step an oracle solver one step at a time; the largest |p| it reaches."""
    scale = 0.0
    for _ in range(steps):
        solver.step(1)
        scale = max(scale, float(np.max(np.abs(solver.get("p")))))
    return scale
