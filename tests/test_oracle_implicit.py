"""CPU checks of the oracle's Crank-Nicolson y lines (IMPLY = 1): the
periodic tridiagonal solver against a dense solve, and the implicit step
against the explicit one (same equations, a second-order-in-time difference,
a projected, divergence-free result)."""
import ctypes as C

import numpy as np
import pytest

from eddy_hybrid_b200 import config


def test_cyclic_solver_matches_dense(oracle):
    lib = oracle.lib()
    P = C.POINTER(C.c_double)
    lib.eo_cyclic.argtypes = [P, P, P, C.c_double, C.c_double, P, P, C.c_int, P]
    rng = np.random.default_rng(3)
    for n in (3, 8, 33, 256):
        a = -rng.uniform(0.1, 1.0, n)
        c = -rng.uniform(0.1, 1.0, n)
        b = 1.0 - a - c + rng.uniform(0.0, 0.5, n)
        r = rng.standard_normal(n)
        alpha, beta = c[n - 1], a[0]
        A = np.diag(b) + np.diag(a[1:], -1) + np.diag(c[:-1], 1)
        A[0, n - 1] += beta
        A[n - 1, 0] += alpha
        want = np.linalg.solve(A, r)
        x = np.zeros(n)
        wk = np.zeros(4 * n)
        lib.eo_cyclic(a.ctypes.data_as(P), b.ctypes.data_as(P), c.ctypes.data_as(P), alpha, beta,
                      r.ctypes.data_as(P), x.ctypes.data_as(P), n, wk.ctypes.data_as(P))
        assert np.max(np.abs(x - want)) < 1e-13 * max(1.0, np.max(np.abs(want))), n


def _run(oracle, imply, steps):
    w = config.small(mx=16, ly=16, nz_=24, noise=0.2, re=500.0, imply=imply)
    o = oracle.OracleSolver(w)
    o.load_initial(config.initial_fields(w, o.grid.get("dens_bg")[: w.nx]))
    o.initialize()
    o.step(steps)
    return o


def test_implicit_y_step_is_projected_and_close_to_explicit(oracle):
    oi, oe = _run(oracle, 1, 4), _run(oracle, 0, 4)
    assert oi.max_divergence() < 1e-12
    for n in ("uo", "vo", "wo", "dens", "p"):
        a, b = oi.get(n)[1:-1, 1:-1, 1:-1], oe.get(n)[1:-1, 1:-1, 1:-1]
        assert np.all(np.isfinite(a)), n
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        # same equations, Crank-Nicolson instead of explicit y diffusion: an
        # O(dt^2) difference, not zero and not large
        assert 0 < d < 5e-3, (n, d)
