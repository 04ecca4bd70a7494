"""The allocation-free max |div u| entry point against the context one.

eddy_max_divergence_noalloc serves callers that cannot call cudaMalloc: it
keeps its scratch in a fixed device array inside the library and takes raw
device pointers.  Two calls in a row (a larger grid, then a smaller one, so a
stale partial from the first call would show up in the second) must each
match eddy_max_divergence on the same fields.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from eddy_hybrid_b200 import config

pytestmark = pytest.mark.gpu


def _fields(oracle, w, steps):
    o = oracle.OracleSolver(w)
    o.load_initial(config.initial_fields(w, o.grid.get("dens_bg")[: w.nx]))
    o.initialize()
    if steps:
        o.step(steps)
    return o


def _noalloc(product, torch, o, w):
    dev = torch.device("cuda", 0)
    t = {n: torch.from_numpy(np.ascontiguousarray(o.get(n).ravel(order="F"))).to(dev) for n in ("uo", "vo", "wo")}
    m = {n: torch.from_numpy(np.ascontiguousarray(o.grid.get(n))).to(dev) for n in ("ap", "bp", "cp")}
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = product.lib().eddy_max_divergence_noalloc(
        w.nx, w.ny, w.nz, C.c_void_p(t["uo"].data_ptr()), C.c_void_p(t["vo"].data_ptr()),
        C.c_void_p(t["wo"].data_ptr()), C.c_void_p(m["ap"].data_ptr()), C.c_void_p(m["bp"].data_ptr()),
        C.c_void_p(m["cp"].data_ptr()), C.c_void_p(out.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 0
    return float(out.item())


def _context(product, o, w):
    g = product.Solver(w)
    for n in ("uo", "vo", "wo"):
        g.upload(n, o.get(n))
    v = g.max_divergence()
    g.close()
    return v


def test_max_divergence_noalloc_two_calls(oracle, product):
    torch = pytest.importorskip("torch")
    big = config.small(mx=24, ly=16, nz_=32, noise=0.3)
    small = config.small(mx=20, ly=16, nz_=24, noise=0.3)
    o1 = _fields(oracle, big, 0)      # initial noise: large divergence
    o2 = _fields(oracle, small, 1)    # projected: divergence at round-off
    a1 = _noalloc(product, torch, o1, big)
    a2 = _noalloc(product, torch, o2, small)
    b1 = _context(product, o1, big)
    b2 = _context(product, o2, small)
    assert b1 > 1.0 and b2 < 1e-10
    assert rel_err(np.array([a1]), np.array([b1])) < 1e-12
    assert rel_err(np.array([a2]), np.array([b2])) < 1e-12


def test_max_divergence_noalloc_rejects_oversize(product):
    n = 1 << 10   # 2^30 cells > EDDY_NOALLOC_MAX_CELLS; rejected before any pointer is touched
    rc = product.lib().eddy_max_divergence_noalloc(n, n, n, C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                                   C.c_void_p(1), C.c_void_p(1), C.c_void_p(1),
                                                   C.c_void_p(1), None)
    assert rc == 1
