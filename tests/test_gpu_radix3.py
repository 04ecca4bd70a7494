"""Periodic extents of 3 x 2^m (the radix-3 factor of FFTPACK): the GPU's
mixed-radix line FFTs (decimation by 3 over radix-2^2 passes) in the plain
and mixed Poisson solves and in full steps, against the oracle (whose
transform of such lengths is a direct DFT, pinned to numpy's FFT on the
CPU)."""
import numpy as np
import pytest

from conftest import P_BAR, P_PROFILE_BAR, p_err, p_profile_err, rel_err, run_with_scale
from eddy_hybrid_b200 import MIXED, config

pytestmark = pytest.mark.gpu


def _rhs(o, w, seed=7):
    rng = np.random.RandomState(seed)
    d = np.zeros((w.nx, w.ny, w.nz), order="F")
    d[1:-1, 1:-1, 1:-1] = rng.randn(w.mx, w.ly, w.nz_)
    ap, cp = o.grid.get("ap"), o.grid.get("cp")
    vol = (1 / ap[1:-1])[:, None, None] * np.ones((1, w.ly, 1)) * (1 / cp[1:-1])[None, None, :]
    inner = d[1:-1, 1:-1, 1:-1]
    inner -= (inner * vol).sum() / vol.sum()
    return d


@pytest.mark.parametrize("ly", [12, 24, 48, 96, 384])
def test_poisson_radix3_plain_and_mixed(oracle, product, ly):
    w = config.small(mx=32, ly=ly, nz_=20, beta=2.5)
    o = oracle.OracleSolver(w)
    d = _rhs(o, w)
    inner = d[1:-1, 1:-1, 1:-1]
    o.set("dp", d)
    o.direct(1)
    xo = o.get("dp")
    g = product.Solver(w)
    x = g.poisson_solve(d)
    r = o.apply_laplacian(x)[1:-1, 1:-1, 1:-1] - inner
    assert np.max(np.abs(r)) / np.max(np.abs(inner)) < 1e-12
    assert rel_err(x, xo) < 1e-12
    g.close()
    gm = product.Solver(w, precision=MIXED, refine_sweeps=2)
    xm = gm.poisson_solve(d)
    rm = o.apply_laplacian(xm)[1:-1, 1:-1, 1:-1] - inner
    assert np.max(np.abs(rm)) / np.max(np.abs(inner)) < 1e-11
    a, b = xm[1:-1, 1:-1, 1:-1], xo[1:-1, 1:-1, 1:-1]
    assert rel_err(a - a.mean(), b - b.mean()) < 1e-10


def test_full_step_parity_radix3(oracle, product):
    w = config.small(mx=16, ly=24, nz_=24, noise=0.2, re=2000.0)
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    o.load_initial(f)
    o.initialize()
    g = product.Solver(w)
    g.load_initial(f)
    g.initialize()
    scale = run_with_scale(o, 10)
    g.step(10)
    for n in ("uo", "vo", "wo", "dens", "tv"):
        e = rel_err(g.download(n), o.get(n))
        assert e < 1e-11, (n, e)
    pg = g.download("p")
    assert p_err(pg, o.get("p"), scale) < P_BAR
    assert p_profile_err(pg, o.get("p"), scale) < P_PROFILE_BAR
    assert g.max_divergence() < 1e-12
