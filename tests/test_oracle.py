"""The CPU oracle against FFTPACK golden vectors, manufactured Poisson
solutions and step invariants (no GPU)."""
import os

import numpy as np
import pytest

from conftest import rel_err
from eddy_hybrid_b200 import config

GOLD = os.path.join(os.path.dirname(__file__), "golden", "fftpack_rfft.npz")


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 256, 6, 12, 30, 384])
def test_fft_matches_fftpack_golden(oracle, n):
    g = np.load(GOLD)
    f = oracle.rfftf(g[f"x{n}"])
    assert np.max(np.abs(f - g[f"f{n}"])) <= 1e-13 * max(1.0, np.max(np.abs(g[f"f{n}"])))
    b = oracle.rfftb(f)
    assert np.max(np.abs(b - g[f"b{n}"])) <= 1e-12 * n
    rb = oracle.rfftb(g[f"r{n}"])
    assert np.max(np.abs(rb - g[f"rb{n}"])) <= 1e-12 * n


def _compatible_rhs(s, w, seed=7):
    rng = np.random.RandomState(seed)
    d = np.zeros((w.nx, w.ny, w.nz), order="F")
    d[1:-1, 1:-1, 1:-1] = rng.randn(w.mx, w.ly, w.nz_)
    ap = s.grid.get("ap")
    cp = s.grid.get("cp")
    vol = (1 / ap[1:-1])[:, None, None] * np.ones((1, w.ly, 1)) * (1 / cp[1:-1])[None, None, :]
    inner = d[1:-1, 1:-1, 1:-1]
    inner -= (inner * vol).sum() / vol.sum()
    return d


@pytest.mark.parametrize("shape", [(8, 4, 10), (12, 8, 16), (20, 16, 14)])
def test_poisson_manufactured_and_two_methods(oracle, shape):
    mx, ly, nz_ = shape
    w = config.small(mx=mx, ly=ly, nz_=nz_, beta=2.5)
    s = oracle.OracleSolver(w)
    d = _compatible_rhs(s, w)
    sols = []
    for method in (0, 1):
        s.set("dp", d)
        assert s.direct(method) == 0
        x = s.get("dp")
        r = s.apply_laplacian(x)
        res = np.max(np.abs(r[1:-1, 1:-1, 1:-1] - d[1:-1, 1:-1, 1:-1])) / np.max(np.abs(d))
        assert res < 1e-12, (method, res)
        # zero-mean k=0 plane convention (direct.f:895-898)
        assert abs(x[1:-1, 1:-1, 1:-1].mean()) < 1e-12 * np.abs(x).max()
        sols.append(x)
    assert rel_err(sols[0], sols[1]) < 1e-12


def test_poisson_ghost_convention(oracle):
    w = config.small(mx=8, ly=8, nz_=8)
    s = oracle.OracleSolver(w)
    s.set("dp", _compatible_rhs(s, w))
    s.direct(0)
    x = s.get("dp")
    assert np.all(x[:, :, 0] == 0) and np.all(x[:, :, -1] == 0)
    np.testing.assert_array_equal(x[0, 1:-1, 1:-1], x[1, 1:-1, 1:-1])
    np.testing.assert_array_equal(x[:, 0, 1:-1], x[:, -2, 1:-1])
    np.testing.assert_array_equal(x[:, -1, 1:-1], x[:, 1, 1:-1])


def _run(oracle, w, steps):
    s = oracle.OracleSolver(w)
    f = config.initial_fields(w, s.grid.get("dens_bg")[: w.nx])
    s.load_initial(f)
    s.initialize()
    s.step(steps)
    return s


def test_step_projection_is_divergence_free(oracle):
    w = config.small(mx=16, ly=8, nz_=24, noise=0.2)
    s = _run(oracle, w, 3)
    for n in ("uo", "vo", "wo", "p", "dens", "tv"):
        assert np.isfinite(s.get(n)).all()
    # post-projection divergence (the src/info.f:32 quantity)
    assert s.max_divergence() < 1e-11


def test_step_dynamic_viscosity_active(oracle):
    w = config.small(mx=16, ly=16, nz_=24, noise=0.5, re=1e4)
    s = _run(oracle, w, 2)
    tv = s.get("tv")
    assert tv[1:-1, 1:-1, 1:-1].max() > 0.0
    assert (tv[1:-1, 1:-1, 1:-1] >= 0).all()


def test_mass_balance_outflow(oracle):
    w = config.small(mx=12, ly=8, nz_=16, noise=0.1)
    s = _run(oracle, w, 2)
    wo = s.get("wo")
    ap = s.grid.get("ap")
    area = (1.0 / ap[1:-1])[:, None] * np.ones((1, w.ly)) * ((w.ylim[1] - w.ylim[0]) / w.ly)
    qin = (wo[1:-1, 1:-1, 0] * area).sum()
    qout = (wo[1:-1, 1:-1, -2] * area).sum()
    assert abs(qin - qout) < 1e-10 * abs(qin)


class _TaylorGreen(config.Workload):
    """Slip walls in x and z, periodic y, no sponges, no SGS, no density."""

    def params(self):
        p = super().params()
        p.update(vspngx1=0, dspngx1=0)
        return p


def _taylor_green(oracle, mx, steps=50, dt=0.01, re=100.0):
    """Known answer: the decaying Taylor-Green vortex of the reference
    (src/boundary.f:996-1044, uvel/wvel/pres_taylor_green on 0 < x, y < pi),
    shifted by pi/2 in x and placed in the x-y plane: u = cos x cos y F,
    v = sin x sin y F, p = (cos 2y - cos 2x) F^2 / 4, F = exp(-2 nu t), on
    x in [-pi/2, pi/2] (u = 0 and dv/dx = 0 at the walls: free slip, type
    60) and y in [-pi, pi] (periodic); uniform in z with w = 0 between slip
    walls.  Returns the max errors of u and v relative to F, max |w|, the
    fitted amplitude of u against F, and max |div u|."""
    import math
    w = _TaylorGreen("taylor_green", mx=mx, ly=2 * mx, nz_=4, xlim=(-math.pi / 2, math.pi / 2),
                     ylim=(-math.pi, math.pi), zlim=(-1.0, 1.0), beta=1e-3, re=re, dt=dt, steps=steps,
                     noise=0.0, isgs=0, idens=0, itype=(60, 60, 500, 500, 60, 60), sphere=False)
    o = oracle.OracleSolver(w)
    xu, xc, yv, yc = (o.grid.get(n) for n in ("xu", "xc", "yv", "yc"))
    sh = (w.nx, w.ny, w.nz)
    one = np.ones(sh)
    U = (np.cos(xu)[:, None] * np.cos(yc)[None, :])[:, :, None] * one
    V = (np.sin(xc)[:, None] * np.sin(yv)[None, :])[:, :, None] * one
    P = (0.25 * (np.cos(2 * yc)[None, :] - np.cos(2 * xc)[:, None]))[:, :, None] * one
    z2 = np.zeros(sh[:2], order="F")
    o.load_initial(dict(uo=np.asfortranarray(U), vo=np.asfortranarray(V), wo=np.zeros(sh, order="F"),
                        p=np.asfortranarray(P), dens=np.zeros(sh, order="F"),
                        planeU=z2, planeV=z2, planeW=z2, planeD=z2))
    o.initialize()
    o.step(steps)
    F = math.exp(-2.0 * steps * dt / re)
    inner = (slice(1, -1), slice(1, -1), slice(1, -1))
    u, v, ww = o.get("uo"), o.get("vo"), o.get("wo")
    eu = float(np.max(np.abs(u[inner] - F * U[inner]))) / F
    ev = float(np.max(np.abs(v[inner] - F * V[inner]))) / F
    amp = float(np.sum(u[inner] * U[inner]) / np.sum(U[inner] ** 2))
    return eu, ev, float(np.max(np.abs(ww[inner]))), amp / F, o.max_divergence()


def test_taylor_green_decay_known_answer(oracle):
    # 16 and 32 cells across pi, 50 steps of dt = 0.01 at Re = 100
    e16 = _taylor_green(oracle, 16)
    e32 = _taylor_green(oracle, 32)
    for e in (e16, e32):
        eu, ev, wmax, amp, div = e
        assert wmax < 1e-12 and div < 1e-12
        assert abs(amp - 1.0) < 1e-4          # decay rate exp(-2 nu t)
    assert e16[0] < 1e-4 and e16[1] < 1e-4    # measured 3.2e-5
    assert e32[0] < 2.5e-5 and e32[1] < 2.5e-5
    # second order in space: the error falls by 4 when the spacing halves
    for a in (0, 1):
        assert 3.5 < e16[a] / e32[a] < 4.5, (e16[a], e32[a])


@pytest.mark.parametrize("n", [6, 12, 24, 48, 96, 384])
def test_fft_non_power_of_two_matches_numpy(oracle, n):
    # lengths 3 x 2^m (the transform of the 384-wide periodic extent): the
    # oracle's transform against numpy's FFT, in FFTPACK's packed order
    x = np.random.RandomState(n).randn(n)
    r = oracle.rfftf(x)
    f = np.fft.rfft(x)
    want = np.empty(n)
    want[0] = f[0].real
    want[1:-1:2] = f[1:n // 2].real
    want[2:-1:2] = f[1:n // 2].imag
    want[-1] = f[n // 2].real
    np.testing.assert_allclose(r, want, rtol=0, atol=1e-12 * np.max(np.abs(want)))
    np.testing.assert_allclose(oracle.rfftb(r), n * x, rtol=0, atol=1e-11 * n * np.max(np.abs(x)))
