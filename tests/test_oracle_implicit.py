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


def _xpair(oracle, implx, imply, steps):
    w = config.small(mx=16, ly=16, nz_=24, noise=0.2, re=500.0, imply=imply, implx=implx)
    o = oracle.OracleSolver(w)
    o.load_initial(config.initial_fields(w, o.grid.get("dens_bg")[: w.nx]))
    o.initialize()
    o.step(steps)
    return o


def test_inversex_lines_solve_their_systems(oracle):
    # every x line after INVERSEX satisfies the Crank-Nicolson system of
    # src/timeindeg.f:441-686 as a numpy restatement assembles it: u with
    # zero wall values at i = 1 and NX-1, v and w with Neumann walls
    w = config.small(mx=16, ly=8, nz_=12, noise=0.3, re=50.0, implx=1)
    o = oracle.OracleSolver(w)
    o.load_initial(config.initial_fields(w, o.grid.get("dens_bg")[: w.nx]))
    o.initialize()
    rng = np.random.default_rng(5)
    tv = np.abs(rng.standard_normal((w.nx, w.ny, w.nz))) * 1e-2
    o.set("tv", np.asfortranarray(tv))
    alf = 2 / 15 * 1e-2
    o.rhs_predictord(alf, 5 / 12 * 1e-2, -17 / 60 * 1e-2)
    before = {n: o.get(n).copy() for n in ("us", "vs", "ws")}
    o.inversex_walls(alf)
    o.inversex(alf)
    after = {n: o.get(n) for n in ("us", "vs", "ws")}
    g = {n: o.grid.get(n) for n in ("ap", "au", "av", "aw")}
    coef, ru1, nx = 0.5 * alf, 1.0 / w.re, w.nx
    worst = 0.0
    for comp in ("us", "vs", "ws"):
        r, x = before[comp], after[comp]
        i = np.arange(2, nx if comp != "us" else nx - 1)  # Fortran indices 2..NX-1 (u: NX-2)
        ks = range(2, w.nz - 1) if comp != "ws" else range(2, w.nz - 2)
        for k in ks:
            for j in range(2, w.ny):
                T = lambda ii, dj=0, dk=0: tv[ii - 1, j - 1 + dj, k - 1 + dk]  # noqa: E731
                if comp == "us":
                    cx = coef * g["au"][i - 1]
                    a = -cx * g["ap"][i - 1] * (2 * T(i) + ru1)
                    c = -cx * g["ap"][i] * (2 * T(i + 1) + ru1)
                    xl = np.concatenate([[0.0], x[i[:-1] - 1, j - 1, k - 1]])
                    xr = np.concatenate([x[i[1:] - 1, j - 1, k - 1], [0.0]])
                else:
                    dj, dk = (1, 0) if comp == "vs" else (0, 1)
                    tp = 0.25 * (T(i, dj, dk) + T(i) + T(i + 1, dj, dk) + T(i + 1)) + ru1
                    tm = 0.25 * (T(i, dj, dk) + T(i) + T(i - 1, dj, dk) + T(i - 1)) + ru1
                    cx = coef * g["av" if comp == "vs" else "aw"][i - 1]
                    a = -cx * g["au"][i - 2] * tm
                    c = -cx * g["au"][i - 1] * tp
                    xs = x[i - 1, j - 1, k - 1]
                    xl = np.concatenate([[xs[0]], xs[:-1]])  # Neumann: ghost = first cell
                    xr = np.concatenate([xs[1:], [xs[-1]]])
                b = 1.0 - a - c
                res = a * xl + b * x[i - 1, j - 1, k - 1] + c * xr - r[i - 1, j - 1, k - 1]
                worst = max(worst, float(np.max(np.abs(res)) / np.max(np.abs(r[i - 1, j - 1, k - 1]))))
        assert not np.array_equal(before[comp], after[comp]), comp
    assert worst < 1e-13, worst


@pytest.mark.parametrize("imply", [0, 1])
def test_implicit_x_step_is_projected_and_close_to_explicit(oracle, imply):
    oi, oe = _xpair(oracle, 1, imply, 4), _xpair(oracle, 0, imply, 4)
    assert oi.max_divergence() < 1e-12
    for n in ("uo", "vo", "wo", "dens", "p"):
        a, b = oi.get(n)[1:-1, 1:-1, 1:-1], oe.get(n)[1:-1, 1:-1, 1:-1]
        assert np.all(np.isfinite(a)), n
        d = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)
        assert 0 < d < 5e-3, (n, d)


def _mode_state(oracle, beta=2.0, **kw):
    w = config.small(mx=32, ly=16, nz_=12, isgs=0, idens=0, re=20.0, beta=beta, **kw)
    o = oracle.OracleSolver(w)
    z = np.zeros((w.nx, w.ny, w.nz), order="F")
    for n in ("uo", "vo", "wo", "p", "tv", "dens", "ua", "va", "wa"):
        o.set(n, z)
    return o, w


def test_crank_nicolson_y_damps_a_y_mode_by_its_factor(oracle):
    # w = sin(k y) is an eigenvector of the periodic y operator, with u = v = 0
    # and p = 0 nothing else acts on it: the predictor's explicit half and
    # INVERSEY's implicit half give w* = w (1 + c lam) / (1 - c lam), c = alfxdt
    # ru1 / 2, lam = -(2 / dy^2)(1 - cos(k dy))
    o, w = _mode_state(oracle, imply=1)
    yc = o.grid.get("yc")
    ly = w.ylim[1] - w.ylim[0]
    dy = ly / w.ly
    for m in (1, 3):
        kk = 2 * np.pi * m / ly
        wo = np.asfortranarray(np.broadcast_to(np.sin(kk * (yc - w.ylim[0]))[None, :, None], (w.nx, w.ny, w.nz)))
        o.set("wo", wo)
        alf = 2 / 15 * 1e-2
        o.rhs_predictord(alf, 8 / 15 * 1e-2, 0.0)
        o.inversey(alf)
        lam = -(2 / dy ** 2) * (1 - np.cos(kk * dy))
        c = 0.5 * alf / w.re
        want = wo * (1 + c * lam) / (1 - c * lam)
        ws = o.get("ws")
        i_end = w.nx - 2 - max(2, w.mx // 24) - 1   # clear of the x sponge
        sl = (slice(1, i_end), slice(1, w.ny - 1), slice(1, w.nz - 2))
        assert np.max(np.abs(ws[sl] - want[sl])) < 1e-12
        assert np.max(np.abs(o.get("us"))) == 0 and np.max(np.abs(o.get("vs")[sl])) == 0


def test_crank_nicolson_x_lines_damp_x_modes_by_their_factor(oracle):
    # on a (nearly) uniform x grid sin(pi m x / Lx) on the u faces (zero at the
    # walls) and cos(pi m x / Lx) at the cell centres (Neumann) are
    # eigenvectors of the x lines of INVERSEX: v* = v / (1 - c lam)
    o, w = _mode_state(oracle, beta=1e-4, implx=1)
    xu, xc = o.grid.get("xu"), o.grid.get("xc")
    lx = w.xlim[1] - w.xlim[0]
    dx = lx / w.mx
    alf = 2 / 15 * 1e-2
    c = 0.5 * alf / w.re
    for m in (1, 2):
        lam = -(2 / dx ** 2) * (1 - np.cos(np.pi * m / w.mx))
        us = np.sin(np.pi * m * (xu - w.xlim[0]) / lx)[:, None, None] * np.ones((1, w.ny, w.nz))
        vs = np.cos(np.pi * m * (xc - w.xlim[0]) / lx)[:, None, None] * np.ones((1, w.ny, w.nz))
        us[-1] = 0.0
        for n, a in (("us", us), ("vs", vs), ("ws", vs)):
            o.set(n, np.asfortranarray(a))
        o.inversex_walls(alf)
        o.inversex(alf)
        f = 1.0 / (1 - c * lam)
        ku = slice(1, w.nz - 1)
        assert np.max(np.abs(o.get("us")[1:w.nx - 2, 1:-1, ku] - f * us[1:w.nx - 2, 1:-1, ku])) < 1e-6
        assert np.max(np.abs(o.get("vs")[1:-1, 1:-1, ku] - f * vs[1:-1, 1:-1, ku])) < 1e-6
        assert np.max(np.abs(o.get("ws")[1:-1, 1:-1, 1:w.nz - 2] - f * vs[1:-1, 1:-1, 1:w.nz - 2])) < 1e-6
