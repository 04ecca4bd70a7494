"""CUDA path against the CPU oracle on the same seeded inputs.

Kernel-level: identical input state in both, one C-ABI entry point, compare
every output.  Stencil kernels compiled with -fmad=false are bit-exact; the
Poisson solve (eigen-transform + DGEMM vs Jacobi eigenvectors in the oracle)
and anything after a reduction is compared at 1e-12 relative.  Step-level:
the whole time advance at the FP64 bar of 1e-11 relative on velocity,
pressure and density and max|div u| < 1e-12.
"""
import numpy as np
import pytest

from conftest import P_BAR, P_PROFILE_BAR, p_err, p_profile_err, rel_err, run_with_scale
from eddy_hybrid_b200 import config

pytestmark = pytest.mark.gpu

STATE = ["uo", "vo", "wo", "p", "dens", "tv", "us", "vs", "ws", "ua", "va", "wa",
         "rha", "planeU", "planeV", "planeW", "planeD"]


def make_pair(oracle, product, w, steps=2):
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    o.load_initial(f)
    o.initialize()
    if steps:
        o.step(steps)
    g = product.Solver(w)
    for n in STATE:
        g.upload(n, o.get(n))
    return o, g


@pytest.fixture(scope="module")
def wsmall():
    return config.small(mx=20, ly=16, nz_=24, noise=0.3, re=2000.0)


def test_rhs_predictord_bit_exact(oracle, product, wsmall):
    o, g = make_pair(oracle, product, wsmall)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.rhs_predictord(alf, gam, rho)
    g.call("eddy_rhs_predictord", alf, gam, rho)
    for n in ("us", "vs", "ws", "ua", "va", "wa"):
        np.testing.assert_array_equal(g.download(n), o.get(n), err_msg=n)


def test_boundary_and_inout(oracle, product, wsmall):
    o, g = make_pair(oracle, product, wsmall)
    alf = 8 / 15 * 1e-3
    o.rhs_predictord(alf, alf, 0.0)
    g.call("eddy_rhs_predictord", alf, alf, 0.0)
    o.boundary(0); o.boundinout(1, alf); o.boundary(0)
    g.call("eddy_boundary", 0); g.call("eddy_boundinout", 1, alf); g.call("eddy_boundary", 0)
    for n in ("us", "vs", "ws"):
        assert rel_err(g.download(n), o.get(n)) < 1e-14, n


def test_direct_poisson(oracle, product, wsmall):
    o, g = make_pair(oracle, product, wsmall)
    alf = 8 / 15 * 1e-3
    for s in (o,):
        s.rhs_predictord(alf, alf, 0.0); s.boundary(0); s.boundinout(1, alf); s.boundary(0)
    for n in ("us", "vs", "ws"):
        g.upload(n, o.get(n))
    o.direct_from_velocity(alf, 0)
    g.call("eddy_direct", alf)
    dpo, dpg = o.get("dp"), g.download("dp")
    assert rel_err(dpg, dpo) < 1e-12


def test_poisson_standalone_manufactured(oracle, product):
    w = config.small(mx=24, ly=16, nz_=20, beta=2.5)
    o = oracle.OracleSolver(w)
    g = product.Solver(w)
    rng = np.random.RandomState(7)
    d = np.zeros((w.nx, w.ny, w.nz), order="F")
    d[1:-1, 1:-1, 1:-1] = rng.randn(w.mx, w.ly, w.nz_)
    ap, cp = o.grid.get("ap"), o.grid.get("cp")
    vol = (1 / ap[1:-1])[:, None, None] * np.ones((1, w.ly, 1)) * (1 / cp[1:-1])[None, None, :]
    inner = d[1:-1, 1:-1, 1:-1]
    inner -= (inner * vol).sum() / vol.sum()
    x = g.poisson_solve(d)
    r = o.apply_laplacian(x)
    assert np.max(np.abs(r[1:-1, 1:-1, 1:-1] - inner)) / np.max(np.abs(inner)) < 1e-12
    o.set("dp", d)
    o.direct(1)
    assert rel_err(x, o.get("dp")) < 1e-12


def test_correct_and_pressure_update_bit_exact(oracle, product, wsmall):
    o, g = make_pair(oracle, product, wsmall)
    alf = 8 / 15 * 1e-3
    o.rhs_predictord(alf, alf, 0.0); o.boundary(0); o.boundinout(1, alf); o.boundary(0)
    o.direct_from_velocity(alf, 0)
    for n in ("us", "vs", "ws", "dp"):
        g.upload(n, o.get(n))
    o.correct(alf); g.call("eddy_correct", alf)
    for n in ("uo", "vo", "wo"):
        np.testing.assert_array_equal(g.download(n), o.get(n), err_msg=n)
    o.pressure_update(); g.call("eddy_pressure_update")
    np.testing.assert_array_equal(g.download("p"), o.get("p"))


def test_density_bit_exact(oracle, product, wsmall):
    o, g = make_pair(oracle, product, wsmall)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.density(alf, gam, rho)
    g.call("eddy_density", alf, gam, rho)
    np.testing.assert_array_equal(g.download("dens"), o.get("dens"))
    np.testing.assert_array_equal(g.download("rha")[1:-1, 1:-1, 1:-1], o.get("rha")[1:-1, 1:-1, 1:-1])


def test_turvis_dynamic(oracle, product, wsmall):
    o, g = make_pair(oracle, product, wsmall)
    o.turvis()
    g.call("eddy_turvis")
    tvo, tvg = o.get("tv"), g.download("tv")
    assert tvo[1:-1, 1:-1, 1:-1].max() > 0
    np.testing.assert_array_equal(tvg, tvo)


@pytest.mark.parametrize("shape", [(16, 8, 24), (24, 16, 32)])
def test_full_step_parity(oracle, product, shape):
    mx, ly, nz_ = shape
    w = config.small(mx=mx, ly=ly, nz_=nz_, noise=0.2, re=2000.0)
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    o.load_initial(f)
    o.initialize()
    g = product.Solver(w)
    g.load_initial(f)
    g.initialize()
    # the outflow mass balance sums in a different order on the device, so
    # from here on the bar is the FP64 parity tolerance, not bit equality
    assert rel_err(g.download("tv"), o.get("tv")) < 1e-12
    scale = run_with_scale(o, 10)
    g.step(10)
    for n in ("uo", "vo", "wo", "dens", "tv"):
        e = rel_err(g.download(n), o.get(n))
        assert e < 1e-11, (n, e)
    pg = g.download("p")
    e = p_err(pg, o.get("p"), scale)
    assert e < P_BAR, ("p", e)
    e = p_profile_err(pg, o.get("p"), scale)
    assert e < P_PROFILE_BAR, ("p profile", e)
    assert g.max_divergence() < 1e-12
    assert o.max_divergence() < 1e-12


@pytest.mark.parametrize("ischm,isgs", [(1, 2), (3, 1), (3, 0)])
def test_step_parity_schemes_and_sgs_models(oracle, product, ischm, isgs):
    # AB2 (one substep, src/inpall.f:218-235), the static Smagorinsky model and
    # no SGS model, 10 steps against the oracle
    w = config.small(mx=16, ly=8, nz_=24, noise=0.2, re=2000.0, ischm=ischm, isgs=isgs)
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    o.load_initial(f)
    o.initialize()
    g = product.Solver(w)
    g.load_initial(f)
    g.initialize()
    scale = run_with_scale(o, 10)
    g.step(10)
    names = ("uo", "vo", "wo", "dens") + (("tv",) if isgs else ())
    for n in names:
        e = rel_err(g.download(n), o.get(n))
        assert e < 1e-11, (n, e)
    if isgs:
        assert float(np.max(o.get("tv")[1:-1, 1:-1, 1:-1])) > 0
    pg = g.download("p")
    assert p_err(pg, o.get("p"), scale) < P_BAR
    assert p_profile_err(pg, o.get("p"), scale) < P_PROFILE_BAR
    assert g.max_divergence() < 1e-12


@pytest.fixture(scope="module")
def wimply():
    # the reference's own input runs the y viscous terms Crank-Nicolson (IMPLY = 1)
    return config.small(mx=20, ly=16, nz_=24, noise=0.3, re=500.0, imply=1)


def test_inversey_bit_exact(oracle, product, wimply):
    o, g = make_pair(oracle, product, wimply)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.rhs_predictord(alf, gam, rho)
    g.call("eddy_rhs_predictord", alf, gam, rho)
    for n in ("us", "vs", "ws", "ua", "va", "wa"):
        np.testing.assert_array_equal(g.download(n), o.get(n), err_msg="predictor " + n)
    o.inversey(alf)
    g.call("eddy_inversey", alf)
    for n in ("us", "vs", "ws"):
        np.testing.assert_array_equal(g.download(n), o.get(n), err_msg="inversey " + n)


def test_density_implicit_y_bit_exact(oracle, product, wimply):
    o, g = make_pair(oracle, product, wimply)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.density(alf, gam, rho)
    g.call("eddy_density", alf, gam, rho)
    np.testing.assert_array_equal(g.download("dens"), o.get("dens"))


@pytest.mark.parametrize("shape", [(16, 16, 24), (24, 32, 32)])
def test_full_step_parity_implicit_y(oracle, product, shape):
    mx, ly, nz_ = shape
    w = config.small(mx=mx, ly=ly, nz_=nz_, noise=0.2, re=500.0, imply=1)
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


@pytest.fixture(scope="module")
def wimplx():
    # IMPLX = 1: the x viscous terms Crank-Nicolson, slip walls on both x sides
    return config.small(mx=20, ly=16, nz_=24, noise=0.3, re=500.0, implx=1)


def test_inversex_bit_exact(oracle, product, wimplx):
    o, g = make_pair(oracle, product, wimplx)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.rhs_predictord(alf, gam, rho)
    g.call("eddy_rhs_predictord", alf, gam, rho)
    for n in ("us", "vs", "ws", "ua", "va", "wa"):
        np.testing.assert_array_equal(g.download(n), o.get(n), err_msg="predictor " + n)
    o.inversex_walls(alf)
    o.inversex(alf)
    g.call("eddy_inversex", alf)
    for n in ("us", "vs", "ws"):
        np.testing.assert_array_equal(g.download(n), o.get(n), err_msg="inversex " + n)


def test_density_implicit_x_bit_exact(oracle, product, wimplx):
    o, g = make_pair(oracle, product, wimplx)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.density(alf, gam, rho)
    g.call("eddy_density", alf, gam, rho)
    np.testing.assert_array_equal(g.download("dens"), o.get("dens"))


@pytest.mark.parametrize("imply", [0, 1])
def test_full_step_parity_implicit_x(oracle, product, imply):
    w = config.small(mx=16, ly=16, nz_=24, noise=0.2, re=500.0, implx=1, imply=imply)
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
    assert abs(g.cfl() - o.calcfl()) < 1e-11 * o.calcfl()


_CONV = [(0, 0, 0, 1), (1, 0, 0, 1), (0, 0, 1, 0), (0, 1, 1, 0), (1, 1, 1, 1)]


@pytest.mark.parametrize("imply,implx,implcx,implcy", _CONV)
def test_line_solves_with_convection_bit_exact(oracle, product, imply, implx, implcx, implcy):
    # IMPLCX / IMPLCY: the convective terms inside the same line solves,
    # linearised about UO / VO and the provisional US / VS
    w = config.small(mx=20, ly=16, nz_=24, noise=0.3, re=500.0, imply=imply, implx=implx, implcx=implcx,
                     implcy=implcy)
    o, g = make_pair(oracle, product, w)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.rhs_predictord(alf, gam, rho)
    g.call("eddy_rhs_predictord", alf, gam, rho)
    for n in ("us", "vs", "ws", "ua", "va", "wa"):
        np.testing.assert_array_equal(g.download(n), o.get(n), err_msg="predictor " + n)
    if imply or implcy:
        o.inversey(alf)
        g.call("eddy_inversey", alf)
        for n in ("us", "vs", "ws"):
            np.testing.assert_array_equal(g.download(n), o.get(n), err_msg="inversey " + n)
    if implx or implcx:
        o.inversex_walls(alf)
        o.inversex(alf)
        g.call("eddy_inversex", alf)
        for n in ("us", "vs", "ws"):
            np.testing.assert_array_equal(g.download(n), o.get(n), err_msg="inversex " + n)


@pytest.mark.parametrize("imply,implx,implcx,implcy", _CONV)
def test_density_with_convection_bit_exact(oracle, product, imply, implx, implcx, implcy):
    # INVERSEYD_NEW when IMPLY and IMPLCY are both on; INVERSEXD with either x flag
    w = config.small(mx=20, ly=16, nz_=24, noise=0.3, re=500.0, imply=imply, implx=implx, implcx=implcx,
                     implcy=implcy)
    o, g = make_pair(oracle, product, w)
    alf, gam, rho = 2 / 15 * 1e-3, 5 / 12 * 1e-3, -17 / 60 * 1e-3
    o.density(alf, gam, rho)
    g.call("eddy_density", alf, gam, rho)
    np.testing.assert_array_equal(g.download("dens"), o.get("dens"))


@pytest.mark.parametrize("imply,implx,implcx,implcy", _CONV)
def test_full_step_parity_implicit_convection(oracle, product, imply, implx, implcx, implcy):
    w = config.small(mx=16, ly=16, nz_=24, noise=0.2, re=500.0, imply=imply, implx=implx, implcx=implcx,
                     implcy=implcy)
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
    assert abs(g.cfl() - o.calcfl()) < 1e-11 * o.calcfl()


@pytest.mark.parametrize("imply,implx,implcx,implcy", [(0, 0, 0, 0), (1, 0, 0, 0), (0, 1, 0, 0), (1, 1, 0, 0),
                                                      (0, 0, 1, 0), (0, 0, 0, 1), (1, 1, 1, 1)])
def test_cfl_and_extrema_bit_exact(oracle, product, imply, implx, implcx, implcy):
    w = config.small(mx=20, ly=16, nz_=24, noise=0.3, re=500.0, imply=imply, implx=implx, implcx=implcx,
                     implcy=implcy)
    o, g = make_pair(oracle, product, w)
    assert g.cfl() == o.calcfl() > 0
    for n in ("uo", "vo", "wo", "p", "dens", "tv"):
        a = o.get(n)[1:-1, 1:-1, 1:-1]
        assert g.extrema(n) == (a.min(), a.max()), n
    # constant-CFL stepping: DTM1 = CFLC / CFLM before every step
    c0 = g.cfl()
    dts = g.step_cfl(0.3, 2)
    assert dts[0] == 0.3 / c0 and g.max_divergence() < 1e-12
