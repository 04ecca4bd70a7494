"""The control-volume body force (calcfrc, src/calcforce.f:3-779) on the GPU
against the oracle, with the moving sphere inside the volume: the same
fields and the same body flags on both sides (flags bit-exact after the
steps), every one of the 56 output terms within the reduction-order
tolerance, including the unsteady term of a second call."""
import numpy as np
import pytest

from eddy_hybrid_b200 import body, config

pytestmark = pytest.mark.gpu

CV = (-1.5, 1.5, -1.5, 2.0)


def _close(g, o):
    scale = float(np.max(np.abs(o)))
    assert scale > 0
    np.testing.assert_allclose(g, o, rtol=1e-11, atol=1e-12 * scale)


def test_body_force_cv_matches_oracle(oracle, product):
    w = config.small(mx=32, ly=16, nz_=40, noise=0.2, re=2000.0)
    vel = (0.0, 0.0, -1.0)
    o = oracle.OracleSolver(w)
    tri, nrm = body.icosphere(3)
    ib = oracle.OracleIB(o, tri, nrm, vel, attach=True)
    g = product.Solver(w)
    g.set_body(tri, nrm, vel)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    o.load_initial(f)
    o.initialize()
    g.load_initial(f)
    g.initialize()
    fb = np.zeros(3)
    for icycle in (0, 1):
        o.step(2)
        g.step(2)
        for q in range(3):
            np.testing.assert_array_equal(g.ib_flags(4 + q), ib.flags(q), err_msg=f"flags {q}")
        for n in ("uo", "vo", "wo", "p"):
            g.upload(n, o.get(n))
        ref = o.calcfrc(CV, w.dt, icycle, fb)
        got = g.body_force_cv(CV, w.dt, icycle)
        # the body sits in the volume: some cells are excluded by the flags
        assert np.count_nonzero(ib.flags(2) > 0) > 0
        _close(got, ref)
    assert abs(ref[20]) > 0  # the unsteady term of the second call


def test_body_force_cv_refuses_outer_planes(product):
    w = config.small(mx=16, ly=8, nz_=16)
    g = product.Solver(w)
    with pytest.raises(product.EddyError):
        g.body_force_cv((-99.0, 1.0, -1.0, 1.0), 1e-3, 0)


@pytest.mark.parametrize("cv", [(-1.5, 1.5, -99.0, 2.0), (-1.5, 1.5, -1.5, 99.0), (-1.5, 1.5, -99.0, 99.0)])
def test_body_force_cv_volumes_past_the_domain(oracle, product, cv):
    # the reference's adjusted ranges when the volume reaches past an end of
    # the domain: the missing face is skipped, the volume clipped
    w = config.small(mx=24, ly=8, nz_=32, noise=0.2, re=2000.0)
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    o.load_initial(f)
    o.initialize()
    o.step(2)
    g = product.Solver(w)
    for n in ("uo", "vo", "wo", "p"):
        g.upload(n, o.get(n))
    fb = np.zeros(3)
    _close(g.body_force_cv(cv, w.dt, 0), o.calcfrc(cv, w.dt, 0, fb))
