"""CPU checks of the oracle's control-volume body force (calcfrc,
src/calcforce.f:3-779, Cartesian branch) on fields whose answer is known:
a uniform stream carries momentum through the inlet and outlet faces and
nothing else, the volume integral is the volume times the velocity, and the
unsteady term is its change over dt; a uniform shear flow's stresses cancel
face against face, so the force on an empty control volume vanishes."""
import numpy as np

from eddy_hybrid_b200 import config

CV = (-1.5, 1.5, -1.5, 2.0)


def _oracle(oracle, **kw):
    w = config.small(mx=24, ly=8, nz_=32, **kw)
    o = oracle.OracleSolver(w)
    return o, w


def _set(o, w, u=0.0, v=0.0, wv=None, p=0.0):
    shape = (w.nx, w.ny, w.nz)
    o.set("uo", np.full(shape, u, order="F"))
    o.set("vo", np.full(shape, v, order="F"))
    o.set("wo", np.asfortranarray(np.broadcast_to(wv, shape)) if wv is not None else np.zeros(shape, order="F"))
    o.set("p", np.full(shape, p, order="F"))


def test_cv_range_follows_closest_and_locate(oracle):
    o, w = _oracle(oracle)
    xu, zw = o.grid.get("xu"), o.grid.get("zw")
    icb, ice, kcb, kce, kbf, kef = o.cv_range(CV)
    assert kbf == 1 and kef == 1
    # the closest x faces, and KCB one past the face below z1
    assert abs(xu[icb - 1] - CV[0]) <= min(abs(xu[icb - 2] - CV[0]), abs(xu[icb] - CV[0]))
    assert abs(xu[ice - 1] - CV[1]) <= min(abs(xu[ice - 2] - CV[1]), abs(xu[ice] - CV[1]))
    assert zw[kcb - 2] <= CV[2] < zw[kcb - 1]
    assert zw[kce - 1] <= CV[3] < zw[kce]
    # past the domain: the reference's adjusted ranges
    assert o.cv_range((-1.5, 1.5, -99.0, 2.0))[2:] == (1, kce, 0, 1)
    assert o.cv_range((-1.5, 1.5, -99.0, 99.0))[2:] == (1, w.nz - 1, 0, 0)
    assert o.cv_range((-1.5, 1.5, 99.0, 99.0))[2:] == (w.nz, 0, 0, 0)


def test_uniform_stream(oracle):
    o, w = _oracle(oracle)
    _set(o, w, wv=1.0)
    xu, zw = o.grid.get("xu"), o.grid.get("zw")
    icb, ice, kcb, kce, _, _ = o.cv_range(CV)
    area = (xu[ice - 1] - xu[icb - 1]) * (w.ylim[1] - w.ylim[0])
    vol = area * (zw[kce - 1] - zw[kcb - 1])
    fb = np.zeros(3)
    out = o.calcfrc(CV, 1e-3, 0, fb)
    fz = out[12:18]
    assert abs(fz[0] + area) < 1e-12 * area and abs(fz[1] - area) < 1e-12 * area
    assert np.all(fz[2:] == 0) and np.all(out[0:6] == 0)
    assert abs(fb[2] - vol) < 1e-12 * vol and fb[0] == 0 and fb[1] == 0
    assert np.all(out[18:21] == 0)                      # icycle 0: no unsteady term
    assert abs(out[23]) < 1e-12 * area                  # inlet and outlet cancel
    # the inlet record: pressure 0, no stress, momentum flux -area
    assert abs(out[24 + 4] + area) < 1e-12 * area and out[24 + 2] == 0 and out[24 + 3] == 0
    # doubled velocity one step later: unsteady term (2V - V) / dt
    _set(o, w, wv=2.0)
    out = o.calcfrc(CV, 1e-3, 1, fb)
    assert abs(out[20] - vol / 1e-3) < 1e-10 * vol / 1e-3


def test_uniform_shear_has_no_net_force(oracle):
    o, w = _oracle(oracle, re=50.0)
    xc = o.grid.get("xc")
    wv = (0.7 * xc)[:, None, None] * np.ones((1, w.ny, w.nz))
    _set(o, w, wv=wv, p=0.3)
    fb = np.zeros(3)
    out = o.calcfrc(CV, 1e-3, 0, fb)
    fx, fz = out[0:6], out[12:18]
    # the shear stress ru1 * dw/dx acts on the x-y and y-z faces and cancels
    # between opposite faces; the pressure cancels likewise
    scale = max(np.max(np.abs(fx)), np.max(np.abs(fz)))
    assert scale > 0 and abs(fx[0]) > 0 and abs(fz[2]) > 0
    assert abs(out[21]) < 1e-12 * scale and abs(out[23]) < 1e-12 * scale
