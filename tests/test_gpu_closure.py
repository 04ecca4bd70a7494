"""Learned closure: tensor-core forward/backward against the FP64 numpy
reference, fused inference against the reference, and what training gains
over the method without the network (a constant-coefficient eddy viscosity)."""
import sys
import os

import numpy as np
import pytest

from eddy_hybrid_b200 import closure as cl
from eddy_hybrid_b200 import config

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_ref  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def flow(product):
    """A small stratified flow with an active dynamic eddy viscosity."""
    w = config.small(mx=32, ly=32, nz_=48, noise=0.5, re=1e4, fr=1.0)
    s = product.Solver(w)
    s.load_initial(config.initial_fields(w, s.metric("dens_bg")[: w.nx]))
    s.initialize()
    snaps = []
    c = cl.Closure(s)
    for _ in range(3):
        s.step(1)
        cells = np.arange(w.mx * w.ly * w.nz_, dtype=np.int64)
        snaps.append(c.harvest(cells))
    return w, s, c, snaps


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def test_gradients_match_fp64_reference(flow):
    w, s, c, snaps = flow
    X, T = snaps[0]
    meta = cl.make_meta(X, T)
    theta = cl.init_theta(3)
    c.set(meta, theta)
    n = 1024
    rng = np.random.RandomState(5)
    idx = rng.choice(len(X), n, replace=False)
    Xb, Yb = X[idx], cl.targets(X[idx], T[idx], meta)[0]
    g, loss = c.grad(Xb, Yb)
    P = cl.unpack(theta)
    cache = mlp_ref.forward(P, mlp_ref.normalise(Xb, meta))
    gref, lref = mlp_ref.backward(cache, Yb.astype(np.float64))
    G = cl.unpack(g)
    assert abs(loss - lref) / lref < 1e-4
    for k in ("W1", "b1", "W2", "b2", "W3", "b3", "W4", "b4"):
        ref = gref[k]
        got = G[k][:ref.shape[0]] if k in ("W4", "b4") else G[k]
        if k == "W4":
            ref, got = ref[:2], got[:2]
        if k == "b4":
            ref, got = ref[:2], got[:2]
        assert rel(got, ref) < 2e-2, (k, rel(got, ref))
    # padding stays exactly zero
    assert np.all(G["W4"][2:] == 0) and np.all(G["b4"][2:] == 0) and np.all(G["W1"][:, 12:] == 0)


def test_fused_inference_matches_reference(flow):
    w, s, c, snaps = flow
    X, T = snaps[2]                # the solver's current state
    meta = cl.make_meta(X, T)
    theta = cl.init_theta(11)
    c.set(meta, theta)
    assert c.apply() == 0          # every cell inside the envelope it was fitted on
    cells = np.arange(w.mx * w.ly * w.nz_, dtype=np.int64)
    Xh, Th = c.harvest(cells)      # Th = nu_t(closure) / Delta
    np.testing.assert_allclose(Xh, X, rtol=0, atol=0)
    out = mlp_ref.forward(cl.unpack(theta), mlp_ref.normalise(X, meta))["out"]
    want = out[:, 0] * meta[4 * cl.NFEAT] * cl.strain_scale(X)
    assert rel(Th, want) < 1e-2, rel(Th, want)
    ka = c.kappa()[1:-1, 1:-1, 1:-1].ravel(order="F")
    nu = s.download("tv")[1:-1, 1:-1, 1:-1].ravel(order="F")
    assert rel(ka / nu, out[:, 1] / out[:, 0]) < 1e-2


def _smag_features(X):
    g = X[:, :9].reshape(-1, 3, 3).astype(np.float64)
    S = 0.5 * (g + np.transpose(g, (0, 2, 1)))
    return np.sqrt(2.0 * np.sum(S * S, axis=(1, 2)))   # Delta |S|


def test_training_gains_over_constant_coefficient(flow):
    w, s, c, snaps = flow
    Xtr = np.concatenate([snaps[0][0], snaps[1][0]])
    Ttr = np.concatenate([snaps[0][1], snaps[1][1]])
    Xte, Tte = snaps[2]
    meta = cl.make_meta(Xtr, Ttr)
    c.set(meta, cl.init_theta(0))
    Y, ok = cl.targets(Xtr, Ttr, meta)
    Xtr, Ttr, Y = Xtr[ok], Ttr[ok], Y[ok]
    Xtr, Ttr, Y = Xtr[: len(Xtr) // 128 * 128], Ttr[: len(Ttr) // 128 * 128], Y[: len(Y) // 128 * 128]
    hist = c.train(Xtr, Y, epochs=40, batch=2048, lr=3e-3, seed=1)
    print("training loss by epoch:", np.round(hist[::5], 4))
    assert hist[-1] < 0.8 * hist[0]
    # held-out snapshot through the fused inference kernel
    m2, th = c.get()
    cache = mlp_ref.forward(cl.unpack(th), mlp_ref.normalise(Xte, meta))
    pred = cache["out"][:, 0] * meta[4 * cl.NFEAT] * cl.strain_scale(Xte)
    err_mlp = rel(pred, Tte)
    # without the network: nu_t/Delta = C * Delta|S| with the best constant C
    q = _smag_features(Xtr)
    C = float(np.dot(q, Ttr) / np.dot(q, q))
    err_const = rel(C * _smag_features(Xte), Tte)
    print(f"held-out nu_t error: network {err_mlp:.3f}, constant coefficient {err_const:.3f}")
    assert err_mlp < err_const
