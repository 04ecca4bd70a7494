"""Learned eddy-viscosity closure: parameter packing, feature normalisation,
training-data harvesting and training driver over the C ABI.

The network (12 -> 64 -> 64 -> 64 -> 2, hard-swish hidden, softplus outputs) maps
local, filter-width-scaled velocity- and density-gradient features to the
eddy-viscosity and diffusivity coefficients C_nu, C_kappa of
nu_t = C_nu Delta^2 |S| and kappa_t = C_kappa Delta^2 |S| (|S| from the same
gradient features), the form of the dynamic procedure's result, so the
closure scales with the local strain like the model it replaces.  It stands in for the test filtering and
coefficient averaging of the dynamic procedure (src/vt.f:172-431); targets
come from that procedure run by the plain solver itself, and kappa_t = nu_t
as in the reference's build (src/Eddy6.f:2959 passes TV as the diffusivity).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

NFEAT, KIN, HID, NOUT = 12, 16, 64, 16
OFF_W1 = 0
OFF_B1 = OFF_W1 + HID * KIN
OFF_W2 = OFF_B1 + HID
OFF_B2 = OFF_W2 + HID * HID
OFF_W3 = OFF_B2 + HID
OFF_B3 = OFF_W3 + HID * HID
OFF_W4 = OFF_B3 + HID
OFF_B4 = OFF_W4 + NOUT * HID
NTHETA = OFF_B4 + NOUT
NMETA = 4 * NFEAT + 2
FEATURES = ["du/dx", "du/dy", "du/dz", "dv/dx", "dv/dy", "dv/dz", "dw/dx", "dw/dy", "dw/dz",
            "|grad rho|", "N^2", "wall distance"]


def unpack(theta: np.ndarray) -> dict:
    t = np.asarray(theta, dtype=np.float32)
    return dict(W1=t[OFF_W1:OFF_B1].reshape(HID, KIN), b1=t[OFF_B1:OFF_W2],
                W2=t[OFF_W2:OFF_B2].reshape(HID, HID), b2=t[OFF_B2:OFF_W3],
                W3=t[OFF_W3:OFF_B3].reshape(HID, HID), b3=t[OFF_B3:OFF_W4],
                W4=t[OFF_W4:OFF_B4].reshape(NOUT, HID), b4=t[OFF_B4:NTHETA])


def init_theta(seed: int = 0) -> np.ndarray:
    """He-style initialisation; padding inputs/outputs stay exactly zero."""
    rng = np.random.RandomState(seed)
    th = np.zeros(NTHETA, dtype=np.float32)
    w1 = rng.randn(HID, KIN) * np.sqrt(2.0 / NFEAT)
    w1[:, NFEAT:] = 0.0
    th[OFF_W1:OFF_B1] = w1.ravel()
    th[OFF_W2:OFF_B2] = (rng.randn(HID, HID) * np.sqrt(2.0 / HID)).ravel()
    th[OFF_W3:OFF_B3] = (rng.randn(HID, HID) * np.sqrt(2.0 / HID)).ravel()
    w4 = np.zeros((NOUT, HID))
    w4[:2] = rng.randn(2, HID) * np.sqrt(1.0 / HID)
    th[OFF_W4:OFF_B4] = w4.ravel()
    return th


def strain_scale(X: np.ndarray) -> np.ndarray:
    """Delta*|S| = Delta*sqrt(2 S_ij S_ij) from the nine Delta-scaled
    velocity-gradient features (row a, column b: Delta du_a/dx_b)."""
    g = X[:, :9].reshape(-1, 3, 3).astype(np.float64)
    S = 0.5 * (g + np.transpose(g, (0, 2, 1)))
    return np.sqrt(2.0 * np.sum(S * S, axis=(1, 2)))


def coefficients(X: np.ndarray, T: np.ndarray):
    """Dynamic coefficient C = (nu_t/Delta) / (Delta|S|) of each sample and a
    mask of the samples where |S| is large enough to define it."""
    q = strain_scale(X)
    ok = q > 1e-8 * max(float(np.median(q)), 1e-30)
    C = np.zeros_like(q)
    C[ok] = T[ok].astype(np.float64) / q[ok]
    return C, ok


def make_meta(X: np.ndarray, T: np.ndarray, margin: float = 1.0) -> np.ndarray:
    """Feature mean/std, the training envelope (min/max of the normalised
    features widened by `margin` standard deviations) and coefficient scales."""
    mean = X.mean(axis=0)
    std = X.std(axis=0)
    std[std < 1e-12] = 1.0
    Z = (X - mean) / std
    lo = Z.min(axis=0) - margin
    hi = Z.max(axis=0) + margin
    C, ok = coefficients(X, T)
    s = float(np.sqrt(np.mean(C[ok] ** 2))) if ok.any() else 1.0
    s = s or 1.0
    return np.concatenate([mean, 1.0 / std, lo, hi, [s, s]]).astype(np.float32)


def targets(X: np.ndarray, T: np.ndarray, meta: np.ndarray):
    """Network targets (C_nu, C_kappa in output-scale units) for the samples
    where the coefficient is defined, and their mask."""
    s_nu, s_ka = meta[4 * NFEAT], meta[4 * NFEAT + 1]
    C, ok = coefficients(X, T)
    return np.stack([C / s_nu, C / s_ka], axis=1).astype(np.float32), ok


def sample_cells(workload, n: int, seed: int) -> np.ndarray:
    ninner = workload.mx * workload.ly * workload.nz_
    rng = np.random.RandomState(seed)
    return np.sort(rng.choice(ninner, size=min(n, ninner), replace=False)).astype(np.int64)


class Closure:
    """The closure network bound to one solver context."""

    def __init__(self, solver):
        self.s = solver
        from . import lib
        self.lib = lib()

    def set(self, meta: np.ndarray, theta: np.ndarray):
        meta = np.ascontiguousarray(meta, dtype=np.float32)
        theta = np.ascontiguousarray(theta, dtype=np.float32)
        self.s._check(self.lib.eddy_closure_set(self.s.h, _fp(meta), _fp(theta)), "eddy_closure_set")

    def get(self):
        meta = np.zeros(NMETA, dtype=np.float32)
        theta = np.zeros(NTHETA, dtype=np.float32)
        self.s._check(self.lib.eddy_closure_get(self.s.h, _fp(meta), _fp(theta)), "eddy_closure_get")
        return meta, theta

    def harvest(self, cells: np.ndarray):
        cells = np.ascontiguousarray(cells, dtype=np.int64)
        n = len(cells)
        X = np.zeros((n, NFEAT), dtype=np.float32)
        T = np.zeros(n, dtype=np.float32)
        self.s._check(self.lib.eddy_closure_harvest(self.s.h, cells.ctypes.data_as(C.c_void_p), n, _fp(X), _fp(T)),
                      "eddy_closure_harvest")
        return X, T

    def grad(self, X: np.ndarray, Y: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.zeros(NTHETA, dtype=np.float32)
        loss = C.c_double(0.0)
        self.s._check(self.lib.eddy_closure_grad(self.s.h, _fp(X), _fp(Y), len(X), _fp(g), C.byref(loss)),
                      "eddy_closure_grad")
        return g, loss.value

    def train(self, X, Y, epochs=5, batch=8192, lr=2e-3, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        hist = np.zeros(epochs)
        self.s._check(self.lib.eddy_closure_train(self.s.h, _fp(X), _fp(Y), len(X), epochs, batch, lr, seed,
                                                  hist.ctypes.data_as(C.POINTER(C.c_double))),
                      "eddy_closure_train")
        return hist

    def apply(self) -> int:
        n = C.c_longlong(0)
        self.s._check(self.lib.eddy_closure_apply(self.s.h, C.byref(n)), "eddy_closure_apply")
        return int(n.value)

    def refresh_fallback(self):
        self.s._check(self.lib.eddy_closure_refresh_fallback(self.s.h), "eddy_closure_refresh_fallback")

    def kappa(self) -> np.ndarray:
        a = np.zeros(self.s.shape, order="F")
        self.s._check(self.lib.eddy_download_kappa(self.s.h, a.ctypes.data_as(C.POINTER(C.c_double))),
                      "eddy_download_kappa")
        return a


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))
