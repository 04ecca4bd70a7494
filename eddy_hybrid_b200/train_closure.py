"""Train the learned eddy-viscosity closure on the GPU from pairs the plain
FP64 solver generates, and write the weights the mixed form loads.

python -m eddy_hybrid_b200.train_closure [--grid 192x128x256] [--frs 0.5,1,2]
        [--noise 0.001,0.3] [--spin 5] [--snaps 4] [--every 5] [--per-snap 800000]
        [--epochs 8] [--out eddy_hybrid_b200/closure_weights.npz]

For each Froude number and initial noise amplitude a plain solver (dynamic
Smagorinsky, src/vt.f:16-442) with the moving sphere runs `spin` steps from the
seeded initial state, then every `every` steps a sample of interior cells is
harvested: the 12 closure features and the dynamic model's nu_t / Delta (the
target).  The small amplitude is the wake workload's own start (activity only
around the body), the large one gives turbulence-like gradients everywhere.
The last snapshot of every run is held out.  Training runs the library's own tensor-core forward and
backward kernels and Adam (eddy_closure_train).  The report records the
held-out relative nu_t error of the network and of the best constant
Smagorinsky coefficient (the method without the network).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import MIXED, PLAIN_FP64, Solver  # noqa: F401
from . import closure as cl
from . import config

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "closure_weights.npz")


smag_scale = cl.strain_scale


def rel(a, b) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def harvest(grid=(192, 128, 256), frs=(0.5, 1.0, 2.0), spin=5, snaps=4, every=5, per_snap=800_000,
            re=1e4, noises=(0.001, 0.3), sphere=True, seed=0, log=print):
    """Run the plain solver at each Froude number and noise amplitude and
    harvest (X, T) samples.  Returns the training and held-out sets and the
    last solver (for training)."""
    mx, ly, nz_ = grid
    train_x, train_t, test_x, test_t = [], [], [], []
    solver = None
    runs = [(fr, noise) for noise in noises for fr in frs]
    for fi, (fr, noise) in enumerate(runs):
        # velocity fluctuations strong enough for the dynamic procedure to
        # produce a non-zero eddy viscosity (its coefficient is clipped at 0)
        w = config.Workload(f"train_fr{fr}", mx=mx, ly=ly, nz_=nz_, re=re, fr=fr, dt=5e-4, sphere=sphere,
                            noise=noise, body_speed=1.0)
        if solver is not None:
            solver.close()
        s = Solver(w)
        if sphere:
            from . import body as bd
            h = float(np.diff(w.faces()[0]).min())
            tri, nrm = bd.icosphere(bd.level_for_spacing(max(h, 0.004)))
            s.set_body(tri, nrm, bd.body_velocity(w))
        s.load_initial(config.initial_fields(w, s.metric("dens_bg")[: w.nx]))
        s.initialize()
        s.step(spin)
        c = cl.Closure(s)
        for k in range(snaps):
            s.step(every)
            cells = cl.sample_cells(w, per_snap, seed + 100 * fi + k)
            X, T = c.harvest(cells)
            ok = np.isfinite(X).all(axis=1) & np.isfinite(T)
            X, T = X[ok], T[ok]
            (test_x if k == snaps - 1 else train_x).append(X)
            (test_t if k == snaps - 1 else train_t).append(T)
            log(f"  Fr={fr} noise={noise} snapshot {k}: {len(X)} samples, mean nu_t/Delta {T.mean():.3e}")
        solver = s
    return (np.concatenate(train_x), np.concatenate(train_t), np.concatenate(test_x), np.concatenate(test_t),
            solver)


def train(solver, X, T, epochs=8, batch=8192, lr=2e-3, seed=1, log=print):
    meta = cl.make_meta(X, T)
    c = cl.Closure(solver)
    c.set(meta, cl.init_theta(seed))
    Y, ok = cl.targets(X, T, meta)
    hist = c.train(X[ok], Y[ok], epochs=epochs, batch=batch, lr=lr, seed=seed)
    log(f"  training loss by epoch: {np.round(hist, 4).tolist()}")
    meta, theta = c.get()
    return meta, theta, hist


def evaluate(meta, theta, X, T):
    """Held-out relative nu_t error of the network (FP32 numpy forward of the
    BF16 weights) and of the best constant coefficient fitted on the same set."""
    P = cl.unpack(theta)
    Z = (X - meta[:cl.NFEAT]) * meta[cl.NFEAT:2 * cl.NFEAT]
    h = Z.astype(np.float64)

    def act(x):  # hard-swish
        return x * np.clip(x / 6.0 + 0.5, 0.0, 1.0)
    pad = np.zeros((len(h), cl.KIN))
    pad[:, :cl.NFEAT] = h
    a = act(pad @ P["W1"].T.astype(np.float64) + P["b1"])
    a = act(a @ P["W2"].T.astype(np.float64) + P["b2"])
    a = act(a @ P["W3"].T.astype(np.float64) + P["b3"])
    o = a @ P["W4"].T.astype(np.float64) + P["b4"]
    nu = np.logaddexp(0.0, o[:, 0]) * meta[4 * cl.NFEAT] * smag_scale(X)
    outside = ((Z < meta[2 * cl.NFEAT:3 * cl.NFEAT]) | (Z > meta[3 * cl.NFEAT:4 * cl.NFEAT])).any(axis=1)
    q = smag_scale(X)
    C = float(np.dot(q, T) / np.dot(q, q))
    return {"nu_t_rel_err_network": rel(nu, T), "nu_t_rel_err_constant_coeff": rel(C * q, T),
            "constant_coeff_C": C, "held_out_samples": int(len(T)),
            "held_out_outside_envelope": float(outside.mean())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", default="192x128x256", help="NX-2 x NY-2 x NZ-2 of the training runs")
    ap.add_argument("--frs", default="0.5,1,2")
    ap.add_argument("--spin", type=int, default=5)
    ap.add_argument("--snaps", type=int, default=4)
    ap.add_argument("--every", type=int, default=5)
    ap.add_argument("--per-snap", type=int, default=800_000)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--noise", default="0.001,0.3", help="initial velocity noise amplitudes (comma list)")
    ap.add_argument("--no-sphere", action="store_true", help="train on flows without the immersed sphere")
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=DEFAULT_OUT)
    a = ap.parse_args()
    grid = tuple(int(v) for v in a.grid.split("x"))
    frs = tuple(float(v) for v in a.frs.split(","))
    t0 = time.time()
    noises = tuple(float(v) for v in a.noise.split(","))
    X, T, Xt, Tt, s = harvest(grid, frs, a.spin, a.snaps, a.every, a.per_snap, noises=noises,
                              sphere=not a.no_sphere)
    t1 = time.time()
    print(f"harvested {len(X)} training / {len(Xt)} held-out samples in {t1 - t0:.1f} s")
    meta, theta, hist = train(s, X, T, a.epochs, a.batch, a.lr)
    t2 = time.time()
    rep = evaluate(meta, theta, Xt, Tt)
    rep.update({"train_samples": int(len(X)), "grid": list(grid), "frs": list(frs), "epochs": a.epochs,
                "noise": list(noises), "sphere": not a.no_sphere, "mean_target": float(T.mean()),
                "loss_by_epoch": [float(v) for v in hist], "harvest_s": t1 - t0, "train_s": t2 - t1})
    print(json.dumps(rep))
    np.savez(a.out, meta=meta, theta=theta, report=json.dumps(rep))
    s.close()
    return 0


def load(path: str = DEFAULT_OUT):
    """(meta, theta, report) of a saved network, or None."""
    if not os.path.exists(path):
        return None
    z = np.load(path)
    return z["meta"], z["theta"], json.loads(str(z["report"]))


if __name__ == "__main__":
    raise SystemExit(main())
