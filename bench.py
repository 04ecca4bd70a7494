"""Throughput of the fractional-step time advance on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = 3 RK substeps (RHS+predictor, boundary fills, divergence + FFT
Poisson solve + projection, pressure update, density) + the eddy viscosity
update, on the 512x384x256 wake grid (streamwise x vertical x periodic) with
the moving sphere, fields resident on the GPU.  Three forms run from the same
state: plain FP64 (dynamic model), mixed (FP32 stencils, FFTs and dynamic
model, FP64-residual refinement and projection) and chosen (mixed with the
learned MLP closure).  Each is held to the accuracy contract against the
plain form; `value` is the fastest form that meets it.  Prints one JSON line.
N > 1 runs N independent replicas (the solver does not shard; one GPU holds
the whole domain): value = all ranks' cell-steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s at 512x384x256: plain FP64 vs FP32-refined+MLP closure, equal accuracy"
UNIT = "Mcell-steps/s"

# algorithmic HBM bytes per interior cell, per launch of each kernel category
# (compulsory reads + writes of 8-byte fields)
ALG_BYTES = {
    "rhs_predictor": 15 * 8,   # R u,v,w,p,rho,nu_t,ua,va,wa  W u*,v*,w*,ua,va,wa
    "div_fft_fwd": 4 * 8,      # R u*,v*,w*  W spectrum
    "transform_fwd": 2 * 8,    # R spectrum W spectrum (plus 2*M flops/cell)
    "z_line_solve": 2 * 8,     # R/W spectrum in place
    "transform_bwd": 2 * 8,
    "fft_bwd": 2 * 8,          # R spectrum W dp
    "correct": 7 * 8,          # R u*,v*,w*,dp  W u,v,w
    "pressure_update": 3 * 8,  # R p,dp W p
    "density": 8 * 8,          # R rho,u,v,w,nu_t,rha  W rho,rha
    "eddy_viscosity": 4 * 8,   # R u,v,w  W nu_t
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--sweeps", type=int, default=2, help="refinement sweeps of the mixed form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--small", action="store_true", help="tiny grid (smoke)")
    ap.add_argument("--medium", action="store_true",
                    help="128x192x128 grid (~3M cells, ~1 GB on the device) for ncu captures")
    ap.add_argument("--profile", default=None, choices=["plain", "mixed"],
                    help="run one form (warm-up + steps, the dynamic model) and exit without timing: the "
                         "command to put under a profiler")
    ap.add_argument("--poisson", action="store_true",
                    help="time the 256^3 Poisson solve alone (plain FP64 and refined FP32)")
    ap.add_argument("--deploy", action="store_true",
                    help="the learned closure deployed on 768x512x384 (Re 2e4, Fr 1, the moving sphere) for "
                         "--deploy-steps steps against a plain FP64 run: nu_t error against the dynamic model and "
                         "the wake-centreline velocity; prints one JSON line")
    ap.add_argument("--deploy-steps", type=int, default=200)
    ap.add_argument("--implicit", action="store_true",
                    help="the plain FP64 step of the wake workload with the y viscous terms Crank-Nicolson "
                         "(imply = 1, the reference input's setting) beside the explicit one; prints one JSON line")
    ap.add_argument("--grid", default=None,
                    help="NZ-2xNX-2xNY-2 of the wake workload, e.g. 64x384x256 (6.3M cells, fields larger "
                         "than L2, a few GB on the device) for ncu captures")
    return ap.parse_args()


def workload(small=False, medium=False, grid=None):
    from eddy_hybrid_b200 import config
    if grid:
        nz_, mx, ly = (int(v) for v in grid.split("x"))
        return config.Workload(f"wake_{nz_}x{mx}x{ly}", mx=mx, ly=ly, nz_=nz_, beta=2.0, re=1e4, fr=1.0,
                               dt=5e-4, body_speed=1.0)
    if medium:
        return config.Workload("wake_128x192x128", mx=192, ly=128, nz_=128, re=1e4, fr=1.0, dt=5e-4,
                               body_speed=1.0)
    if small:
        return config.Workload("wake_64x48x32", mx=48, ly=32, nz_=64, re=1e4, fr=1.0, dt=5e-4,
                               body_speed=1.0)
    return config.wake_512x384x256()


def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                smax = float(c[2])
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def _cpu_sample(grid, threads):
    """The CPU oracle (FP64 restatement of the reference loops, OpenMP over
    `threads` host cores) on the wake workload's equations and parameters on
    a coarser grid (streamwise x vertical x periodic), with the moving sphere
    regenerated every step, initialised and ready to step."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import eddy_oracle
    from eddy_hybrid_b200 import body as bd
    from eddy_hybrid_b200 import config
    nz_, mx, ly = grid
    w = config.Workload(f"wake_sample_{nz_}x{mx}x{ly}", mx=mx, ly=ly, nz_=nz_, re=1e4, fr=1.0, dt=5e-4,
                        body_speed=1.0)
    s = eddy_oracle.OracleSolver(w, threads=threads)
    xu = np.diff(w.faces()[0])
    tri, nrm = bd.icosphere(bd.level_for_spacing(max(float(xu.min()), 0.004)))
    ib = eddy_oracle.OracleIB(s, tri, nrm, bd.body_velocity(w), attach=True)
    s.load_initial(config.initial_fields(w, s.grid.get("dens_bg")[: w.nx]))
    s.initialize()
    return w, s, ib, len(tri)


CPU_GRID = (256, 192, 128)      # 1/8 of the cells of 512x384x256 (the all-core sample)
CPU_GRID_1CORE = (128, 96, 64)  # 1/64 of the cells (the one-core sample)


def cpu_baseline(steps=2):
    """Reported CPU baseline: the oracle port timed on the host cores, all
    cores on a 1/8 sample and one core on a 1/64 sample of the workload."""
    cores = len(os.sched_getaffinity(0))
    w, s, ib, ntri = _cpu_sample(CPU_GRID, cores)
    t0 = time.perf_counter()
    s.step(steps)
    dt = time.perf_counter() - t0
    w1, s1, ib1, ntri1 = _cpu_sample(CPU_GRID_1CORE, 1)
    t1 = time.perf_counter()
    s1.step(1)
    dt1 = time.perf_counter() - t1
    return {"value": w.ncell * steps / dt / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} full step(s) of the wake workload's equations on a {w.nz_}x{w.mx}x{w.ly} grid "
                      f"(1/8 of the cells) with the moving sphere ({ntri} triangles, tags and stencils "
                      f"regenerated every step) after initialisation; {dt:.2f} s on {cores} threads",
            "one_core": {"value": w1.ncell / dt1 / 1e6, "unit": UNIT, "cores": 1,
                         "sample": f"1 step on a {w1.nz_}x{w1.mx}x{w1.ly} grid (1/64 of the cells) with the "
                                   f"moving sphere ({ntri1} triangles); {dt1:.2f} s"}}


def run_reference(args):
    """The reference arm: the reference's CPU path, restated (the Fortran
    cannot be built here), timed on all host cores; one step = one time step
    of the 1/8-size sample with the moving sphere."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0))
    w, s, ib, ntri = _cpu_sample(CPU_GRID, cores)
    s.step(args.warmup)
    t0 = time.perf_counter()
    s.step(args.steps)
    dt = time.perf_counter() - t0
    v = w.ncell * args.steps / dt / 1e6
    cb = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
          "sample": f"{args.steps} timed step(s) after {args.warmup} warm-up step(s) of the wake workload's "
                    f"equations on a {w.nz_}x{w.mx}x{w.ly} grid (1/8 of the cells) with the moving sphere "
                    f"({ntri} triangles, regenerated every step); {dt:.2f} s on {cores} threads"}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / max(args.steps, 1) * 1e3, "ms_per_step_of": f"the {w.nz_}x{w.mx}x{w.ly} sample",
            "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"wake_512x384x256 sampled on {w.nz_}x{w.mx}x{w.ly}",
                       "form": "plain FP64 (CPU oracle port of the reference loops)",
                       "immersed_body": "moving sphere, regenerated every step"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# algorithmic bytes per interior cell per launch in the mixed forms (FP32
# stencil fields, FP64 masters, residual, solution and pressure)
ALG_BYTES_MIXED = {
    "rhs_predictor": 15 * 4,   # R 9 FP32 fields  W u*,v*,w*,ua,va,wa FP32
    "div_fft_fwd": 3 * 4 + 8 + 4,  # R u*,v*,w* FP32  W d FP64, spectrum FP32
    "refine_residual": 8 + 8 + 4,  # R phi, d FP64  W spectrum FP32
    "transform_fwd": 2 * 4,
    "z_line_solve": 5 * 4,     # R rhs, W eliminated; R eliminated, c' table, W solution (FP32)
    "transform_bwd": 2 * 4,
    "fft_bwd": 4 + 8,          # R spectrum FP32  W solution FP64 (the corrections also R it: below)
    "correct": 3 * 4 + 8 + 3 * 8 + 3 * 4,  # R u*,v*,w* FP32, dp  W u,v,w FP64 + FP32 copies
    "pressure_update": 8 + 8 + 8 + 4,      # R p,dp  W p FP64, p FP32
    "density": 6 * 4 + 2 * 4,              # R rho,kappa,u,v,w,rha  W rho,rha (FP32)
    "precision_copy": 4 + 8,               # one FP32<->FP64 copy
}


def step_alg_bytes(alg, sweeps, mixed):
    """Algorithmic bytes per cell of one step, the sum of the per-launch
    figures above: three substeps of RHS + predictor, divergence + FFT, the
    Poisson solve (mixed: 1 + sweeps solves, sweeps residuals, the backward
    passes writing (then adding to) the FP64 solution), CORRECT, the pressure
    update and the density, then the eddy viscosity (R u, v, w, W nu_t; the
    mixed form's FP32 copy of nu_t included)."""
    sub = alg["rhs_predictor"] + alg["div_fft_fwd"] + alg["correct"] + alg["pressure_update"] + alg["density"]
    solve = alg["transform_fwd"] + alg["z_line_solve"] + alg["transform_bwd"]
    if mixed:
        sub += (1 + sweeps) * solve + sweeps * alg["refine_residual"] + 12 + 20 * sweeps
        return 3 * sub + 3 * 4 + 8 + alg["precision_copy"]
    return 3 * (sub + solve + alg["fft_bwd"]) + alg["eddy_viscosity"]


# the learned closure: R u,v,w,rho FP32  W nu_t,kappa_t FP64 + FP32 copies
CLOSURE_BYTES = 4 * 4 + 2 * 8 + 2 * 4
MLP_FLOP_PER_CELL = 2 * (12 * 64 + 64 * 64 + 64 * 64 + 64 * 2)   # algorithmic (unpadded) 12-64-64-64-2
# the dynamic procedure is bound by arithmetic, not bytes: floating-point
# operations per interior cell (centring 6, strain and |S| 68, the 12 products
# 12, 22 quantities x 3 separable passes x 5, M_ij and M.M 42, L.M 24,
# averages 2), each a separate instruction (the reference's order, no FMA)
SGS_OPS_PER_CELL = 6 + 68 + 12 + 22 * 3 * 5 + 42 + 24 + 2
# nominal B200 non-tensor instruction rates (148 SMs x lanes x 1965 MHz):
# FP64 64 lanes, FP32 128 lanes per SM
FP64_OPS_PEAK = 148 * 64 * 1.965e9
FP32_OPS_PEAK = 148 * 128 * 1.965e9
# the accuracy contract every form is held to against the plain FP64 form
GATE = {"velocity_rms": 1e-4, "max_div_u": 1e-10, "nu_t_rel_err": 0.05}


def timed_steps(g, steps, stream, torch, device):
    """K steps bracketed by CUDA events on the solver's stream, profiled,
    with the clocks sampled during the timed region."""
    g.sync()
    torch.cuda.synchronize()
    g.profile_enable(0xFFFF)
    l0 = g.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = Clocks(device)
    e0.record(stream)
    g.step(steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    prof = g.profile_read()
    g.profile_enable(0)
    return ms, prof, g.launches - l0, clk


def kernel_table(prof, steps, ncell, alg, hbm=None, sgs_peak=None):
    """Per category: time per step, launches, share of the summed category
    times (the regeneration runs on a second stream, overlapped with the
    predictor, so shares of a step are not additive), and for the HBM-bound
    ones the algorithmic GB/s and its fraction of the measured copy
    bandwidth; for the dynamic procedure its operation rate."""
    total = sum(v[0] for v in prof.values())
    out = {}
    for c, (ms, n) in prof.items():
        if not n:
            continue
        e = {"ms_per_step": ms / steps, "launches": n, "share_of_category_sum": ms / total if total else None}
        if c in alg:
            e["gbs"] = alg[c] * ncell / (ms / n / 1e3) / 1e9
            if hbm:
                e["hbm_frac"] = e["gbs"] / hbm
        if c == "eddy_viscosity" and sgs_peak:
            e["ops_per_s"] = SGS_OPS_PER_CELL * ncell / (ms / n / 1e3)
            e["op_frac_of_nominal"] = e["ops_per_s"] / sgs_peak
        if c == "ib_regen":
            e["stream"] = "second (overlapped with the predictor)"
        out[c] = e
    return out


def field_errors(a, b, names):
    import numpy as np
    rep = {}
    for n in names:
        x, y = a.download(n)[1:-1, 1:-1, 1:-1], b.download(n)[1:-1, 1:-1, 1:-1]
        d = x - y
        rep[n] = {"rms": float(np.sqrt(np.mean(d * d))), "max": float(np.max(np.abs(d))),
                  "rel_rms": float(np.sqrt(np.mean(d * d)) / max(np.sqrt(np.mean(y * y)), 1e-300))}
    return rep


def gate(acc, closure):
    """The accuracy contract: velocity RMS error, max|div u| and, for the
    learned closure, nu_t against the dynamic model."""
    checks = {"velocity_rms": max(acc[n]["rms"] for n in ("uo", "vo", "wo")) < GATE["velocity_rms"],
              "max_div_u": acc["max_div_u"] < GATE["max_div_u"]}
    if closure:
        checks["nu_t_rel_err"] = acc["nu_t_rel_err_vs_dynamic"] < GATE["nu_t_rel_err"]
    return {"ok": all(checks.values()), "checks": checks, "limits": GATE}


def closure_weights(g_plain, w, log):
    """Saved network, or one trained now on pairs harvested from the plain run."""
    from eddy_hybrid_b200 import train_closure as tc
    from eddy_hybrid_b200 import closure as cl
    got = tc.load()
    if got is not None:
        meta, theta, rep = got
        rep = dict(rep)
        rep["source"] = "eddy_hybrid_b200/closure_weights.npz"
        return meta, theta, rep
    c = cl.Closure(g_plain)
    X, T = c.harvest(cl.sample_cells(w, 2_000_000, 5))
    meta, theta, hist = tc.train(g_plain, X, T, epochs=4, log=log)
    rep = {"source": "trained in this run on 2e6 cells of the plain run's state", "loss_by_epoch":
           [float(v) for v in hist]}
    return meta, theta, rep


def run_deploy(args):
    """The learned closure deployed on the 768x512x384 wake (streamwise x
    vertical x periodic; Re 2e4, Fr 1, the sphere moving at U = 1) with the
    dynamic-model fallback outside the training envelope, against a plain
    FP64 run with the dynamic model from the same start.  The plain run steps
    at constant CFL 1 (icfl = 1: a fixed step of 5e-4 is unstable there once
    the dynamic model's eddy viscosity grows in the near wake) and the
    closure run replays its time steps, so both reach the same times.  After
    the steps: the closure's nu_t against the dynamic model's on the closure
    run's state, and the streamwise velocity along the wake centreline (the
    line through the body centre, x = y = 0) of the two runs."""
    import numpy as np
    import eddy_hybrid_b200 as eb
    from eddy_hybrid_b200 import body as bd
    from eddy_hybrid_b200 import closure as cl
    from eddy_hybrid_b200 import config
    log = lambda *a: print(*a, file=sys.stderr, flush=True)  # noqa: E731
    w = config.Workload("wake_768x512x384", mx=512, ly=384, nz_=768, re=2e4, fr=1.0, dt=5e-4, body_speed=1.0)
    xu = np.diff(w.faces()[0])
    tri, nrm = bd.icosphere(bd.level_for_spacing(max(float(xu.min()), 0.004)))
    vel = bd.body_velocity(w)
    out = {"workload": w.name, "cells": w.ncell, "steps": args.deploy_steps, "re": w.re, "fr": w.fr,
           "triangles": int(len(tri))}
    runs = {}
    dts = []
    for form in ("plain", "closure"):
        g = eb.Solver(w, precision=eb.PLAIN_FP64 if form == "plain" else eb.MIXED, refine_sweeps=args.sweeps,
                      closure=1 if form == "closure" else 0)
        g.set_body(tri, nrm, vel)
        if form == "closure":
            meta, theta, rep = closure_weights(None, w, log)
            cl.Closure(g).set(meta, theta)
            out["closure_weights"] = rep.get("source")
        g.load_initial(config.initial_fields(w, g.metric("dens_bg")[: w.nx]))
        g.initialize()
        t0 = time.time()
        if form == "plain":
            dts = g.step_cfl(1.0, args.deploy_steps)
            out["dt_min"], out["dt_max"], out["time_reached"] = min(dts), max(dts), float(sum(dts))
        else:
            for dt in dts:
                g.step(1, dt)
        g.sync()
        out[f"{form}_s_per_step"] = (time.time() - t0) / args.deploy_steps
        xc, yc = g.metric("xc")[: w.nx], g.metric("yc")[: w.ny]
        ic, jc = int(np.argmin(np.abs(xc))), int(np.argmin(np.abs(yc)))
        wo = g.download("wo")
        runs[form] = {"line": np.array(wo[ic, jc, 1:-1]), "ymean": np.array(wo[ic, 1:-1, 1:-1].mean(axis=0))}
        if form == "closure":
            c = cl.Closure(g)
            nout = c.apply()
            nu_c = g.download("tv")[1:-1, 1:-1, 1:-1]
            c.refresh_fallback()
            nu_d = g.download("tv")[1:-1, 1:-1, 1:-1]
            out["nu_t_rel_err_vs_dynamic"] = float(np.linalg.norm(nu_c - nu_d) / max(np.linalg.norm(nu_d), 1e-300))
            out["cells_outside_envelope"] = int(nout)
            out["max_div_u"] = g.max_divergence()
        log(f"deploy {form}: {out[f'{form}_s_per_step'] * 1e3:.1f} ms/step (wall)")
        g.close()
        del g
    for key in ("line", "ymean"):
        a, b = runs["closure"][key], runs["plain"][key]
        out[f"centreline_w_{key}"] = {"max_abs_diff": float(np.max(np.abs(a - b))),
                                      "rms_diff": float(np.sqrt(np.mean((a - b) ** 2))),
                                      "plain_min": float(b.min()), "closure_min": float(a.min())}
    out["note"] = ("streamwise velocity w along the centreline (x = y = 0, and averaged over the periodic y at "
                   "x = 0) after the steps, free stream 1; wall-clock seconds per step include the host's "
                   "step loop (and, in the plain run, the CFL reduction before every step)")
    print(json.dumps({"deploy": out}), flush=True)


def run_poisson(args):
    """The Poisson solve in isolation on the 256^3 grid stretched 2.5 along x
    and z around the periodic y (seed-7 N(0,1) right-hand side, its
    volume-weighted mean removed): the plain FP64 solve and the mixed form's
    FP32 transforms with two FP64-residual sweeps, timed on the device (CUDA
    events around repeated solves of a device-resident right-hand side).  Their
    accuracy against the oracle is the parity tests' (config 1)."""
    import ctypes
    import numpy as np
    import torch
    import eddy_hybrid_b200 as eb
    from eddy_hybrid_b200 import config
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    w = config.poisson_256x256x256()
    rng = np.random.RandomState(7)
    d = np.zeros((w.nx, w.ny, w.nz), order="F")
    d[1:-1, 1:-1, 1:-1] = rng.randn(w.mx, w.ly, w.nz_)
    out = {"workload": w.name, "cells": w.ncell, "repeats": args.steps, "warmup": args.warmup}
    for name, prec in (("plain_fp64", eb.PLAIN_FP64), ("refined_fp32_2_sweeps", eb.MIXED)):
        g = eb.Solver(w, precision=prec, refine_sweeps=2)
        ap, cp = g.metric("ap")[: w.nx], g.metric("cp")[: w.nz]
        vol = (1 / ap[1:-1])[:, None, None] * np.ones((1, w.ly, 1)) * (1 / cp[1:-1])[None, None, :]
        dd = d.copy(order="F")
        inner = dd[1:-1, 1:-1, 1:-1]
        inner -= (inner * vol).sum() / vol.sum()
        rhs = torch.from_numpy(dd.ravel(order="F").copy()).to(dev)
        sol = torch.empty_like(rhs)
        pr = ctypes.cast(rhs.data_ptr(), ctypes.POINTER(ctypes.c_double))
        ps = ctypes.cast(sol.data_ptr(), ctypes.POINTER(ctypes.c_double))
        stream = torch.cuda.ExternalStream(g.stream, device=dev)

        def solve():
            g._check(eb.lib().eddy_poisson_solve(g.h, pr, ps, 1), "eddy_poisson_solve")

        torch.cuda.synchronize()
        for _ in range(args.warmup):
            solve()
        g.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            solve()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        r = {"ms_per_solve": ms, "Mcells_per_s": w.ncell / (ms / 1e3) / 1e6}
        if prec == eb.MIXED:
            r["pre_sweep_residuals_relative"] = [float(v) / float(np.max(np.abs(inner)))
                                                 for v in g.refine_residuals()[:2]]
        out[name] = r
        g.close()
        del g
    print(json.dumps({"poisson": out}), flush=True)


# C.N. line solves, per launch (one velocity component's lines): R right-hand
# side, W solution, R nu_t (the faces' viscosities) -- the bytes a one-pass
# solve would move; the Thomas + Sherman-Morrison sweeps move more (their
# multipliers and correction vector go through two scratch fields)
CN_LINE_BYTES = 3 * 8


def run_implicit(args):
    """The plain FP64 step of the wake workload (the moving sphere) with the y
    viscous terms Crank-Nicolson (imply = 1: INVERSEY on the three velocity
    components, INVERSEYD on the density, the implicit pressure terms) and
    the same step explicit, both timed on the device like the main bench."""
    import numpy as np
    import torch
    import eddy_hybrid_b200 as eb
    from eddy_hybrid_b200 import body as bd
    from eddy_hybrid_b200 import config
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    out = {}
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm = peaks.get("hbm_gbs") or 6650.0
    for name, imply in (("explicit", 0), ("imply_1", 1)):
        w = workload(args.small, args.medium, args.grid)
        w.imply = imply
        xu = np.diff(w.faces()[0])
        tri, nrm = bd.icosphere(bd.level_for_spacing(max(float(xu.min()), 0.004)))
        g = eb.Solver(w, precision=eb.PLAIN_FP64)
        if w.sphere:
            g.set_body(tri, nrm, bd.body_velocity(w))
        g.load_initial(config.initial_fields(w, g.metric("dens_bg")[: w.nx]))
        g.initialize()
        g.step(args.warmup)
        st = torch.cuda.ExternalStream(g.stream, device=dev)
        ms, prof, launches, clk = timed_steps(g, args.steps, st, torch, 0)
        alg = dict(ALG_BYTES, cn_line_solve=CN_LINE_BYTES)
        out[name] = {"ms_per_step": ms / args.steps, "value": w.ncell * args.steps / (ms / 1e3) / 1e6,
                     "unit": UNIT, "launches": launches, "clocks": clk,
                     "kernels": kernel_table(prof, args.steps, w.ncell, alg, hbm, FP64_OPS_PEAK),
                     "max_div_u": g.max_divergence()}
        g.close()
        del g
    print(json.dumps({"workload": workload(args.small, args.medium, args.grid).name, "form": "plain FP64",
                      "steps": args.steps, "warmup": args.warmup, "hbm_peak_gbs": hbm, **out}), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.deploy:
        return run_deploy(args)
    if args.poisson:
        return run_poisson(args)
    if args.implicit:
        return run_implicit(args)
    rank, world, local, dist = dist_init(args.gpus)
    import numpy as np
    import torch

    import eddy_hybrid_b200 as eb
    from eddy_hybrid_b200 import closure as cl
    from eddy_hybrid_b200 import config

    log = (lambda *a: print(*a, file=sys.stderr, flush=True)) if rank == 0 else (lambda *a: None)
    dev_i = local if world > 1 else 0
    dev = torch.device("cuda", dev_i)
    torch.cuda.set_device(dev)
    w = workload(args.small, args.medium, args.grid)
    ncell = w.ncell
    sweeps = args.sweeps

    # the sphere (D = 1 at the origin) as a triangulated immersed body, moving
    # at the workload's body speed; tags and stencils regenerated every step
    from eddy_hybrid_b200 import body as bd
    xu = np.diff(w.faces()[0])
    blevel = bd.level_for_spacing(max(float(xu.min()), 0.004))
    tri, nrm = bd.icosphere(blevel)
    vel = bd.body_velocity(w)

    def make(precision, closure):
        g = eb.Solver(w, device=dev_i, precision=precision, refine_sweeps=sweeps, closure=closure)
        if w.sphere:
            g.set_body(tri, nrm, vel)
        return g

    def run(g):
        g.load_initial(fields)
        g.initialize()
        g.step(args.warmup)
        st = torch.cuda.ExternalStream(g.stream, device=dev)
        if dist:
            dist.barrier()
        ms, prof, launches, clk = timed_steps(g, args.steps, st, torch, dev_i)
        if dist:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return {"ms": ms, "prof": prof, "launches": launches, "clocks": clk, "stream": st}

    if args.profile:
        g = make(eb.PLAIN_FP64 if args.profile == "plain" else eb.MIXED, 0)
        g.load_initial(config.initial_fields(w, g.metric("dens_bg")[: w.nx]))
        g.initialize()
        g.step(args.warmup)
        g.step(args.steps)
        g.sync()
        log(f"profile run: {args.profile} form, {args.warmup} + {args.steps} steps of {w.name}")
        return

    # ---- plain FP64 form (the accuracy reference: bit-exact / 1e-11 against the CPU oracle) ----
    g0 = make(eb.PLAIN_FP64, 0)
    fields = config.initial_fields(w, g0.metric("dens_bg")[: w.nx])
    r0 = run(g0)
    log(f"plain FP64: {r0['ms'] / args.steps:.2f} ms/step")

    # ---- mixed precision with the dynamic model ----
    g1 = make(eb.MIXED, 0)
    r1 = run(g1)
    log(f"mixed + dynamic model: {r1['ms'] / args.steps:.2f} ms/step")
    g1.sync()
    acc1 = field_errors(g1, g0, ["uo", "vo", "wo", "p", "dens", "tv"])
    acc1["max_div_u"] = g1.max_divergence()
    acc1["refine_residuals_last_solve"] = [float(v) for v in g1.refine_residuals()[:sweeps]]

    # ---- mixed precision with the learned closure ----
    meta, theta, wrep = closure_weights(g0, w, log)
    g2 = make(eb.MIXED, 1)
    cl.Closure(g2).set(meta, theta)
    r2 = run(g2)
    log(f"mixed + learned closure: {r2['ms'] / args.steps:.2f} ms/step")
    acc2 = field_errors(g2, g0, ["uo", "vo", "wo", "p", "dens"])
    acc2["max_div_u"] = g2.max_divergence()
    c2 = cl.Closure(g2)
    nout = c2.apply()
    nu_closure = g2.download("tv")[1:-1, 1:-1, 1:-1]
    c2.refresh_fallback()                     # the dynamic model on the same state
    nu_dyn = g2.download("tv")[1:-1, 1:-1, 1:-1]
    acc2["nu_t_rel_err_vs_dynamic"] = float(np.linalg.norm(nu_closure - nu_dyn) /
                                            max(np.linalg.norm(nu_dyn), 1e-300))
    acc2["cells_outside_envelope"] = nout
    c2.apply()                                # the closure's viscosity again

    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    mixed_alg = dict(ALG_BYTES_MIXED)
    # of the 1 + sweeps backward passes per solve, the corrections add their
    # result to the FP64 solution (R and W): the mean bytes per launch
    mixed_alg["fft_bwd"] = (12 + 20 * sweeps) / (1 + sweeps)
    forms = {
        "plain": {"solver": g0, "r": r0, "dtype": "f64", "closure": False,
                  "desc": "plain FP64 (dynamic model)",
                  "kernels": kernel_table(r0["prof"], args.steps, ncell, ALG_BYTES, hbm, FP64_OPS_PEAK),
                  "accuracy": {"note": "the accuracy reference (the GPU parity tests hold it bit-exact / 1e-11 "
                                       "to the CPU oracle)"},
                  "gate": {"ok": True, "checks": {}, "limits": GATE}},
        "mixed_dynamic": {"solver": g1, "r": r1, "dtype": "f32 stencils/FFTs/dynamic model + f64 solve/projection",
                          "closure": False,
                          "desc": f"FP32 stencils, FFTs and dynamic model, FP64-residual refinement ({sweeps} sweeps), "
                                  "FP64 projection",
                          "kernels": kernel_table(r1["prof"], args.steps, ncell, mixed_alg, hbm, FP32_OPS_PEAK),
                          "accuracy": acc1, "gate": gate(acc1, False)},
        "chosen": {"solver": g2, "r": r2, "dtype": "f32 stencils/FFTs + f64 solve/projection, bf16 MLP",
                   "closure": True,
                   "desc": f"FP32 stencils and FFTs, FP64-residual refinement ({sweeps} sweeps), learned MLP closure",
                   "kernels": kernel_table(r2["prof"], args.steps, ncell, dict(mixed_alg, eddy_viscosity=CLOSURE_BYTES),
                                           hbm),
                   "accuracy": acc2, "gate": gate(acc2, True)},
    }
    # the headline: the fastest form that meets the accuracy contract
    passing = [k for k in ("chosen", "mixed_dynamic", "plain") if forms[k]["gate"]["ok"]]
    head = min(passing, key=lambda k: forms[k]["r"]["ms"])
    H = forms[head]
    gH = H["solver"]
    msH = H["r"]["ms"]
    value = world * ncell * args.steps / (msH / 1e3) / 1e6

    # end to end through the public API with host buffers (headline form): per
    # step upload the state from pinned host memory, step, read the state back
    io = ["uo", "vo", "wo", "p", "dens", "tv"]
    pinned = {}
    for n in io:
        t = torch.empty(w.nx * w.ny * w.nz, dtype=torch.float64, pin_memory=True)
        a = t.numpy().reshape((w.nx, w.ny, w.nz), order="F")
        a[...] = gH.download(n)
        pinned[n] = (t, a)
    sH = H["r"]["stream"]
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2.record(sH)
    for _ in range(args.e2e_steps):
        for n in io:
            gH.upload(n, pinned[n][1])
        gH.step(1)
        for n in io:
            gH.download(n, out=pinned[n][1])
    e3.record(sH)
    e3.synchronize()
    ems = e2.elapsed_time(e3)
    if dist:
        t = torch.tensor([ems], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e = world * ncell * args.e2e_steps / (ems / 1e3) / 1e6
    fbytes = 8 * w.nx * w.ny * w.nz

    # roofline of the headline form's dominant HBM-bound kernel (the dynamic
    # procedure is arithmetic-bound and reported by its operation rate)
    prof = H["r"]["prof"]
    alg = ALG_BYTES if head == "plain" else dict(mixed_alg, **({"eddy_viscosity": CLOSURE_BYTES}
                                                               if H["closure"] else {}))
    cands = [c for c in alg if c in prof and prof[c][1] and not (c == "eddy_viscosity" and not H["closure"])]
    dom = max(cands, key=lambda c: prof[c][0])
    dms, dn = prof[dom]
    achieved = alg[dom] * ncell / (dms / dn / 1e3) / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(dom)
    roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "traffic": traffic, "peak_source": peak_src,
                "algorithmic_bytes_per_cell": alg[dom], "form": head}
    step_bytes = step_alg_bytes(ALG_BYTES if head == "plain" else mixed_alg, sweeps, head != "plain")
    roofline["whole_step"] = {"algorithmic_bytes_per_cell_step": step_bytes,
                              "achieved_gbs": step_bytes * ncell / (msH / args.steps / 1e3) / 1e9,
                              "frac": step_bytes * ncell / (msH / args.steps / 1e3) / 1e9 / hbm}
    tpk = peaks.get("bf16_tflops_sustained") or 1400.0
    mlp = forms["chosen"]["r"]["prof"].get("eddy_viscosity", (0.0, 0))
    mlp_ms = mlp[0] / max(mlp[1], 1)

    def summary(k):
        F = forms[k]
        v = world * ncell * args.steps / (F["r"]["ms"] / 1e3) / 1e6
        return {"value": v, "ms_per_step": F["r"]["ms"] / args.steps, "dtype": F["dtype"], "form": F["desc"],
                "accuracy_ok": F["gate"]["ok"], "gate": F["gate"], "accuracy": F["accuracy"],
                "launches": F["r"]["launches"], "clocks": F["r"]["clocks"], "kernels": F["kernels"]}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": msH / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": H["dtype"], "data": "synthetic",
        "config": {"workload": w.name + " (NZ-2=512 streamwise, NX-2=384 vertical, NY-2=256 periodic)",
                   "form": f"{head}: {H['desc']}",
                   "headline_rule": "the fastest form that meets the accuracy contract (velocity RMS < 1e-4 and "
                                    "max|div u| < 1e-10 against the plain FP64 form after the timed steps; nu_t "
                                    "within 5% of the dynamic model for the learned closure)",
                   "global_batch": world * ncell, "steps_per_rank": args.steps,
                   "re": w.re, "fr": w.fr, "dt": w.dt,
                   "immersed_body": (f"sphere D=1, {len(tri)} triangles, velocity {vel}, moved and its tags "
                                     "and stencils regenerated once per step" if w.sphere else "none"),
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (~20 GB state)"},
        "forms": {k: summary(k) for k in ("plain", "mixed_dynamic", "chosen")},
        "speedup_vs_plain": {k: r0["ms"] / forms[k]["r"]["ms"] for k in ("mixed_dynamic", "chosen")},
        "closure": wrep,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": len(io) * fbytes,
                "d2h_bytes_per_step": len(io) * fbytes, "form": head},
        "gpu_launches": H["r"]["launches"],
        "roofline": roofline,
        "mlp_tensor": {"tflops": MLP_FLOP_PER_CELL * ncell / (mlp_ms / 1e3) / 1e12 if mlp_ms else None,
                       "peak_tflops_sustained": tpk, "flop_per_cell": MLP_FLOP_PER_CELL,
                       "frac": (MLP_FLOP_PER_CELL * ncell / (mlp_ms / 1e3) / 1e12 / tpk) if mlp_ms else None},
        "clocks": H["r"]["clocks"],
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not (args.small or args.medium or args.grid):
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    for F in forms.values():
        F["solver"].close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
