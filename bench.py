"""Throughput of the fractional-step time advance on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = 3 RK substeps (RHS+predictor, boundary fills, divergence + FFT
Poisson solve + projection, pressure update, density) + the eddy viscosity
update, on the 512x384x256 wake grid (streamwise x vertical x periodic),
fields resident on the GPU.  Both forms run from the same state: the plain
FP64 form (dynamic model) and the chosen form (FP32 stencils and FFTs, FP64
residual refinement and projection, learned MLP closure); `value` is the
chosen form, `plain` the FP64 form, `accuracy` the chosen form's error against
the plain one.  Prints one JSON line.
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
OWN = [k for k in ALG_BYTES if not k.startswith("transform")]  # cuBLAS does the transforms


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


def cpu_baseline(steps=1):
    """The CPU oracle (restatement of the reference CPU path, FP64, OpenMP
    over the host cores) on a bounded sample of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import eddy_oracle
    from eddy_hybrid_b200 import config
    cores = len(os.sched_getaffinity(0))
    w = config.Workload("wake_sample_256x192x128", mx=192, ly=128, nz_=256, re=1e4, fr=1.0,
                        dt=5e-4, sphere=False)
    s = eddy_oracle.OracleSolver(w, threads=cores)
    s.load_initial(config.initial_fields(w, s.grid.get("dens_bg")[: w.nx]))
    s.initialize()
    t0 = time.perf_counter()
    s.step(steps)
    dt = time.perf_counter() - t0
    return {"value": w.ncell * steps / dt / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} full step(s) of a 256x192x128 grid (1/8 of the cells, same "
                      f"equations and parameters) after initialisation; {dt:.2f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from eddy_hybrid_b200 import config  # noqa: F401
    for _ in range(args.warmup):
        cpu_baseline(1)
    vals = [cpu_baseline(1) for _ in range(args.steps)]
    v = statistics.mean(x["value"] for x in vals)
    cb = dict(vals[0])
    cb["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "wake_512x384x256 (CPU sample, see cpu_baseline)",
                       "form": "plain FP64 (CPU oracle port of the reference loops)"},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# algorithmic bytes per interior cell per launch in the mixed form (FP32
# stencil fields, FP64 masters, residual, solution and pressure)
ALG_BYTES_MIXED = {
    "rhs_predictor": 15 * 4,   # R 9 FP32 fields  W u*,v*,w*,ua,va,wa FP32
    "div_fft_fwd": 3 * 4 + 8 + 4,  # R u*,v*,w* FP32  W d FP64, spectrum FP32
    "refine_residual": 8 + 8 + 4,  # R phi, d FP64  W spectrum FP32
    "transform_fwd": 2 * 4,
    "z_line_solve": 2 * 4,
    "transform_bwd": 2 * 4,
    "correct": 3 * 4 + 8 + 3 * 8 + 3 * 4,  # R u*,v*,w* FP32, dp  W u,v,w FP64 + FP32 copies
    "pressure_update": 8 + 8 + 8 + 4,      # R p,dp  W p FP64, p FP32
    "density": 6 * 4 + 2 * 4,              # R rho,kappa,u,v,w,rha  W rho,rha (FP32)
    "eddy_viscosity": 4 * 4 + 2 * 8 + 2 * 4,  # R u,v,w,rho FP32  W nu_t,kappa_t FP64 + FP32 copies
    "precision_copy": 4 + 8,               # one FP32<->FP64 copy
}
OWN_MIXED = ["rhs_predictor", "div_fft_fwd", "refine_residual", "z_line_solve", "fft_bwd", "correct",
             "pressure_update", "density", "eddy_viscosity", "precision_copy"]
MLP_FLOP_PER_CELL = 2 * (16 * 64 + 64 * 64 + 64 * 64 + 64 * 16)


def timed_steps(g, steps, stream, torch):
    """K steps bracketed by CUDA events on the solver's stream, profiled."""
    g.sync()
    torch.cuda.synchronize()
    g.profile_enable(0x7FFF)
    l0 = g.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    prof = g.profile_read()
    g.profile_enable(0)
    return ms, prof, g.launches - l0


def kernel_table(prof, steps, ncell, alg, hbm=None):
    """Per category: time per step, launches, share of the summed category
    time, and for the HBM-bound ones the algorithmic GB/s and its fraction of
    the measured copy bandwidth."""
    total = sum(v[0] for v in prof.values())
    out = {}
    for c, (ms, n) in prof.items():
        if not n:
            continue
        e = {"ms_per_step": ms / steps, "launches": n, "share": ms / total if total else None}
        if c in alg:
            e["gbs"] = alg[c] * ncell / (ms / n / 1e3) / 1e9
            if hbm:
                e["hbm_frac"] = e["gbs"] / hbm
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


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
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

    # ---- plain FP64 form ----
    g0 = make(eb.PLAIN_FP64, 0)
    fields = config.initial_fields(w, g0.metric("dens_bg")[: w.nx])
    g0.load_initial(fields)
    g0.initialize()
    g0.step(args.warmup)
    s0 = torch.cuda.ExternalStream(g0.stream, device=dev)
    if dist:
        dist.barrier()
    ms0, prof0, _ = timed_steps(g0, args.steps, s0, torch)
    log(f"plain FP64: {ms0 / args.steps:.2f} ms/step")

    # ---- mixed precision with the dynamic model (precision error alone) ----
    g1 = make(eb.MIXED, 0)
    g1.load_initial(fields)
    g1.initialize()
    g1.step(args.warmup + args.steps)
    g1.sync()
    acc_mixed = field_errors(g1, g0, ["uo", "vo", "wo", "p", "dens", "tv"])
    acc_mixed["max_div_u"] = g1.max_divergence()
    acc_mixed["refine_residuals_last_solve"] = [float(v) for v in g1.refine_residuals()[:sweeps]]
    g1.close()

    # ---- chosen form: mixed precision + learned closure ----
    meta, theta, wrep = closure_weights(g0, w, log)
    g2 = make(eb.MIXED, 1)
    cl.Closure(g2).set(meta, theta)
    g2.load_initial(fields)
    g2.initialize()
    g2.step(args.warmup)
    s2 = torch.cuda.ExternalStream(g2.stream, device=dev)
    if dist:
        dist.barrier()
    clocks = Clocks(dev_i)
    ms2, prof2, launches = timed_steps(g2, args.steps, s2, torch)
    clk = clocks.stop()
    log(f"chosen form: {ms2 / args.steps:.2f} ms/step")
    acc_chosen = field_errors(g2, g0, ["uo", "vo", "wo", "p", "dens"])
    acc_chosen["max_div_u"] = g2.max_divergence()
    nu_closure = g2.download("tv")[1:-1, 1:-1, 1:-1]
    c2 = cl.Closure(g2)
    nout = c2.apply()
    nu_closure = g2.download("tv")[1:-1, 1:-1, 1:-1]
    c2.refresh_fallback()                     # the dynamic model on the same state
    nu_dyn = g2.download("tv")[1:-1, 1:-1, 1:-1]
    acc_chosen["nu_t_rel_err_vs_dynamic"] = float(np.linalg.norm(nu_closure - nu_dyn) /
                                                  max(np.linalg.norm(nu_dyn), 1e-300))
    acc_chosen["cells_outside_envelope"] = nout
    # restore the closure's viscosity before the end-to-end run
    c2.apply()
    if dist:
        t = torch.tensor([ms0, ms2], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms0, ms2 = (float(v) for v in t.tolist())
    value = world * ncell * args.steps / (ms2 / 1e3) / 1e6
    value_plain = world * ncell * args.steps / (ms0 / 1e3) / 1e6

    # end to end through the public API with host buffers: per step upload the
    # state from pinned host memory, step, read the state back
    io = ["uo", "vo", "wo", "p", "dens", "tv"]
    pinned = {}
    for n in io:
        t = torch.empty(w.nx * w.ny * w.nz, dtype=torch.float64, pin_memory=True)
        a = t.numpy().reshape((w.nx, w.ny, w.nz), order="F")
        a[...] = g2.download(n)
        pinned[n] = (t, a)
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e2.record(s2)
    for _ in range(args.e2e_steps):
        for n in io:
            g2.upload(n, pinned[n][1])
        g2.step(1)
        for n in io:
            g2.download(n, out=pinned[n][1])
    e3.record(s2)
    e3.synchronize()
    ems = e2.elapsed_time(e3)
    if dist:
        t = torch.tensor([ems], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    e2e = world * ncell * args.e2e_steps / (ems / 1e3) / 1e6
    fbytes = 8 * w.nx * w.ny * w.nz

    # roofline of the dominant kernel among our own (chosen form)
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    k2 = kernel_table(prof2, args.steps, ncell, ALG_BYTES_MIXED, hbm)
    dom = max((c for c in OWN_MIXED if c in k2 and c in ALG_BYTES_MIXED), key=lambda c: prof2[c][0])
    dms, dn = prof2[dom]
    achieved = ALG_BYTES_MIXED[dom] * ncell / (dms / dn / 1e3) / 1e9 if dn else None
    traffic = None
    tf = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tf):
        traffic = json.load(open(tf)).get(dom)
    mlp_ms = prof2["eddy_viscosity"][0] / max(prof2["eddy_viscosity"][1], 1)
    tpk = peaks.get("bf16_tflops_sustained")
    tpk_src = "measured (sustained)" if tpk else "fallback (sustained)"
    tpk = tpk or 1400.0
    if dom == "eddy_viscosity":
        # the closure kernel is a tensor-core MLP: its roofline is the tensor
        # peak (sustained, the kernel runs inside a long step); HBM alongside
        ach_t = MLP_FLOP_PER_CELL * ncell / (dms / dn / 1e3) / 1e12 if dn else None
        roofline = {"kernel": dom, "bound": "tensor", "achieved": ach_t, "peak": tpk, "unit": "TFLOP/s",
                    "frac": (ach_t / tpk) if ach_t else None, "traffic": traffic, "peak_source": tpk_src,
                    "algorithmic_flop_per_cell": MLP_FLOP_PER_CELL,
                    "hbm": {"achieved": achieved, "peak": hbm, "unit": "GB/s",
                            "frac": (achieved / hbm) if achieved else None,
                            "algorithmic_bytes_per_cell": ALG_BYTES_MIXED[dom]}}
    else:
        roofline = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                    "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
                    "peak_source": peak_src, "algorithmic_bytes_per_cell": ALG_BYTES_MIXED[dom]}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms2 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 stencils/FFTs + f64 solve/projection, bf16 MLP",
        "data": "synthetic",
        "config": {"workload": w.name + " (NZ-2=512 streamwise, NX-2=384 vertical, NY-2=256 periodic)",
                   "form": f"chosen: FP32 stencils+FFTs, FP64-residual refinement ({sweeps} sweeps), "
                           "learned MLP closure",
                   "global_batch": world * ncell, "steps_per_rank": args.steps,
                   "re": w.re, "fr": w.fr, "dt": w.dt,
                   "immersed_body": (f"sphere D=1, {len(tri)} triangles, velocity {vel}, moved and its tags "
                                     "and stencils regenerated once per step" if w.sphere else "none"),
                   "parallelism": f"replicas x{world}", "l2": "inputs larger than L2 (~20 GB state)"},
        "plain": {"value": value_plain, "ms_per_step": ms0 / args.steps, "dtype": "f64",
                  "kernels": kernel_table(prof0, args.steps, ncell, ALG_BYTES, hbm)},
        "speedup_chosen_vs_plain": ms0 / ms2,
        "accuracy": {"reference": "plain FP64 GPU form (bit-exact/1e-11 vs the CPU oracle) from the "
                                  f"same state after {args.warmup + args.steps} steps",
                     "mixed_dynamic": acc_mixed, "chosen": acc_chosen, "closure": wrep},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": len(io) * fbytes,
                "d2h_bytes_per_step": len(io) * fbytes},
        "gpu_launches": launches,
        "roofline": roofline,
        "mlp_tensor": {"tflops": MLP_FLOP_PER_CELL * ncell / (mlp_ms / 1e3) / 1e12 if mlp_ms else None,
                       "peak_tflops": peaks.get("bf16_tflops"), "flop_per_cell": MLP_FLOP_PER_CELL},
        "kernels": k2,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not (args.small or args.medium):
        line["cpu_baseline"] = cpu_baseline(1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    g2.close()
    g0.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
