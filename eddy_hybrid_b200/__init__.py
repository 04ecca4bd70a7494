"""B200-native fractional-step time advance of the eddy-hybrid LES solver.

Host-side mirror of the reference's Fortran driver over the C ABI in
include/eddy_b200.h (libeddy_b200.so, built in-tree by
``eddy_hybrid_b200.build``).  The CUDA library is the only compute path: if
it cannot be loaded every call raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import config  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeddy_b200.so")

FIELDS = ["uo", "vo", "wo", "p", "dp", "dens", "tv", "us", "vs", "ws", "ua",
          "va", "wa", "ub", "vb", "wb", "rha", "rhb", "rs", "planeU", "planeV",
          "planeW", "planeD"]
FID = {n: i for i, n in enumerate(FIELDS)}
METRICS = ["xu", "xc", "ap", "au", "av", "aw", "yv", "yc", "bp", "bu", "bv",
           "bw", "zw", "zc", "cp", "cu", "cv", "cw", "whx", "why", "whz",
           "dfxu", "dfxw", "dfxul", "dfxwl", "dfxd", "dfxdl", "dens_bg"]
ERRORS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "non-finite value",
          4: "singular system", 5: "refinement did not converge", 6: "timeout",
          7: "out of memory"}
PLAIN_FP64, MIXED = 0, 1


class EddyError(RuntimeError):
    pass


class Params(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("itype", C.c_int * 7), ("ischm", C.c_int), ("isgs", C.c_int),
                ("idens", C.c_int), ("ru1", C.c_double), ("prn", C.c_double),
                ("denP1", C.c_double), ("grav", C.c_double), ("dpdx", C.c_double),
                ("dpdy", C.c_double), ("dpdz", C.c_double), ("eps", C.c_double),
                ("css", C.c_double), ("vspngx1", C.c_int), ("dspngx1", C.c_int),
                ("vspngx3in", C.c_int), ("vspngx3out", C.c_int),
                ("dspngx3in", C.c_int), ("dspngx3out", C.c_int),
                ("precision", C.c_int), ("refine_sweeps", C.c_int),
                ("closure", C.c_int), ("imply", C.c_int), ("implx", C.c_int),
                ("implcx", C.c_int), ("implcy", C.c_int)]


def make_params(d: dict, precision: int = PLAIN_FP64, refine_sweeps: int = 2,
                closure: int = 0) -> Params:
    p = Params()
    for k, v in d.items():
        if k == "itype":
            p.itype = (C.c_int * 7)(0, *v)
        else:
            setattr(p, k, v)
    p.precision = precision
    p.refine_sweeps = refine_sweeps
    p.closure = closure
    return p


_lib = None
_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)

# exported symbols and their argument types (must match include/eddy_b200.h)
SIGNATURES = {
    "eddy_create": ([C.POINTER(C.c_void_p), C.POINTER(Params), _DP, C.c_double, C.c_double, _DP, C.c_int], C.c_int),
    "eddy_destroy": ([C.c_void_p], C.c_int),
    "eddy_upload": ([C.c_void_p, C.c_int, _DP], C.c_int),
    "eddy_download": ([C.c_void_p, C.c_int, _DP], C.c_int),
    "eddy_get_metric": ([C.c_void_p, C.c_int, _DP, C.c_int], C.c_int),
    "eddy_grid_metric": ([C.POINTER(Params), _DP, C.c_double, C.c_double, _DP, C.c_int, _DP, C.c_int], C.c_int),
    "eddy_rhs_predictord": ([C.c_void_p, C.c_double, C.c_double, C.c_double], C.c_int),
    "eddy_inversey": ([C.c_void_p, C.c_double], C.c_int),
    "eddy_inversex": ([C.c_void_p, C.c_double], C.c_int),
    "eddy_body_force_cv": ([C.c_void_p, _DP, C.c_double, C.c_int, _DP], C.c_int),
    "eddy_body_force_cv_reset": ([C.c_void_p], C.c_int),
    "eddy_cfl": ([C.c_void_p, _DP], C.c_int),
    "eddy_field_extrema": ([C.c_void_p, C.c_int, _DP, _DP], C.c_int),
    "eddy_ioscalar_write": ([C.c_char_p, C.c_int, C.c_int, C.c_int, _DP, C.c_int, C.c_double, C.c_double,
                             C.c_double], C.c_int),
    "eddy_ioscalar_read": ([C.c_char_p, C.c_int, C.c_int, C.c_int, _DP, C.POINTER(C.c_int), _DP, _DP, _DP],
                           C.c_int),
    "eddy_save_field": ([C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.c_double, C.c_double], C.c_int),
    "eddy_read_hybrid_plane": ([C.c_char_p, C.c_int, C.c_int, _DP, _DP, _DP, _DP, _DP, C.POINTER(C.c_int), _DP],
                               C.c_int),
    "eddy_inflow_sequence": ([C.c_void_p, C.c_int, _DP, C.c_int, C.c_int], C.c_int),
    "eddy_inflow_cycle": ([C.c_void_p, C.c_int], C.c_int),
    "eddy_set_time": ([C.c_void_p, C.c_double], C.c_int),
    "eddy_get_time": ([C.c_void_p, _DP], C.c_int),
    "eddy_probes_set": ([C.c_void_p, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "eddy_probes_read": ([C.c_void_p, _DP, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "eddy_plane": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, _DP], C.c_int),
    "eddy_load_field": ([C.c_void_p, C.c_int, C.c_char_p, C.POINTER(C.c_int), _DP, _DP, _DP], C.c_int),
    "eddy_boundary": ([C.c_void_p, C.c_int], C.c_int),
    "eddy_boundinout": ([C.c_void_p, C.c_int, C.c_double], C.c_int),
    "eddy_direct": ([C.c_void_p, C.c_double], C.c_int),
    "eddy_correct": ([C.c_void_p, C.c_double], C.c_int),
    "eddy_pressure_update": ([C.c_void_p], C.c_int),
    "eddy_density": ([C.c_void_p, C.c_double, C.c_double, C.c_double], C.c_int),
    "eddy_turvis": ([C.c_void_p], C.c_int),
    "eddy_initialize": ([C.c_void_p, C.c_double], C.c_int),
    "eddy_substep": ([C.c_void_p, C.c_int, C.c_double], C.c_int),
    "eddy_step": ([C.c_void_p, C.c_double, C.c_int], C.c_int),
    "eddy_poisson_solve": ([C.c_void_p, _DP, _DP, C.c_int], C.c_int),
    "eddy_max_divergence": ([C.c_void_p, _DP], C.c_int),
    "eddy_refine_residuals": ([C.c_void_p, _DP, C.c_int], C.c_int),
    "eddy_ib_set_body": ([C.c_void_p, C.c_int, _DP, _DP, _DP], C.c_int),
    "eddy_ib_move": ([C.c_void_p, C.c_double], C.c_int),
    "eddy_ib_set_cadence": ([C.c_void_p, C.c_int], C.c_int),
    "eddy_ib_regen": ([C.c_void_p], C.c_int),
    "eddy_ib_momforc": ([C.c_void_p], C.c_int),
    "eddy_ib_correct": ([C.c_void_p, C.c_int], C.c_int),
    "eddy_ib_flags": ([C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    "eddy_ib_limits": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "eddy_ib_stencils": ([C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p, C.c_void_p,
                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "eddy_ib_stencil_kinds": ([C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "eddy_profile_enable": ([C.c_void_p, C.c_uint], C.c_int),
    "eddy_profile_read": ([C.c_void_p, _DP, C.POINTER(C.c_longlong)], C.c_int),
    "eddy_selftest_wait_bound": ([C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double)], C.c_int),
    "eddy_max_divergence_noalloc": ([C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "eddy_umma_gemm_bf16": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, _FP, C.c_int], C.c_int),
    "eddy_closure_set": ([C.c_void_p, _FP, _FP], C.c_int),
    "eddy_closure_get": ([C.c_void_p, _FP, _FP], C.c_int),
    "eddy_closure_harvest": ([C.c_void_p, C.c_void_p, C.c_int, _FP, _FP], C.c_int),
    "eddy_closure_grad": ([C.c_void_p, _FP, _FP, C.c_int, _FP, _DP], C.c_int),
    "eddy_closure_train": ([C.c_void_p, _FP, _FP, C.c_longlong, C.c_int, C.c_int, C.c_float, C.c_ulonglong, _DP],
                           C.c_int),
    "eddy_closure_apply": ([C.c_void_p, C.POINTER(C.c_longlong)], C.c_int),
    "eddy_closure_refresh_fallback": ([C.c_void_p], C.c_int),
    "eddy_download_kappa": ([C.c_void_p, _DP], C.c_int),
    "eddy_sync": ([C.c_void_p], C.c_int),
    "eddy_last_error": ([C.c_void_p, C.c_char_p, C.c_int], C.c_int),
    "eddy_launch_count": ([C.c_void_p], C.c_int64),
    "eddy_stream": ([C.c_void_p], C.c_void_p),
}


def lib():
    """Load libeddy_b200.so (raises if it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EddyError(f"CUDA library not built: {LIB_PATH} (run python -m eddy_hybrid_b200.build)")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def write_ioscalar(path: str, a: np.ndarray, nstep: int, time: float, dtm1: float, grav: float):
    """Host array (NX,NY,NZ) to a restart file in the IOSCALAR layout."""
    a = np.asfortranarray(a, dtype=np.float64)
    nx, ny, nz = a.shape
    rc = lib().eddy_ioscalar_write(path.encode(), nx, ny, nz, _ptr(a), nstep, time, dtm1, grav)
    if rc:
        raise EddyError(f"eddy_ioscalar_write failed ({rc})")


def read_ioscalar(path: str, shape) -> tuple:
    """Restart file to a host array of `shape`; returns (array, nstep, time, dtm1, grav)."""
    a = np.zeros(shape, order="F")
    ns, t, dt, gr = C.c_int(0), C.c_double(0.), C.c_double(0.), C.c_double(0.)
    rc = lib().eddy_ioscalar_read(path.encode(), shape[0], shape[1], shape[2], _ptr(a), C.byref(ns), C.byref(t),
                                  C.byref(dt), C.byref(gr))
    if rc:
        raise EddyError(f"eddy_ioscalar_read failed ({rc}): missing, truncated or another grid")
    return a, ns.value, t.value, dt.value, gr.value


def write_hybrid_plane(path: str, u, v, w, d, p=None, icycle: int = 0, time: float = 0.0, dtm1: float = 0.0,
                       grav: float = 0.0, rho: float = 0.0, re: float = 0.0, pr: float = 0.0, index: int = 0,
                       xc=None, xu=None, yc=None, yv=None, zcg: float = 0.0, zwg: float = 0.0):
    """An inflow-plane file in the layout the reference's read_hybrid reads
    (src/hybrid.f:162-200): Fortran unformatted sequential records with
    4-byte length markers; the planes are (NX, NY) arrays."""
    import struct
    u = np.asfortranarray(u, dtype=np.float64)
    nx, ny = u.shape
    zero = np.zeros((nx, ny))
    planes = [u, v, w, zero if p is None else p, d]
    xc = np.zeros(nx) if xc is None else xc
    xu = np.zeros(nx) if xu is None else xu
    yc = np.zeros(ny) if yc is None else yc
    yv = np.zeros(ny) if yv is None else yv

    def rec(f, payload: bytes):
        f.write(struct.pack("<I", len(payload)) + payload + struct.pack("<I", len(payload)))

    with open(path, "wb") as f:
        rec(f, struct.pack("<i", icycle))
        rec(f, struct.pack("<6d", time, dtm1, grav, rho, re, pr))
        rec(f, struct.pack("<3i", 3, 0, index))
        rec(f, struct.pack("<2d", zcg, zwg))
        rec(f, struct.pack("<3i", nx, 0, ny))
        rec(f, np.concatenate([np.asarray(xc, np.float64), np.asarray(xu, np.float64)]).tobytes())
        rec(f, np.concatenate([np.asarray(yc, np.float64), np.asarray(yv, np.float64)]).tobytes())
        for a in planes:
            rec(f, np.asfortranarray(a, dtype=np.float64).tobytes(order="F"))


def read_hybrid_plane(path: str, nx: int, ny: int) -> dict:
    """An inflow-plane file (read_hybrid's layout) through the library's
    reader: planes u, v, w, p, d of shape (NX, NY), icycle and time."""
    out = {k: np.zeros((nx, ny), order="F") for k in ("u", "v", "w", "p", "d")}
    ic, t = C.c_int(0), C.c_double(0.)
    rc = lib().eddy_read_hybrid_plane(path.encode(), nx, ny, *(_ptr(out[k]) for k in ("u", "v", "w", "p", "d")),
                                      C.byref(ic), C.byref(t))
    if rc:
        raise EddyError(f"eddy_read_hybrid_plane failed ({rc}): missing, truncated or another grid")
    out["icycle"], out["time"] = ic.value, t.value
    return out


def _ptr(a: np.ndarray):
    if a.dtype != np.float64:
        raise TypeError("float64 arrays required")
    if not (a.flags.f_contiguous or a.ndim == 1):
        raise ValueError("Fortran-ordered arrays required")
    return a.ctypes.data_as(_DP)


def grid_metric(workload, name: str) -> np.ndarray:
    """Metric array built by the library's host code (no GPU needed)."""
    p = make_params(workload.params())
    xf, zf = workload.faces()
    xf = np.ascontiguousarray(xf, dtype=np.float64)
    zf = np.ascontiguousarray(zf, dtype=np.float64)
    n = 3 * (max(workload.nx, workload.ny, workload.nz) + 2) + workload.nx * workload.ny
    out = np.zeros(n)
    m = lib().eddy_grid_metric(C.byref(p), _ptr(xf), workload.ylim[0], workload.ylim[1], _ptr(zf),
                               METRICS.index(name), _ptr(out), n)
    if m < 0:
        raise EddyError("eddy_grid_metric failed")
    return out[:m].copy()


class Solver:
    """One device-resident solver context (one CUDA stream)."""

    def __init__(self, workload, device: int = 0, precision: int = PLAIN_FP64,
                 refine_sweeps: int = 2, closure: int = 0):
        self.w = workload
        self.params = workload.params()
        self._p = make_params(self.params, precision, refine_sweeps, closure)
        xf, zf = workload.faces()
        xf = np.ascontiguousarray(xf, dtype=np.float64)
        zf = np.ascontiguousarray(zf, dtype=np.float64)
        h = C.c_void_p()
        rc = lib().eddy_create(C.byref(h), C.byref(self._p), _ptr(xf), workload.ylim[0],
                               workload.ylim[1], _ptr(zf), device)
        self.h = h
        self._check(rc, "eddy_create")
        self.shape = (self.params["nx"], self.params["ny"], self.params["nz"])

    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = ""
            if self.h:
                buf = C.create_string_buffer(512)
                lib().eddy_last_error(self.h, buf, 512)
                msg = buf.value.decode(errors="replace")
            raise EddyError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")

    def metric(self, name: str) -> np.ndarray:
        n = 3 * (max(self.shape) + 2) + self.shape[0] * self.shape[1]
        out = np.zeros(n)
        m = lib().eddy_get_metric(self.h, METRICS.index(name), _ptr(out), n)
        if m < 0:
            raise EddyError("eddy_get_metric failed")
        return out[:m].copy()

    def upload(self, name: str, a: np.ndarray):
        a = np.asfortranarray(a, dtype=np.float64)
        self._check(lib().eddy_upload(self.h, FID[name], _ptr(a)), "eddy_upload")

    def download(self, name: str, out: np.ndarray | None = None) -> np.ndarray:
        """Copy field `name` to the host.  `out`: optional preallocated
        Fortran-ordered float64 array of the field's shape (for example a view
        of pinned memory, which the copy then reaches at full link speed);
        a new array otherwise."""
        shape = self.shape[:2] if name.startswith("plane") else self.shape
        if out is None:
            a = np.zeros(shape, order="F")
        else:
            if out.dtype != np.float64 or tuple(out.shape) != tuple(shape) or not out.flags.f_contiguous:
                raise ValueError(f"download({name!r}): out must be a Fortran-ordered float64 array of shape {shape}")
            if not out.flags.writeable:
                raise ValueError(f"download({name!r}): out is read-only")
            a = out
        self._check(lib().eddy_download(self.h, FID[name], _ptr(a)), "eddy_download")
        return a

    # restart files: the reference's set and names, <dir>/<field>_<step:08d>.res
    # (src/Eddy6.f:3391-3408), in the IOSCALAR layout
    RESTART_FIELDS = ("uo", "vo", "wo", "p", "tv", "dens")
    RESTART_NAMES = {"uo": "u", "vo": "v", "wo": "w", "p": "p", "tv": "tv", "dens": "dens"}

    def save_restart(self, directory: str, step: int, time: float, dt: float | None = None):
        dt = self.w.dt if dt is None else dt
        for n in self.RESTART_FIELDS:
            path = os.path.join(directory, f"{self.RESTART_NAMES[n]}_{step:08d}.res").encode()
            self._check(lib().eddy_save_field(self.h, FID[n], path, step, time, dt), "eddy_save_field")

    def load_restart(self, directory: str, step: int) -> dict:
        ns, t, dt, gr = C.c_int(0), C.c_double(0.), C.c_double(0.), C.c_double(0.)
        for n in self.RESTART_FIELDS:
            path = os.path.join(directory, f"{self.RESTART_NAMES[n]}_{step:08d}.res").encode()
            self._check(lib().eddy_load_field(self.h, FID[n], path, C.byref(ns), C.byref(t), C.byref(dt),
                                              C.byref(gr)), "eddy_load_field")
        return {"nstep": ns.value, "time": t.value, "dtm1": dt.value, "grav": gr.value}

    def set_inflow_sequence(self, planes, iref: int, nstep: int = 0):
        """The hybrid inlet's plane sequence, (n, 4, NX, NY) u, v, w, rho in
        feed order, kept on the device and cycled by the steps; cells with
        x index >= iref take the last plane; the step counter starts at nstep."""
        a = np.ascontiguousarray(np.asarray(planes, dtype=np.float64).transpose(0, 1, 3, 2))
        n = a.shape[0]
        self._check(lib().eddy_inflow_sequence(self.h, n, a.ctypes.data_as(_DP), iref, nstep),
                    "eddy_inflow_sequence")

    @property
    def time(self) -> float:
        t = C.c_double(0.)
        self._check(lib().eddy_get_time(self.h, C.byref(t)), "eddy_get_time")
        return t.value

    @time.setter
    def time(self, t: float):
        self._check(lib().eddy_set_time(self.h, t), "eddy_set_time")

    def set_probes(self, ijk, capacity: int = 1024):
        """Time probes at 1-based cells ijk (n, 3), recorded on the device
        after every step."""
        a = np.ascontiguousarray(np.asarray(ijk, dtype=np.int32).reshape(-1, 3))
        self._check(lib().eddy_probes_set(self.h, a.shape[0], a.ctypes.data_as(C.c_void_p), capacity),
                    "eddy_probes_set")
        self._nprobe = a.shape[0]

    def read_probes(self, max_samples: int = 1 << 20) -> np.ndarray:
        """The recorded samples, (nsamples, nprobe, 5): time, u, v, w, p."""
        n = getattr(self, "_nprobe", 0)
        out = np.zeros(max(1, max_samples * n * 5))
        cnt = C.c_int(0)
        self._check(lib().eddy_probes_read(self.h, out.ctypes.data_as(_DP), max_samples, C.byref(cnt)),
                    "eddy_probes_read")
        m = min(cnt.value, max_samples)
        return out[: m * n * 5].reshape(m, n, 5)

    def plane(self, name: str, axis: int, index: int, center: int = 0) -> np.ndarray:
        """One plane of a field computed on the device (center: the
        yface_velocity mode 0..4); axis 1, 2, 3 hold i, j, k at index."""
        nx, ny, nz = self.w.nx, self.w.ny, self.w.nz
        shape = {1: (ny, nz), 2: (nx, nz), 3: (nx, ny)}[axis]
        out = np.zeros(shape, order="F")
        self._check(lib().eddy_plane(self.h, FID[name], center, axis, index, _ptr(out)), "eddy_plane")
        return out

    def body_force_cv(self, cvlim, dt: float, icycle: int) -> np.ndarray:
        """calcfrc (src/calcforce.f:3): the 56 control-volume force terms of
        eddy_body_force_cv; the volume's momentum of this call is kept for the
        next call's unsteady term."""
        cv = np.ascontiguousarray(cvlim, dtype=np.float64)
        if cv.shape != (4,):
            raise ValueError("cvlim holds (x1, x2, z1, z2)")
        out = np.zeros(56)
        self._check(lib().eddy_body_force_cv(self.h, _ptr(cv), float(dt), int(icycle), _ptr(out)),
                    "eddy_body_force_cv")
        return out

    def body_force_cv_reset(self):
        self._check(lib().eddy_body_force_cv_reset(self.h), "eddy_body_force_cv_reset")

    def set_cycle(self, icycle: int):
        self._check(lib().eddy_inflow_cycle(self.h, icycle), "eddy_inflow_cycle")

    def cfl(self) -> float:
        v = C.c_double(0.)
        self._check(lib().eddy_cfl(self.h, C.byref(v)), "eddy_cfl")
        return v.value

    def step_cfl(self, cflc: float, nsteps: int = 1) -> list:
        """Constant-CFL stepping (icfl = 1): before every step DTM1 = CFLC / CFLM
        (src/Eddy6.f:2114-2128); returns the time steps taken."""
        dts = []
        for _ in range(nsteps):
            dt = cflc / self.cfl()
            if dt <= 1e-6:
                raise EddyError(f"constant-CFL time step {dt:.3e} <= 1e-6 (the reference stops here)")
            self.step(1, dt)
            dts.append(dt)
        return dts

    def extrema(self, name: str) -> tuple:
        lo, hi = C.c_double(0.), C.c_double(0.)
        self._check(lib().eddy_field_extrema(self.h, FID[name], C.byref(lo), C.byref(hi)), "eddy_field_extrema")
        return lo.value, hi.value

    def load_initial(self, fields: dict):
        for k, v in fields.items():
            self.upload(k, v)

    def initialize(self):
        self._check(lib().eddy_initialize(self.h, self.w.dt), "eddy_initialize")

    def step(self, nsteps: int = 1, dt: float | None = None):
        self._check(lib().eddy_step(self.h, self.w.dt if dt is None else dt, nsteps), "eddy_step")

    def substep(self, is_: int, dt: float | None = None):
        self._check(lib().eddy_substep(self.h, is_, self.w.dt if dt is None else dt), "eddy_substep")

    def call(self, name: str, *args):
        self._check(getattr(lib(), name)(self.h, *args), name)

    def poisson_solve(self, rhs: np.ndarray) -> np.ndarray:
        rhs = np.asfortranarray(rhs, dtype=np.float64)
        out = np.zeros(self.shape, order="F")
        self._check(lib().eddy_poisson_solve(self.h, _ptr(rhs), _ptr(out), 0), "eddy_poisson_solve")
        return out

    def max_divergence(self) -> float:
        v = C.c_double(0.0)
        self._check(lib().eddy_max_divergence(self.h, C.byref(v)), "eddy_max_divergence")
        return v.value

    # ---- immersed body ----
    def set_body(self, tri: np.ndarray, normals: np.ndarray, velocity=(0.0, 0.0, 0.0)):
        # C order [triangle][vertex][x, y, z] and [triangle][x, y, z]
        tri = np.ascontiguousarray(tri, dtype=np.float64).reshape(-1)
        nrm = np.ascontiguousarray(normals, dtype=np.float64).reshape(-1)
        vel = np.ascontiguousarray(velocity, dtype=np.float64).reshape(-1)
        self._check(lib().eddy_ib_set_body(self.h, len(tri) // 9, _ptr(tri), _ptr(nrm), _ptr(vel)),
                    "eddy_ib_set_body")

    def ib_flags(self, which: int) -> np.ndarray:
        out = np.zeros(self.shape[0] * self.shape[1] * self.shape[2], dtype=np.int8)
        self._check(lib().eddy_ib_flags(self.h, which, out.ctypes.data_as(C.c_void_p)), "eddy_ib_flags")
        return out.reshape(self.shape, order="F")

    def ib_limits(self):
        lim = (C.c_int * 6)()
        self._check(lib().eddy_ib_limits(self.h, lim), "eddy_ib_limits")
        return tuple(lim)

    def ib_stencils(self, q: int) -> dict:
        n, nl = C.c_int(0), C.c_int(0)
        self._check(lib().eddy_ib_stencils(self.h, q, C.byref(n), C.byref(nl), None, None, None, None, None, None),
                    "eddy_ib_stencils")
        m = n.value
        ijk = np.zeros(3 * max(m, 1), np.int32)
        dijk = np.zeros(3 * max(m, 1), np.int32)
        lev = np.zeros(max(m, 1), np.int32)
        xn = np.zeros(3 * max(m, 1))
        lu = np.zeros(4 * max(m, 1))
        indx = np.zeros(2 * max(m, 1), np.int32)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        self._check(lib().eddy_ib_stencils(self.h, q, C.byref(n), C.byref(nl), vp(ijk), vp(dijk), vp(lev), vp(xn),
                                           vp(lu), vp(indx)), "eddy_ib_stencils")
        mrk = np.zeros(max(m, 1), np.int32)
        dr = np.zeros(max(m, 1), np.int32)
        xe = np.zeros(3 * max(m, 1))
        self._check(lib().eddy_ib_stencil_kinds(self.h, q, vp(mrk), vp(dr), vp(xe)), "eddy_ib_stencil_kinds")
        return {"n": m, "nlev": nl.value, "ijk": ijk[:3 * m].reshape(m, 3), "dijk": dijk[:3 * m].reshape(m, 3),
                "lev": lev[:m], "xn": xn[:3 * m].reshape(m, 3), "lu": lu[:4 * m].reshape(m, 4),
                "indx": indx[:2 * m].reshape(m, 2), "mrk": mrk[:m], "dir": dr[:m], "xe": xe[:3 * m].reshape(m, 3)}

    def refine_residuals(self) -> np.ndarray:
        """max |d - L phi| before each refinement sweep of the last mixed solve."""
        out = np.zeros(4)
        self._check(lib().eddy_refine_residuals(self.h, _ptr(out), 4), "eddy_refine_residuals")
        return out

    PROFILE_CATEGORIES = ["rhs_predictor", "boundary", "div_fft_fwd", "transform_fwd",
                          "z_line_solve", "transform_bwd", "fft_bwd", "correct",
                          "pressure_update", "density", "eddy_viscosity", "refine_residual",
                          "precision_copy", "ib_regen", "ib_force", "cn_line_solve"]

    def profile_enable(self, mask: int = 0xFFFF):
        self._check(lib().eddy_profile_enable(self.h, mask), "eddy_profile_enable")

    def profile_read(self) -> dict:
        ms = (C.c_double * len(self.PROFILE_CATEGORIES))()
        n = (C.c_longlong * len(self.PROFILE_CATEGORIES))()
        self._check(lib().eddy_profile_read(self.h, ms, n), "eddy_profile_read")
        return {c: (ms[i], n[i]) for i, c in enumerate(self.PROFILE_CATEGORIES)}

    def sync(self):
        self._check(lib().eddy_sync(self.h), "eddy_sync")

    @property
    def launches(self) -> int:
        return int(lib().eddy_launch_count(self.h))

    @property
    def stream(self) -> int:
        return int(lib().eddy_stream(self.h) or 0)

    def close(self):
        if getattr(self, "h", None):
            lib().eddy_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
