"""ctypes front end of the CPU FP64 oracle (libeddy_oracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker; the product never imports it.
The library is built by oracle/Makefile into oracle/_build/.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libeddy_oracle.so")

FIELDS = ["uo", "vo", "wo", "p", "dp", "dens", "tv", "us", "vs", "ws", "ua",
          "va", "wa", "ub", "vb", "wb", "rha", "rhb", "rs", "planeU", "planeV",
          "planeW", "planeD"]
FID = {n: i for i, n in enumerate(FIELDS)}
GRID_ARRAYS = ["xu", "xc", "ap", "au", "av", "aw", "yv", "yc", "bp", "bu", "bv",
               "bw", "zw", "zc", "cp", "cu", "cv", "cw", "whx", "why", "whz",
               "dfxu", "dfxw", "dfxul", "dfxwl", "dfxd", "dfxdl", "dens_bg"]


class Params(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("itype", C.c_int * 7), ("ischm", C.c_int), ("isgs", C.c_int),
                ("idens", C.c_int), ("ru1", C.c_double), ("prn", C.c_double),
                ("denP1", C.c_double), ("grav", C.c_double), ("dpdx", C.c_double),
                ("dpdy", C.c_double), ("dpdz", C.c_double), ("eps", C.c_double),
                ("css", C.c_double), ("vspngx1", C.c_int), ("dspngx1", C.c_int),
                ("vspngx3in", C.c_int), ("vspngx3out", C.c_int),
                ("dspngx3in", C.c_int), ("dspngx3out", C.c_int), ("imply", C.c_int),
                ("implx", C.c_int), ("implcx", C.c_int), ("implcy", C.c_int)]


class IBSet(C.Structure):
    _fields_ = [("n", C.c_int), ("nlev", C.c_int)] + \
        [(f, C.POINTER(C.c_int)) for f in ("i", "j", "k", "di", "dj", "dk", "lev", "indx")] + \
        [(f, C.POINTER(C.c_double)) for f in ("xn", "yn", "zn", "lu")] + [("lev_start", C.POINTER(C.c_int))] + \
        [(f, C.POINTER(C.c_int)) for f in ("mrk", "dir")] + [(f, C.POINTER(C.c_double)) for f in ("xe", "ye", "ze")]


def make_params(d: dict) -> Params:
    p = Params()
    for k, v in d.items():
        if k == "itype":
            arr = (C.c_int * 7)(0, *v)
            p.itype = arr
        else:
            setattr(p, k, v)
    return p


_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.eo_grid_create.restype = C.c_void_p
        L.eo_grid_create.argtypes = [C.POINTER(Params), dp, C.c_double, C.c_double, dp]
        L.eo_grid_free.argtypes = [C.c_void_p]
        L.eo_grid_get.argtypes = [C.c_void_p, C.c_int, dp, C.c_int]
        L.eo_state_create.restype = C.c_void_p
        L.eo_state_create.argtypes = [C.POINTER(Params), C.c_void_p]
        L.eo_state_free.argtypes = [C.c_void_p]
        L.eo_set.argtypes = [C.c_void_p, C.c_int, dp]
        L.eo_get.argtypes = [C.c_void_p, C.c_int, dp]
        L.eo_initialize.argtypes = [C.c_void_p, C.c_double]
        L.eo_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
        L.eo_substep.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.eo_direct.argtypes = [C.c_void_p, C.c_int]
        L.eo_direct.restype = C.c_int
        L.eo_apply_laplacian.argtypes = [C.c_void_p, dp, dp]
        L.eo_rfftf.argtypes = [C.c_int, dp]
        L.eo_rfftb.argtypes = [C.c_int, dp]
        L.eo_turvis.argtypes = [C.c_void_p]
        L.eo_filtersize.argtypes = [C.c_void_p]
        L.eo_set_threads.argtypes = [C.c_int]
        for name in ("eo_predictord", "eo_density"):
            getattr(L, name).argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.eo_correct.argtypes = [C.c_void_p, C.c_double]
        L.eo_pressure_update.argtypes = [C.c_void_p]
        L.eo_rhs_density.argtypes = [C.c_void_p]
        L.eo_call_rhs_predictord.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.eo_inversey.argtypes = [C.c_void_p, C.c_double]
        L.eo_inversex.argtypes = [C.c_void_p, C.c_double]
        L.eo_inversex_walls.argtypes = [C.c_void_p, C.c_double]
        L.eo_calcfl.argtypes = [C.c_void_p]
        L.eo_calcfl.restype = C.c_double
        _P = C.POINTER(C.c_double)
        L.eo_calcfrc.argtypes = [C.c_void_p, _P, C.c_double, C.c_int, _P, _P]
        L.eo_cv_range.argtypes = [C.c_void_p, _P, C.POINTER(C.c_int)]
        L.eo_call_density.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.eo_call_boundary.argtypes = [C.c_void_p, C.c_int]
        L.eo_call_boundinout.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.eo_call_direct.argtypes = [C.c_void_p, C.c_double, C.c_int]
        L.eo_call_direct.restype = C.c_int
        L.eo_max_divergence.argtypes = [C.c_void_p]
        L.eo_max_divergence.restype = C.c_double
        vp = C.c_void_p
        L.eo_ib_create.restype = vp
        L.eo_ib_create.argtypes = [vp, C.c_int, dp, dp, dp]
        L.eo_ib_free.argtypes = [vp]
        for name in ("eo_ib_regen", "eo_ib_limimb", "eo_ib_flagp"):
            getattr(L, name).argtypes = [vp]
        L.eo_ib_tag.argtypes = [vp, C.c_int]
        L.eo_ib_taguo.argtypes = [vp, C.c_int, C.c_int]
        L.eo_ib_geom.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.eo_ib_move.argtypes = [vp, C.c_double]
        L.eo_ib_set_cadence.argtypes = [vp, C.c_int]
        L.eo_ib_set_brute.argtypes = [vp, C.c_int]
        L.eo_ib_force.argtypes = [vp, C.c_int, dp, C.c_double]
        L.eo_ib_interior.argtypes = [vp, C.c_int, dp, C.c_double]
        L.eo_ib_limits.restype = C.POINTER(C.c_int)
        L.eo_ib_limits.argtypes = [vp]
        L.eo_ib_tags.restype = C.POINTER(C.c_byte)
        L.eo_ib_tags.argtypes = [vp, C.c_int]
        L.eo_ib_flags.restype = C.POINTER(C.c_byte)
        L.eo_ib_flags.argtypes = [vp, C.c_int]
        L.eo_ib_stencils.restype = C.POINTER(IBSet)
        L.eo_ib_stencils.argtypes = [vp, C.c_int]
        L.eo_ib_body.argtypes = [vp, dp, dp]
        L.eo_state_set_ib.argtypes = [vp, vp]
        L.eo_feed_set.argtypes = [vp, C.c_int, dp, C.c_int, C.c_int]
        L.eo_feed_position.argtypes = [C.c_int, C.c_int]
        L.eo_feed_position.restype = C.c_int
        L.eo_locate.restype = C.c_int
        L.eo_locate.argtypes = [dp, C.c_int, C.c_double]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1)
    return a.ctypes.data_as(C.POINTER(C.c_double))


def yface_velocity(u: np.ndarray, mode: int) -> np.ndarray:
    """yface_velocity (src/Planes.f:481-543) of an (NX,NY,NZ) field, 0-based
    arrays: mode 1 the average over (i-1, i) x (j, j+1) for i = 2..NX-1, j =
    1..NY-1, k = 2..NZ-1 (1-based), 3 over (k-1, k) x (j, j+1), 4 over (j,
    j+1) for j = 1..NY-1; 0 and 2 the field itself; zero elsewhere."""
    u = np.asarray(u, dtype=np.float64)
    out = np.zeros_like(u)
    if mode in (0, 2):
        return u.copy()
    if mode == 1:
        out[1:-1, :-1, 1:-1] = 0.250 * (((u[1:-1, :-1, 1:-1] + u[:-2, :-1, 1:-1]) + u[1:-1, 1:, 1:-1])
                                        + u[:-2, 1:, 1:-1])
    elif mode == 3:
        out[1:-1, :-1, 1:-1] = 0.250 * (((u[1:-1, :-1, 1:-1] + u[1:-1, :-1, :-2]) + u[1:-1, 1:, 1:-1])
                                        + u[1:-1, 1:, :-2])
    elif mode == 4:
        out[:, :-1, :] = 0.50 * (u[:, :-1, :] + u[:, 1:, :])
    return out


def rfftf(x: np.ndarray) -> np.ndarray:
    r = np.ascontiguousarray(x, dtype=np.float64).copy()
    lib().eo_rfftf(len(r), _ptr(r))
    return r


def rfftb(x: np.ndarray) -> np.ndarray:
    r = np.ascontiguousarray(x, dtype=np.float64).copy()
    lib().eo_rfftb(len(r), _ptr(r))
    return r


class OracleGrid:
    def __init__(self, params: dict, xfaces, ymin, ymax, zfaces):
        self.params = params
        self._p = make_params(params)
        xf = np.ascontiguousarray(xfaces[:params["nx"] - 1], dtype=np.float64)
        zf = np.ascontiguousarray(zfaces[:params["nz"] - 1], dtype=np.float64)
        self.h = lib().eo_grid_create(C.byref(self._p), _ptr(xf), ymin, ymax, _ptr(zf))

    def get(self, name: str) -> np.ndarray:
        which = GRID_ARRAYS.index(name)
        n = 3 * (max(self.params["nx"], self.params["ny"], self.params["nz"]) + 2)
        n = max(n, self.params["nx"] * self.params["ny"])
        out = np.zeros(n)
        m = lib().eo_grid_get(self.h, which, _ptr(out), n)
        return out[:m].copy()

    def __del__(self):
        if getattr(self, "h", None):
            lib().eo_grid_free(self.h)
            self.h = None


class OracleSolver:
    """Whole-state oracle of the reference driver's time advance."""

    def __init__(self, workload, threads: int = 0):
        self.w = workload
        params = workload.params()
        xf, zf = workload.faces()
        self.grid = OracleGrid(params, xf, workload.ylim[0], workload.ylim[1], zf)
        self._p = make_params(params)
        self.h = lib().eo_state_create(C.byref(self._p), self.grid.h)
        if threads:
            lib().eo_set_threads(threads)
        self.shape = (params["nx"], params["ny"], params["nz"])

    def set(self, name: str, a: np.ndarray):
        a = np.asfortranarray(a, dtype=np.float64)
        lib().eo_set(self.h, FID[name], _ptr(a))

    def get(self, name: str) -> np.ndarray:
        shape = self.shape[:2] if name.startswith("plane") else self.shape
        a = np.zeros(shape, order="F")
        lib().eo_get(self.h, FID[name], _ptr(a))
        return a

    def load_initial(self, fields: dict):
        for k, v in fields.items():
            self.set(k, v)

    def initialize(self):
        lib().eo_initialize(self.h, self.w.dt)

    def step(self, nsteps: int = 1, poisson_method: int = 0):
        lib().eo_step(self.h, self.w.dt, nsteps, poisson_method)

    def direct(self, method: int = 0) -> int:
        return lib().eo_direct(self.h, method)

    def apply_laplacian(self, x: np.ndarray) -> np.ndarray:
        x = np.asfortranarray(x, dtype=np.float64)
        out = np.zeros(self.shape, order="F")
        lib().eo_apply_laplacian(self.h, _ptr(x), _ptr(out))
        return out

    def turvis(self):
        lib().eo_turvis(self.h)

    # one method per product C-ABI entry point
    def rhs_predictord(self, alf, gam, rho):
        lib().eo_call_rhs_predictord(self.h, alf, gam, rho)

    def inversey(self, alf):
        lib().eo_inversey(self.h, alf)

    def inversex_walls(self, alf):
        """UB, VB, WB wall planes before the line solves (src/Eddy6.f:2582-2591)."""
        lib().eo_inversex_walls(self.h, alf)

    def inversex(self, alf):
        lib().eo_inversex(self.h, alf)

    def calcfl(self) -> float:
        return lib().eo_calcfl(self.h)

    def calcfrc(self, cvlim, dt: float, icycle: int, fb: np.ndarray) -> np.ndarray:
        """calcfrc (src/calcforce.f:3): the 56 force terms; fb (3,) the
        control volume's momentum of the previous call, updated in place."""
        P = C.POINTER(C.c_double)
        cv = np.ascontiguousarray(cvlim, dtype=np.float64)
        assert fb.dtype == np.float64 and fb.flags.c_contiguous and fb.shape == (3,)
        out = np.zeros(56)
        lib().eo_calcfrc(self.h, cv.ctypes.data_as(P), dt, icycle, fb.ctypes.data_as(P), out.ctypes.data_as(P))
        return out

    def cv_range(self, cvlim) -> tuple:
        """ICB, ICE, KCB, KCE, KBFLAG, KEFLAG of the control volume."""
        cv = np.ascontiguousarray(cvlim, dtype=np.float64)
        r = (C.c_int * 6)()
        lib().eo_cv_range(self.grid.h, cv.ctypes.data_as(C.POINTER(C.c_double)), r)
        return tuple(r)

    def boundary(self, set_):
        lib().eo_call_boundary(self.h, set_)

    def boundinout(self, idiv, alf):
        lib().eo_call_boundinout(self.h, idiv, alf)

    def direct_from_velocity(self, alf, method=0):
        return lib().eo_call_direct(self.h, alf, method)

    def correct(self, alf):
        lib().eo_correct(self.h, alf)

    def pressure_update(self):
        lib().eo_pressure_update(self.h)

    def density(self, alf, gam, rho):
        lib().eo_call_density(self.h, alf, gam, rho)

    def substep(self, is_):
        lib().eo_substep(self.h, is_, self.w.dt)

    def max_divergence(self):
        return lib().eo_max_divergence(self.h)

    def set_inflow_sequence(self, planes: np.ndarray, iref: int, nstep: int = 0):
        """planes: (n, 4, NX, NY) inflow planes u, v, w, rho in feed order"""
        a = np.ascontiguousarray(np.asarray(planes, dtype=np.float64).transpose(0, 1, 3, 2))
        lib().eo_feed_set(self.h, a.shape[0], a.ctypes.data_as(C.POINTER(C.c_double)), iref, nstep)

    def __del__(self):
        if getattr(self, "h", None):
            lib().eo_state_free(self.h)
            self.h = None


class OracleIB:
    """Immersed body attached to an OracleSolver (restated TAG3D_MOD, taguo,
    flagp, grid-line geom/mtrx, momforc/correctpres, RBM translation)."""

    VARS = ("u", "v", "w", "p")

    def __init__(self, solver: "OracleSolver", tri: np.ndarray, normals: np.ndarray, vel=(0.0, 0.0, 0.0),
                 attach: bool = True):
        self.s = solver
        tri = np.ascontiguousarray(tri, dtype=np.float64).reshape(-1)
        nrm = np.ascontiguousarray(normals, dtype=np.float64).reshape(-1)
        v = np.ascontiguousarray(vel, dtype=np.float64)
        self.nb = len(tri) // 9
        self.h = lib().eo_ib_create(solver.grid.h, self.nb, _ptr(tri), _ptr(nrm), _ptr(v))
        if attach:
            lib().eo_state_set_ib(solver.h, self.h)

    def regen(self):
        lib().eo_ib_regen(self.h)

    def set_cadence(self, every_substep: int):
        lib().eo_ib_set_cadence(self.h, every_substep)

    def set_brute(self, brute: int):
        lib().eo_ib_set_brute(self.h, brute)

    def move(self, t: float):
        lib().eo_ib_move(self.h, t)

    def limits(self):
        p = lib().eo_ib_limits(self.h)
        return tuple(p[a] for a in range(6))

    def _grid3(self, ptr):
        nx, ny, nz = self.s.shape
        a = np.ctypeslib.as_array(ptr, shape=(nx * ny * nz,)).copy()
        return a.reshape((nx, ny, nz), order="F")

    def tags(self, q: int) -> np.ndarray:
        return self._grid3(lib().eo_ib_tags(self.h, q))

    def flags(self, fq: int) -> np.ndarray:
        return self._grid3(lib().eo_ib_flags(self.h, fq))

    def stencils(self, q: int) -> dict:
        S = lib().eo_ib_stencils(self.h, q).contents
        n = S.n
        out = {"n": n, "nlev": S.nlev}
        for f in ("i", "j", "k", "di", "dj", "dk", "lev", "mrk", "dir"):
            out[f] = np.ctypeslib.as_array(getattr(S, f), shape=(n,)).copy() if n else np.zeros(0, np.int32)
        for f in ("xn", "yn", "zn", "xe", "ye", "ze"):
            out[f] = np.ctypeslib.as_array(getattr(S, f), shape=(n,)).copy() if n else np.zeros(0)
        out["lu"] = np.ctypeslib.as_array(S.lu, shape=(4 * n,)).copy().reshape(n, 4) if n else np.zeros((0, 4))
        out["indx"] = np.ctypeslib.as_array(S.indx, shape=(2 * n,)).copy().reshape(n, 2) if n else \
            np.zeros((0, 2), np.int32)
        out["lev_start"] = np.ctypeslib.as_array(S.lev_start, shape=(S.nlev + 1,)).copy()
        return out

    def force(self, q: int, a: np.ndarray, b0: float) -> np.ndarray:
        a = np.asfortranarray(a, dtype=np.float64).copy(order="F")
        lib().eo_ib_force(self.h, q, _ptr(a), b0)
        return a

    def interior(self, fq: int, a: np.ndarray, value: float) -> np.ndarray:
        a = np.asfortranarray(a, dtype=np.float64).copy(order="F")
        lib().eo_ib_interior(self.h, fq, _ptr(a), value)
        return a

    def body(self):
        v = np.zeros(9 * self.nb)
        c = np.zeros(3 * self.nb)
        lib().eo_ib_body(self.h, _ptr(v), _ptr(c))
        return v.reshape(self.nb, 3, 3), c.reshape(self.nb, 3)
