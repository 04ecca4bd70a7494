"""Workload definitions and host-side grid/initial-field generation.

The reference never generates stretched grids: it reads face coordinates
from text files of the form ``N`` followed by ``i x_i`` lines
(src/grid.f:21-25, e.g. run/x1_grid.in).  ``tanh_faces`` defines the
two-sided tanh clustering used by the workloads here and ``write_grid_file``
writes it in that format, so a Fortran driver and this library consume the
same coordinates.

Axis convention (the reference's): x = x_ref (stretched, slip walls, gravity
direction), y = y_ref (uniform, periodic, FFT axis), z = z_ref (stretched,
streamwise, hybrid inlet type 305 / convective outlet type 730).  A workload
named ``Nx x Ny x Nz`` in streamwise/vertical/periodic order maps to
NX-2 = Ny (vertical), NY-2 = Nz (periodic), NZ-2 = Nx (streamwise).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

# Reference boundary-type codes (src/boundary.f: 60 slip wall, 500 periodic,
# 305 hybrid inlet plane, 730 convective outlet with mass balance).
ITYPE_WAKE = (60, 60, 500, 500, 305, 730)


def tanh_faces(a: float, b: float, c: float, n: int, beta: float) -> np.ndarray:
    """n+1 face coordinates on [a,b], clustered at c by a two-sided tanh map.

    On each side of c the normalised index t in [0,1] maps to
    x = c + side*(1 - tanh(beta*(1-t))/tanh(beta)); the cell counts on the two
    sides are proportional to the side lengths so the spacing is continuous at
    c.  Spacing ratio max/min is cosh(beta)**2.
    """
    if not (a < c < b):
        raise ValueError("cluster point must lie inside the interval")
    na = int(round(n * (c - a) / (b - a)))
    na = min(max(na, 1), n - 1)
    nb = n - na
    ta = np.arange(na + 1, dtype=np.float64) / na
    tb = np.arange(nb + 1, dtype=np.float64) / nb
    tb_ = math.tanh(beta)
    left = c - (c - a) * (1.0 - np.tanh(beta * (1.0 - ta)) / tb_)
    right = c + (b - c) * (1.0 - np.tanh(beta * (1.0 - tb)) / tb_)
    x = np.concatenate([left[::-1], right[1:]])
    x[0], x[-1] = a, b
    return x


def write_grid_file(path: str, faces: np.ndarray) -> None:
    """Write faces in the reference grid-file format (src/grid.f:23-24)."""
    with open(path, "w") as f:
        f.write(f"{len(faces)}\n")
        for i, x in enumerate(faces, start=1):
            f.write(f"{i} {x:.17e}\n")


@dataclasses.dataclass
class Workload:
    """One configuration in the reference's axis convention."""
    name: str
    mx: int            # interior cells along x_ref (vertical)
    ly: int            # interior cells along y_ref (periodic)
    nz_: int           # interior cells along z_ref (streamwise)
    xlim: tuple = (-4.0, 4.0)
    ylim: tuple = (-4.0, 4.0)
    zlim: tuple = (-4.0, 12.0)
    beta: float = 2.0
    re: float = 1000.0
    fr: float = 0.5
    pr: float = 1.0
    dt: float = 1e-3
    steps: int = 10
    seed: int = 42
    noise: float = 1e-3
    isgs: int = 2
    ischm: int = 3          # 3 RK3, 1 AB2 (src/inpall.f:218-235)
    idens: int = 1
    itype: tuple = ITYPE_WAKE
    sphere: bool = True
    body_speed: float = 0.0
    imply: int = 0     # Crank-Nicolson viscous terms along y (the reference input's IMPLY)
    implx: int = 0     # Crank-Nicolson viscous terms along x (IMPLX)
    implcx: int = 0    # Crank-Nicolson convective terms along x (IMPLCX)
    implcy: int = 0    # Crank-Nicolson convective terms along y (IMPLCY)

    @property
    def nx(self) -> int:
        return self.mx + 2

    @property
    def ny(self) -> int:
        return self.ly + 2

    @property
    def nz(self) -> int:
        return self.nz_ + 2

    @property
    def ncell(self) -> int:
        return self.mx * self.ly * self.nz_

    def faces(self):
        xf = tanh_faces(self.xlim[0], self.xlim[1], 0.0, self.mx, self.beta)
        zf = tanh_faces(self.zlim[0], self.zlim[1], 0.0, self.nz_, self.beta)
        return xf, zf

    def params(self) -> dict:
        """Solver parameters (names as the reference's COMMON blocks)."""
        return dict(
            nx=self.nx, ny=self.ny, nz=self.nz, itype=self.itype, ischm=self.ischm,
            isgs=self.isgs, idens=self.idens, ru1=1.0 / self.re, prn=self.pr,
            # Fr = N D / U with D = U = 1 and N^2 = -grav*denP1, denP1 = -1
            denP1=-1.0, grav=self.fr ** 2, dpdx=0.0, dpdy=0.0, dpdz=0.0,
            eps=1e-16, css=0.1,
            vspngx1=max(2, self.mx // 24), dspngx1=max(2, self.mx // 24),
            vspngx3in=0, vspngx3out=0, dspngx3in=0,
            dspngx3out=max(4, self.nz_ // 14),
            imply=self.imply, implx=self.implx, implcx=self.implcx, implcy=self.implcy,
        )


# Named workloads (streamwise x vertical x periodic in the names).
def sphere_128x96x64(**kw) -> Workload:
    return Workload("sphere_128x96x64", mx=96, ly=64, nz_=128, beta=2.0, re=1000.0,
                    fr=0.5, dt=1e-3, steps=10, **kw)


def poisson_256x256x256(**kw) -> Workload:
    return Workload("poisson_256x256x256", mx=256, ly=256, nz_=256, beta=2.5, re=1000.0,
                    fr=1.0, dt=1e-3, steps=1, sphere=False, **kw)


def wake_512x384x256(**kw) -> Workload:
    return Workload("wake_512x384x256", mx=384, ly=256, nz_=512, beta=2.0, re=10000.0,
                    fr=1.0, dt=5e-4, steps=100, body_speed=1.0, **kw)


def small(mx=24, ly=16, nz_=32, **kw) -> Workload:
    """A small case for parity tests (seconds on the CPU oracle)."""
    kw.setdefault("sphere", False)
    return Workload(f"small_{nz_}x{mx}x{ly}", mx=mx, ly=ly, nz_=nz_, **kw)


def splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)).astype(np.uint64)
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)).astype(np.uint64)
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)).astype(np.uint64)
    return x ^ (x >> np.uint64(31))


def uniform(seed: int, counters: np.ndarray) -> np.ndarray:
    """Counter-based U[0,1): splitmix64(splitmix64(seed) ^ counter)."""
    with np.errstate(over="ignore"):
        s = splitmix64(np.array([seed], dtype=np.uint64))[0]
        h = splitmix64(np.bitwise_xor(counters.astype(np.uint64), s))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def initial_fields(w: Workload, dens_bg_x: np.ndarray) -> dict:
    """Start-from-scratch fields (src/hybrid.f:119-146 with a uniform inlet
    plane u=v=0, w=1, dens=background): velocity plus white noise
    noise*(U-0.5) on the interior (after devel.f:4913-4915), Fortran order."""
    nx, ny, nz = w.nx, w.ny, w.nz
    shape = (nx, ny, nz)
    n = nx * ny * nz
    u = np.zeros(shape, order="F")
    v = np.zeros(shape, order="F")
    ww = np.ones(shape, order="F")
    idx = np.arange(n, dtype=np.uint64).reshape(shape, order="F")
    inner = (slice(1, nx - 1), slice(1, ny - 1), slice(1, nz - 1))
    for c, f in enumerate((u, v, ww)):
        r = uniform(w.seed, idx + np.uint64(c * n))
        f[inner] += w.noise * (r[inner] - 0.5)
    dens = np.empty(shape, order="F")
    dens[:] = dens_bg_x[:, None, None]
    p = np.zeros(shape, order="F")
    planeU = np.zeros((nx, ny), order="F")
    planeV = np.zeros((nx, ny), order="F")
    planeW = np.ones((nx, ny), order="F")
    planeD = np.empty((nx, ny), order="F")
    planeD[:] = dens_bg_x[:, None]
    return dict(uo=u, vo=v, wo=ww, dens=dens, p=p, planeU=planeU, planeV=planeV,
                planeW=planeW, planeD=planeD)
