"""Immersed body geometry: a triangulated sphere (icosphere).

The reference reads its bodies from STL files (src/object.f, run/stl.input);
the sphere of the workloads (diameter D = 1 at the origin) is generated here
instead: an icosahedron subdivided `level` times with every vertex projected
onto the sphere, triangles ordered with outward normals.  Arrays use the
solver's axes (x vertical, y periodic, z streamwise): vertices (nb, 3, 3) as
[triangle][vertex a, b, c][x, y, z], unit outward normals (nb, 3).
"""
from __future__ import annotations

import numpy as np


def icosphere(level: int = 3, radius: float = 0.5, center=(0.0, 0.0, 0.0)):
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]
        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    P = np.array(verts) * radius + np.asarray(center, dtype=np.float64)
    tri = P[np.array(faces)]                       # (nb, 3, 3)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    cen = tri.mean(axis=1)
    flip = np.einsum("ij,ij->i", n, cen - np.asarray(center)) < 0
    tri[flip] = tri[flip][:, [0, 2, 1]]
    n[flip] = -n[flip]
    n /= np.linalg.norm(n, axis=1)[:, None]
    return np.ascontiguousarray(tri), np.ascontiguousarray(n)


def level_for_spacing(h: float, radius: float = 0.5) -> int:
    """Smallest subdivision level whose edges are no longer than about 2h."""
    lev = 0
    edge = 1.05 * radius  # icosahedron edge on the unit sphere ~1.05
    while edge > 2.0 * h and lev < 8:
        edge *= 0.5
        lev += 1
    return lev


def body_velocity(workload) -> tuple:
    """Translation velocity of the sphere (x, y, z): upstream along z at the
    workload's body speed (the inflow is w = 1 downstream)."""
    return (0.0, 0.0, -float(getattr(workload, "body_speed", 0.0)))
