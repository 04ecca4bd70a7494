"""Immersed-boundary oracle checks on the CPU (no GPU): the analytic sphere.

The reference's only IB record (run/stats_imb.dat) needs a grid and STL that
are not in the repository, so the restated tagging is pinned by invariants of
a sphere at the origin: mirror symmetry of the tags across x = 0 (the x grid
and the icosphere are exactly symmetric), the interior volume against the
sphere volume, and the forcing-point stencils reproducing linear data.
"""
import numpy as np
import pytest

from eddy_hybrid_b200 import body, config


@pytest.fixture(scope="module")
def sphere_ib(oracle):
    w = config.small(mx=40, ly=32, nz_=48)
    o = oracle.OracleSolver(w)
    tri, nrm = body.icosphere(3)
    ib = oracle.OracleIB(o, tri, nrm, attach=False)
    ib.regen()
    return w, o, ib


def test_tags_mirror_symmetric_in_x(sphere_ib):
    w, o, ib = sphere_ib
    for q in (1, 3):   # v and p grids: x at cell centres, symmetric about 0
        T = ib.tags(q)
        xc = o.grid.get("xc")            # xc(1..NX)
        np.testing.assert_array_equal(xc, -xc[::-1])
        np.testing.assert_array_equal(T, T[::-1], err_msg=f"var {q}")


def test_interior_volume_matches_sphere(sphere_ib):
    w, o, ib = sphere_ib
    T = ib.tags(3)
    ap, bp, cp = o.grid.get("ap"), o.grid.get("bp"), o.grid.get("cp")
    vol = (1 / ap[:w.nx])[:, None, None] * (1 / bp[:w.ny])[None, :, None] * (1 / cp[:w.nz])[None, None, :]
    inside = (T == -1)
    inside[:, 0, :] = inside[:, -1, :] = False   # periodic ghosts
    v = float((vol * inside).sum())
    assert abs(v - np.pi / 6) / (np.pi / 6) < 0.1, v


def test_flags_and_stencils_consistent(sphere_ib):
    w, o, ib = sphere_ib
    for q, fq in ((0, 0), (1, 1), (2, 2), (3, 4)):
        F = ib.flags(fq)
        S = ib.stencils(q)
        assert S["n"] > 0 and S["nlev"] >= 1
        # every stencil point is a forcing point, every extension point is not interior
        for a in range(S["n"]):
            i, j, k = S["i"][a] - 1, S["j"][a] - 1, S["k"][a] - 1
            assert F[i, j, k] == -1
            e = (i + S["di"][a], j + S["dj"][a], k + S["dk"][a])
            assert F[e] <= 0
        # levels are non-decreasing along the list
        assert np.all(np.diff(S["lev"]) >= 0)


def test_velocity_stencil_reproduces_linear_data(sphere_ib):
    """u(s) = c0 + c1 s along the stencil line: forcing with the body value and
    the extension value of a linear field returns its value at the point."""
    w, o, ib = sphere_ib
    S = ib.stencils(0)
    # 1-based coordinate lookups
    xu, yc, zc = (np.concatenate([[0.0], o.grid.get(n)]) for n in ("xu", "yc", "zc"))
    for a in range(0, S["n"], max(1, S["n"] // 25)):
        i, j, k = S["i"][a], S["j"][a], S["k"][a]
        p = np.array([xu[i], yc[j], zc[k]])
        e = np.array([xu[i + S["di"][a]], yc[j + S["dj"][a]], zc[k + S["dk"][a]]])
        xn = np.array([S["xn"][a], S["yn"][a], S["zn"][a]])
        so, s1 = -np.linalg.norm(p - xn), np.linalg.norm(p - e)
        c0, c1 = 0.7, -1.3
        A = S["lu"][a]
        # rebuild L U with the pivot and solve, as lubksb does
        L = np.array([[1.0, 0.0], [A[1], 1.0]])
        U = np.array([[A[0], A[2]], [0.0, A[3]]])
        b = np.array([c0 + c1 * so, c0 + c1 * s1])
        P = S["indx"][a]
        b[[0, P[0]]] = b[[P[0], 0]]
        x = np.linalg.solve(U, np.linalg.solve(L, b))
        assert abs(x[0] - c0) < 1e-12


@pytest.mark.parametrize("level,shift", [(3, (0.0, 0.0, 0.0)), (5, (0.013, -0.021, 0.37))])
def test_binned_searches_equal_exhaustive(oracle, level, shift):
    # the oracle prunes TAG3D candidates and nearest-centroid lists with exact
    # spatial bins (the reference prunes with ANN kd-trees); tags, flags and
    # every stencil must equal those of the exhaustive searches
    w = config.small(mx=40, ly=32, nz_=48)
    tri, nrm = body.icosphere(level)
    tri = tri + np.asarray(shift)[None, None, :]
    out = []
    for brute in (1, 0):
        o = oracle.OracleSolver(w)
        ib = oracle.OracleIB(o, tri, nrm, attach=False)
        ib.set_brute(brute)
        ib.regen()
        out.append((ib, [ib.tags(q) for q in range(4)], [ib.flags(f) for f in range(5)],
                    [ib.stencils(q) for q in range(4)]))
    (_, t0, f0, s0), (_, t1, f1, s1) = out
    for a, b in zip(t0 + f0, t1 + f1):
        np.testing.assert_array_equal(a, b)
    for a, b in zip(s0, s1):
        assert a["n"] == b["n"] and a["n"] > 0
        for key in ("i", "j", "k", "di", "dj", "dk", "lev", "xn", "yn", "zn", "lu", "indx"):
            np.testing.assert_array_equal(a[key], b[key], err_msg=key)


def test_locate_contract(oracle):
    # the table search keeps LOCATE's contract (src/numrec.f:390-422)
    import ctypes as C
    lib = oracle.lib()
    lib.eo_locate.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_double]
    lib.eo_locate.restype = C.c_int
    xs = np.array([0.0, -1.0, -0.5, 0.0, 0.0, 0.25, 1.0, 2.0])  # 1-based table xx[1..7], a repeated entry
    n = 7
    p = xs.ctypes.data_as(C.POINTER(C.c_double))
    def ref(x):
        if xs[1] == x:
            return 1
        return int(np.sum(xs[1:n + 1] < x))
    for x in (-2.0, -1.0, -0.7, -0.5, -0.1, 0.0, 0.1, 0.25, 0.9, 1.0, 2.0, 3.0):
        assert lib.eo_locate(p, n, x) == ref(x), x
    d = xs.copy()
    d[1:n + 1] = xs[1:n + 1][::-1]
    pd = d.ctypes.data_as(C.POINTER(C.c_double))
    for x in (-2.0, -0.5, 0.0, 0.3, 2.0, 3.0):
        want = 1 if d[1] == x else int(np.sum(d[1:n + 1] >= x))
        assert lib.eo_locate(pd, n, x) == want, x
