"""Host-side pieces that need no GPU: grid generation, the library's metric
builder against the oracle (bit-exact), and the C ABI's exported symbols."""
import ctypes
import os
import re

import numpy as np
import pytest

from eddy_hybrid_b200 import config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tanh_faces_properties():
    f = config.tanh_faces(-4.0, 12.0, 0.0, 512, 2.0)
    assert len(f) == 513 and f[0] == -4.0 and f[-1] == 12.0
    assert np.all(np.diff(f) > 0)
    h = np.diff(f)
    assert h.max() / h.min() == pytest.approx(np.cosh(2.0) ** 2, rel=0.05)
    assert np.argmin(h) in (127, 128)  # clustered at the origin


def test_grid_file_format(tmp_path):
    f = config.tanh_faces(-4.0, 4.0, 0.0, 16, 2.0)
    p = tmp_path / "x1_grid.in"
    config.write_grid_file(str(p), f)
    lines = p.read_text().splitlines()
    assert int(lines[0]) == 17
    idx, x = lines[5].split()
    assert int(idx) == 5 and float(x) == f[4]


@pytest.mark.parametrize("mk", [lambda: config.small(mx=12, ly=8, nz_=16),
                                lambda: config.sphere_128x96x64()])
def test_metrics_bit_exact_vs_oracle(oracle, product, mk):
    w = mk()
    g = oracle.OracleGrid(w.params(), *w.faces()[:1], w.ylim[0], w.ylim[1], w.faces()[1])
    for name in product.METRICS:
        a = product.grid_metric(w, name)
        b = g.get(name)
        assert a.shape == b.shape, name
        np.testing.assert_array_equal(a, b, err_msg=name)


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "eddy_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(eddy_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(product):
    lib = ctypes.CDLL(product.LIB_PATH)
    syms = _declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    # and the Python mirror binds them all
    assert set(syms) <= set(product.SIGNATURES)


def test_create_fails_cleanly_without_valid_config(product):
    w = config.small(mx=12, ly=8, nz_=16)
    w.itype = (60, 60, 60, 60, 305, 730)   # y not periodic: refused
    with pytest.raises(product.EddyError):
        product.Solver(w)
    # the implicit x terms are built for slip walls on both x sides and the
    # plain FP64 form only: anything else is refused before any device work
    for kw in ({"implx": 1, "itype": (60, 82, 500, 500, 305, 730)}, {"implx": 2},
               {"implcx": 1, "itype": (82, 60, 500, 500, 305, 730)}, {"implcx": -1}, {"implcy": 2}):
        w = config.small(mx=12, ly=8, nz_=16)
        for k, v in kw.items():
            setattr(w, k, v)
        with pytest.raises(product.EddyError):
            product.Solver(w)
    for kw in ({"implx": 1}, {"implcx": 1}, {"implcy": 1}):
        with pytest.raises(product.EddyError):
            product.Solver(config.small(mx=12, ly=8, nz_=16, **kw), precision=product.MIXED)


def test_download_checks_the_callers_buffer_before_copying(product):
    # a caller's buffer must be a Fortran-ordered float64 array of the field's
    # shape; anything else is refused before the library is called (no GPU)
    s = object.__new__(product.Solver)
    s.shape = (6, 5, 7)
    s.h = None
    ro = np.empty((6, 5, 7), order="F")
    ro.flags.writeable = False
    for bad in (np.empty((6, 5, 7)),                        # C order
                np.empty((6, 5, 6), order="F"),             # wrong shape
                np.empty((6, 5, 7), order="F", dtype=np.float32),
                ro):                                        # read-only
        with pytest.raises(ValueError):
            s.download("uo", out=bad)


def test_restart_file_layout_is_ioscalars(product, tmp_path):
    # the reference's IOSCALAR (src/io.f:150-175, serial): Fortran unformatted
    # records framed by 4-byte lengths -- (NX, NY, NZ, 1), one NX*NY plane per
    # k, nstep, TIME, (DTM1, grav)
    nx, ny, nz = 5, 4, 3
    a = np.asfortranarray(np.arange(nx * ny * nz, dtype=np.float64).reshape((nx, ny, nz), order="F") * 0.25 - 3.0)
    path = str(tmp_path / "u_00000042.res")
    product.write_ioscalar(path, a, 42, 1.5, 5e-4, 1.0)
    raw = open(path, "rb").read()
    pos = 0

    def rec(nbytes):
        nonlocal pos
        n0 = int(np.frombuffer(raw, np.int32, 1, pos)[0])
        assert n0 == nbytes
        body = raw[pos + 4: pos + 4 + nbytes]
        n1 = int(np.frombuffer(raw, np.int32, 1, pos + 4 + nbytes)[0])
        assert n1 == nbytes
        pos += nbytes + 8
        return body

    assert list(np.frombuffer(rec(16), np.int32)) == [nx, ny, nz, 1]
    for k in range(nz):
        np.testing.assert_array_equal(np.frombuffer(rec(8 * nx * ny), np.float64), a[:, :, k].ravel(order="F"))
    assert int(np.frombuffer(rec(4), np.int32)[0]) == 42
    assert float(np.frombuffer(rec(8), np.float64)[0]) == 1.5
    assert list(np.frombuffer(rec(16), np.float64)) == [5e-4, 1.0]
    assert pos == len(raw)
    b, ns, t, dt, gr = product.read_ioscalar(path, (nx, ny, nz))
    np.testing.assert_array_equal(a, b)
    assert (ns, t, dt, gr) == (42, 1.5, 5e-4, 1.0)
    # another grid, or a truncated file, is refused
    with pytest.raises(product.EddyError):
        product.read_ioscalar(path, (nx, ny, nz + 1))
    open(path, "wb").write(raw[:-10])
    with pytest.raises(product.EddyError):
        product.read_ioscalar(path, (nx, ny, nz))
