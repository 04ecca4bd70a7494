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
