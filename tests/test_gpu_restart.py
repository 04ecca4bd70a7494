"""Restart files (the reference's IOSCALAR layout): a run saved after some
steps and read back into a fresh solver continues bit-identically."""
import numpy as np
import pytest

from eddy_hybrid_b200 import config

pytestmark = pytest.mark.gpu


def test_restart_roundtrip_continues_bit_identically(product, tmp_path):
    w = config.small(mx=20, ly=16, nz_=24, noise=0.2, re=2000.0)
    f = config.initial_fields(w, product.Solver(w).metric("dens_bg")[: w.nx])
    a = product.Solver(w)
    a.load_initial(f)
    a.initialize()
    a.step(3)
    a.save_restart(str(tmp_path), 3, 3 * w.dt)
    b = product.Solver(w)
    b.load_initial(f)          # the inlet planes
    info = b.load_restart(str(tmp_path), 3)
    assert info["nstep"] == 3 and info["time"] == 3 * w.dt and info["dtm1"] == w.dt
    for n in a.RESTART_FIELDS:
        np.testing.assert_array_equal(b.download(n), a.download(n), err_msg=n)
    a.step(3)
    b.step(3)
    for n in a.RESTART_FIELDS:
        np.testing.assert_array_equal(b.download(n), a.download(n), err_msg=n)
