"""Post-processing on device fields: time probes recorded every step
(rec_timeprobes_all, src/stats.f:132-185) and planes of the y-face-centred
fields (WRITE_PLANES / yface_velocity, src/Planes.f:1-543)."""
import numpy as np
import pytest

from eddy_hybrid_b200 import config

pytestmark = pytest.mark.gpu


def _solver(product, oracle):
    w = config.small(mx=24, ly=16, nz_=32, noise=0.1)
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    g = product.Solver(w)
    g.load_initial(f)
    g.initialize()
    return w, g


def test_time_probes_record_every_step(product, oracle):
    w, g = _solver(product, oracle)
    ijk = np.array([[2, 2, 2], [w.nx // 2, w.ny // 2, w.nz // 2], [w.nx - 1, w.ny - 1, w.nz - 1], [5, 3, 11]])
    g.set_probes(ijk, capacity=8)
    want = []
    t = 0.0
    for n in range(3):
        g.step(1)
        t += w.dt
        fl = {k: g.download(k) for k in ("uo", "vo", "wo", "p")}
        want.append([[t] + [fl[k][i - 1, j - 1, k_ - 1] for k in ("uo", "vo", "wo", "p")] for i, j, k_ in ijk])
    got = g.read_probes()
    assert got.shape == (3, 4, 5)
    np.testing.assert_array_equal(got, np.array(want))
    # consumed by the read; the capacity bounds what is kept
    assert g.read_probes().shape[0] == 0
    for _ in range(10):
        g.step(1)
    assert g.read_probes().shape[0] == 8


@pytest.mark.parametrize("mode,name", [(0, "p"), (1, "uo"), (2, "vo"), (3, "wo"), (4, "dens")])
def test_planes_match_yface_velocity(product, oracle, mode, name):
    w, g = _solver(product, oracle)
    g.step(2)
    full = oracle.yface_velocity(g.download(name), mode)
    for axis, index in ((1, 3), (2, 5), (2, w.ny), (3, w.nz // 2), (3, 1)):
        pl = g.plane(name, axis, index, center=mode)
        want = {1: full[index - 1, :, :], 2: full[:, index - 1, :], 3: full[:, :, index - 1]}[axis]
        np.testing.assert_array_equal(pl, want, err_msg=f"axis {axis} index {index}")
