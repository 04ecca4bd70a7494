"""A device-resident sequence of inflow planes at the hybrid inlet
(sequence_hybrid, src/hybrid.f:213-260, loaded after every substep,
src/Eddy6.f:2985-2991): GPU steps against the oracle's."""
import numpy as np
import pytest

from conftest import P_BAR, P_PROFILE_BAR, p_err, p_profile_err, rel_err, run_with_scale
from eddy_hybrid_b200 import MIXED, config

pytestmark = pytest.mark.gpu


def _sequence(w, f, n, seed=3):
    rng = np.random.RandomState(seed)
    base = np.stack([f["planeU"], f["planeV"], f["planeW"], f["planeD"]])
    return np.stack([base + 0.05 * rng.randn(*base.shape) for _ in range(n)])


@pytest.mark.parametrize("nstep0", [0, 7])
def test_inflow_sequence_steps(oracle, product, nstep0):
    w = config.small(mx=24, ly=16, nz_=32, noise=0.1)
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    seq = _sequence(w, f, 3)
    iref = w.nx // 2
    o.load_initial(f)
    o.set_inflow_sequence(seq, iref, nstep0)
    o.initialize()
    g = product.Solver(w)
    g.load_initial(f)
    g.set_inflow_sequence(seq, iref, nstep0)
    g.initialize()
    for n in ("planeU", "planeV", "planeW", "planeD"):
        np.testing.assert_array_equal(g.download(n), o.get(n))
    scale = run_with_scale(o, 5)
    g.step(5)
    # the planes of the last cycle, the far field (x index >= iref) from the last plane
    c = nstep0 + 5
    pos = c % 3
    for q, n in enumerate(("planeU", "planeV", "planeW", "planeD")):
        want = np.array(seq[pos, q])
        want[iref - 1:, :] = seq[2, q, iref - 1:, :]
        np.testing.assert_array_equal(o.get(n), want)
        np.testing.assert_array_equal(g.download(n), want)
    for n in ("uo", "vo", "wo", "dens", "tv"):
        e = rel_err(g.download(n), o.get(n))
        assert e < 1e-11, (n, e)
    pg = g.download("p")
    assert p_err(pg, o.get("p"), scale) < P_BAR
    assert p_profile_err(pg, o.get("p"), scale) < P_PROFILE_BAR


def test_inflow_sequence_mixed_form(product, oracle):
    w = config.small(mx=24, ly=16, nz_=32, noise=0.1)
    o = oracle.OracleSolver(w)
    f = config.initial_fields(w, o.grid.get("dens_bg")[: w.nx])
    seq = _sequence(w, f, 4)
    g = product.Solver(w, precision=MIXED, refine_sweeps=2)
    g.load_initial(f)
    g.set_inflow_sequence(seq, w.nx + 1, 0)
    g.initialize()
    g.step(2)
    # after step 2 the planes are those of cycle 2
    np.testing.assert_array_equal(g.download("planeW"), seq[2, 2])
    assert g.max_divergence() < 1e-10
