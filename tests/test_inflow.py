"""The hybrid inlet's inflow planes (src/hybrid.f:162-260) on the host: the
plane file layout read_hybrid reads, and the sequence position of a cycle."""
import math

import numpy as np
import pytest

import eddy_hybrid_b200 as eh


def _planes(nx, ny, seed=1):
    rng = np.random.RandomState(seed)
    return {k: rng.randn(nx, ny) for k in "uvwpd"}


def test_plane_file_roundtrip(tmp_path):
    nx, ny = 7, 5
    pl = _planes(nx, ny)
    path = str(tmp_path / "hybrid_k0001_n00000012.interp")
    eh.write_hybrid_plane(path, pl["u"], pl["v"], pl["w"], pl["d"], p=pl["p"], icycle=12, time=3.25,
                          xc=np.arange(nx) * 0.5, yc=np.arange(ny) * 0.25)
    r = eh.read_hybrid_plane(path, nx, ny)
    for k in "uvwpd":
        np.testing.assert_array_equal(r[k], pl[k])
    assert r["icycle"] == 12 and r["time"] == 3.25


def test_plane_file_refused(tmp_path):
    nx, ny = 7, 5
    pl = _planes(nx, ny)
    path = str(tmp_path / "p.interp")
    eh.write_hybrid_plane(path, pl["u"], pl["v"], pl["w"], pl["d"])
    with pytest.raises(eh.EddyError):
        eh.read_hybrid_plane(path, nx, ny + 1)          # another grid
    data = open(path, "rb").read()
    short = str(tmp_path / "short.interp")
    open(short, "wb").write(data[:-20])
    with pytest.raises(eh.EddyError):
        eh.read_hybrid_plane(short, nx, ny)             # truncated
    with pytest.raises(eh.EddyError):
        eh.read_hybrid_plane(str(tmp_path / "missing.interp"), nx, ny)


def _icycle_feed(icycle, start, end, stride):
    # sequence_hybrid, src/hybrid.f:224-232, as written there
    num = (end - start) // stride + 1
    n_feed_cycles = math.floor(icycle / num)
    return int(start + stride * icycle - stride * n_feed_cycles * num)


@pytest.mark.parametrize("start,end,stride", [(0, 40, 10), (100, 100, 1), (3, 21, 2)])
def test_feed_position_follows_sequence_hybrid(oracle, start, end, stride):
    num = (end - start) // stride + 1
    for c in range(-2 * num - 1, 3 * num + 2):
        pos = oracle.lib().eo_feed_position(c, num)
        assert 0 <= pos < num
        assert start + stride * pos == _icycle_feed(c, start, end, stride), c
