"""Every barrier wait in the library's kernels is bounded: a wait on a barrier
that nothing completes returns after about 2 s instead of hanging the GPU, so
an error path ends with a status the host can read (no fault is caused)."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def test_barrier_wait_gives_up_in_bounded_time(product):
    gave_up, seconds = C.c_int(-1), C.c_double(-1.0)
    rc = product.lib().eddy_selftest_wait_bound(0, C.byref(gave_up), C.byref(seconds))
    assert rc == 0
    assert gave_up.value == 1
    # the wall-time cap is 2 s, checked every 256 polls
    assert 1.9 < seconds.value < 10.0, seconds.value
