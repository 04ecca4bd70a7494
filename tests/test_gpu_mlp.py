"""Tensor-core (tcgen05, BF16 in / FP32 accumulate) kernels of the learned
closure against numpy on the same BF16-rounded operands."""
import ctypes as C

import numpy as np
import pytest

from eddy_hybrid_b200 import config

pytestmark = pytest.mark.gpu


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even FP32 -> BF16 bit patterns."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
    return r


def bf16_val(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32)


@pytest.fixture(scope="module")
def solver(product):
    return product.Solver(config.small(mx=12, ly=8, nz_=16))


@pytest.mark.parametrize("mnk", [(128, 64, 16), (256, 64, 64), (128, 16, 64), (384, 128, 192), (128, 256, 32)])
def test_umma_gemm_matches_numpy(product, solver, mnk):
    M, N, K = mnk
    rng = np.random.RandomState(M + N + K)
    a = bf16_bits(rng.randn(M, K).astype(np.float32))
    b = bf16_bits(rng.randn(N, K).astype(np.float32))
    d0 = rng.randn(M, N).astype(np.float32)
    ref = bf16_val(a).astype(np.float64) @ bf16_val(b).astype(np.float64).T
    for acc in (0, 1):
        d = d0.copy()
        rc = product.lib().eddy_umma_gemm_bf16(solver.h, M, N, K, a.ctypes.data_as(C.c_void_p),
                                               b.ctypes.data_as(C.c_void_p),
                                               d.ctypes.data_as(C.POINTER(C.c_float)), acc)
        assert rc == 0
        want = ref + (d0 if acc else 0)
        err = np.max(np.abs(d - want)) / np.max(np.abs(want))
        assert err < 1e-5, (acc, err)
