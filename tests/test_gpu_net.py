"""Warm-start network kernels: the tcgen05 tensor-core core against numpy."""
import numpy as np
import pytest

import qesb

pytestmark = pytest.mark.gpu


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bfloat16 bit patterns."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_value(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("N,K,a_mn,b_mn", [(16, 64, 0, 0), (32, 128, 0, 0), (64, 448, 0, 0), (128, 192, 0, 0),
                                           (256, 64, 0, 0), (64, 128, 1, 0), (64, 128, 0, 1), (128, 256, 1, 1),
                                           (16, 64, 1, 1)])
def test_umma_gemm_core(N, K, a_mn, b_mn):
    import ctypes as C

    rng = np.random.default_rng(N * 1000 + K + 7 * a_mn + 13 * b_mn)
    A = bf16_bits(rng.standard_normal((128, K)).astype(np.float32))
    B = bf16_bits(rng.standard_normal((N, K)).astype(np.float32))
    Af, Bf = bf16_value(A).astype(np.float64), bf16_value(B).astype(np.float64)
    ref = Af @ Bf.T
    Ain = np.ascontiguousarray(A.T) if a_mn else A
    Bin = np.ascontiguousarray(B.T) if b_mn else B
    out = np.zeros((128, N), np.float32)
    qesb.check(qesb.lib().qesb_umma_selftest(Ain.ctypes.data_as(C.c_void_p), Bin.ctypes.data_as(C.c_void_p),
                                             out.ctypes.data_as(C.c_void_p), N, K, a_mn, b_mn))
    np.testing.assert_allclose(out, ref, rtol=1e-5, atol=1e-4 * np.sqrt(K))
