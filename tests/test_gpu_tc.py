"""The tensor-core building block of the warm-start network (tcgen05 UMMA,
BF16 x BF16 -> FP32 in TMEM) against an FP64 product of the same BF16
values.  Tolerance: FP32 accumulation of K <= 128 exact BF16 products,
|D - ref| <= 1e-5 * sum_k |a_k b_k| per entry."""
import ctypes as C

import numpy as np
import pytest

from cffc_b200 import capi

pytestmark = pytest.mark.gpu


def to_bf16_bits(x):
    """float32 -> bfloat16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_bf16_bits(b):
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("N,K", [(16, 16), (128, 128), (64, 32), (256, 128), (16, 128)])
def test_tc_gemm(N, K):
    lib = capi.load_library()
    rng = np.random.default_rng(N * 1000 + K)
    A = to_bf16_bits(rng.standard_normal((128, K)))
    B = to_bf16_bits(rng.standard_normal((N, K)))
    D = np.zeros((128, N), np.float32)
    lib.e2d_tc_selftest.argtypes = [C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), C.POINTER(C.c_float),
                                    C.c_int, C.c_int]
    rc = lib.e2d_tc_selftest(A.ctypes.data_as(C.POINTER(C.c_uint16)), B.ctypes.data_as(C.POINTER(C.c_uint16)),
                             D.ctypes.data_as(C.POINTER(C.c_float)), N, K)
    assert rc == 0
    a, b = from_bf16_bits(A).astype(np.float64), from_bf16_bits(B).astype(np.float64)
    ref = a @ b.T
    scale = np.abs(a) @ np.abs(b).T
    assert np.all(np.abs(D - ref) <= 1e-5 * scale + 1e-30)
