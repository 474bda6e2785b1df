"""GPU test: the fast FP64 path's Newton-refined reciprocal, reciprocal
square root and square root stay within a few units in the last place of
IEEE division and square root over the value range of the path."""
import ctypes as C

import numpy as np
import pytest
import torch

from cffc_b200 import capi

pytestmark = pytest.mark.gpu


def test_fast_reciprocal_and_sqrt_error_bounds():
    lib = capi.load_library()
    f = lib.e2d_fastmath_check
    f.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    f.restype = C.c_int
    rng = np.random.default_rng(5)
    x = np.concatenate([10.0 ** rng.uniform(-12, 12, 200000), rng.uniform(0.5, 2.0, 200000),
                        [1.0, 2.0, 0.25, 3.0, 1e-300 * 1e10]])
    xd = torch.from_numpy(x).cuda()
    out = (C.c_double * 3)()
    assert f(C.c_void_p(xd.data_ptr()), len(x), out) == 0
    eps = np.finfo(np.float64).eps
    assert out[0] <= 2 * eps, out[0]   # 1/x
    assert out[1] <= 2 * eps, out[1]   # 1/sqrt(x)
    assert out[2] <= 2 * eps, out[2]   # sqrt(x)
