"""GPU test of e2d_residual_norms_static, the residual-norm entry point that
allocates no device memory (its scratch is a fixed device array in the
library).  It serves callers that cannot allocate device memory when they
need the norms — e.g. a solver loop where cudaMalloc could stall the device,
or a plugin whose host process owns the whole device-memory budget.

The test calls it through the C ABI on two block sets of different sizes in
a row, and checks each result against the allocating entry point e2d_norms:
each call's result must depend on its own input only, whatever the shared
scratch held before.  It also checks the property the entry point exists
for: once the first call on the device has been made (that call may load the
library's device code, which can allocate), a further call leaves the free
device memory unchanged.  It runs alone in a fresh process as well as after
the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from cffc_b200 import capi, cases

pytestmark = pytest.mark.gpu

RTOL = 1e-13  # the norm tolerance of the explicit-step parity tests


def _declare(lib):
    f = lib.e2d_residual_norms_static
    f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _device_dudt(h):
    d = C.POINTER(C.c_double)()
    assert h.lib.e2d_device_state(h.h, None, None, C.byref(d)) == 0
    return C.cast(d, C.c_void_p)


def test_static_norms_match_allocating_norms_twice():
    lib = capi.load_library()
    norms_static = _declare(lib)
    stream = torch.cuda.current_stream()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    for bs in (cases.periodic_box_bumps(nb=4, nc=32, seed=21),
               cases.channel(nbi=2, nbj=1, nci=8, ncj=6, seed=22)):
        h = capi.Handle(bs)
        h.lib.e2d_set_stream.argtypes = [C.c_void_p, C.c_void_p]
        assert h.lib.e2d_set_stream(h.h, C.c_void_p(stream.cuda_stream)) == 0
        h.set_state()
        h.residual()
        rc, _ = h.rk_steps(2)
        assert rc == 0
        expected = h.norms()
        out.fill_(-1.0)
        rc = norms_static(_device_dudt(h), bs.nblk, bs.nci, bs.ncj,
                          C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(expected > 0)
        np.testing.assert_allclose(got, expected, rtol=RTOL, atol=0)
        # after the first call: no device allocation by a further call
        free_before, _ = torch.cuda.mem_get_info()
        rc = norms_static(_device_dudt(h), bs.nblk, bs.nci, bs.ncj,
                          C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert rc == 0 and free_after == free_before
        np.testing.assert_allclose(out.cpu().numpy(), expected, rtol=RTOL, atol=0)
        h.close()


def test_static_norms_reject_too_many_blocks():
    lib = capi.load_library()
    norms_static = _declare(lib)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = norms_static(C.c_void_p(out.data_ptr()), 4097, 8, 8, C.c_void_p(out.data_ptr()), None)
    assert rc == -1
    rc = norms_static(None, 4, 8, 8, C.c_void_p(out.data_ptr()), None)
    assert rc == -1
