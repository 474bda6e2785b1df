"""The ILU(k) level-of-fill pattern of the library (e2d_ilu_pattern, host
code) against a restatement of BPKIT's symbolic_ilu (oracle/ilu_pattern.py)
on the reference's block matrix: integer work, compared exactly.  The
numerical factors built on this pattern are compared with the reference's
Block_Preconditioner on the GPU (tests/test_gpu_precon.py)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from cffc_b200 import capi

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import ilu_pattern  # noqa: E402


def library_pattern(nci, ncj, level):
    lib = capi.load_library()
    f = lib.e2d_ilu_pattern
    f.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int32,
                  C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    row_ptr = np.zeros(nci * ncj + 1, dtype=np.int32)
    nnz, levels = C.c_int32(0), (C.c_int32 * 2)()
    as_p = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
    assert f(nci, ncj, level, as_p(row_ptr), None, 0, C.byref(nnz), levels) == 0
    col = np.zeros(nnz.value, dtype=np.int32)
    assert f(nci, ncj, level, as_p(row_ptr), as_p(col), nnz.value, C.byref(nnz), levels) == 0
    return row_ptr, col, (levels[0], levels[1])


@pytest.mark.parametrize("nci,ncj,level", [(6, 5, 0), (8, 6, 1), (8, 6, 2), (10, 7, 4), (12, 8, 7), (5, 9, 16)])
def test_pattern_matches_symbolic_ilu(nci, ncj, level):
    row_ptr, col, _ = library_pattern(nci, ncj, level)
    want_ptr, want_col = ilu_pattern.interior_pattern(nci, ncj, level)
    assert row_ptr.tolist() == want_ptr
    assert col.tolist() == want_col


def test_level_zero_is_the_five_point_stencil():
    nci, ncj = 7, 5
    row_ptr, col, levels = library_pattern(nci, ncj, 0)
    for r in range(nci * ncj):
        x, y = r % nci, r // nci
        want = sorted(q for q, ok in ((r - nci, y > 0), (r - 1, x > 0), (r, True), (r + 1, x < nci - 1),
                                      (r + nci, y < ncj - 1)) if ok)
        assert col[row_ptr[r]:row_ptr[r + 1]].tolist() == want
    # natural order: forward levels along anti-diagonals
    assert levels == (nci + ncj - 1, nci + ncj - 1)


def test_fill_grows_with_level():
    sizes = [library_pattern(12, 10, k)[1].size for k in range(6)]
    assert all(a < b for a, b in zip(sizes, sizes[1:]))


def test_bad_arguments_are_rejected():
    lib = capi.load_library()
    n = C.c_int32(0)
    rp = (C.c_int32 * 64)()
    for args in ((0, 4, 0), (4, 4, -1), (4, 4, 17)):
        assert lib.e2d_ilu_pattern(*args, rp, None, 0, C.byref(n), None) != 0
