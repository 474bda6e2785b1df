"""CPU tests of the Newton-Krylov host surface: the C structs' layout, the
argument checks of e2d_nks (no device work), and the SER time-step and GMRES
forcing rules checked against the reference's own printed history in the
golden fixtures."""
import ctypes

import numpy as np
import pytest

from cffc_b200 import capi
from helpers import fixtures, load


def test_struct_layouts_match_header():
    # e2d_nks_params: 4 int32 + 6 double + 1 pointer + 2 int32 + 1 pointer;
    # e2d_nks_step: 7 double + 4 int32
    assert ctypes.sizeof(capi.NksParams) == 88
    assert capi.NksParams.l2_reference.offset == 64
    assert capi.NksParams.ilu_level_of_fill.offset == 72
    assert capi.NksParams.cfl_reference.offset == 80
    assert ctypes.sizeof(capi.NksStep) == 72
    assert capi.NksStep.gmres_iters.offset == 56


def test_nks_null_handle_is_rejected():
    lib = capi.load_library()
    p = capi.nks_params(3)
    n = ctypes.c_int(7)
    assert lib.e2d_nks(None, ctypes.byref(p), None, ctypes.byref(n)) == -1
    assert n.value == 0


@pytest.mark.parametrize("name", fixtures("nks"))
def test_fixture_history_follows_ser_rule(name):
    """CFL_n = CFL_0 * max(1, 1/ratio_n) (Finite_Time_Step, NKS2D.h:1316-1340)
    and ratio_n = L2_n / L2_1 in the reference's own output."""
    _, ref, _, _ = load(name)
    newton = ref["newton"]
    cfl0 = ref["params"][3]
    for l2, ratio, cfl in newton:
        assert abs(ratio - l2 / newton[0, 0]) <= 1e-9 * ratio
        assert abs(cfl - cfl0 * max(1.0, 1.0 / ratio)) <= 1e-9 * cfl


@pytest.mark.parametrize("name", fixtures("nks"))
def test_fixture_gmres_counts(name):
    """The printed GMRES lines are consistent: resid = relres * resid0, the
    iteration count never exceeds the cap, and a count below the cap means
    the forcing tolerance (the GMRES tolerance, 1e-5 by default, with the
    initial and final tolerances equal, NKS2D.h:1034-1036) was met."""
    _, ref, _, _ = load(name)
    cap = ref["params"][2]
    tol = float(ref["params"][5]) if len(ref["params"]) > 5 else 1e-5
    for iters, r0, r, rr in ref["gmres"]:
        assert abs(r - rr * r0) <= 1e-8 * r
        assert iters <= cap
        if iters < cap:
            assert rr <= tol
