"""The Newton step's block preconditioner alone (e2d_block_precon_apply
through the C ABI) against the compiled reference's Block_Preconditioner:
Create_Preconditioner, Update_Jacobian_and_Preconditioner and
Apply_Preconditioner (NewtonKrylovSchwarz2D/Block_Preconditioner2D.h:261,
352, 787) with BPKIT's BJacobi or BILUK(k) (bpkit/src/BILUK.cc:55-205), on
seeded vectors (golden fixtures made by tests/golden/make_golden.py).

Tolerance.  The factors are products of 4x4 blocks and exact inverses of
the U diagonal blocks; the device inverts by its own LU with partial
pivoting, the reference by LAPACK dgetrf/dgetri, so inverses differ in
their last bits (scaled by the blocks' condition numbers, up to about 1e4
after normalization here) and the triangular solves carry that through the
rows.  RTOL_PRECON bounds |z - z_ref| / (|z_ref| + max |z_ref| of the
variable) per entry."""
import dataclasses

import numpy as np
import pytest

from cffc_b200 import capi
from helpers import fixtures, load, rel_err

pytestmark = pytest.mark.gpu

RTOL_PRECON = 1e-10
EXACT = 2
FAST = 0


def apply(name, precision=EXACT):
    bs, ref, _, _ = load(name)
    bs = dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=precision))
    cfl, level, _ = ref["params"]
    p = capi.nks_params(1, ilu_level=None if level < 0 else int(level))
    h = capi.Handle(bs)
    h.set_state()
    z = h.block_precon_apply(p, float(cfl), ref["v"])
    W0, _ = h.get_state()
    h.close()
    return bs, ref, z, W0


@pytest.mark.parametrize("name", fixtures("precon"))
def test_precon_matches_reference(name):
    bs, ref, z, _ = apply(name)
    g = bs.ng
    ghost = z.copy()
    ghost[:, g:-g, g:-g, :] = 0.0
    assert not np.any(ghost)  # identity rows on zero ghost entries
    err = rel_err(z, ref["z"], axis_var=3)
    assert err <= RTOL_PRECON, err


def test_precon_fast_path_dt():
    """The fast FP64 path's CFL step feeds the same preconditioner."""
    bs, ref, z, _ = apply("precon_bump_iluk2", FAST)
    assert rel_err(z, ref["z"], axis_var=3) <= 1e-8


def test_precon_is_repeatable_and_leaves_state():
    bs, ref, z1, W1 = apply("precon_bump_iluk4")
    h = capi.Handle(bs)
    h.set_state()
    cfl, level, _ = ref["params"]
    p = capi.nks_params(1, ilu_level=int(level))
    z2 = h.block_precon_apply(p, float(cfl), ref["v"])
    z3 = h.block_precon_apply(p, float(cfl), ref["v"])
    W, _ = h.get_state()
    h.close()
    assert np.array_equal(z1, z2) and np.array_equal(z2, z3)
    assert np.array_equal(bs.interior(W), bs.interior(bs.W))


def test_precon_rejects_unsupported_options():
    bs, ref, _, _ = load("precon_bump_iluk0")
    h = capi.Handle(bs)
    h.set_state()
    v = ref["v"]
    for kw in (dict(ilu_level=17), dict(ilu_level=-2), dict(jacobian_order=2)):
        p = capi.nks_params(1, **{"ilu_level": 0, **kw})
        with pytest.raises(RuntimeError):
            h.block_precon_apply(p, 1.0, v)
    p = capi.nks_params(1, ilu_level=0)
    p.block_preconditioner = 2
    with pytest.raises(RuntimeError):
        h.block_precon_apply(p, 1.0, v)
    h.close()


def test_source_terms_only_jacobian_is_diagonal():
    """Jacobian_Order Source_Terms_Only: -I/dt alone, normalized; ILU(k) of a
    block-diagonal matrix is its block inverse, equal to block Jacobi's."""
    bs, ref, _, _ = load("precon_bump_iluk2")
    out = []
    for level in (None, 3):
        h = capi.Handle(bs)
        h.set_state()
        p = capi.nks_params(1, ilu_level=level, jacobian_order=capi.JACOBIAN_SOURCE_TERMS_ONLY)
        out.append(h.block_precon_apply(p, 10.0, ref["v"]))
        h.close()
    assert np.array_equal(out[0], out[1])
    assert np.any(out[0])
