"""CPU tests: the C restatement (oracle/e2d_oracle.c) against the golden
vectors the compiled CFFC reference produced (tests/golden/make_golden.py).
The restatement must reproduce the reference bit for bit."""
import numpy as np
import pytest

from helpers import fixtures, load

import e2d_oracle


@pytest.mark.parametrize("name", fixtures("residual"))
def test_oracle_residual_bitwise(name):
    bs, ref, _, lean = load(name)
    o = e2d_oracle.Oracle(bs)
    o.set_state()
    dUdt = o.residual()
    if lean:
        assert np.array_equal(bs.interior(dUdt), ref["dUdt"])
        return
    W, _ = o.get_state()
    gx, gy, phi = o.reconstruction()
    assert np.array_equal(W, ref["W"]), "ghost fill differs"
    assert np.array_equal(dUdt, ref["dUdt"])
    # reconstruction is compared where the reference reconstructs (ring 1 and interior)
    g = bs.ng
    sl = (slice(None), slice(None), slice(g - 1, bs.NCj - g + 1), slice(g - 1, bs.NCi - g + 1))
    for a, r in ((gx, ref["dWdx"]), (gy, ref["dWdy"]), (phi, ref["phi"])):
        assert np.array_equal(a[sl], r[sl])


@pytest.mark.parametrize("name", fixtures("explicit"))
def test_oracle_explicit_bitwise(name):
    bs, ref, steps, lean = load(name)
    o = e2d_oracle.Oracle(bs)
    o.set_state()
    rc, hist = o.rk_steps(steps)
    assert rc == int(ref["err"]) == 0
    _, U = o.get_state()
    assert np.array_equal(hist, ref["hist"])
    if lean:
        assert np.array_equal(bs.interior(U), ref["U"])
    else:
        assert np.array_equal(bs.interior(U), bs.interior(ref["U"]))


def test_oracle_negative_density_is_reported():
    """A planted non-physical state makes the update fail the way
    Update_Solution_Multistage_Explicit does (non-zero error return)."""
    from cffc_b200 import cases
    bs = cases.channel(seed=3)
    W = bs.W.copy()
    W[0, 3, 4, 4] = -5.0  # negative pressure in one interior cell
    o = e2d_oracle.Oracle(bs)
    o.set_state(W)
    rc, _ = o.rk_steps(3)
    assert rc > 0
