"""Batched handles (e2d_create_batch): several independent cases with uneven
block counts in one handle.  Every case must come out exactly as it does on
a handle of its own — explicit steps and Newton-Krylov solves alike (the
reductions are per block, then per case in block order)."""
import dataclasses

import numpy as np
import pytest

from cffc_b200 import capi, cases

pytestmark = pytest.mark.gpu


def with_scheme(bs, **kw):
    return dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, **kw))


def explicit_cases(precision):
    sc = dict(limiter=cases.LIMITER_VENKATAKRISHNAN, n_stage=2, local_dt=0, cfl=0.5, precision=precision)
    return [with_scheme(cases.periodic_box_bumps(nb=2, nc=16, seed=31), **sc),
            with_scheme(cases.periodic_box_bumps(nb=3, nc=16, seed=32), **sc),
            with_scheme(cases.bump_channel(nbi=4, nbj=2, nci=16, ncj=16), **sc)]


@pytest.mark.parametrize("precision", [2, 0])
def test_batched_explicit_equals_solo(precision):
    cs = explicit_cases(precision)
    hb = capi.BatchHandle(cs)
    hb.set_state()
    rc, hist = hb.rk_steps(25)
    assert rc == 0
    states = hb.get_state()
    hb.close()
    for c, bs in enumerate(cs):
        h = capi.Handle(bs)
        h.set_state()
        rc1, h1 = h.rk_steps(25)
        W1, U1 = h.get_state()
        h.close()
        assert rc1 == 0
        assert np.array_equal(bs.interior(states[c][1]), bs.interior(U1)), c
        assert np.array_equal(hist[:, c, 0], h1[:, 0])          # time-step minima: exact
        np.testing.assert_allclose(hist[:, c, 1:], h1[:, 1:], rtol=1e-12, atol=0)  # atomically summed norms


def nks_cases():
    sc = dict(limiter=cases.LIMITER_ZERO, local_dt=1, precision=0)
    return [with_scheme(cases.bump_channel(nbi=6, nbj=2, nci=16, ncj=16, mach=1.4, h=0.04), **sc),
            with_scheme(cases.bump_channel(nbi=4, nbj=2, nci=16, ncj=16, mach=1.5, h=0.03), **sc),
            with_scheme(cases.bump_channel(nbi=6, nbj=3, nci=16, ncj=16, mach=1.3, h=0.05), **sc)]


@pytest.mark.parametrize("ilu_level", [None, 2])
def test_batched_nks_equals_solo(ilu_level):
    """Block Jacobi and ILU(k) alike: the preconditioner is built and applied
    block by block, so a case's solve is the same in a batch as alone."""
    cs = nks_cases()
    p = capi.nks_params(30, gmres_restart=20, max_gmres=120, overall_tol=1e-10, cfl0=10.0, gmres_tol=0.1,
                        ilu_level=ilu_level)
    hb = capi.BatchHandle(cs)
    hb.set_state()
    rc, hists = hb.nks(p)
    assert rc == 0
    states = hb.get_state()
    hb.close()
    for c, bs in enumerate(cs):
        h = capi.Handle(bs)
        h.set_state()
        rc1, h1 = h.nks(p)
        _, U1 = h.get_state()
        h.close()
        assert rc1 == 0
        assert hists[c] == h1, c
        assert np.array_equal(bs.interior(states[c][1]), bs.interior(U1)), c
    # cases leave the batch at different Newton steps (converged or not)
    assert sum(x[-1]["ratio"] <= 1e-10 for x in hists) >= 1
    assert len({len(x) for x in hists}) > 1


def test_mixed_block_shapes_equal_solo():
    """Cases of different block shapes in one batch run as one sub-batch per
    shape: explicit steps and Newton-Krylov solves give every case what a
    handle of its own gives (state bitwise; explicit norms to 1e-12), with
    histories, norms and states in the order the cases were given."""
    sc = dict(limiter=cases.LIMITER_VENKATAKRISHNAN, n_stage=2, local_dt=0, cfl=0.5, precision=0)
    ex = [with_scheme(cases.periodic_box_bumps(nb=2, nc=16, seed=31), **sc),
          with_scheme(cases.periodic_box_bumps(nb=3, nc=8, seed=32), **sc),
          with_scheme(cases.periodic_box_bumps(nb=2, nc=16, seed=33), **sc)]
    hb = capi.BatchHandle(ex)
    hb.lib.e2d_batch_cases.argtypes = [capi.C.c_void_p]
    assert hb.lib.e2d_batch_cases(hb.h) == 3
    hb.set_state()
    rc, hist = hb.rk_steps(15)
    assert rc == 0
    states = hb.get_state()
    hb.close()
    for c, bs in enumerate(ex):
        h = capi.Handle(bs)
        h.set_state()
        rc1, h1 = h.rk_steps(15)
        _, U1 = h.get_state()
        h.close()
        assert rc1 == 0
        assert np.array_equal(bs.interior(states[c][1]), bs.interior(U1)), c
        assert np.array_equal(hist[:, c, 0], h1[:, 0])
        np.testing.assert_allclose(hist[:, c, 1:], h1[:, 1:], rtol=1e-12, atol=0)
    sn = dict(limiter=cases.LIMITER_ZERO, local_dt=1, precision=0)
    nk = [with_scheme(cases.bump_channel(nbi=6, nbj=2, nci=16, ncj=16, mach=1.4, h=0.04), **sn),
          with_scheme(cases.bump_channel(nbi=4, nbj=2, nci=32, ncj=16, mach=1.5, h=0.03), **sn),
          with_scheme(cases.bump_channel(nbi=4, nbj=2, nci=16, ncj=16, mach=1.3, h=0.05), **sn)]
    p = capi.nks_params(30, gmres_restart=20, max_gmres=120, overall_tol=1e-10, cfl0=10.0, gmres_tol=0.1,
                        ilu_level=2)
    hb = capi.BatchHandle(nk)
    hb.set_state()
    rc, hists = hb.nks(p)
    assert rc == 0
    states = hb.get_state()
    hb.close()
    for c, bs in enumerate(nk):
        h = capi.Handle(bs)
        h.set_state()
        rc1, h1 = h.nks(p)
        _, U1 = h.get_state()
        h.close()
        assert rc1 == 0
        assert hists[c] == h1, c
        assert np.array_equal(bs.interior(states[c][1]), bs.interior(U1)), c


def _sweep_l2(bs, ref, U):
    """Relative L2 difference of density and total energy between a solved
    state and the reference's (every cell, or the fixture's subsample)."""
    got = bs.interior(U)
    if "U_sub" in ref:
        got, want = got[..., ::4, ::4], ref["U_sub"]
    else:
        want = bs.interior(ref["U"])
    return [float(np.sqrt(np.sum((got[:, v] - want[:, v]) ** 2) / np.sum(want[:, v] ** 2))) for v in (0, 3)]


def test_sweep_cases_match_reference_fp64_and_mixed():
    """Three cases of the 512-case supersonic sweep (reference fixtures
    nks_sweep*: the compiled reference's Newton-Krylov with ILU(2) to a 1e-10
    drop) solved together in one batch, first in FP64 throughout, then with
    the FP32 reconstruction and flux down to a 1e-4 drop followed by FP64 to
    1e-10 (the sweep's mixed-precision solve).  Each case's converged state
    must agree with the reference's FP64 answer to 1e-9 (relative L2 of
    density and energy) either way."""
    from helpers import fixtures, load
    names = fixtures("nks_sweep")
    assert len(names) >= 3
    loaded = [load(n) for n in names]
    cs = [with_scheme(bs, precision=0) for bs, _, _, _ in loaded]
    refs = [r for _, r, _, _ in loaded]
    p64 = capi.nks_params(40, gmres_restart=30, max_gmres=200, overall_tol=1e-10, cfl0=10.0, gmres_tol=0.1,
                          ilu_level=2)
    p32 = capi.nks_params(40, gmres_restart=30, max_gmres=200, overall_tol=1e-4, cfl0=10.0, gmres_tol=0.1,
                          ilu_level=2, epsilon0=1e-2)
    hb = capi.BatchHandle(cs)
    hb.set_state()
    rc, h64 = hb.nks(p64)
    assert rc == 0
    s64 = hb.get_state()
    hb.set_state()
    hb.set_precision(1)
    rcA, hA = hb.nks(p32)
    assert rcA == 0
    hb.set_precision(0)
    rcB, hB = hb.nks(p64, [h[0]["l2"] for h in hA])
    assert rcB == 0
    smix = hb.get_state()
    hb.close()
    for c, (bs, ref) in enumerate(zip(cs, refs)):
        assert h64[c][-1]["ratio"] <= 1e-10 and hB[c][-1]["ratio"] <= 1e-10, c
        e64, emix = _sweep_l2(bs, ref, s64[c][1]), _sweep_l2(bs, ref, smix[c][1])
        print(f"{names[c]}: L2 vs reference fp64 {e64[0]:.1e} {e64[1]:.1e}, mixed {emix[0]:.1e} {emix[1]:.1e}")
        assert max(e64) <= 1e-9 and max(emix) <= 1e-9, (names[c], e64, emix)
