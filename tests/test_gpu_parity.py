"""GPU parity of the CUDA path (through the C ABI) against the compiled
reference's golden vectors and the C restatement.

* precision E2D_PREC_FP64_EXACT: bit-identical to the reference, except
  that a case reaching pow (characteristic BCs, Godunov and HLLC fluxes)
  agrees within helpers.RTOL_POW (one-ulp differences between CUDA's and
  glibc's pow);
* precision E2D_PREC_FP64 (FMA contraction): per cell
  |x - ref| <= 1e-12 * (|ref| + max|ref| of the variable)  (helpers.rel_err),
  1e-11 for the flux functions other than Roe (helpers.rtol_fast).
"""
import dataclasses

import numpy as np
import pytest

from cffc_b200 import capi, cases
from helpers import RTOL_FP64, RTOL_POW, assert_exact, fixtures, load, reaches_pow, rel_err, rtol_fast

import e2d_oracle

pytestmark = pytest.mark.gpu

EXACT = 2
FAST = 0


def with_precision(bs, prec):
    bs2 = dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=prec))
    return bs2


@pytest.mark.parametrize("name", fixtures("residual"))
def test_residual_exact_is_bitwise(name):
    bs, ref, _, lean = load(name)
    h = capi.Handle(with_precision(bs, EXACT))
    h.set_state()
    dUdt = h.residual()
    if lean:
        assert_exact(bs, bs.interior(dUdt), ref["dUdt"])
        return
    W, _ = h.get_state()
    assert_exact(bs, W, ref["W"])
    assert_exact(bs, dUdt, ref["dUdt"])
    gx, gy, phi = h.reconstruction()
    g = bs.ng
    sl = (slice(None), slice(None), slice(g - 1, bs.NCj - g + 1), slice(g - 1, bs.NCi - g + 1))
    assert_exact(bs, gx[sl], ref["dWdx"][sl])
    assert_exact(bs, gy[sl], ref["dWdy"][sl])
    assert_exact(bs, phi[sl], ref["phi"][sl])


@pytest.mark.parametrize("name", fixtures("residual"))
def test_residual_fast_within_tolerance(name):
    bs, ref, _, lean = load(name)
    h = capi.Handle(with_precision(bs, FAST))
    h.set_state()
    dUdt = bs.interior(h.residual())
    r = ref["dUdt"] if lean else bs.interior(ref["dUdt"])
    err = rel_err(dUdt, r)
    assert err <= rtol_fast(bs), err


def per_value_relative(got, ref):
    """Pure relative error |x - ref| / |ref| of every value that is not
    round-off (|ref| >= 1e-8 of its variable's largest |ref|, floored at 1e-3
    of the largest over all variables, as helpers.rel_err), and the ratio
    scale / |ref| of each such value."""
    scale = np.max(np.abs(ref), axis=tuple(a for a in range(ref.ndim) if a != 1), keepdims=True)
    scale = np.maximum(scale, 1e-3 * np.max(np.abs(ref)))
    scale = np.broadcast_to(scale, ref.shape)
    sig = np.abs(ref) >= 1e-8 * scale
    return np.abs(got[sig] - ref[sig]) / np.abs(ref[sig]), scale[sig] / np.abs(ref[sig])


@pytest.mark.parametrize("name", fixtures("residual"))
def test_residual_fast_relative_per_value(name):
    """The fast path's residual read value by value: the pure relative error
    against the reference.  The median is at most 1e-12; a value whose cell's
    fluxes cancel (|ref| small against its variable's scale) carries the
    cancellation, so each value's relative error is at most
    1e-12 (1 + scale / |ref|) (the flux functions other than Roe: 1e-11).
    The statistics (median, largest, count above 1e-12) are printed."""
    bs, ref, _, lean = load(name)
    h = capi.Handle(with_precision(bs, FAST))
    h.set_state()
    dUdt = bs.interior(h.residual())
    r = ref["dUdt"] if lean else bs.interior(ref["dUdt"])
    rel, amp = per_value_relative(dUdt, r)
    print(f"{name}: {rel.size} values, median {np.median(rel):.2e}, max {rel.max():.2e}, "
          f"above 1e-12: {int((rel > 1e-12).sum())}")
    assert np.median(rel) <= 1e-12
    assert np.all(rel <= rtol_fast(bs) * (1.0 + amp))


@pytest.mark.parametrize("name", fixtures("explicit"))
def test_explicit_exact_is_bitwise(name):
    bs, ref, steps, lean = load(name)
    h = capi.Handle(with_precision(bs, EXACT))
    h.set_state()
    rc, hist = h.rk_steps(steps)
    assert rc == 0
    _, U = h.get_state()
    r = ref["U"] if lean else bs.interior(ref["U"])
    assert_exact(bs, bs.interior(U), r)
    # dt history is bitwise; the norms are reductions in another order
    if reaches_pow(bs):
        np.testing.assert_allclose(hist[:, 0], ref["hist"][:, 0], rtol=RTOL_POW)
    else:
        assert np.array_equal(hist[:, 0], ref["hist"][:, 0])
    np.testing.assert_allclose(hist[:, 1:], ref["hist"][:, 1:], rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("name", fixtures("explicit"))
def test_explicit_fast_within_tolerance(name):
    bs, ref, steps, lean = load(name)
    h = capi.Handle(with_precision(bs, FAST))
    h.set_state()
    rc, hist = h.rk_steps(steps)
    assert rc == 0
    _, U = h.get_state()
    r = ref["U"] if lean else bs.interior(ref["U"])
    # state after `steps` RK2 steps: the FMA differences of every step accumulate
    err = rel_err(bs.interior(U), r)
    assert err <= 1e-11, err
    np.testing.assert_allclose(hist[:, 0], ref["hist"][:, 0], rtol=1e-12)


def test_negative_density_reported_like_reference():
    bs = cases.channel(seed=3)
    W = bs.W.copy()
    W[0, 3, 4, 4] = -5.0
    o = e2d_oracle.Oracle(bs)
    o.set_state(W)
    rc_o, _ = o.rk_steps(3)
    h = capi.Handle(with_precision(bs, EXACT))
    h.set_state(W)
    rc_g, _ = h.rk_steps(3)
    assert rc_o > 0 and rc_g > 0
    assert h.status() == rc_g


def test_curvilinear_full_size_residual_matches_oracle():
    """The benchmark block set (256 blocks of 64x64 cells): the exact kernels
    match the C restatement bit for bit over a million cells."""
    bs = cases.curvilinear_mach2()
    o = e2d_oracle.Oracle(bs)
    o.set_state()
    ro = o.residual()
    h = capi.Handle(with_precision(bs, EXACT))
    h.set_state()
    rg = h.residual()
    assert np.array_equal(rg, ro)
    hf = capi.Handle(with_precision(bs, FAST))
    hf.set_state()
    err = rel_err(bs.interior(hf.residual()), bs.interior(ro))
    assert err <= RTOL_FP64, err


def test_curvilinear_full_size_steps_conserve_mass():
    """Size-independent property at full size: with periodic boundaries the
    finite-volume update conserves sum(A * rho) to round-off."""
    bs = cases.curvilinear_mach2()
    o = e2d_oracle.Oracle(bs)
    _, _, area = o.geometry()
    h = capi.Handle(bs)
    h.set_state()
    _, U0 = h.get_state()
    rc, _ = h.rk_steps(20)
    assert rc == 0
    _, U1 = h.get_state()
    m0 = np.sum(bs.interior(area) * bs.interior(U0[:, 0]))
    m1 = np.sum(bs.interior(area) * bs.interior(U1[:, 0]))
    assert abs(m1 - m0) <= 1e-12 * abs(m0), (m0, m1)


@pytest.mark.parametrize("prec", [EXACT, FAST])
def test_curvilinear_full_size_steps_match_oracle(prec):
    """Full-size explicit steps (many CTA waves per stage): the exact kernels
    stay bit-identical to the C restatement, the fast ones within tolerance."""
    bs = with_precision(cases.curvilinear_mach2(), prec)
    o = e2d_oracle.Oracle(bs)
    o.set_state()
    rco, ho = o.rk_steps(3)
    h = capi.Handle(bs)
    h.set_state()
    rcg, hg = h.rk_steps(3)
    assert rco == rcg == 0
    _, Uo = o.get_state()
    _, Ug = h.get_state()
    if prec == EXACT:
        assert np.array_equal(bs.interior(Ug), bs.interior(Uo))
        assert np.array_equal(hg[:, 0], ho[:, 0])
    else:
        err = rel_err(bs.interior(Ug), bs.interior(Uo))
        assert err <= 1e-12, err


def test_full_size_residual_against_reference_digest():
    """The full 1,048,576-cell bench set (cases.curvilinear_mach2()) against
    the compiled reference's own residual, kept as digests
    (tests/golden/digest_residual_curv_256x64.npz): the exact path's interior
    dUdt must hash to the reference's per block (bit-identical), and the fast
    path must meet the per-value bound of the fast residual on the stored
    subsample (every 8th interior cell in i and j)."""
    import hashlib
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "digest_residual_curv_256x64.npz"))
    bs = cases.curvilinear_mach2()
    inputs = hashlib.sha256(np.ascontiguousarray(bs.W).tobytes() + np.ascontiguousarray(bs.node_x).tobytes() +
                            np.ascontiguousarray(bs.node_y).tobytes()).digest()
    assert inputs == z["inputs_sha256"].tobytes(), "the case differs from the one the reference saw"
    sub = int(z["sub"])
    h = capi.Handle(with_precision(bs, EXACT))
    h.set_state()
    inner = np.ascontiguousarray(bs.interior(h.residual()))
    h.close()
    got = np.array([np.frombuffer(hashlib.sha256(inner[b].tobytes()).digest(), np.uint8) for b in range(bs.nblk)])
    bad = [b for b in range(bs.nblk) if not np.array_equal(got[b], z["dUdt_block_sha256"][b])]
    assert not bad, f"{len(bad)} blocks differ from the reference, first {bad[:5]}"
    assert np.array_equal(inner[..., ::sub, ::sub], z["dUdt_sub"])
    h = capi.Handle(with_precision(bs, FAST))
    h.set_state()
    fast = bs.interior(h.residual())[..., ::sub, ::sub]
    h.close()
    rel, amp = per_value_relative(fast, z["dUdt_sub"])
    print(f"1M-cell fast residual on {rel.size} values: median {np.median(rel):.2e}, max {rel.max():.2e}")
    assert np.median(rel) <= 1e-12
    assert np.all(rel <= rtol_fast(bs) * (1.0 + amp))
