"""Both stage kernels against the reference's golden vectors, whichever
one the handle's autotuner would choose: CFFC_E2D_STAGE_KERNEL=tiled /
march fixes the kernel when a handle is created.  The column-marching kernel
serves blocks of even width (every flux function); other block sets keep
the tiled kernel whatever the setting.

* fast FP64 precision: tolerances as tests/test_gpu_parity.py (residual per
  cell within helpers.rtol_fast and per value within 1e-12 (1 + scale /
  |ref|); explicit runs within 1e-11 with the time-step history to 1e-12);
* exact FP64 precision: each kernel bit-identical to the reference
  (helpers.assert_exact), the reconstruction it exports included.
"""
import dataclasses

import numpy as np
import pytest

from cffc_b200 import capi, cases
from helpers import RTOL_POW, assert_exact, fixtures, load, reaches_pow, rel_err, rtol_fast

pytestmark = pytest.mark.gpu

FAST = 0
EXACT = 2
KERNELS = {"tiled": 0, "march": 1}


def fast_handle(bs, kernel, monkeypatch, precision=FAST):
    monkeypatch.setenv("CFFC_E2D_STAGE_KERNEL", kernel)
    h = capi.Handle(dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=precision)))
    monkeypatch.delenv("CFFC_E2D_STAGE_KERNEL")
    k, _, _ = h.stage_config()
    marchable = bs.nci % 2 == 0
    assert k == (KERNELS[kernel] if marchable else 0), (kernel, k)
    return h


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", fixtures("residual"))
def test_residual_fast_each_kernel(name, kernel, monkeypatch):
    bs, ref, _, lean = load(name)
    h = fast_handle(bs, kernel, monkeypatch)
    h.set_state()
    dUdt = bs.interior(h.residual())
    h.close()
    r = ref["dUdt"] if lean else bs.interior(ref["dUdt"])
    assert rel_err(dUdt, r) <= rtol_fast(bs)
    scale = np.max(np.abs(r), axis=(0, 2, 3), keepdims=True)
    scale = np.broadcast_to(np.maximum(scale, 1e-3 * np.max(np.abs(r))), r.shape)
    sig = np.abs(r) >= 1e-8 * scale
    rel = np.abs(dUdt[sig] - r[sig]) / np.abs(r[sig])
    assert np.all(rel <= rtol_fast(bs) * (1.0 + scale[sig] / np.abs(r[sig])))


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", fixtures("explicit"))
def test_explicit_fast_each_kernel(name, kernel, monkeypatch):
    bs, ref, steps, lean = load(name)
    h = fast_handle(bs, kernel, monkeypatch)
    h.set_state()
    rc, hist = h.rk_steps(steps)
    _, U = h.get_state()
    h.close()
    assert rc == 0
    r = ref["U"] if lean else bs.interior(ref["U"])
    assert rel_err(bs.interior(U), r) <= 1e-11
    np.testing.assert_allclose(hist[:, 0], ref["hist"][:, 0], rtol=1e-12)


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", fixtures("residual"))
def test_residual_exact_each_kernel(name, kernel, monkeypatch):
    bs, ref, _, lean = load(name)
    h = fast_handle(bs, kernel, monkeypatch, EXACT)
    h.set_state()
    dUdt = h.residual()
    if lean:
        h.close()
        assert_exact(bs, bs.interior(dUdt), ref["dUdt"])
        return
    gx, gy, phi = h.reconstruction()
    h.close()
    assert_exact(bs, dUdt, ref["dUdt"])
    g = bs.ng
    sl = (slice(None), slice(None), slice(g - 1, bs.NCj - g + 1), slice(g - 1, bs.NCi - g + 1))
    assert_exact(bs, gx[sl], ref["dWdx"][sl])
    assert_exact(bs, gy[sl], ref["dWdy"][sl])
    assert_exact(bs, phi[sl], ref["phi"][sl])


@pytest.mark.parametrize("kernel", sorted(KERNELS))
@pytest.mark.parametrize("name", fixtures("explicit"))
def test_explicit_exact_each_kernel(name, kernel, monkeypatch):
    bs, ref, steps, lean = load(name)
    h = fast_handle(bs, kernel, monkeypatch, EXACT)
    h.set_state()
    rc, hist = h.rk_steps(steps)
    _, U = h.get_state()
    h.close()
    assert rc == 0
    r = ref["U"] if lean else bs.interior(ref["U"])
    assert_exact(bs, bs.interior(U), r)
    if reaches_pow(bs):
        np.testing.assert_allclose(hist[:, 0], ref["hist"][:, 0], rtol=RTOL_POW)
    else:
        assert np.array_equal(hist[:, 0], ref["hist"][:, 0])


@pytest.mark.parametrize("name", fixtures("residual")[:6])
def test_switch_to_exact_on_a_live_handle(name, monkeypatch):
    """A handle created in the fast precision and switched to the exact one
    (e2d_set_precision) runs the exact build of its stage kernel with the
    exact geometry: bit-identical to the reference; switched back, the fast
    result again."""
    bs, ref, _, lean = load(name)
    h = fast_handle(bs, "march", monkeypatch)
    h.set_state()
    fast = h.residual().copy()
    h.set_precision(EXACT)
    h.set_state()
    dUdt = h.residual()
    h.set_precision(FAST)
    h.set_state()
    again = h.residual()
    h.close()
    r = ref["dUdt"] if lean else bs.interior(ref["dUdt"])
    assert_exact(bs, bs.interior(dUdt), r)
    assert np.array_equal(again, fast)
