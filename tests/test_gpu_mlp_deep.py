"""The deep warm-start network's tcgen05 kernels (e2d_mlp_deep_*: 5 features
padded to 16 -> 4 x 256 GELU -> 4 outputs) against the numpy oracle
(oracle/mlp_deep_oracle.py, BF16 rounding at the same points as the kernels):

* forward: max |y - y_ref| <= 2e-3 * max |y_ref|;
* gradient: per parameter group ||g - g_ref|| <= 3e-2 ||g_ref||, loss to
  1e-3 relative (FP32 accumulation order and tanhf against tanh can flip an
  occasional BF16 rounding of an activation or delta, and four layers carry
  such flips further than the shallow network's two);
* training on minibatches reduces the loss on a smooth target.
"""
import os
import sys

import numpy as np
import pytest

from cffc_b200 import warmstart

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_deep_oracle as oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def data(n, seed):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 16), np.float32)
    X[:, :5] = rng.standard_normal((n, 5)).astype(np.float32)
    T = (0.5 * np.tanh(X[:, :4] @ rng.standard_normal((4, 4)))).astype(np.float32)
    return X, T


def test_deep_forward_matches_oracle():
    import torch
    net = warmstart.MlpDeep(seed=3)
    p = net.params().astype(np.float64)
    X, _ = data(300, 1)
    Y = net.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    ref, _ = oracle.forward(p, X.astype(np.float64))
    assert np.max(np.abs(Y - ref)) <= 2e-3 * np.max(np.abs(ref))
    net.close()


def test_deep_gradient_matches_oracle():
    import torch
    net = warmstart.MlpDeep(seed=5)
    p = net.params().astype(np.float64)
    X, T = data(333, 2)  # two full tiles of 128 rows and a partial one
    loss, g = net.gradient(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    lref, gref = oracle.gradient(p, X.astype(np.float64), T.astype(np.float64))
    assert abs(loss - lref) <= 1e-3 * lref
    k = 0
    for name, shape in oracle.SIZES:
        n = int(np.prod(shape))
        a, b = g[k:k + n].astype(np.float64), gref[k:k + n]
        if np.linalg.norm(b) > 0:
            assert np.linalg.norm(a - b) <= 3e-2 * np.linalg.norm(b), (name, np.linalg.norm(a - b) / np.linalg.norm(b))
        else:
            assert np.all(a == 0), name
        k += n
    net.close()


def test_deep_training_reduces_loss():
    import torch
    net = warmstart.MlpDeep(seed=7)
    X, T = data(4096, 3)
    hist = net.train(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda(), steps=300, batch=1024, lr=1e-3)
    assert np.all(np.isfinite(hist))
    assert hist[-20:].mean() < 0.2 * hist[:5].mean()
    net.close()
