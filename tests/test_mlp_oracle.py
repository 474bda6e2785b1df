"""CPU check of the warm-start networks' numpy oracles (oracle/mlp_oracle.py,
oracle/mlp_deep_oracle.py), which the GPU tests use as the checker of the
tensor-core kernels: with the BF16 rounding points switched off, each
oracle's analytic gradient must agree with central finite differences of its
own loss."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_deep_oracle  # noqa: E402
import mlp_oracle  # noqa: E402


def _loss(mod, p, X, T):
    y, _ = mod.forward(p, X)
    return float(np.sum((y - T) ** 2) / X.shape[0])


@pytest.mark.parametrize("mod", [mlp_oracle, mlp_deep_oracle], ids=["shallow", "deep"])
def test_oracle_gradient_matches_finite_differences(mod, monkeypatch):
    monkeypatch.setattr(mod, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(11)
    nf = getattr(mod, "F", getattr(mod, "MF", None))
    n_out = getattr(mod, "O_USED", getattr(mod, "MO_USED", None))
    p = rng.normal(0.0, 0.15, mod.NPARAM)
    X = np.zeros((48, nf))
    X[:, :5] = rng.uniform(-1.0, 1.0, (48, 5))
    T = rng.normal(0.0, 0.5, (48, n_out))
    loss, g = mod.gradient(p, X, T)
    assert abs(loss - _loss(mod, p, X, T)) <= 1e-12 * max(1.0, loss)
    # trained parameters only: the padded outputs' rows carry no gradient
    idx = rng.choice(np.flatnonzero(g != 0.0), 24, replace=False)
    h = 1e-6
    for k in idx:
        e = np.zeros_like(p)
        e[k] = h
        fd = (_loss(mod, p + e, X, T) - _loss(mod, p - e, X, T)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])), (int(k), fd, g[k])
