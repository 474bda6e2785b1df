"""The warm-start network's tcgen05 kernels against the numpy oracle
(oracle/mlp_oracle.py, BF16 rounding at the same points as the kernels):

* forward: max |y - y_ref| <= 2e-3 * max |y_ref|;
* gradient: per parameter group ||g - g_ref|| <= 2e-2 ||g_ref||, loss to
  1e-4 relative (FP32 accumulation order and tanhf vs tanh can flip an
  occasional BF16 rounding of a hidden activation);
* training reduces the loss on a smooth target;
* end to end: trained on solutions the solver produced, the prediction
  seeds held-out cases that the solver drives to the same residual level
  and the same steady state as from the freestream, in fewer Newton steps.
"""
import os
import sys

import numpy as np
import pytest

from cffc_b200 import capi, cases, warmstart

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle  # noqa: E402

pytestmark = pytest.mark.gpu


def data(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, 16)).astype(np.float32)
    T = (0.5 * np.tanh(X[:, :4] @ rng.standard_normal((4, 4)))).astype(np.float32)
    return X, T


def test_forward_matches_oracle():
    import torch
    net = warmstart.Mlp(seed=3)
    p = net.params().astype(np.float64)
    X, _ = data(300, 1)
    Y = net.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    ref, _ = mlp_oracle.forward(p, X.astype(np.float64))
    assert np.max(np.abs(Y - ref)) <= 2e-3 * np.max(np.abs(ref))


def test_gradient_matches_oracle():
    import torch
    net = warmstart.Mlp(seed=5)
    p = net.params().astype(np.float64)
    X, T = data(333, 2)  # three partial tiles' worth: 2 full + 1 partial
    loss, g = net.gradient(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    lref, gref = mlp_oracle.gradient(p, X.astype(np.float64), T.astype(np.float64))
    assert abs(loss - lref) <= 1e-4 * lref
    k = 0
    for name, shape in mlp_oracle.SIZES:
        n = int(np.prod(shape))
        a, b = g[k:k + n].astype(np.float64), gref[k:k + n]
        if np.linalg.norm(b) > 0:
            assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b), name
        else:
            assert np.all(a == 0), name
        k += n


def test_training_is_deterministic():
    import torch
    X, T = data(20000, 4)
    Xd, Td = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    a = warmstart.Mlp(seed=9)
    b = warmstart.Mlp(seed=9)
    a.train(Xd, Td, 20, 1e-3)
    b.train(Xd, Td, 20, 1e-3)
    assert np.array_equal(a.params(), b.params())


def test_training_reduces_loss():
    import torch
    net = warmstart.Mlp(seed=7)
    X, T = data(4096, 3)
    hist = net.train(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda(), 300, 3e-3)
    assert hist[-1] < 0.1 * hist[0]


def test_warm_start_reaches_same_solution_faster():
    import torch
    p = capi.nks_params(30, gmres_restart=30, max_gmres=150, overall_tol=1e-10, cfl0=10.0, gmres_tol=0.1)
    train = cases.bump_family(10, seed=101, nc=16)
    test = cases.bump_family(3, seed=202, nc=16)
    rc, _, states = warmstart.solve_family(train, p)
    assert rc == 0
    X, T = warmstart.build_training_set(train, states)
    net = warmstart.Mlp(seed=11)
    hist = net.train(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda(), 1500, 2e-3)
    assert hist[-1] < 0.05 * hist[0]
    rc, cold, cold_states = warmstart.solve_family(test, p)
    assert rc == 0
    rc, warm, warm_states, fallback = warmstart.warm_solve(net, test, p)
    assert rc == 0
    for c, bs in enumerate(test):
        assert cold[c][-1]["ratio"] <= 1e-10 and warm[c][-1]["ratio"] <= 1e-10
        # the same steady state
        assert warmstart.l2_cells(bs.interior(warm_states[c][1]), bs.interior(cold_states[c][1])) < 1e-7
    assert sum(len(h) for h in warm) < sum(len(h) for h in cold)
    assert not fallback
