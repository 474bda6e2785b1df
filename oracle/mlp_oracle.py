"""Test infrastructure: a CPU (numpy) restatement of the warm-start network's
forward and backward passes, rounding to BF16 exactly where the tensor-core
kernels stage an operand in shared memory (inputs, weights, the hidden
activations, and the backward deltas), with FP32/FP64 arithmetic elsewhere.
It checks the gradients of cffc_b200/csrc/e2d_mlp.cu; the product never
uses it.

Parameter layout (flat): W1[128][16], b1[128], W2[128][128], b2[128],
W3[16][128], b3[16]; only the first four outputs are trained."""
from __future__ import annotations

import numpy as np

MF, MH, MO, MO_USED = 16, 128, 16, 4
SIZES = [("W1", (MH, MF)), ("b1", (MH,)), ("W2", (MH, MH)), ("b2", (MH,)), ("W3", (MO, MH)), ("b3", (MO,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(p):
    out, k = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[k:k + n], dtype=np.float64).reshape(shape)
        k += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SIZES])


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, X):
    w = unpack(p)
    x = bf16(X)
    h1 = np.tanh(x @ bf16(w["W1"]).T + w["b1"])
    h1b = bf16(h1)
    h2 = np.tanh(h1b @ bf16(w["W2"]).T + w["b2"])
    h2b = bf16(h2)
    y = h2b @ bf16(w["W3"]).T + w["b3"]
    return y[:, :MO_USED], (x, h1b, h2b, y)


def gradient(p, X, T):
    """(loss, grad) of loss = sum((y - t)^2) / n over the four outputs."""
    w = unpack(p)
    n = X.shape[0]
    _, (x, h1b, h2b, y) = forward(p, X)
    e = np.zeros_like(y)
    e[:, :MO_USED] = y[:, :MO_USED] - T
    loss = float(np.sum(e * e) / n)
    dy = 2.0 * e / n
    dyb = bf16(dy)
    g = {k: np.zeros(s) for k, s in SIZES}
    g["W3"] = (h2b.T @ dyb).T
    g["b3"] = dy.sum(axis=0)
    dz2 = (dyb @ bf16(w["W3"])) * (1.0 - h2b * h2b)
    dz2b = bf16(dz2)
    g["W2"] = dz2b.T @ h1b
    g["b2"] = dz2.sum(axis=0)
    dz1 = (dz2b @ bf16(w["W2"])) * (1.0 - h1b * h1b)
    g["W1"] = bf16(dz1).T @ x
    g["b1"] = dz1.sum(axis=0)
    g["W3"][MO_USED:] = 0.0
    g["b3"][MO_USED:] = 0.0
    return loss, pack(g)
