"""Test infrastructure: a CPU (numpy) restatement of the deep warm-start
network's forward and backward passes -- 5 input features (padded to 16),
four hidden layers of 256 with GELU (tanh form), 4 outputs (padded to 16) --
rounding to BF16 exactly where the tensor-core kernels of
cffc_b200/csrc/e2d_mlp_deep.cu stage an operand (inputs, weights, the hidden
activations and the backward deltas) and keeping FP32/FP64 elsewhere (the
pre-activations, bias gradients summed from the rounded deltas).  It checks
the device gradients; the product never uses it.

Parameter layout (flat, FP32): W1[256][16], b1[256], W2..W4[256][256],
b2..b4[256], W5[16][256], b5[16]; only the first four outputs are trained.

GELU, tanh form: g(z) = z/2 (1 + tanh(c (z + 0.044715 z^3))), c = sqrt(2/pi)."""
from __future__ import annotations

import math

import numpy as np

F, H, O, O_USED, NL = 16, 256, 16, 4, 4
SIZES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)), ("b3", (H,)),
         ("W4", (H, H)), ("b4", (H,)), ("W5", (O, H)), ("b5", (O,))]
NPARAM = sum(int(np.prod(s)) for _, s in SIZES)
C_GELU = math.sqrt(2.0 / math.pi)


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


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(C_GELU * (z + 0.044715 * z ** 3)))


def gelu_prime(z):
    t = np.tanh(C_GELU * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * z * z)


def forward(p, X):
    """X [n][16] -> (y [n][4], intermediates)."""
    w = unpack(p)
    a = bf16(X)
    acts, zs = [a], []
    for layer in range(1, NL + 1):
        z = a @ bf16(w[f"W{layer}"]).T + w[f"b{layer}"]
        zs.append(z)
        a = bf16(gelu(z))
        acts.append(a)
    y = a @ bf16(w["W5"]).T + w["b5"]
    return y[:, :O_USED], (acts, zs, y)


def gradient(p, X, T):
    """(loss, grad) of loss = sum((y - t)^2) / n over the four outputs."""
    w = unpack(p)
    n = X.shape[0]
    _, (acts, zs, y) = forward(p, X)
    e = np.zeros_like(y)
    e[:, :O_USED] = y[:, :O_USED] - T
    loss = float(np.sum(e * e) / n)
    d = bf16(2.0 * e / n)
    g = {}
    g["W5"] = d.T @ acts[NL]
    g["b5"] = d.sum(axis=0)
    wnext = w["W5"]
    for layer in range(NL, 0, -1):
        dz = bf16((d @ bf16(wnext)) * gelu_prime(zs[layer - 1]))
        g[f"W{layer}"] = dz.T @ acts[layer - 1]
        g[f"b{layer}"] = dz.sum(axis=0)
        d, wnext = dz, w[f"W{layer}"]
    g["W5"][O_USED:] = 0.0
    g["b5"][O_USED:] = 0.0
    return loss, pack(g)
