"""Learned warm start for batched Newton-Krylov solves of the supersonic
bump-channel family (cases.bump_family).

A per-cell network (e2d_mlp_*, tcgen05 kernels) maps flow parameters and
cell geometry to the converged state, normalised by the freestream; it is
trained on converged solutions the solver itself produced.  Its prediction
seeds e2d_set_state; the solver then drives each case to the same absolute
residual level as a run from the freestream (the ratio is taken against the
case's freestream residual), so the answer is still the solver's.

Features (16 per cell): Mach and bump height (centred, scaled), x, the
wall-normal coordinate y_rel = (y - y_w(x)) / (1 - y_w(x)), y_w / 0.05, the
bump's normalised slope, sin/cos(k pi x / 1.5) for k = 1..3, sin/cos(pi
y_rel), x times the scaled Mach, and the scaled height times x.
Outputs: rho/rho_inf - 1, u/u_inf - 1, v/u_inf, p/p_inf - 1.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import capi, cases

NF = 16
NOUT = 4


def _declare(lib):
    vp = C.c_void_p
    lib.e2d_mlp_create.argtypes = [C.c_uint64, C.POINTER(C.c_int)]
    lib.e2d_mlp_create.restype = vp
    lib.e2d_mlp_destroy.argtypes = [vp]
    lib.e2d_mlp_destroy.restype = None
    lib.e2d_mlp_nparams.argtypes = []
    lib.e2d_mlp_nparams.restype = C.c_int
    lib.e2d_mlp_params.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.e2d_mlp_forward.argtypes = [vp, vp, C.c_int, vp, vp]
    lib.e2d_mlp_gradient.argtypes = [vp, vp, vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_double), vp]
    lib.e2d_mlp_train.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_float, C.POINTER(C.c_float), vp]
    for f in ("e2d_mlp_params", "e2d_mlp_forward", "e2d_mlp_gradient", "e2d_mlp_train"):
        getattr(lib, f).restype = C.c_int


class Mlp:
    """The warm-start network (device parameters).  X, T, Y are torch CUDA
    float32 tensors."""

    def __init__(self, seed: int = 1, lib=None):
        self.lib = lib or capi.load_library()
        _declare(self.lib)
        err = C.c_int(0)
        self.m = self.lib.e2d_mlp_create(seed, C.byref(err))
        if not self.m:
            raise RuntimeError(f"e2d_mlp_create failed: {err.value}")
        self.nparam = self.lib.e2d_mlp_nparams()

    def close(self):
        if getattr(self, "m", None):
            self.lib.e2d_mlp_destroy(self.m)
            self.m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self, new=None):
        out = np.zeros(self.nparam, np.float32)
        pin = None
        if new is not None:
            new = np.ascontiguousarray(new, dtype=np.float32)
            pin = new.ctypes.data_as(C.POINTER(C.c_float))
        rc = self.lib.e2d_mlp_params(self.m, out.ctypes.data_as(C.POINTER(C.c_float)), pin)
        if rc:
            raise RuntimeError(f"e2d_mlp_params: {rc}")
        return out

    def forward(self, X):
        import torch
        Y = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device=X.device)
        rc = self.lib.e2d_mlp_forward(self.m, X.data_ptr(), X.shape[0], Y.data_ptr(), None)
        if rc:
            raise RuntimeError(f"e2d_mlp_forward: {rc}")
        return Y

    def gradient(self, X, T):
        g = np.zeros(self.nparam, np.float32)
        loss = C.c_double(0.0)
        rc = self.lib.e2d_mlp_gradient(self.m, X.data_ptr(), T.data_ptr(), X.shape[0],
                                       g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss), None)
        if rc:
            raise RuntimeError(f"e2d_mlp_gradient: {rc}")
        return loss.value, g

    def train(self, X, T, steps: int, lr: float):
        hist = np.zeros(max(steps, 1), np.float32)
        rc = self.lib.e2d_mlp_train(self.m, X.data_ptr(), T.data_ptr(), X.shape[0], steps, lr,
                                    hist.ctypes.data_as(C.POINTER(C.c_float)), None)
        if rc:
            raise RuntimeError(f"e2d_mlp_train: {rc}")
        return hist[:steps]


NF_DEEP = 16  # the deep network's input width: 5 features, padded


def _declare_deep(lib):
    vp = C.c_void_p
    lib.e2d_mlp_deep_create.argtypes = [C.c_uint64, C.POINTER(C.c_int)]
    lib.e2d_mlp_deep_create.restype = vp
    lib.e2d_mlp_deep_destroy.argtypes = [vp]
    lib.e2d_mlp_deep_destroy.restype = None
    lib.e2d_mlp_deep_nparams.argtypes = []
    lib.e2d_mlp_deep_nparams.restype = C.c_int
    lib.e2d_mlp_deep_params.argtypes = [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]
    lib.e2d_mlp_deep_forward.argtypes = [vp, vp, C.c_int, vp, vp]
    lib.e2d_mlp_deep_gradient.argtypes = [vp, vp, vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_double), vp]
    lib.e2d_mlp_deep_train.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                       C.POINTER(C.c_float), vp]
    for f in ("e2d_mlp_deep_params", "e2d_mlp_deep_forward", "e2d_mlp_deep_gradient", "e2d_mlp_deep_train"):
        getattr(lib, f).restype = C.c_int


class MlpDeep:
    """The deep warm-start network (e2d_mlp_deep_*): 5 features (h, Mach,
    x, y, wall distance; padded to 16) -> 4 hidden layers of 256 (GELU) ->
    (rho, u, v, p) normalised.  X, T, Y are torch CUDA float32 tensors."""

    def __init__(self, seed: int = 1, lib=None):
        self.lib = lib or capi.load_library()
        _declare_deep(self.lib)
        err = C.c_int(0)
        self.m = self.lib.e2d_mlp_deep_create(seed, C.byref(err))
        if not self.m:
            raise RuntimeError(f"e2d_mlp_deep_create failed: {err.value}")
        self.nparam = self.lib.e2d_mlp_deep_nparams()

    def close(self):
        if getattr(self, "m", None):
            self.lib.e2d_mlp_deep_destroy(self.m)
            self.m = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self, new=None):
        out = np.zeros(self.nparam, np.float32)
        pin = None
        if new is not None:
            new = np.ascontiguousarray(new, dtype=np.float32)
            pin = new.ctypes.data_as(C.POINTER(C.c_float))
        rc = self.lib.e2d_mlp_deep_params(self.m, out.ctypes.data_as(C.POINTER(C.c_float)), pin)
        if rc:
            raise RuntimeError(f"e2d_mlp_deep_params: {rc}")
        return out

    def forward(self, X):
        import torch
        Y = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device=X.device)
        rc = self.lib.e2d_mlp_deep_forward(self.m, X.data_ptr(), X.shape[0], Y.data_ptr(), None)
        if rc:
            raise RuntimeError(f"e2d_mlp_deep_forward: {rc}")
        return Y

    def gradient(self, X, T):
        g = np.zeros(self.nparam, np.float32)
        loss = C.c_double(0.0)
        rc = self.lib.e2d_mlp_deep_gradient(self.m, X.data_ptr(), T.data_ptr(), X.shape[0],
                                            g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss), None)
        if rc:
            raise RuntimeError(f"e2d_mlp_deep_gradient: {rc}")
        return loss.value, g

    def train(self, X, T, steps: int, batch: int, lr: float, seed: int = 7):
        hist = np.zeros(max(steps, 1), np.float32)
        rc = self.lib.e2d_mlp_deep_train(self.m, X.data_ptr(), T.data_ptr(), X.shape[0], steps, batch, lr, seed,
                                         hist.ctypes.data_as(C.POINTER(C.c_float)), None)
        if rc:
            raise RuntimeError(f"e2d_mlp_deep_train: {rc}")
        return hist[:steps]


def case_params(bs):
    """(Mach, bump height) of a bump_family case from its name."""
    parts = bs.name.split("_")
    return float(parts[1][1:]), float(parts[2][1:])


def features(bs, mach: float, height: float):
    """[nblk * ncj * nci, 16] float32 features of the interior cells, in the
    block / j / i order of the cell arrays."""
    g = bs.ng
    X, Y = bs.node_x, bs.node_y
    xc = 0.25 * (X[:, :-1, :-1] + X[:, :-1, 1:] + X[:, 1:, 1:] + X[:, 1:, :-1])[:, g:g + bs.ncj, g:g + bs.nci]
    yc = 0.25 * (Y[:, :-1, :-1] + Y[:, :-1, 1:] + Y[:, 1:, 1:] + Y[:, 1:, :-1])[:, g:g + bs.ncj, g:g + bs.nci]
    x, y = xc.ravel(), yc.ravel()
    inb = np.abs(x) <= 0.5
    yw = np.where(inb, height * np.sin(np.pi * (x + 0.5)) ** 2, 0.0)
    slope = np.where(inb, np.sin(2.0 * np.pi * (x + 0.5)), 0.0)
    yr = (y - yw) / (1.0 - yw)
    mn = (mach - 1.475) / 0.125
    hn = (height - 0.0325) / 0.0125
    xs = x / 1.5
    cols = [np.full_like(x, mn), np.full_like(x, hn), xs, yr, yw / 0.05, slope]
    for k in (1, 2, 3):
        cols += [np.sin(k * np.pi * xs), np.cos(k * np.pi * xs)]
    cols += [np.sin(np.pi * yr), np.cos(np.pi * yr), xs * mn, hn * xs]
    return np.stack(cols, axis=1).astype(np.float32)


def features_deep(bs, mach: float, height: float):
    """[cells, 16] float32 inputs of the deep network, the five quantities of
    the sweep's learned start -- bump height, Mach number, cell-centre x and
    y, and the distance to the nearer wall (the bump below, y = 1 above) --
    scaled to O(1), then zeros to the network's 16 input columns."""
    g = bs.ng
    X, Y = bs.node_x, bs.node_y
    xc = 0.25 * (X[:, :-1, :-1] + X[:, :-1, 1:] + X[:, 1:, 1:] + X[:, 1:, :-1])[:, g:g + bs.ncj, g:g + bs.nci]
    yc = 0.25 * (Y[:, :-1, :-1] + Y[:, :-1, 1:] + Y[:, 1:, 1:] + Y[:, 1:, :-1])[:, g:g + bs.ncj, g:g + bs.nci]
    x, y = xc.ravel(), yc.ravel()
    yw = np.where(np.abs(x) <= 0.5, height * np.sin(np.pi * (x + 0.5)) ** 2, 0.0)
    dwall = np.minimum(y - yw, 1.0 - y)
    out = np.zeros((x.size, NF_DEEP), np.float32)
    out[:, 0] = (height - 0.0325) / 0.0125
    out[:, 1] = (mach - 1.475) / 0.125
    out[:, 2] = x / 1.5
    out[:, 3] = 2.0 * y - 1.0
    out[:, 4] = 4.0 * dwall
    return out


def freestream(bs):
    """(rho, u, v, p) of the case's freestream (its West reference state)."""
    return bs.wo_w[0, :, 0]


def targets(bs, W):
    """Normalised converged state [cells, 4] from a cell array W."""
    r0, u0, _, p0 = freestream(bs)
    g = bs.ng
    w = W[:, :, g:g + bs.ncj, g:g + bs.nci].transpose(0, 2, 3, 1).reshape(-1, 4)
    return np.stack([w[:, 0] / r0 - 1.0, w[:, 1] / u0 - 1.0, w[:, 2] / u0, w[:, 3] / p0 - 1.0],
                    axis=1).astype(np.float32)


def state_from(bs, out):
    """Cell array W (ghosts at the freestream) from predicted outputs."""
    r0, u0, v0, p0 = freestream(bs)
    W = np.empty(bs.cell_shape())
    W[:, 0], W[:, 1], W[:, 2], W[:, 3] = r0, u0, v0, p0
    o = out.reshape(bs.nblk, bs.ncj, bs.nci, 4)
    g = bs.ng
    W[:, 0, g:g + bs.ncj, g:g + bs.nci] = r0 * (1.0 + o[..., 0])
    W[:, 1, g:g + bs.ncj, g:g + bs.nci] = u0 * (1.0 + o[..., 1])
    W[:, 2, g:g + bs.ncj, g:g + bs.nci] = u0 * o[..., 2]
    W[:, 3, g:g + bs.ncj, g:g + bs.nci] = p0 * (1.0 + o[..., 3])
    return W


def solve_family(fam, params, Ws=None, l2_ref=None, device=0, handle=None):
    """Batched Newton-Krylov solve of a list of cases from Ws (or the
    freestream); l2_ref: per-case reference L2 for the tolerance and CFL
    ratio (None: each case's first residual).  Uses `handle` (a BatchHandle
    of fam) when given.  Returns (rc, hists, states)."""
    hb = handle or capi.BatchHandle(fam, device=device)
    hb.set_state(Ws)
    rc, hists = hb.nks(params, l2_ref)
    states = hb.get_state()
    if handle is None:
        hb.close()
    return rc, hists, states


def freestream_l2(fam, device=0, handle=None):
    """Density-residual L2 of each case at its freestream state (on `handle`,
    a BatchHandle of fam, when given)."""
    hb = handle or capi.BatchHandle(fam, device=device)
    hb.set_state()
    hb.residual()
    out = np.zeros(3 * len(fam))
    hb.lib.e2d_norms.argtypes = [C.c_void_p, capi._dp]
    rc = hb.lib.e2d_norms(hb.h, capi.ptr(out))
    if handle is None:
        hb.close()
    if rc:
        raise RuntimeError(f"e2d_norms: {rc}")
    return out.reshape(-1, 3)[:, 1]


def feature_fn(net):
    """The input features a network was trained on."""
    return features_deep if isinstance(net, MlpDeep) else features


def build_training_set(fam, states, feat=features):
    Xs, Ts = [], []
    for bs, (W, _) in zip(fam, states):
        m, h = case_params(bs)
        Xs.append(feat(bs, m, h))
        Ts.append(targets(bs, W))
    return np.concatenate(Xs), np.concatenate(Ts)


def predict_states(net, fam):
    import torch
    feat = feature_fn(net)
    Ws = []
    for bs in fam:
        m, h = case_params(bs)
        X = torch.from_numpy(feat(bs, m, h)).cuda()
        Ws.append(state_from(bs, net.forward(X).cpu().numpy().astype(np.float64)))
    return Ws


def current_l2(fam, handle):
    """Density-residual L2 of each case at the handle's current state."""
    handle.residual()
    out = np.zeros(3 * len(fam))
    handle.lib.e2d_norms.argtypes = [C.c_void_p, capi._dp]
    rc = handle.lib.e2d_norms(handle.h, capi.ptr(out))
    if rc:
        raise RuntimeError(f"e2d_norms: {rc}")
    return out.reshape(-1, 3)[:, 1]


def l2_cells(a, b):
    return float(math.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def warm_solve(net, fam, params, smooth_steps: int = 150, device=0, handle=None, own_cfl: bool = False):
    """The warm-started batched solve: freestream residuals (the reference
    level), the network's prediction, smooth_steps explicit local-time-step
    RK steps that damp its high-frequency error, then Newton-Krylov to the
    cold start's absolute residual level.  A case the warm start does not
    bring to the tolerance is solved again from the freestream (the plain
    method is the fallback), so every answer meets the tolerance.  Uses
    `handle` (a BatchHandle of fam) when given.  Returns (rc, hists, states,
    fallback case indices).  own_cfl: the pseudo-time step grows from the
    warm state's own residual (cfl_reference) rather than the freestream's,
    so the first Newton steps are not taken at the huge CFL the small ratio
    to the freestream residual would give."""
    hb = handle or capi.BatchHandle(fam, device=device)
    l2 = freestream_l2(fam, handle=hb)
    hb.set_state(predict_states(net, fam))
    rc, hists, states = 0, [], []
    if smooth_steps:
        rc, _ = hb.rk_steps(smooth_steps, history=False)
    if rc == 0:
        cref = current_l2(fam, hb) if own_cfl else None
        rc, hists = hb.nks(params, l2, cref)
        states = hb.get_state()
    if handle is None:
        hb.close()
    if rc:
        return rc, hists, states, []
    tol = params.overall_tol
    bad = [c for c, h in enumerate(hists) if not (h and h[-1]["ratio"] <= tol)]
    if bad:
        sub = [fam[c] for c in bad]
        rc, h2, s2 = solve_family(sub, params, device=device)
        for k, c in enumerate(bad):
            hists[c] = hists[c] + h2[k]
            states[c] = s2[k]
    return rc, hists, states, bad


def solve_in_batches(fam, params, device=0, per_batch=256):
    """Cold batched solves of a list of cases, per_batch cases a handle.
    Returns (rc, hists, states)."""
    hists, states = [], []
    for k in range(0, len(fam), per_batch):
        rc, h, st = solve_family(fam[k:k + per_batch], params, device=device)
        if rc:
            return rc, hists, states
        hists += h
        states += st
    return 0, hists, states


def train_network_deep(train_fam, params, steps=((1e-3, 2000), (3e-4, 1500), (1e-4, 500)), batch=8192, seed=11,
                       device=0, per_batch=256, row_stride=1):
    """Solves the training cases (batched, per_batch cases a handle, from the
    freestream), builds the per-cell training set of the deep network
    (features_deep; every row_stride-th cell of each case, so that large
    training families stay within host memory; each batch's states are
    dropped once its rows are taken) and trains it on minibatches.  Returns
    (net, info)."""
    import time

    import torch
    t0 = time.perf_counter()
    Xs, Ts, hists = [], [], []
    for k in range(0, len(train_fam), per_batch):
        sub = train_fam[k:k + per_batch]
        rc, h, states = solve_family(sub, params, device=device)
        if rc:
            raise RuntimeError(f"training-set solve failed: {rc}")
        X, T = build_training_set(sub, states, features_deep)
        Xs.append(X[::row_stride])
        Ts.append(T[::row_stride])
        hists += h
        del states
    t_solve = time.perf_counter() - t0
    X, T = np.concatenate(Xs), np.concatenate(Ts)
    del Xs, Ts
    Xd, Td = torch.from_numpy(X).cuda(device), torch.from_numpy(T).cuda(device)
    net = MlpDeep(seed=seed)
    t0 = time.perf_counter()
    losses = []
    for k, (lr, n) in enumerate(steps):
        losses.append(net.train(Xd, Td, n, batch, lr, seed=seed + k))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    loss = np.concatenate(losses)
    return net, {"network": "5 features -> 4 x 256 GELU -> 4 (BF16 tcgen05, FP32 accumulation)",
                 "cases": len(train_fam), "cells": int(X.shape[0]), "solve_seconds": round(t_solve, 3),
                 "train_seconds": round(t_train, 3), "adam_steps": int(loss.size), "batch_rows": batch,
                 "loss_first": float(loss[0]), "loss_last": float(np.mean(loss[-20:])),
                 "converged": int(sum(h[-1]["ratio"] <= params.overall_tol for h in hists))}


def train_network(train_fam, params, steps=((3e-3, 1500), (1e-3, 1500), (3e-4, 1000)), seed=11, device=0):
    """Solves the training cases (batched, from the freestream), builds the
    per-cell training set from their converged states and trains a network
    on it.  Returns (net, info)."""
    import time

    import torch
    t0 = time.perf_counter()
    rc, hists, states = solve_family(train_fam, params, device=device)
    t_solve = time.perf_counter() - t0
    if rc:
        raise RuntimeError(f"training-set solve failed: {rc}")
    X, T = build_training_set(train_fam, states)
    Xd, Td = torch.from_numpy(X).cuda(device), torch.from_numpy(T).cuda(device)
    net = Mlp(seed=seed)
    t0 = time.perf_counter()
    losses = []
    for lr, n in steps:
        losses.append(net.train(Xd, Td, n, lr))
    t_train = time.perf_counter() - t0
    loss = np.concatenate(losses)
    return net, {"cases": len(train_fam), "cells": int(X.shape[0]), "solve_seconds": round(t_solve, 3),
                 "train_seconds": round(t_train, 3), "adam_steps": int(loss.size),
                 "loss_first": float(loss[0]), "loss_last": float(loss[-1]),
                 "converged": int(sum(h[-1]["ratio"] <= params.overall_tol for h in hists))}
