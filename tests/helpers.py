"""Shared helpers of the test suite: golden fixtures and comparisons."""
from __future__ import annotations

import glob
import os

import numpy as np

from cffc_b200 import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Tolerance of the fast FP64 path (FMA contraction) against the reference:
# per cell, |x - ref| <= RTOL * (|ref| + scale), scale = max |ref| of that
# variable over the block set (so cells where the residual nearly cancels are
# judged against the field's magnitude, not their own).
RTOL_FP64 = 1e-12


def fixtures(kind=None):
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
    return [n for n in names if kind is None or n.startswith(kind)]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    nci, ncj, ng = (int(x) for x in z["dims"])
    sc = z["scheme"]
    scf = z["scheme_f"]
    scheme = cases.Scheme(limiter=int(sc[0]), flux=int(sc[1]), n_stage=int(sc[2]),
                          local_dt=int(sc[3]), precision=int(sc[4]), cfl=float(scf[0]),
                          gamma=float(scf[1]))
    bs = cases.BlockSet(nci, ncj, z["neighbour"], z["bc_w"], z["bc_e"], z["bc_s"], z["bc_n"],
                        z["node_x"], z["node_y"], z["wo_w"], z["wo_e"], z["wo_s"], z["wo_n"],
                        z["W"], scheme, name, ng).contiguous()
    ref = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    return bs, ref, int(z["steps"]), bool(z["lean"]) if "lean" in z.files else False


def rel_err(x, ref, axis_var=1):
    """max over cells of |x - ref| / (|ref| + scale_v).

    scale_v = max(max |ref| of variable v, 1e-3 * max |ref| of all variables):
    a variable whose residual is pure round-off everywhere (e.g. the
    y-momentum residual of a uniform-pressure, v = 0 state, ~1e-14) is judged
    against the residual magnitude of the other variables, not itself."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    red = tuple(a for a in range(ref.ndim) if a != axis_var)
    scale = np.max(np.abs(ref), axis=red, keepdims=True)
    scale = np.maximum(scale, 1e-3 * np.max(np.abs(ref)))
    scale = np.where(scale == 0, 1.0, scale)
    return float(np.max(np.abs(x - ref) / (np.abs(ref) + scale)))
