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
# measured against the field's magnitude, not their own).
RTOL_FP64 = 1e-12
# The other flux functions have more cancellation in their dissipation terms
# (differences of products, then scaled): FMA contraction moves their
# residuals by up to 3.3e-12 (Godunov), 2e-12 (AUSM+, HLLC), 1.7e-12 (Linde)
# on the curvilinear Mach-2 grid.
RTOL_FP64_OTHER_FLUX = 1e-11

# Paths through pow.  CUDA's pow and glibc's pow are both faithfully rounded
# but need not round to the same neighbour (glibc's own pow differs from the
# correctly rounded power in about 5 of 10^4 calls on the arguments these
# paths take), so a case that reaches pow -- the characteristic boundary
# condition, the Godunov and HLLC fluxes -- reproduces the reference up to
# those one-ulp differences and what the steps carry them into (measured
# 1e-15 .. 1.2e-13 after 20 steps); every other case is bit for bit.
RTOL_POW = 1e-12


def reaches_pow(bs):
    if bs.scheme.flux in (cases.FLUX_GODUNOV, cases.FLUX_HLLC):
        return True
    return any(np.any(np.asarray(a) == cases.BC_CHARACTERISTIC) for a in (bs.bc_w, bs.bc_e, bs.bc_s, bs.bc_n))


def rtol_fast(bs):
    return RTOL_FP64 if bs.scheme.flux == cases.FLUX_ROE else RTOL_FP64_OTHER_FLUX


def assert_exact(bs, got, want):
    """Bit for bit, or within RTOL_POW where the case reaches pow."""
    if reaches_pow(bs):
        err = rel_err(got, want)
        assert err <= RTOL_POW, err
    else:
        assert np.array_equal(got, want)


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
    if len(sc) > 5:  # time integration, residual smoothing, limiter freezing
        scheme = cases.Scheme(**{**scheme.__dict__, "time_integration": int(sc[5]), "rs_iterations": int(sc[6]),
                                 "freeze_limiter": int(sc[7]), "rs_epsilon": float(scf[2]),
                                 "freeze_level": float(scf[3])})
    bs = cases.BlockSet(nci, ncj, z["neighbour"], z["bc_w"], z["bc_e"], z["bc_s"], z["bc_n"],
                        z["node_x"], z["node_y"], z["wo_w"], z["wo_e"], z["wo_s"], z["wo_n"],
                        z["W"], scheme, name, ng).contiguous()
    ref = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    return bs, ref, int(z["steps"]), bool(z["lean"]) if "lean" in z.files else False


def rel_err(x, ref, axis_var=1):
    """max over cells of |x - ref| / (|ref| + scale_v).

    scale_v = max(max |ref| of variable v, 1e-3 * max |ref| of all variables):
    a variable whose residual is pure round-off everywhere (e.g. the
    y-momentum residual of a uniform-pressure, v = 0 state, ~1e-14) is measured
    against the residual magnitude of the other variables, not itself."""
    x = np.asarray(x)
    ref = np.asarray(ref)
    red = tuple(a for a in range(ref.ndim) if a != axis_var)
    scale = np.max(np.abs(ref), axis=red, keepdims=True)
    scale = np.maximum(scale, 1e-3 * np.max(np.abs(ref)))
    scale = np.where(scale == 0, 1.0, scale)
    return float(np.max(np.abs(x - ref) / (np.abs(ref) + scale)))
