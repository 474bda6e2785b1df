"""ctypes binding of the C ABI in ``include/cffc_e2d.h``.

This is the reference-side binding a Python caller of the library uses: the
descriptor structs, the loader for ``libcffc_e2d.so`` (built in-tree next to
this file) and a thin handle class whose methods are the C entry points.
There is no fallback: if the shared library is missing or a CUDA device is
unavailable the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .cases import BlockSet, Scheme

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcffc_e2d.so")

E2D_ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory",
              -4: "NaN/Inf in residual", -5: "GMRES breakdown"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class BlocksDesc(C.Structure):
    _fields_ = [("nblk", C.c_int32), ("nci", C.c_int32), ("ncj", C.c_int32), ("ng", C.c_int32),
                ("neighbour", _ip), ("bc_w", _ip), ("bc_e", _ip), ("bc_s", _ip), ("bc_n", _ip),
                ("node_x", _dp), ("node_y", _dp),
                ("wo_w", _dp), ("wo_e", _dp), ("wo_s", _dp), ("wo_n", _dp)]


class SchemeDesc(C.Structure):
    _fields_ = [("limiter", C.c_int32), ("flux", C.c_int32), ("n_stage", C.c_int32),
                ("local_dt", C.c_int32), ("precision", C.c_int32), ("time_integration", C.c_int32),
                ("rs_iterations", C.c_int32), ("freeze_limiter", C.c_int32),
                ("cfl", C.c_double), ("gamma", C.c_double), ("rs_epsilon", C.c_double),
                ("freeze_level", C.c_double)]


def ptr(a: np.ndarray | None, kind=_dp):
    if a is None:
        return C.cast(None, kind)
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(kind)


def make_desc(bs: BlockSet):
    """Returns (BlocksDesc, keep-alive list)."""
    bs.contiguous()
    keep = [bs.neighbour, bs.bc_w, bs.bc_e, bs.bc_s, bs.bc_n, bs.node_x, bs.node_y,
            bs.wo_w, bs.wo_e, bs.wo_s, bs.wo_n]
    d = BlocksDesc(bs.nblk, bs.nci, bs.ncj, bs.ng,
                   ptr(bs.neighbour, _ip), ptr(bs.bc_w, _ip), ptr(bs.bc_e, _ip),
                   ptr(bs.bc_s, _ip), ptr(bs.bc_n, _ip), ptr(bs.node_x), ptr(bs.node_y),
                   ptr(bs.wo_w), ptr(bs.wo_e), ptr(bs.wo_s), ptr(bs.wo_n))
    return d, keep


def make_scheme(sc: Scheme) -> SchemeDesc:
    s = SchemeDesc()
    s.limiter, s.flux, s.n_stage, s.local_dt, s.precision = (
        sc.limiter, sc.flux, sc.n_stage, sc.local_dt, sc.precision)
    s.time_integration, s.rs_iterations, s.freeze_limiter = (
        sc.time_integration, sc.rs_iterations, sc.freeze_limiter)
    s.cfl, s.gamma, s.rs_epsilon, s.freeze_level = sc.cfl, sc.gamma, sc.rs_epsilon, sc.freeze_level
    return s


class NksParams(C.Structure):
    """e2d_nks_params: the NKS_Input_Parameters fields the solver reads
    (NewtonKrylovSchwarz2D/NKSInput2D.h:125-172 for the defaults)."""
    _fields_ = [("max_newton", C.c_int32), ("gmres_restart", C.c_int32), ("max_gmres", C.c_int32),
                ("block_preconditioner", C.c_int32), ("overall_tol", C.c_double), ("cfl0", C.c_double),
                ("gmres_tol_initial", C.c_double), ("gmres_tol_final", C.c_double),
                ("epsilon0", C.c_double), ("min_ratio", C.c_double),
                ("l2_reference", C.POINTER(C.c_double)), ("ilu_level_of_fill", C.c_int32),
                ("jacobian_order", C.c_int32), ("cfl_reference", C.POINTER(C.c_double))]


PRECON_BLOCK_JACOBI = 0    # GMRES_Block_Preconditioner Diagonal
PRECON_BLOCK_ILUK = 1      # GMRES_Block_Preconditioner ILUK
JACOBIAN_FIRST_ORDER_HLLE = 0
JACOBIAN_SOURCE_TERMS_ONLY = 1


class NksStep(C.Structure):
    """e2d_nks_step: one Newton step of the history."""
    _fields_ = [("l1", C.c_double), ("l2", C.c_double), ("lmax", C.c_double), ("ratio", C.c_double),
                ("cfl", C.c_double), ("gmres_resid0", C.c_double), ("gmres_relres", C.c_double),
                ("gmres_iters", C.c_int32), ("gmres_restarts", C.c_int32), ("gmres_failed", C.c_int32),
                ("pad", C.c_int32)]


def nks_params(max_newton: int, gmres_restart: int = 30, max_gmres: int = 100, overall_tol: float = 1e-5,
               cfl0: float = 1.0, gmres_tol: float = 1e-5, gmres_tol_final: float | None = None,
               epsilon0: float = 1e-6, min_ratio: float = 1e-10, ilu_level: int | None = None,
               jacobian_order: int = 0) -> NksParams:
    """ilu_level None: block Jacobi (the reference's default); k: ILU(k)."""
    p = NksParams()
    p.max_newton, p.gmres_restart, p.max_gmres = max_newton, gmres_restart, max_gmres
    p.block_preconditioner = PRECON_BLOCK_JACOBI if ilu_level is None else PRECON_BLOCK_ILUK
    p.ilu_level_of_fill = 0 if ilu_level is None else ilu_level
    p.jacobian_order = jacobian_order
    p.overall_tol, p.cfl0, p.gmres_tol_initial = overall_tol, cfl0, gmres_tol
    p.gmres_tol_final = gmres_tol if gmres_tol_final is None else gmres_tol_final
    p.epsilon0, p.min_ratio = epsilon0, min_ratio
    return p


def declare(lib, prefix: str) -> None:
    """Argument/return types of the handle API under `prefix` (e2d_ or e2d_oracle_)."""
    vp = C.c_void_p
    sig = {
        "set_state": [vp, _dp], "get_state": [vp, _dp, _dp], "fill_ghosts": [vp],
        "residual": [vp, _dp], "get_reconstruction": [vp, _dp, _dp, _dp],
        "rk_steps": [vp, C.c_int, _dp],
    }
    for name, args in sig.items():
        f = getattr(lib, prefix + name)
        f.argtypes = args
        f.restype = C.c_int
    getattr(lib, prefix + "destroy").argtypes = [vp]
    getattr(lib, prefix + "destroy").restype = None


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libcffc_e2d.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with __graft_entry__.build()")
        lib = C.CDLL(path)
        declare(lib, "e2d_")
        lib.e2d_create.argtypes = [C.POINTER(BlocksDesc), C.POINTER(SchemeDesc), C.c_int,
                                   C.POINTER(C.c_int)]
        lib.e2d_create.restype = C.c_void_p
        for name in ("norms",):
            getattr(lib, "e2d_" + name).argtypes = [C.c_void_p, _dp]
            getattr(lib, "e2d_" + name).restype = C.c_int
        lib.e2d_status.argtypes = [C.c_void_p]
        lib.e2d_status.restype = C.c_int
        lib.e2d_device_state.argtypes = [C.c_void_p, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp)]
        lib.e2d_device_state.restype = C.c_int
        lib.e2d_nks.argtypes = [C.c_void_p, C.POINTER(NksParams), C.POINTER(NksStep), C.POINTER(C.c_int)]
        lib.e2d_nks.restype = C.c_int
        _lib = lib
    return _lib


class Handle:
    """A block set resident on the GPU (one e2d_handle)."""

    prefix = "e2d_"

    def __init__(self, bs: BlockSet, device: int = 0, lib=None):
        self.lib = lib or load_library()
        self.bs = bs
        self._desc, self._keep = make_desc(bs)
        self._scheme = make_scheme(bs.scheme)
        self.h = self._create(device)

    def _create(self, device):
        err = C.c_int(0)
        h = self.lib.e2d_create(C.byref(self._desc), C.byref(self._scheme), device, C.byref(err))
        if not h:
            raise RuntimeError(f"e2d_create failed: {E2D_ERRORS.get(err.value, err.value)}")
        return h

    def _call(self, name, *args):
        rc = getattr(self.lib, self.prefix + name)(self.h, *args)
        if rc < 0:
            raise RuntimeError(f"{self.prefix}{name} failed: {E2D_ERRORS.get(rc, rc)}")
        return rc

    def close(self):
        if getattr(self, "h", None):
            getattr(self.lib, self.prefix + "destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- entry points -----------------------------------------------------
    def set_state(self, W: np.ndarray | None = None) -> None:
        W = np.ascontiguousarray(self.bs.W if W is None else W, dtype=np.float64)
        self._call("set_state", ptr(W))

    def get_state(self):
        W = np.empty(self.bs.cell_shape())
        U = np.empty(self.bs.cell_shape())
        self._call("get_state", ptr(W), ptr(U))
        return W, U

    def fill_ghosts(self) -> None:
        self._call("fill_ghosts")

    def residual(self) -> np.ndarray:
        out = np.empty(self.bs.cell_shape())
        self._call("residual", ptr(out))
        return out

    def reconstruction(self):
        a, b, c = (np.empty(self.bs.cell_shape()) for _ in range(3))
        self._call("get_reconstruction", ptr(a), ptr(b), ptr(c))
        return a, b, c

    def rk_steps(self, n: int, history: bool = True):
        hist = np.zeros((n, 4)) if history else None
        rc = self._call("rk_steps", n, ptr(hist))
        return rc, hist

    def norms(self):
        out = np.zeros(3)
        self._call("norms", ptr(out))
        return out

    def set_precision(self, precision: int) -> None:
        """e2d_set_precision: E2D_PREC_FP64 (0), _FP32 (1) or _FP64_EXACT (2)
        for the calls that follow."""
        self.lib.e2d_set_precision.argtypes = [C.c_void_p, C.c_int]
        self._call("set_precision", precision)

    def stage_config(self):
        """e2d_stage_config: (kernel, rows per chunk, tuned microseconds per
        explicit stage) the autotuner chose for the current precision;
        kernel 0 = tiled, 1 = column-marching."""
        k, r, us = C.c_int(0), C.c_int(0), C.c_double(0.0)
        self.lib.e2d_stage_config.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                              C.POINTER(C.c_double)]
        self._call("stage_config", C.byref(k), C.byref(r), C.byref(us))
        return k.value, r.value, us.value

    def nks(self, params: NksParams):
        """Newton-Krylov steady solve from the resident state.  Returns
        (rc, history) with one dict per Newton step evaluated."""
        steps = (NksStep * max(params.max_newton, 1))()
        n = C.c_int(0)
        rc = self._call("nks", C.byref(params), steps, C.byref(n))
        hist = [{f: getattr(steps[k], f) for f, _ in NksStep._fields_ if f != "pad"} for k in range(n.value)]
        return rc, hist

    def block_precon_apply(self, params: NksParams, cfl: float, v: np.ndarray) -> np.ndarray:
        """e2d_block_precon_apply: z = M^-1 v with the Newton step's
        preconditioner at the current state (dt = cfl x the CFL step); v, z
        in the GMRES layout [nblk][NCj][NCi][4]."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        z = np.zeros_like(v)
        self.lib.e2d_block_precon_apply.argtypes = [C.c_void_p, C.POINTER(NksParams), C.c_double,
                                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
        rc = self.lib.e2d_block_precon_apply(self.h, C.byref(params), cfl, ptr(v), ptr(z))
        if rc != 0:
            raise RuntimeError(f"e2d_block_precon_apply failed: {rc}")
        return z

    def status(self) -> int:
        return self.lib.e2d_status(self.h)


class BatchHandle(Handle):
    """Several independent cases on one handle (e2d_create_batch): their
    blocks end to end in case order; per-case histories and Newton-Krylov
    solves.  The scheme must agree across cases; cases of different block
    shapes run as one sub-batch per shape, and the host arrays are each
    case's array in its own shape, concatenated in case order."""

    def __init__(self, cases: list[BlockSet], device: int = 0, lib=None):
        self.lib = lib or load_library()
        if not cases:
            raise ValueError("no cases")
        self.cases = cases
        self.bs = cases[0]
        descs, self._keep = [], []
        for bs in cases:
            d, k = make_desc(bs)
            descs.append(d)
            self._keep += k
        self._descs = (BlocksDesc * len(cases))(*descs)
        self._scheme = make_scheme(cases[0].scheme)
        self.lib.e2d_create_batch.argtypes = [C.POINTER(BlocksDesc), C.c_int, C.POINTER(SchemeDesc), C.c_int,
                                              C.POINTER(C.c_int)]
        self.lib.e2d_create_batch.restype = C.c_void_p
        err = C.c_int(0)
        self.h = self.lib.e2d_create_batch(self._descs, len(cases), C.byref(self._scheme), device, C.byref(err))
        if not self.h:
            raise RuntimeError(f"e2d_create_batch failed: {E2D_ERRORS.get(err.value, err.value)}")
        self.nblk = sum(bs.nblk for bs in cases)
        self.offsets = np.cumsum([0] + [bs.nblk for bs in cases])
        self._shapes = [(bs.nblk, 4, bs.NCj, bs.NCi) for bs in cases]
        self._sizes = [int(np.prod(sh)) for sh in self._shapes]
        self._flat_off = np.cumsum([0] + self._sizes)

    def split(self, a):
        """Per-case views of a concatenated host array."""
        a = a.ravel()
        return [a[self._flat_off[c]:self._flat_off[c + 1]].reshape(self._shapes[c]) for c in range(len(self.cases))]

    def _flat(self):
        return np.empty(int(self._flat_off[-1]))

    def set_state(self, Ws=None) -> None:
        Ws = [bs.W for bs in self.cases] if Ws is None else Ws
        W = np.ascontiguousarray(np.concatenate([np.asarray(w, dtype=np.float64).ravel() for w in Ws]))
        self._call("set_state", ptr(W))

    def get_state(self):
        W, U = self._flat(), self._flat()
        self._call("get_state", ptr(W), ptr(U))
        return list(zip(self.split(W), self.split(U)))

    def residual(self):
        out = self._flat()
        self._call("residual", ptr(out))
        return self.split(out)

    def rk_steps(self, n: int, history: bool = True):
        hist = np.zeros((n, len(self.cases), 4)) if history else None
        rc = self._call("rk_steps", n, ptr(hist))
        return rc, hist

    def nks(self, params: NksParams, l2_reference=None, cfl_reference=None):
        C_ = len(self.cases)
        ref = cref = None
        if l2_reference is not None:
            ref = np.ascontiguousarray(l2_reference, dtype=np.float64)
            params.l2_reference = ref.ctypes.data_as(C.POINTER(C.c_double))
        if cfl_reference is not None:
            cref = np.ascontiguousarray(cfl_reference, dtype=np.float64)
            params.cfl_reference = cref.ctypes.data_as(C.POINTER(C.c_double))
        m = max(params.max_newton, 1)
        steps = (NksStep * (m * C_))()
        counts = (C.c_int * C_)()
        self.lib.e2d_nks.argtypes = [C.c_void_p, C.POINTER(NksParams), C.POINTER(NksStep), C.POINTER(C.c_int)]
        rc = self._call("nks", C.byref(params), steps, counts)
        hists = [[{f: getattr(steps[c * m + k], f) for f, _ in NksStep._fields_ if f != "pad"}
                  for k in range(counts[c])] for c in range(C_)]
        params.l2_reference = None
        params.cfl_reference = None
        return rc, hists
