"""ctypes binding of the C restatement (oracle/e2d_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  It exposes the same methods as
cffc_b200.capi.Handle so a test can run a case through either.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from cffc_b200 import capi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "libe2d_oracle.so")
HARNESS = os.path.join(HERE, "_ref", "e2d_ref_harness")

_lib = None


def build() -> str:
    """Compiles the restatement (needs only gcc)."""
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        capi.declare(lib, "e2d_oracle_")
        lib.e2d_oracle_create.argtypes = [C.POINTER(capi.BlocksDesc), C.POINTER(capi.SchemeDesc),
                                          C.POINTER(C.c_int)]
        lib.e2d_oracle_create.restype = C.c_void_p
        lib.e2d_oracle_geometry.argtypes = [C.c_void_p] + [C.POINTER(C.c_double)] * 3
        lib.e2d_oracle_geometry.restype = C.c_int
        _lib = lib
    return _lib


class Oracle(capi.Handle):
    prefix = "e2d_oracle_"

    def __init__(self, bs):
        super().__init__(bs, lib=load())

    def _create(self, device):
        err = C.c_int(0)
        h = self.lib.e2d_oracle_create(C.byref(self._desc), C.byref(self._scheme), C.byref(err))
        if not h:
            raise RuntimeError(f"e2d_oracle_create failed ({err.value})")
        return h

    def status(self) -> int:
        return 0

    def geometry(self):
        import numpy as np
        shp = (self.bs.nblk, self.bs.NCj, self.bs.NCi)
        xc, yc, a = np.empty(shp), np.empty(shp), np.empty(shp)
        self.lib.e2d_oracle_geometry(self.h, capi.ptr(xc), capi.ptr(yc), capi.ptr(a))
        return xc, yc, a
