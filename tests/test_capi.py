"""CPU tests of the C ABI library: it loads, exports every entry point the
public header declares, and rejects invalid descriptions without touching a
GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from cffc_b200 import capi, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "include")


def declared_symbols():
    syms = set()
    for fn in os.listdir(HEADER_DIR):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        syms |= set(re.findall(r"\b(e2d_[a-z0-9_]+)\s*\(", text))
    return sorted(syms)


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("e2d_create", "e2d_destroy", "e2d_set_state", "e2d_residual", "e2d_rk_steps",
              "e2d_norms", "e2d_status"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = capi.load_library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_create_rejects_bad_arguments_before_any_device_work():
    lib = capi.load_library()
    bs = cases.channel()
    d, keep = capi.make_desc(bs)
    sc = capi.make_scheme(bs.scheme)
    err = ctypes.c_int(0)
    d.ng = 3  # only two ghost layers are supported, as in the reference's configs
    assert not lib.e2d_create(ctypes.byref(d), ctypes.byref(sc), 0, ctypes.byref(err))
    assert err.value == -1
    d.ng = 2
    sc.flux = 99
    assert not lib.e2d_create(ctypes.byref(d), ctypes.byref(sc), 0, ctypes.byref(err))
    assert err.value == -1
    sc.flux = cases.FLUX_ROE
    bc = bs.bc_w.copy()
    bc[0, 3] = 1234  # unsupported BC code
    d.bc_w = capi.ptr(bc, ctypes.POINTER(ctypes.c_int32))
    assert not lib.e2d_create(ctypes.byref(d), ctypes.byref(sc), 0, ctypes.byref(err))
    assert err.value == -1
    del keep


def test_null_handle_calls_fail_cleanly():
    lib = capi.load_library()
    assert lib.e2d_set_state(None, None) == -1
    assert lib.e2d_rk_steps(None, 1, None) == -1
    out = np.zeros(3)
    assert lib.e2d_norms(None, capi.ptr(out)) == -1
