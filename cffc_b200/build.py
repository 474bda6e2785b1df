"""Builds libcffc_e2d.so in-tree with nvcc for sm_100a.

Per-file flags matter: the exact FP64 kernels (and the ghost-fill, time-step,
norm and state-conversion kernels every path shares) are compiled with
-fmad=false so they round as the reference's x86-64 build does; the fast
FP64 kernels are compiled with contraction on.  The C++ host layer
(cffc_b200/host, include/cffc_euler2d.hpp) is compiled with the host compiler
and linked into the same library.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcffc_e2d.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
HOST = os.path.join(HERE, "host")
ROOT_DIR = os.path.dirname(HERE)
HOST_SOURCES = ["euler2d_host.cc"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
          "--expt-relaxed-constexpr"]
SOURCES = {
    "e2d_exact.cu": ["-fmad=false"],
    "e2d_fast.cu": ["-fmad=true"],
    "e2d_f32.cu": ["-fmad=true", "-prec-div=false", "-prec-sqrt=false"],
    "e2d_capi.cu": ["-fmad=false"],
    "e2d_noalloc.cu": ["-fmad=false"],
    "e2d_nks.cu": ["-fmad=false"],
    "e2d_mlp.cu": ["-fmad=true"],
    "e2d_mlp_deep.cu": ["-fmad=true"],
}
HEADERS = ["e2d_device.cuh", "e2d_stage.cuh", "e2d_aux.cuh", "e2d_geom.cuh", "e2d_launch.h",
           "e2d_fastmath.cuh", "e2d_handle.h", "e2d_tc.cuh", "e2d_smooth.cuh", "e2d_ilu.cuh",
           "e2d_march.cuh", "e2d_march_args.h", os.path.join("..", "..", "include", "cffc_e2d.h")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in HEADERS]
    objs, cmds = [], []
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if ptxas_info or _newer(o, [s, __file__] + headers):
            cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            if verbose:
                print(" ".join(cmd), flush=True)
            cmds.append(cmd)
    # the translation units compile independently: run them side by side
    # (the marching-kernel units dominate; one process each)
    from concurrent.futures import ThreadPoolExecutor
    workers = max(1, min(len(cmds), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        for r in list(pool.map(lambda c: subprocess.run(c), cmds)):
            if r.returncode != 0:
                raise subprocess.CalledProcessError(r.returncode, r.args)
    # C++ host layer (include/cffc_euler2d.hpp): plain host code, without
    # contraction so the restart files' cell geometry is the reference's
    inc = os.path.join(ROOT_DIR, "include")
    for src in HOST_SOURCES:
        s = os.path.join(HOST, src)
        o = os.path.join(BUILD, src.replace(".cc", ".o"))
        objs.append(o)
        if _newer(o, [s, __file__, os.path.join(inc, "cffc_euler2d.hpp"), os.path.join(inc, "cffc_e2d.h")]):
            cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", inc, "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
