"""Generates the golden vectors in tests/golden/ by running the compiled CFFC
reference (oracle/_ref/e2d_ref_harness, built by `make -C oracle reference`
from the reference sources) on seeded block sets.

Each fixture is a compressed .npz holding the case's inputs (so the test does
not need to rebuild the case bit for bit) and what the reference computed:

* residual fixtures: W after ghost fill, dUdt, dWdx, dWdy, phi
  (dUdt_Residual_Evaluation, src_2D/Euler2D/Euler2DQuad.cc:814);
* explicit fixtures: final U, last dUdt and the per-step dt/L1/L2/Max history
  of the explicit loop (src_2D/Euler2D/Euler2DQuadSolvers.cc:657-898).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import dataclasses
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cffc_b200 import cases  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "e2d_ref_harness")
OUT = os.path.dirname(os.path.abspath(__file__))


def run_residual(bs):
    with tempfile.TemporaryDirectory() as td:
        cp, op = os.path.join(td, "c.bin"), os.path.join(td, "o.bin")
        cases.write_case(cp, bs)
        subprocess.run([HARNESS, "residual", cp, op], check=True)
        raw = np.fromfile(op, dtype="<f8").reshape(bs.nblk, 5, 4, bs.NCj, bs.NCi)
    return dict(W=raw[:, 0], dUdt=raw[:, 1], dWdx=raw[:, 2], dWdy=raw[:, 3], phi=raw[:, 4])


def run_explicit(bs, nsteps):
    with tempfile.TemporaryDirectory() as td:
        cp, op = os.path.join(td, "c.bin"), os.path.join(td, "o.bin")
        cases.write_case(cp, bs)
        subprocess.run([HARNESS, "explicit", cp, str(nsteps), op], check=True)
        buf = open(op, "rb").read()
    n, err = np.frombuffer(buf[:8], dtype="<i4")
    hist = np.frombuffer(buf[8:8 + 32 * n], dtype="<f8").reshape(n, 4)
    rest = np.frombuffer(buf[8 + 32 * n:], dtype="<f8").reshape(bs.nblk, 2, 4, bs.NCj, bs.NCi)
    return dict(U=rest[:, 0], dUdt=rest[:, 1], hist=hist, err=np.int32(err))


def case_arrays(bs):
    d = {f.name: getattr(bs, f.name) for f in dataclasses.fields(bs)
         if isinstance(getattr(bs, f.name), np.ndarray)}
    sc = bs.scheme
    d["scheme"] = np.array([sc.limiter, sc.flux, sc.n_stage, sc.local_dt, sc.precision], np.int32)
    d["scheme_f"] = np.array([sc.cfl, sc.gamma])
    d["dims"] = np.array([bs.nci, bs.ncj, bs.ng], np.int32)
    return d


def golden_cases():
    """(name, block set, kind, steps) of every fixture."""
    small_box = cases.periodic_box_bumps(nb=2, nc=8, seed=11)
    box = cases.periodic_box_bumps()  # 4x4 blocks of 32x32
    ch = cases.channel()
    ch_char = cases.channel(bc=dict(W=cases.BC_CHARACTERISTIC, E=cases.BC_CHARACTERISTIC,
                                    S=cases.BC_REFLECTION, N=cases.BC_CONSTANT_EXTRAPOLATION),
                            seed=8)
    ch_bj = cases.channel(seed=9, scheme=cases.Scheme(limiter=cases.LIMITER_BARTH_JESPERSEN,
                                                      cfl=0.4, n_stage=2, local_dt=1))
    curv = cases.curvilinear_mach2(nbi=4, nbj=2, nc=16, seed=5)
    return [
        ("residual_box_2x2x8", small_box, "residual", 0),
        ("residual_box_4x4x32", box, "residual", 0),
        ("residual_channel", ch, "residual", 0),
        ("residual_channel_char", ch_char, "residual", 0),
        ("residual_curv_4x2x16", curv, "residual", 0),
        ("explicit_box_4x4x32_200", box, "explicit", 200),
        ("explicit_channel_local_bj_40", ch_bj, "explicit", 40),
        ("explicit_channel_char_40", ch_char, "explicit", 40),
        ("explicit_curv_4x2x16_30", curv, "explicit", 30),
    ]


def main():
    if not os.path.exists(HARNESS):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "reference"], check=True)
    for name, bs, kind, steps in golden_cases():
        out = case_arrays(bs)
        res = run_residual(bs) if kind == "residual" else run_explicit(bs, steps)
        if bs.nblk * bs.nci * bs.ncj > 8192:
            # keep the large fixtures small: the interior of the main output only
            keep = "dUdt" if kind == "residual" else "U"
            res = {k: (bs.interior(v) if k == keep else v) for k, v in res.items()
                   if k in (keep, "hist", "err")}
            out["lean"] = np.int32(1)
        out.update({"ref_" + k: v for k, v in res.items()})
        out["steps"] = np.int32(steps)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main()
