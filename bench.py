"""Benchmark of the Euler2D explicit path on B200.

Workload (one bench "step"): the curvilinear Mach-2 case — 256 blocks of
64x64 cells (1,048,576 cells, [0,4]x[0,1], seeded sinusoidal node
displacement, 5% seeded density perturbation, periodic) advanced by 500
explicit RK2 time steps (Roe flux, least-squares reconstruction,
Venkatakrishnan limiter, CFL 0.5, global time step), FP64.
Metric: Mcell-updates/s (interior cells x time steps / second).

  value     device time (CUDA events) with the state resident in HBM
  e2e       the same through the C ABI from pinned host memory: upload W,
            500 steps, download U, every bench step
  roofline  the fused stage kernel: algorithmic bytes per launch (80 B/cell
            for RK stage 1, 112 B/cell for stage 2) / mean launch time,
            against the measured HBM copy bandwidth
  cpu_baseline  the compiled CFFC reference (oracle/_ref) on the host cores

With --gpus N (torchrun) every rank runs its own replica (the path's blocks
live on one GPU; independent cases are the unit of scale-out): weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

RK_STEPS = 500


PRECISION = {"fp64": 0, "fp32": 1, "exact": 2}  # E2D_PREC_*


def fp32_error(bs, nsteps, device):
    """Relative L2 error of density and total energy after nsteps of the FP32
    reconstruction/flux path against the FP64 path, same initial state."""
    import dataclasses

    import numpy as np

    from cffc_b200 import capi
    out = {}
    for prec in (0, 1):
        b2 = dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=prec))
        h = capi.Handle(b2, device=device)
        h.set_state()
        rc, _ = h.rk_steps(nsteps, history=False)
        assert rc == 0, rc
        out[prec] = bs.interior(h.get_state()[1])
        h.close()
    err = {}
    for name, v in (("density", 0), ("energy", 3)):
        ref, x = out[0][:, v], out[1][:, v]
        err[name] = float(np.sqrt(np.sum((x - ref) ** 2) / np.sum(ref ** 2)))
    return err


def fp32_leg(bs, rk_steps, device, steps=3):
    """The FP32 reconstruction/flux path on the bench workload: its
    throughput (device time over `steps` calls of rk_steps RK2 steps) and the
    density / total-energy L2 error against the FP64 path after rk_steps."""
    import dataclasses

    import torch

    from cffc_b200 import capi
    b32 = dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=PRECISION["fp32"]))
    h = capi.Handle(b32, device=device)
    h.set_state()
    rc, _ = h.rk_steps(rk_steps, history=False)
    assert rc == 0, rc
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        rc, _ = h.rk_steps(rk_steps, history=False)
        assert rc == 0, rc
    secs = (time.perf_counter() - t0) / steps
    h.close()
    return {"value": round(bs.n_interior * rk_steps / secs * 1e-6, 3), "unit": "Mcell-updates/s",
            "timing": "host clock around e2d_rk_steps (returns after the device finished)",
            "l2_error_vs_fp64": dict(fp32_error(bs, rk_steps, device), steps=rk_steps)}


def exact_leg(bs, rk_steps, device, steps=2):
    """The exact FP64 path (the reference's arithmetic, bit-identical to its
    residual and explicit steps: tests/test_gpu_parity.py,
    tests/test_gpu_kernels.py) on the bench workload: throughput over `steps`
    calls of rk_steps RK2 steps, the stage kernel its handle runs and that
    kernel's mean CUDA-event time per launch."""
    import dataclasses

    import numpy as np
    import torch

    from cffc_b200 import capi
    bx = dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=PRECISION["exact"]))
    h = capi.Handle(bx, device=device)
    h.set_state()
    rc, _ = h.rk_steps(rk_steps, history=False)
    assert rc == 0, rc
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        rc, _ = h.rk_steps(rk_steps, history=False)
        assert rc == 0, rc
    secs = (time.perf_counter() - t0) / steps
    kt = np.zeros(6)
    h.lib.e2d_kernel_times.argtypes = [capi.C.c_void_p, capi.C.c_int, capi._dp]
    assert h.lib.e2d_kernel_times(h.h, 10, capi.ptr(kt)) == 0
    kind, rows, _ = h.stage_config()
    h.close()
    hbm, peak_kind = peaks()
    achieved = bs.n_interior * 0.5 * (80 + 112) / (0.5 * (kt[1] + kt[2]) * 1e-3) / 1e9
    return {"value": round(bs.n_interior * rk_steps / secs * 1e-6, 3), "unit": "Mcell-updates/s",
            "timing": "host clock around e2d_rk_steps (returns after the device finished)",
            "stage_kernel": f"march_kernel, {rows} rows per chunk" if kind == 1 else "stage_kernel (tiled)",
            "stage_ms": [round(kt[1], 5), round(kt[2], 5)],
            "roofline": {"achieved": round(achieved, 2), "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4)}}


def parity_leg(bs, device):
    """Per-cell relative error of the fast FP64 residual (the benchmarked
    kernels) against the exact FP64 path, which reproduces the reference's
    residual bit for bit (tests/test_gpu_parity.py), on the bench workload."""
    import dataclasses

    import numpy as np

    from cffc_b200 import capi
    out = {}
    # the state after 20 exact RK2 steps: the initial state has v = 0 and a
    # uniform pressure, where the y-momentum residual is round-off only
    h = capi.Handle(dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=PRECISION["exact"])),
                    device=device)
    h.set_state()
    rc, _ = h.rk_steps(20, history=False)
    assert rc == 0, rc
    W, _ = h.get_state()
    h.close()
    for prec in (PRECISION["exact"], PRECISION["fp64"]):
        h = capi.Handle(dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=prec)), device=device)
        h.set_state(W)
        out[prec] = bs.interior(h.residual())
        h.close()
    ref, got = out[PRECISION["exact"]], out[PRECISION["fp64"]]
    # per variable: the largest |dUdt| (at least 1e-3 of the largest over all
    # variables, as tests/helpers.py rel_err); a value below 1e-8 of it is the
    # round-off left where the fluxes of a cell cancel, whose own relative
    # error says nothing about the kernel
    scale = np.max(np.abs(ref), axis=(0, 2, 3), keepdims=True)
    scale = np.maximum(scale, 1e-3 * np.max(np.abs(ref)))
    sig = np.abs(ref) >= 1e-8 * scale
    rel = np.abs(got[sig] - ref[sig]) / np.abs(ref[sig])
    scaled = np.abs(got - ref) / (np.abs(ref) + scale)
    l2 = np.sqrt(np.sum((got - ref) ** 2, axis=(0, 2, 3)) / np.sum(ref ** 2, axis=(0, 2, 3)))
    # a variable none of whose values is significant is round-off everywhere
    # (the y-momentum here: the density perturbation of a uniform-pressure,
    # v = 0 stream is a contact wave, which keeps p uniform and v = 0)
    l2 = [float(x) if sig[:, v].any() else None for v, x in enumerate(l2)]
    return {"quantity": "dUdt per cell and variable, fast FP64 vs exact FP64 (= the reference), "
                        "on the state after 20 RK2 steps",
            "values": int(ref.size), "values_above_1e-8_of_variable_max": int(sig.sum()),
            "max_rel_err": float(rel.max()), "p99_rel_err": float(np.quantile(rel, 0.99)),
            "median_rel_err": float(np.median(rel)),
            "above_1e-12_rel": int((rel > 1e-12).sum()), "above_1e-10_rel": int((rel > 1e-10).sum()),
            "max_scaled_err": float(scaled.max()),
            "rel_l2_per_variable": l2,
            "rel_l2_note": "null: the variable's residual is round-off in every cell (y-momentum of this state)"}


C2_FIXTURES = {None: "nks_c2_bump_12x4x64x32_bj", 4: "nks_c2_bump_12x4x64x32_iluk4"}


def nks_c2_measure(precision, device, cpu):
    """The 98,304-cell subsonic bump channel (12 x 4 blocks of 64 x 32, bump
    height 0.1, Mach 0.5) from the freestream, as the reference's fixtures
    run it: block Jacobi for 40 Newton steps (GMRES(30), at most 60
    iterations) and ILU(4) for 12.  Seconds per Newton step on the device,
    the history next to the reference's (from the committed fixtures), and
    the compiled reference's seconds per Newton step on one host core (two
    steps)."""
    import numpy as np

    from cffc_b200 import capi, cases
    out = {"workload": "subsonic bump channel, 12 x 4 blocks x 64x32 (98,304 cells), h 0.1, Mach 0.5, "
                       "freestream start, tolerance 1e-10"}
    for level, fx in C2_FIXTURES.items():
        path = os.path.join(ROOT, "tests", "golden", fx + ".npz")
        if not os.path.exists(path):
            continue
        z = np.load(path)
        par = z["ref_params"]
        max_newton, restart, max_gmres, cfl0, tol = par[:5]
        gtol = float(par[5]) if len(par) > 5 else 1e-5
        bs = cases.bump_channel()
        bs.scheme.precision = precision
        p = capi.nks_params(int(max_newton), gmres_restart=int(restart), max_gmres=int(max_gmres),
                            overall_tol=float(tol), cfl0=float(cfl0), gmres_tol=gtol, ilu_level=level)
        h = capi.Handle(bs, device=device)
        h.set_state()
        h.nks(capi.nks_params(1, gmres_restart=int(restart), max_gmres=5, ilu_level=level))  # warm-up
        t0 = time.perf_counter()
        h.set_state()
        rc, hist = h.nks(p)
        secs = time.perf_counter() - t0
        h.close()
        ref_ratio = z["ref_newton"][:, 1]
        n = min(len(hist), len(ref_ratio))
        dev = [abs(hist[k]["ratio"] - ref_ratio[k]) / ref_ratio[k] for k in range(n)]
        leg = {"preconditioner": "block Jacobi" if level is None else f"ILU({level})",
               "newton_steps": len(hist), "seconds": round(secs, 4),
               "seconds_per_newton_step": round(secs / max(1, len(hist)), 5),
               "gmres_iterations": int(sum(st["gmres_iters"] for st in hist)),
               "converged": bool(rc == 0 and hist and hist[-1]["ratio"] <= float(tol)),
               "final_ratio": hist[-1]["ratio"] if hist else None,
               "reference_final_ratio": float(z["ref_final"][2]),
               "ratio_history": [round(st["ratio"], 6) for st in hist],
               "max_rel_dev_ratio_vs_reference": float(max(dev)) if dev else None,
               "gmres_counts_equal_to_reference": int(sum(hist[k]["gmres_iters"] == int(z["ref_gmres"][k, 0])
                                                          for k in range(n)))}
        harness = os.path.join(ROOT, "oracle", "_ref", "e2d_ref_harness")
        if cpu and os.path.exists(harness):
            with tempfile.TemporaryDirectory() as td:
                cp, op = os.path.join(td, "c.bin"), os.path.join(td, "o.bin")
                cases.write_case(cp, bs)
                extra = [] if level is None else ["ILUK", str(level)]
                r = subprocess.run([harness, "nks", cp, op, "2", str(int(restart)), str(int(max_gmres)),
                                    str(float(cfl0)), str(float(tol)), str(gtol)] + extra,
                                   capture_output=True, text=True)
                try:
                    ref_s = float(r.stderr.strip().split(",")[-1].split()[0])
                    leg["cpu_reference"] = {"seconds_per_newton_step": round(ref_s / 2, 3), "cores": 1,
                                            "kind": "reference", "sample": "2 Newton steps"}
                except (ValueError, IndexError):
                    pass
        out["iluk4" if level else "block_jacobi"] = leg
    return out


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="fp64", choices=["fp64", "exact", "fp32"])
    p.add_argument("--rk-steps", type=int, default=RK_STEPS)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-nks", action="store_true", help="skip the Newton-Krylov s-to-steady measurement")
    p.add_argument("--sweep-cases", type=int, default=512, help="cases of the batched Newton-Krylov sweep")
    return p.parse_args(argv)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.rows = []
        self.stop = threading.Event()
        self.th = threading.Thread(target=self.run, daemon=True)

    def run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.th.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.th.join(timeout=10)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_reference_run(bs, nsteps, threads):
    """Times the compiled reference's explicit loop (oracle/_ref harness)."""
    from cffc_b200 import cases
    harness = os.path.join(ROOT, "oracle", "_ref", "e2d_ref_harness")
    if not os.path.exists(harness):
        return None
    with tempfile.TemporaryDirectory() as td:
        cp = os.path.join(td, "case.bin")
        cases.write_case(cp, bs)
        out = subprocess.run([harness, "time", cp, str(nsteps), str(threads)], capture_output=True,
                             text=True, check=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def cpu_port_run(bs, nsteps):
    """Fallback when the compiled reference is absent: the C restatement."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import e2d_oracle
    o = e2d_oracle.Oracle(bs)
    o.set_state()
    t0 = time.perf_counter()
    rc, _ = o.rk_steps(nsteps)
    s = time.perf_counter() - t0
    return {"seconds": s, "steps": nsteps, "cells": bs.n_interior, "threads": 1,
            "mcell_updates_per_s": bs.n_interior * nsteps / s * 1e-6, "error": rc}


CPU_DETAIL = {
    "reference": "the compiled reference's own per-block routines (BCs, dUdt_Multistage_Explicit, "
                 "Update_Solution_Multistage_Explicit, CFL, norms) on {n} pthreads over blocks, with a "
                 "restated same-resolution exchange; the reference itself runs one thread per process",
    "port": "the C restatement of the path (oracle/e2d_oracle.c) on one thread",
}


def cpu_baseline(bs, nsteps=12):
    threads = os.cpu_count() or 1
    r = cpu_reference_run(bs, nsteps, threads)
    kind = "reference"
    if r is None:
        r = cpu_port_run(bs, max(2, nsteps // 4))
        kind = "port"
    sample = (f"{r['steps']} RK2 steps of the same 1,048,576-cell block set "
              f"({r['cells'] * r['steps'] / 1e6:.1f} M cell-updates, {r['seconds']:.1f} s)")
    return {"value": round(r["mcell_updates_per_s"], 4), "unit": "Mcell-updates/s",
            "cores": r["threads"], "kind": kind, "detail": CPU_DETAIL[kind].format(n=r["threads"]),
            "sample": sample}


NKS_PARAMS = dict(max_newton=40, gmres_restart=30, max_gmres=200, overall_tol=1e-10, cfl0=10.0,
                  gmres_tol=0.1)


def nks_workload():
    """Steady supersonic (Mach 1.4) flow over a 4 % sin^2 bump, first order
    (limiter zero), local time stepping: 6 x 2 blocks of 32 x 32 cells.  The
    reference's block-Jacobi Newton-Krylov converges this case to a 1e-10
    L2 drop (it stalls on the subsonic bump and on larger grids)."""
    from cffc_b200 import cases
    return cases.bump_channel(nbi=6, nbj=2, nci=32, ncj=32, mach=1.4, h=0.04,
                              scheme=cases.Scheme(limiter=cases.LIMITER_ZERO, local_dt=1))


def nks_measure(precision, device, cpu, ilu_level=None):
    """Seconds to a 1e-10 L2 density drop: the device solve end to end (host
    W in, Newton loop with its per-iteration host round trips), and the
    compiled reference's Newton_Krylov_Schwarz_Solver on one host core, both
    with block Jacobi (ilu_level None) or ILU(ilu_level)."""
    from cffc_b200 import capi
    bs = nks_workload()
    bs.scheme.precision = precision
    p = capi.nks_params(**NKS_PARAMS, ilu_level=ilu_level)
    h = capi.Handle(bs, device=device)
    h.set_state()
    h.nks(capi.nks_params(2, gmres_restart=30, max_gmres=20, ilu_level=ilu_level))  # warm-up: allocation, first launches
    t0 = time.perf_counter()
    h.set_state()
    rc, hist = h.nks(p)
    secs = time.perf_counter() - t0
    h.close()
    iters = sum(st["gmres_iters"] for st in hist)
    out = {"workload": "supersonic bump, 6 x 2 blocks x 32x32 (12,288 cells), first order, "
                       "GMRES(30) tol 0.1, CFL0 10, " + ("block-Jacobi" if ilu_level is None else
                                                         "ILU(%d)" % ilu_level),
           "tolerance": NKS_PARAMS["overall_tol"], "seconds_to_steady": round(secs, 4),
           "converged": bool(rc == 0 and hist and hist[-1]["ratio"] <= NKS_PARAMS["overall_tol"]),
           "newton_steps": len(hist) - 1, "gmres_iterations": iters,
           "residual_evaluations": len(hist) + iters + sum(st["gmres_restarts"] for st in hist),
           "final_ratio": hist[-1]["ratio"] if hist else None}
    harness = os.path.join(ROOT, "oracle", "_ref", "e2d_ref_harness")
    if cpu and os.path.exists(harness):
        from cffc_b200 import cases
        with tempfile.TemporaryDirectory() as td:
            cp, op = os.path.join(td, "c.bin"), os.path.join(td, "o.bin")
            cases.write_case(cp, bs)
            a = NKS_PARAMS
            extra = [] if ilu_level is None else ["ILUK", str(ilu_level)]
            r = subprocess.run([harness, "nks", cp, op, str(a["max_newton"]), str(a["gmres_restart"]),
                                str(a["max_gmres"]), str(a["cfl0"]), str(a["overall_tol"]), str(a["gmres_tol"])]
                               + extra, capture_output=True, text=True)
            secs_ref = float(r.stderr.strip().split(",")[-1].split()[0])
            end = [l for l in r.stdout.split("\n") if "End of Newton Steps" in l]
            out["cpu_reference"] = {"seconds_to_steady": round(secs_ref, 3), "cores": 1, "kind": "reference",
                                    "summary": end[0].strip() if end else None}
    return out


def nks_batch_measure(precision, device, n_cases=16, ilu_level=None):
    """A sweep of steady cases (cases.bump_family: Mach, bump height and
    block layout drawn per case, 8-48 blocks of 32x32 cells) solved to a
    1e-10 drop as one batched handle, and one after another on single-case
    handles (the plain GPU path), from the freestream; block Jacobi
    (ilu_level None) or ILU(ilu_level)."""
    from cffc_b200 import capi, cases
    fam = cases.bump_family(n_cases, precision=precision)
    p = capi.nks_params(**NKS_PARAMS, ilu_level=ilu_level)
    # handles (device allocation) are made before the clock starts; each
    # timed solve uploads the freestream state and runs to convergence
    hb = capi.BatchHandle(fam, device=device)
    solo = [capi.Handle(bs, device=device) for bs in fam]
    hb.set_state()
    hb.nks(capi.nks_params(1, gmres_restart=30, max_gmres=5, ilu_level=ilu_level))  # warm-up: work arrays
    t0 = time.perf_counter()
    hb.set_state()
    rc, hists = hb.nks(p)
    t_batch = time.perf_counter() - t0
    hb.close()
    for h in solo:
        h.set_state()
        h.nks(capi.nks_params(1, gmres_restart=30, max_gmres=5, ilu_level=ilu_level))
    t0 = time.perf_counter()
    solo_ok = 0
    for h in solo:
        h.set_state()
        rc1, h1 = h.nks(p)
        solo_ok += int(rc1 == 0 and h1[-1]["ratio"] <= NKS_PARAMS["overall_tol"])
    t_solo = time.perf_counter() - t0
    for h in solo:
        h.close()
    conv = sum(int(x and x[-1]["ratio"] <= NKS_PARAMS["overall_tol"]) for x in hists)
    return {"workload": f"{n_cases} supersonic bump cases (cases.bump_family, 8-48 blocks of 32x32, "
                        f"{sum(b.n_interior for b in fam)} cells in all), first order, to a 1e-10 drop, "
                        + ("block-Jacobi" if ilu_level is None else "ILU(%d)" % ilu_level),
            "batched_seconds": round(t_batch, 3), "sequential_seconds": round(t_solo, 3),
            "speedup": round(t_solo / t_batch, 2), "converged": conv, "converged_sequential": solo_ok,
            "newton_steps": [len(x) - 1 for x in hists],
            "gmres_iterations": sum(st["gmres_iters"] for x in hists for st in x)}


def nks_sweep_measure(device, n_cases=512, ilu_level=2, fp32_tol=1e-4, fp32_eps0=1e-2):
    """The batched sweep: n_cases supersonic bump-channel cases
    (cases.bump_family, 8 to 96 blocks of 32 x 32 cells, Mach and bump height
    drawn per case) solved to a 1e-10 drop as ONE batch on one handle, with
    ILU(ilu_level).  Mixed precision: Newton-Krylov with the FP32
    reconstruction and flux down to a fp32_tol drop (near the single-precision
    floor of the residual), then FP64 on the same state to 1e-10
    (e2d_set_precision), the ratio still taken against the freestream
    residual.  The FP32 phase's Frechet derivatives use a larger perturbation
    (epsilon0 = fp32_eps0): single-precision round-off in the residual
    difference divided by the default 1e-6 would swamp the product.
    Compared with the same batch solved in FP64 throughout: time, and the
    per-case relative L2 difference of density and total energy between the
    two converged states."""
    import numpy as np

    from cffc_b200 import capi, cases
    fam = cases.bump_family(n_cases, layouts=cases.LAYOUTS_8_96)
    cells = sum(b.n_interior for b in fam)
    tol = NKS_PARAMS["overall_tol"]
    p64 = capi.nks_params(**NKS_PARAMS, ilu_level=ilu_level)
    p32 = capi.nks_params(**dict(NKS_PARAMS, overall_tol=fp32_tol), epsilon0=fp32_eps0, ilu_level=ilu_level)
    hb = capi.BatchHandle(fam, device=device)
    tiles = {}
    for prec, name in ((PRECISION["fp64"], "fp64"), (PRECISION["fp32"], "fp32")):
        hb.set_precision(prec)
        k, r, us = hb.stage_config()
        tiles[name] = {"kernel": "column-marching" if k == 1 else "tiled", "rows_per_chunk": r,
                       "tuned_us_per_explicit_stage": round(us, 1)}
    hb.set_precision(PRECISION["fp64"])
    hb.set_state()
    hb.nks(capi.nks_params(1, gmres_restart=30, max_gmres=5, ilu_level=ilu_level))  # warm-up
    t0 = time.perf_counter()
    hb.set_state()
    rc64, h64 = hb.nks(p64)
    t64 = time.perf_counter() - t0
    s64 = hb.get_state()
    t0 = time.perf_counter()
    hb.set_state()
    hb.set_precision(PRECISION["fp32"])
    rcA, hA = hb.nks(p32)
    l2ref = [h[0]["l2"] for h in hA]
    hb.set_precision(PRECISION["fp64"])
    rcB, hB = hb.nks(p64, l2ref)
    tmix = time.perf_counter() - t0
    smix = hb.get_state()
    hb.close()
    err_d, err_e = [], []
    for bs, a, b in zip(fam, smix, s64):
        ua, ub = bs.interior(a[1]), bs.interior(b[1])
        err_d.append(float(np.sqrt(np.sum((ua[:, 0] - ub[:, 0]) ** 2) / np.sum(ub[:, 0] ** 2))))
        err_e.append(float(np.sqrt(np.sum((ua[:, 3] - ub[:, 3]) ** 2) / np.sum(ub[:, 3] ** 2))))
    ok64 = [bool(x) and x[-1]["ratio"] <= tol for x in h64]
    okmix = [bool(x) and x[-1]["ratio"] <= tol for x in hB]
    conv64, convmix = sum(ok64), sum(okmix)
    both = [c for c in range(n_cases) if ok64[c] and okmix[c]]

    def unconverged(hs, ok):
        return [{"case": c, "blocks": fam[c].nblk, "newton_steps": len(hs[c]),
                 "final_ratio": hs[c][-1]["ratio"] if hs[c] else None} for c in range(n_cases) if not ok[c]]
    return {"workload": f"{n_cases} supersonic bump cases (cases.bump_family, 8-96 blocks of 32x32, "
                        f"{cells} cells in all), first order, ILU({ilu_level}), to a 1e-10 drop, one batch",
            "cases": n_cases, "cells": cells, "stage_kernel": tiles,
            "fp64": {"seconds": round(t64, 3), "cases_per_s": round(n_cases / t64, 2), "converged": conv64,
                     "newton_steps": int(sum(len(x) - 1 for x in h64)), "rc": rc64},
            "fp32_then_fp64": {"seconds": round(tmix, 3), "cases_per_s": round(n_cases / tmix, 2),
                               "converged": convmix, "fp32_tol": fp32_tol,
                               "newton_steps_fp32": int(sum(len(x) for x in hA)),
                               "newton_steps_fp64": int(sum(len(x) - 1 for x in hB)), "rc": [rcA, rcB]},
            "speedup_mixed_vs_fp64": round(t64 / tmix, 3),
            "unconverged_fp64": unconverged(h64, ok64), "unconverged_fp32_then_fp64": unconverged(hB, okmix),
            "l2_vs_fp64_over": f"{len(both)} cases converged both ways",
            "max_l2_density_vs_fp64": max(err_d[c] for c in both) if both else None,
            "max_l2_energy_vs_fp64": max(err_e[c] for c in both) if both else None,
            "median_l2_density_vs_fp64": float(np.median([err_d[c] for c in both])) if both else None,
            "l2_vs_reference": sweep_vs_reference(fam, s64, smix)}


def sweep_vs_reference(fam, s64, smix):
    """Per-case relative L2 (density, total energy) of the sweep's converged
    states, FP64 and mixed, against the compiled reference's FP64
    Newton-Krylov answers for the cases with a committed fixture
    (tests/golden/nks_sweep*: ILU(2) to 1e-10; large cases keep every 4th
    interior cell)."""
    import glob

    import numpy as np
    out = {}
    for path in sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "nks_sweep*.npz"))):
        z = np.load(path)
        k = int(z["sweep_index"])
        if k >= len(fam):
            continue
        bs = fam[k]
        want = z["ref_U_sub"] if "ref_U_sub" in z.files else bs.interior(z["ref_U"])
        sub = np.s_[..., ::4, ::4] if "ref_U_sub" in z.files else np.s_[...]
        row = {}
        for name, st in (("fp64", s64), ("fp32_then_fp64", smix)):
            got = bs.interior(st[k][1])[sub]
            row[name] = [float(np.sqrt(np.sum((got[:, v] - want[:, v]) ** 2) / np.sum(want[:, v] ** 2)))
                         for v in (0, 3)]
        out[f"case{k}_{bs.nblk}blocks"] = row
    return out


def nks_learned_measure(device, n_train=256, n_test=32, per_batch=256, n_sample=64, row_stride=1):
    """Learned + batched against plain, on the sweep family (8-96 blocks of
    32 x 32, seeded Mach and bump height): the deep network (5 features ->
    4 x 256 GELU -> 4, trained by the library's tcgen05 kernels on the
    converged states of n_train solved cases, every row_stride-th cell)
    seeds n_test held-out cases; seconds to the same absolute residual level
    (1e-10 of each case's freestream residual) for the warm-started batches
    and the cold batches (per_batch cases a handle), and the plain GPU path
    (cold single-case solves one after another) on the first n_sample test
    cases, with the block-Jacobi preconditioner (the reference's default)
    and with ILU(2); and the relative L2 difference of the warm answers
    against the exact-precision path's cold solve (the reference's FP64
    arithmetic) on those n_sample cases.  With n_test > n_sample the
    sequential time of all cases is the sample's per-case time times n_test
    (reported as such)."""
    from cffc_b200 import capi, cases, warmstart
    tol = NKS_PARAMS["overall_tol"]
    train = cases.bump_family(n_train, seed=101, layouts=cases.LAYOUTS_8_96)
    test = cases.bump_family(n_test, seed=202, layouts=cases.LAYOUTS_8_96)
    net, info = warmstart.train_network_deep(train, capi.nks_params(**NKS_PARAMS, ilu_level=2), device=device,
                                             per_batch=per_batch, row_stride=row_stride)
    n_sample = min(n_sample, n_test)
    out = {"workload": f"{n_test} held-out cases of the sweep family (seed 202, 8-96 blocks of 32x32), "
                       f"network trained on {n_train} (seed 101), to the cold start's residual level",
           "training": dict(info, row_stride=row_stride)}
    sample = test[:n_sample]
    exact = [dataclasses_replace_precision(bs, PRECISION["exact"]) for bs in sample]
    for name, ilu in (("block_jacobi", None), ("iluk2", 2)):
        p = capi.nks_params(**NKS_PARAMS, ilu_level=ilu)
        warm_p = capi.nks_params(1, gmres_restart=30, max_gmres=5, ilu_level=ilu)
        t_cold = t_warm = 0.0
        cold, warm, warm_states, fallback, rcs = [], [], [], [], [0, 0]
        for k in range(0, n_test, per_batch):
            sub = test[k:k + per_batch]
            hb = capi.BatchHandle(sub, device=device)
            hb.set_state()
            hb.nks(warm_p)  # warm-up
            t0 = time.perf_counter()
            rc_c, c_h, _ = warmstart.solve_family(sub, p, handle=hb)
            t_cold += time.perf_counter() - t0
            t0 = time.perf_counter()
            rc_w, w_h, w_s, fb = warmstart.warm_solve(net, sub, p, handle=hb)
            t_warm += time.perf_counter() - t0
            hb.close()
            cold += c_h
            warm += w_h
            warm_states += w_s[:max(0, n_sample - k)]
            fallback += [k + c for c in fb]
            rcs = [rcs[0] or rc_w, rcs[1] or rc_c]
        solo = [capi.Handle(bs, device=device) for bs in sample]
        for h in solo:
            h.set_state()
            h.nks(warm_p)
        t0 = time.perf_counter()
        for h in solo:
            h.set_state()
            h.nks(p)
        t_seq_sample = time.perf_counter() - t0
        for h in solo:
            h.close()
        t_seq = t_seq_sample * n_test / n_sample
        # the exact-precision cold solve: the reference's arithmetic
        rc_x, _, exact_states = warmstart.solve_family(exact, p, device=device)
        err_x = max(warmstart.l2_cells(bs.interior(a[1]), bs.interior(b[1]))
                    for bs, a, b in zip(sample, warm_states, exact_states))
        out[name] = {"warm_batched_seconds": round(t_warm, 3), "cold_batched_seconds": round(t_cold, 3),
                     "cold_sequential_seconds": round(t_seq, 3),
                     "cold_sequential_measured_on": f"{n_sample} cases ({round(t_seq_sample, 3)} s)",
                     "speedup_vs_plain_sequential": round(t_seq / t_warm, 2),
                     "speedup_vs_cold_batched": round(t_cold / t_warm, 2),
                     "newton_steps_warm": int(sum(len(x) - 1 for x in warm)),
                     "newton_steps_cold": int(sum(len(x) - 1 for x in cold)),
                     "gmres_iterations_warm": int(sum(st["gmres_iters"] for x in warm for st in x)),
                     "gmres_iterations_cold": int(sum(st["gmres_iters"] for x in cold for st in x)),
                     "converged_warm": int(sum(x[-1]["ratio"] <= tol for x in warm)),
                     "converged_cold": int(sum(x[-1]["ratio"] <= tol for x in cold)),
                     "fallback_cases": len(fallback), "rc": rcs + [rc_x],
                     "max_l2_error_warm_vs_exact_cold": float(err_x),
                     "l2_error_measured_on": f"{n_sample} cases"}
    net.close()
    return out


def dataclasses_replace_precision(bs, precision):
    import dataclasses
    return dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, precision=precision))


def workload():
    from cffc_b200 import cases
    return cases.curvilinear_mach2()


def config(bs, n, args):
    return {"workload": f"curvilinear Mach-2, {bs.nblk} blocks x {bs.nci}x{bs.ncj} cells "
                        f"({bs.n_interior} cells), {args.rk_steps} RK2 steps per bench step",
            "blocks": bs.nblk, "cells_per_block": [bs.nci, bs.ncj], "cells": bs.n_interior,
            "rk_steps_per_step": args.rk_steps, "scheme": "Roe + LSQ + Venkatakrishnan, RK2, CFL 0.5",
            "precision": args.precision, "parallelism": f"replicas x{n}",
            "l2": "working set (~170 MB per stage) larger than the 126 MB L2; no flush"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    bs = workload()
    vals = []
    sample_steps = 4
    for k in range(args.warmup + args.steps):
        r = cpu_reference_run(bs, sample_steps, os.cpu_count() or 1)
        kind = "reference"
        if r is None:
            r = cpu_port_run(bs, 2)
            kind = "port"
        if k >= args.warmup:
            vals.append(r)
    v = statistics.median(x["mcell_updates_per_s"] for x in vals)
    # one step of this arm is one sample of sample_steps RK2 steps: its
    # measured time, not a projection to the GPU arm's step length
    ms = statistics.median(x["seconds"] * 1e3 for x in vals)
    line = {"impl": "reference", "metric": "Mcell-updates/s (Roe+limiter residual, explicit RK2)",
            "value": round(v, 4), "unit": "Mcell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 reconstruction+flux / f64 state" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded)", "config": config(bs, 1, args),
            "cpu_baseline": {"value": round(v, 4), "unit": "Mcell-updates/s",
                             "cores": vals[0]["threads"], "kind": kind,
                             "detail": CPU_DETAIL[kind].format(n=vals[0]["threads"]),
                             "sample": f"{sample_steps} RK2 steps of the 1,048,576-cell block set per bench step",
                             "sample_rk_steps": sample_steps},
            "e2e": {"value": round(v, 4), "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def max_over_ranks(x, world, device):
    """The largest x over the ranks (replicas: each rank times its own
    device, the job takes as long as the slowest); every rank gets it."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, cell_updates, ms):
    """Mcell-updates/s of the whole job: world replicas, each advancing
    cell_updates per step, in ms per step (the slowest rank's)."""
    return world * cell_updates / (ms * 1e-3) * 1e-6


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from cffc_b200 import capi
    bs = workload()
    bs.scheme.precision = PRECISION[args.precision]
    h = capi.Handle(bs, device=local)
    stream = torch.cuda.current_stream()
    h.lib.e2d_set_stream.argtypes = [capi.C.c_void_p, capi.C.c_void_p]
    h.lib.e2d_set_stream(h.h, capi.C.c_void_p(stream.cuda_stream))
    h.set_state()

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        rc, _ = h.rk_steps(args.rk_steps, history=False)
        assert rc == 0, rc
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            rc, _ = h.rk_steps(args.rk_steps, history=False)
            assert rc == 0, rc
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, "cuda")
    cell_updates = bs.n_interior * args.rk_steps
    value = job_throughput(world, cell_updates, ms)

    # per-kernel device times of the fused stage kernel (launch by launch)
    kt = np.zeros(6)
    h.lib.e2d_kernel_times.argtypes = [capi.C.c_void_p, capi.C.c_int, capi._dp]
    rc = h.lib.e2d_kernel_times(h.h, 20, capi.ptr(kt))
    assert rc == 0, rc
    hbm, peak_kind = peaks()
    kind, rows, _ = h.stage_config()
    stage_name = (f"march_kernel (column-marching LSQ+limiter+Roe+update, {rows} rows per chunk)" if kind == 1
                  else "stage_kernel (tiled LSQ+limiter+Roe+update)")
    stage_ms = 0.5 * (kt[1] + kt[2])
    stage_bytes = bs.n_interior * 0.5 * (80 + 112)  # per launch, mean of the two stages
    achieved = stage_bytes / (stage_ms * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("bytes_per_launch")
        except Exception:
            traffic = None

    # end to end through the C ABI: pinned host W in, U out, every step
    Wh = torch.from_numpy(np.ascontiguousarray(bs.W)).pin_memory()
    Uh = torch.empty(bs.cell_shape(), dtype=torch.float64).pin_memory()
    Wp = capi.C.cast(Wh.data_ptr(), capi._dp)
    Up = capi.C.cast(Uh.data_ptr(), capi._dp)
    nbytes = Wh.numel() * 8
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        assert h.lib.e2d_set_state(h.h, Wp) == 0
        rc, _ = h.rk_steps(args.rk_steps, history=False)
        assert rc == 0
        assert h.lib.e2d_get_state(h.h, capi.C.cast(None, capi._dp), Up) == 0
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps, world, "cuda")
    e2e = job_throughput(world, cell_updates, e2e_ms)

    line = None
    if rank == 0:
        # per time step: slot init, (ghost fill + stage) per stage, step end;
        # per e2d_rk_steps call: slot init, CFL, two norm kernels
        launches_per_rk = 2 + 2 * bs.scheme.n_stage
        line = {
            "metric": "Mcell-updates/s (Roe+limiter residual, explicit RK2)",
            "value": round(value, 3), "unit": "Mcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 reconstruction+flux / f64 state" if args.precision == "fp32" else "f64",
            "data": "synthetic (seeded curvilinear grid and perturbation)",
            "config": config(bs, world, args),
            "e2e": {"value": round(e2e, 3), "unit": "Mcell-updates/s",
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes},
            "roofline": {"bound": "hbm", "kernel": stage_name,
                         "achieved": round(achieved, 2), "peak": hbm, "peak_kind": peak_kind,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": traffic,
                         "algorithmic_bytes_per_launch": stage_bytes,
                         "launch_ms": {"ghost_fill": round(kt[0], 5), "stage1": round(kt[1], 5),
                                       "stage2": round(kt[2], 5), "cfl": round(kt[3], 5),
                                       "norms": round(kt[4], 5), "step": round(kt[5], 5)}},
            "path_roofline": {"bytes_per_cell_update": 240,
                              "achieved_gbs": round(240 * cell_updates / (ms * 1e-3) / 1e9, 2),
                              "frac": round(240 * cell_updates / (ms * 1e-3) / 1e9 / hbm, 4)},
            "gpu_launches": args.steps * (args.rk_steps * launches_per_rk + 4),
            "clocks": clk.summary(),
        }
        if args.precision == "fp32":
            line["l2_error_vs_fp64"] = dict(fp32_error(bs, args.rk_steps, local), steps=args.rk_steps)
        elif world == 1:
            line["fp32"] = fp32_leg(bs, args.rk_steps, local)
        if world == 1:
            line["exact"] = exact_leg(bs, args.rk_steps, local)
            line["parity"] = parity_leg(bs, local)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(bs)
        if world == 1 and not args.no_nks:
            line["nks_c2"] = nks_c2_measure(PRECISION[args.precision], local, not args.no_cpu_baseline)
            line["nks"] = nks_measure(PRECISION[args.precision], local, not args.no_cpu_baseline)
            line["nks_iluk"] = nks_measure(PRECISION[args.precision], local, not args.no_cpu_baseline, ilu_level=2)
            line["nks_batch"] = nks_batch_measure(PRECISION[args.precision], local)
            line["nks_batch_iluk"] = nks_batch_measure(PRECISION[args.precision], local, ilu_level=2)
            line["nks_sweep"] = nks_sweep_measure(local, n_cases=args.sweep_cases)
            line["nks_learned"] = nks_learned_measure(local)
        print(json.dumps(line), flush=True)
    h.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
