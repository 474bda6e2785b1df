"""Generates the golden vectors in tests/golden/ by running the compiled CFFC
reference (oracle/_ref/e2d_ref_harness, built by `make -C oracle reference`
from the reference sources) on seeded block sets.

Each fixture is a compressed .npz holding the case's inputs (so the test does
not need to rebuild the case bit for bit) and what the reference computed:

* residual fixtures: W after ghost fill, dUdt, dWdx, dWdy, phi
  (dUdt_Residual_Evaluation, src_2D/Euler2D/Euler2DQuad.cc:814);
* explicit fixtures: final U, last dUdt and the per-step dt/L1/L2/Max history
  of the explicit loop (src_2D/Euler2D/Euler2DQuadSolvers.cc:657-898);
* nks fixtures: final U of Newton_Krylov_Schwarz_Solver
  (src_2D/NewtonKrylovSchwarz2D/NKS2D.h:136) and, per Newton step, the L2
  norm, ratio and CFL and the GMRES iterations / resid0 / resid / relative
  residual it prints (10 significant digits, NKS2D.h:938-945 and
  GMRES2D.h:1515-1520), and the closing "End of Newton Steps" line (steps
  taken, final L2 and ratio, NKS2D.h:1150-1153); plus the same run from the initial density scaled
  by (1 + 2^-46) ("pert_"), which measures how far the reference's own
  history moves under a round-off-sized change of its input.

Run from the repository root:  python tests/golden/make_golden.py [NAME ...]
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
NKS_SUB = 4  # large NKS fixtures keep the final state on every 4th cell in i and j
SWEEP_SIZE, SWEEP_CASES = 512, (3, 11, 5)  # sweep cases with a reference fixture (8, 12, 16 blocks)


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


def run_nks(bs, params):
    """params: (max_newton, restart, max_gmres, cfl0, overall_tol[, gmres_tol[, ilu_level]]);
    ilu_level k >= 0 selects GMRES_Block_Preconditioner ILUK with level of fill k."""
    res = run_nks_once(bs, params)
    W = bs.W.copy()
    W[:, 0] *= 1.0 + 2.0 ** -46
    pert = run_nks_once(dataclasses.replace(bs, W=W), params)
    res.update({"pert_" + k: pert[k] for k in ("U", "newton", "gmres", "final")})
    return res


def run_nks_once(bs, params):
    with tempfile.TemporaryDirectory() as td:
        cp, op = os.path.join(td, "c.bin"), os.path.join(td, "o.bin")
        cases.write_case(cp, bs)
        args = [str(v) for v in params[:6]]
        if len(params) > 6 and params[6] >= 0:
            args += ["ILUK", str(params[6])]
        r = subprocess.run([HARNESS, "nks", cp, op] + args, check=True, capture_output=True, text=True)
        buf = open(op, "rb").read()
    err = np.frombuffer(buf[:8], dtype="<i4")[0]
    U = np.frombuffer(buf[16:], dtype="<f8").reshape(bs.nblk, 4, bs.NCj, bs.NCi)
    newton, gmres, final = [], [], []
    for line in r.stdout.split("\n"):
        t = line.split()
        if line.strip().startswith("Newton Step (Outer It.)"):
            newton.append([float(t[t.index("L2norm") + 2]), float(t[t.index("L2norm_ratio") + 2]),
                           float(t[t.index("CFL") + 2])])
        elif line.strip().startswith("End of Newton Steps"):
            final = [float(t[t.index("Steps") + 2]), float(t[t.index("L2norm") + 2]),
                     float(t[t.index("L2norm_ratio") + 2])]
        elif line.strip().startswith("Finished GMRES"):
            gmres.append([float(t[t.index("Iterations)") + 2]), float(t[t.index("resid0") + 2]),
                          float(t[t.index("resid") + 2]), float(t[t.index("relative_residual") + 2])])
    return dict(U=U, newton=np.array(newton), gmres=np.array(gmres), final=np.array(final),
                err=np.int32(err), params=np.array(params, dtype=np.float64))


def precon_vector(bs, seed):
    """Seeded GMRES-layout vector [nblk][NCj][NCi][4], ghost entries zero."""
    v = np.zeros((bs.nblk, bs.NCj, bs.NCi, 4))
    g = bs.ng
    v[:, g:-g, g:-g, :] = np.random.default_rng(seed).standard_normal((bs.nblk, bs.ncj, bs.nci, 4))
    return v


def run_precon(bs, params):
    """params: (cfl, ilu_level, seed); ilu_level -1 is block Jacobi.  The
    reference's Newton-step preconditioner applied to a seeded vector."""
    cfl, level, seed = params
    v = precon_vector(bs, int(seed))
    with tempfile.TemporaryDirectory() as td:
        cp, op, vp = (os.path.join(td, n) for n in ("c.bin", "o.bin", "v.bin"))
        cases.write_case(cp, bs)
        v.astype("<f8").tofile(vp)
        kind = "ILUK" if level >= 0 else "Diagonal"
        subprocess.run([HARNESS, "precon", cp, op, repr(float(cfl)), kind, str(max(int(level), 0)), vp],
                       check=True, capture_output=True, text=True)
        z = np.fromfile(op, dtype="<f8").reshape(v.shape)
    return dict(v=v, z=z, params=np.array(params, dtype=np.float64))


def case_arrays(bs):
    d = {f.name: getattr(bs, f.name) for f in dataclasses.fields(bs)
         if isinstance(getattr(bs, f.name), np.ndarray)}
    sc = bs.scheme
    d["scheme"] = np.array([sc.limiter, sc.flux, sc.n_stage, sc.local_dt, sc.precision, sc.time_integration,
                            sc.rs_iterations, sc.freeze_limiter], np.int32)
    d["scheme_f"] = np.array([sc.cfl, sc.gamma, sc.rs_epsilon, sc.freeze_level])
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
    bump = cases.bump_channel(nbi=6, nbj=2, nci=16, ncj=16)
    bump_bj = cases.bump_channel(nbi=4, nbj=2, nci=16, ncj=8, mach=0.6,
                                 scheme=cases.Scheme(limiter=cases.LIMITER_BARTH_JESPERSEN, local_dt=0))
    bump_m14 = cases.bump_channel(nbi=6, nbj=2, nci=16, ncj=16, mach=1.4, h=0.04,
                                  scheme=cases.Scheme(limiter=cases.LIMITER_ZERO, local_dt=1))
    c2 = cases.bump_channel()  # 12 x 4 blocks of 64 x 32, h 0.1, Mach 0.5
    box21 = cases.periodic_box_bumps(nb=2, nbj=1, nc=16, seed=31)
    box11 = cases.periodic_box_bumps(nb=1, nc=16, seed=32)
    sweep = cases.bump_family(SWEEP_SIZE, layouts=cases.LAYOUTS_8_96)
    ch_ms = cases.channel(nbi=2, nbj=2, nci=12, ncj=10, seed=9,
                          scheme=cases.Scheme(limiter=cases.LIMITER_VENKATAKRISHNAN, cfl=0.8, n_stage=4, local_dt=1))
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
        # periodic boxes with a single block across a direction: BC_PERIODIC
        # edges, and for 2 x 1 no wrap in i (the reference's periodic-box
        # wiring needs several blocks in both directions)
        ("residual_box_2x1x16", box21, "residual", 0),
        ("explicit_box_2x1x16_20", box21, "explicit", 20),
        ("explicit_box_1x1x16_20", box11, "explicit", 20),
        # Newton steps, GMRES restart, GMRES iteration cap, initial CFL, tolerance
        ("nks_bump_6x2x16_6", bump, "nks", (6, 30, 60, 1.0, 1e-10)),
        # global time step, Barth-Jespersen, GMRES restarts and its iteration cap
        ("nks_bump_bj_global_4", bump_bj, "nks", (4, 10, 25, 5.0, 1e-10)),
        # supersonic, first order, inexact Newton (GMRES tolerance 0.1): converges to 1e-10
        ("nks_bump_m14_converged", bump_m14, "nks", (30, 30, 120, 10.0, 1e-10, 0.1)),
        # the same solve with the HLLE flux in the residual
        ("nks_bump_m14_hlle", with_flux(bump_m14, cases.FLUX_HLLE), "nks", (30, 30, 120, 10.0, 1e-10, 0.1)),
        # the subsonic bump that stalls under block Jacobi, with the ILU(4)
        # preconditioner of the reference's NKS example decks
        ("nks_bump_iluk4", bump, "nks", (12, 30, 120, 10.0, 1e-10, 0.1, 4)),
        # global time step, Barth-Jespersen, restarts, with ILU(0)
        ("nks_bump_bj_global_iluk0", bump_bj, "nks", (4, 10, 25, 5.0, 1e-10, 1e-5, 0)),
        # the 98,304-cell subsonic bump channel (12 x 4 blocks of 64 x 32,
        # h 0.1, Mach 0.5) from the freestream: GMRES(30) with block Jacobi,
        # 40 Newton steps of the reference's stalling history, and the ILU(4)
        # preconditioner of the reference's example decks
        ("nks_c2_bump_12x4x64x32_bj", c2, "nks", (40, 30, 60, 1.0, 1e-10)),
        ("nks_c2_bump_12x4x64x32_iluk4", c2, "nks", (12, 30, 120, 10.0, 1e-10, 0.1, 4)),
    ] + [
        # three cases of the 512-case supersonic sweep (cases.bump_family with
        # the 8-96 block layouts), solved to 1e-10 with ILU(2) as the batched
        # sweep runs them: the FP64 reference answer each case of a batch is
        # compared with ("sweep_index" in the fixture)
        (f"nks_sweep{k:03d}_{sweep[k].name.rsplit('_', 1)[1]}", sweep[k], "nks",
         (40, 30, 200, 10.0, 1e-10, 0.1, 2)) for k in SWEEP_CASES
    ] + [
        # the Newton step's preconditioner alone: (CFL, ILU level or -1 for
        # block Jacobi, vector seed)
        ("precon_bump_jacobi", bump, "precon", (10.0, -1, 1)),
        ("precon_bump_iluk0", bump, "precon", (10.0, 0, 2)),
        ("precon_bump_iluk2", bump, "precon", (10.0, 2, 3)),
        ("precon_bump_iluk4", bump, "precon", (100.0, 4, 4)),
        ("precon_bump_bj_global_iluk1", bump_bj, "precon", (5.0, 1, 5)),
        ("precon_curv_iluk3", curv, "precon", (3.0, 3, 6)),
        # one 64x60 channel block: the solve's vector and descriptors exceed
        # shared memory, so the device works them in global memory
        ("precon_channel64_iluk1", cases.channel(nbi=1, nbj=1, nci=64, ncj=60, seed=7), "precon", (2.0, 1, 7)),
    ] + [
        # the other explicit schemes (optimally smoothing multistage, RK4, RK5),
        # implicit residual smoothing and limiter freezing
        (name, dataclasses.replace(ch_ms, scheme=dataclasses.replace(ch_ms.scheme, **kw)), "explicit", steps)
        for name, kw, steps in (
            ("explicit_os4_channel_30", dict(time_integration=cases.TIME_OPTIMAL_SMOOTHING, n_stage=4), 30),
            ("explicit_os5_zero_channel_30", dict(time_integration=cases.TIME_OPTIMAL_SMOOTHING, n_stage=5,
                                                  limiter=cases.LIMITER_ZERO), 30),
            ("explicit_os2_global_channel_30", dict(time_integration=cases.TIME_OPTIMAL_SMOOTHING, n_stage=2,
                                                    local_dt=0, cfl=0.4), 30),
            ("explicit_rk4_channel_20", dict(time_integration=cases.TIME_RUNGE_KUTTA, n_stage=4, local_dt=0), 20),
            ("explicit_rk5_channel_20", dict(time_integration=cases.TIME_RUNGE_KUTTA, n_stage=5), 20),
            ("explicit_os3_smoothing_channel_30", dict(time_integration=cases.TIME_OPTIMAL_SMOOTHING, n_stage=3,
                                                       rs_epsilon=0.125, rs_iterations=2), 30),
            ("explicit_pc_smoothing_channel_30", dict(time_integration=cases.TIME_PREDICTOR_CORRECTOR, n_stage=2,
                                                      rs_epsilon=0.25, rs_iterations=1, cfl=0.6), 30),
            ("explicit_os4_freeze_channel_30", dict(time_integration=cases.TIME_OPTIMAL_SMOOTHING, n_stage=4,
                                                    freeze_limiter=1, freeze_level=0.0463), 30),
            ("explicit_os5_smoothing_freeze_channel_30", dict(
                time_integration=cases.TIME_OPTIMAL_SMOOTHING, n_stage=5, rs_epsilon=0.125, rs_iterations=2,
                freeze_limiter=1, freeze_level=0.0484), 30))
    ] + [
        # every other flux function: a supersonic curvilinear residual, explicit
        # steps in the subsonic channel with fixed inflow and reflecting walls,
        # and in the channel with characteristic inflow/outflow
        case for f, nm in FLUX_NAMES.items() for case in (
            (f"residual_{nm}_curv_4x2x8", with_flux(cases.curvilinear_mach2(nbi=4, nbj=2, nc=8, seed=6), f),
             "residual", 0),
            (f"explicit_{nm}_channel_20", with_flux(ch, f), "explicit", 20),
            (f"explicit_{nm}_channel_char_20", with_flux(ch_char, f), "explicit", 20))
    ]


FLUX_NAMES = {cases.FLUX_GODUNOV: "godunov", cases.FLUX_RUSANOV: "rusanov", cases.FLUX_HLLE: "hlle",
              cases.FLUX_LINDE: "linde", cases.FLUX_HLLC: "hllc", cases.FLUX_VANLEER: "vanleer",
              cases.FLUX_AUSM: "ausm", cases.FLUX_AUSMPLUS: "ausmplus"}


def with_flux(bs, flux):
    return dataclasses.replace(bs, scheme=dataclasses.replace(bs.scheme, flux=flux))


# Decks of the restart fixture, run by the reference's own solver
# (Euler2DQuadSolver).  A: the reference's Bump_Channel_Flow grid (4 x 2
# blocks of 8 x 4 cells, circular-arc bump spline), 20 predictor-corrector
# steps from the Mach 1.4 freestream, restart files written at the end.
# B: a restart from A's files for 10 more steps.
RESTART_DECK = """# supersonic bump channel, explicit predictor-corrector
Time_Integration_Type =
Explicit_Predictor_Corrector
Time_Accurate =
0
Local_Time_Stepping =
1
CFL_Number =
0.5
Maximum_Number_of_Time_Steps =
{steps}
Reconstruction_Type =
Least_Squares
Limiter_Type =
Venkatakrishnan
Flux_Function_Type =
Roe
ICs_Type =
{ics}
Mach_Number =
1.40
{grid}Number_of_Cells_Idir =
8
Number_of_Cells_Jdir =
4
Number_of_Blocks_Per_Processor =
8
Restart_File_Name =
bump
Output_File_Name =
bump
{extra}Execute
Write_Restart
Terminate
"""


BUMP_GRID = "Grid_Type =\nBump_Channel_Flow\nSmooth_Bump =\nOFF\n"
# (Grid_File_Name after Output_File_Name, which also sets the grid file name)
DATA_GRID = "Grid_Type =\nRead_From_Data_File\n"
DATA_GRID_FILE = "Grid_File_Name =\nbumpgrid\n"


def restart_deck(restart, extra="", grid=BUMP_GRID):
    return RESTART_DECK.format(steps=10 if restart else 20, ics="Restart" if restart else "Uniform", extra=extra,
                               grid=grid)


# deck D: Newton-Krylov with the ILU(2) preconditioner, first order, from the
# freestream on the grid data file (no explicit steps)
NKS_ILU_EXTRA = ("Maximum_Number_of_NKS_Iterations =\n12\nNKS_Overall_Tolerance =\n1e-10\n"
                 "NKS_Finite_Time_Step_Initial_CFL =\n10.0\nGMRES_Tolerance =\n0.1\nGMRES_Restart =\n30\n"
                 "Maximum_Number_of_GMRES_Iterations =\n100\nGMRES_Block_Preconditioner =\nILUK\n"
                 "GMRES_ILUK_Level_of_Fill =\n2\nJacobian_Order =\nFirst_Order_Inviscid_HLLE\n")


def nks_deck():
    text = restart_deck(False, extra=DATA_GRID_FILE + NKS_ILU_EXTRA, grid=DATA_GRID)
    text = text.replace("Limiter_Type =\nVenkatakrishnan", "Limiter_Type =\nZero")
    return text.replace("Maximum_Number_of_Time_Steps =\n20", "Maximum_Number_of_Time_Steps =\n0")


def make_restart_fixture():
    """tests/golden/restart.tar.gz: restart files the reference wrote and what
    its own reader (Read_QuadTree + Read_Restart_Solution) makes of them
    (read.bin, layout of the harness's restart_read):
      chan/   Write_Restart_Solution of the channel case with characteristic
              inflow/outflow (17 steps, time 0.25)
      bump0/  deck A's restart files (boundary splines in the grid)
      bump1/  deck B's, a restart from bump0 continued for 10 steps
      bump2/  deck C's: deck A on the grid data file bumpgrid.grid (bump0's
              grids as Write_Quad_Block writes them) read back by the
              reference (Grid_Type Read_From_Data_File)
      bump3/  deck D's: Newton-Krylov with ILU(2), first order, on the same
              grid data file, from the freestream
      grid/   grid data files of the channel case and of a periodic box
    and the four decks."""
    import shutil
    import tarfile
    ch_char = cases.channel(bc=dict(W=cases.BC_CHARACTERISTIC, E=cases.BC_CHARACTERISTIC,
                                    S=cases.BC_REFLECTION, N=cases.BC_CONSTANT_EXTRAPOLATION), seed=8)
    with tempfile.TemporaryDirectory() as td:
        root = os.path.join(td, "restart")
        for d in ("chan", "bump0", "bump1", "bump2", "bump3", "grid"):
            os.makedirs(os.path.join(root, d))
        grid = os.path.join(root, "grid")
        for name, bs in (("chan", ch_char), ("box", cases.periodic_box_bumps(nb=2, nc=8, seed=11))):
            cp = os.path.join(td, name + ".case")
            cases.write_case(cp, bs)
            subprocess.run([HARNESS, "grid_write", cp, os.path.join(grid, name + ".grid")], check=True)
        chan = os.path.join(root, "chan")
        cp = os.path.join(td, "chan.case")
        cases.write_case(cp, ch_char)
        subprocess.run([HARNESS, "restart_write", cp, "chan", "17", "0.25"], cwd=chan, check=True)
        subprocess.run([HARNESS, "restart_read", cp, "chan", "read.bin"], cwd=chan, check=True)
        for name, text in (("deck_a.in", restart_deck(False)), ("deck_b.in", restart_deck(True)),
                           ("deck_c.in", restart_deck(False, extra=DATA_GRID_FILE, grid=DATA_GRID)),
                           ("deck_d.in", nks_deck())):
            with open(os.path.join(root, name), "w") as f:
                f.write(text)
        dummy = os.path.join(td, "bump.case")  # block count and wiring for restart_read
        cases.write_case(dummy, cases.channel(nbi=4, nbj=2))
        run = os.path.join(td, "run")
        os.makedirs(run)
        for stage, deck in (("bump0", "deck_a.in"), ("bump1", "deck_b.in"), ("bump2", "deck_c.in"),
                            ("bump3", "deck_d.in")):
            subprocess.run([HARNESS, "solve", os.path.join(root, deck)], cwd=run, check=True,
                           capture_output=True)
            dst = os.path.join(root, stage)
            for fn in sorted(os.listdir(run)):
                if fn.startswith("bump_blk") or fn == "bump_quadtree.tree":
                    shutil.copy(os.path.join(run, fn), dst)
            extra = [os.path.join(run, "bumpgrid.grid")] if stage == "bump0" else []
            subprocess.run([HARNESS, "restart_read", dummy, "bump", "read.bin"] + extra, cwd=dst, check=True)
            if extra:
                shutil.copy(extra[0], os.path.join(root, "bump2"))
        with tarfile.open(os.path.join(OUT, "restart.tar.gz"), "w:gz") as t:
            t.add(root, arcname="restart")
    print("restart.tar.gz")


BIG_SUB = 8  # the 1M-cell residual digest keeps dUdt on every 8th interior cell in i and j


def block_digests(bs, dUdt):
    """SHA-256 of each block's interior dUdt bytes ([nblk][32] uint8)."""
    import hashlib
    inner = np.ascontiguousarray(bs.interior(dUdt))
    return np.array([np.frombuffer(hashlib.sha256(inner[b].tobytes()).digest(), np.uint8)
                     for b in range(bs.nblk)])


def make_big_residual():
    """The reference's residual of the full 1,048,576-cell curvilinear Mach-2
    block set (cases.curvilinear_mach2()), kept as digests: SHA-256 of each
    block's interior dUdt (a bit-exact comparison without storing 34 MB),
    dUdt on every BIG_SUB-th interior cell, and SHA-256 of the inputs the
    reference saw (W and the nodes), so a test can check that it rebuilt the
    same case."""
    import hashlib
    bs = cases.curvilinear_mach2()
    res = run_residual(bs)
    inputs = hashlib.sha256(np.ascontiguousarray(bs.W).tobytes() + np.ascontiguousarray(bs.node_x).tobytes() +
                            np.ascontiguousarray(bs.node_y).tobytes()).digest()
    np.savez_compressed(os.path.join(OUT, "digest_residual_curv_256x64.npz"),
                        dUdt_block_sha256=block_digests(bs, res["dUdt"]),
                        dUdt_sub=np.ascontiguousarray(bs.interior(res["dUdt"])[..., ::BIG_SUB, ::BIG_SUB]),
                        inputs_sha256=np.frombuffer(inputs, np.uint8), sub=np.int32(BIG_SUB))
    print("digest_residual_curv_256x64", bs.nblk, "blocks")


def main():
    if not os.path.exists(HARNESS):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "reference"], check=True)
    only = set(sys.argv[1:])
    if not only or "restart" in only:
        make_restart_fixture()
    if not only or "digest_residual_curv_256x64" in only:
        make_big_residual()
    for name, bs, kind, steps in golden_cases():
        if only and name not in only:
            continue
        out = case_arrays(bs)
        if kind == "nks":
            res = run_nks(bs, steps)
            steps = steps[0]
        elif kind == "precon":
            res = run_precon(bs, steps)
            steps = 0
        else:
            res = run_residual(bs) if kind == "residual" else run_explicit(bs, steps)
        if kind == "nks" and bs.nblk * bs.nci * bs.ncj > 8192:
            # large Newton-Krylov fixtures: the whole history, and the final
            # states on every NKS_SUB-th interior cell in i and j
            for k in ("U", "pert_U"):
                res[k + "_sub"] = np.ascontiguousarray(bs.interior(res.pop(k))[..., ::NKS_SUB, ::NKS_SUB])
            out["lean"] = np.int32(1)
        elif bs.nblk * bs.nci * bs.ncj > 8192:
            # keep the large fixtures small: the interior of the main output only
            keep = "dUdt" if kind == "residual" else "U"
            res = {k: (bs.interior(v) if k == keep else v) for k, v in res.items()
                   if k in (keep, "hist", "err")}
            out["lean"] = np.int32(1)
        out.update({"ref_" + k: v for k, v in res.items()})
        if name.startswith("nks_sweep"):
            out["sweep_index"] = np.int32(int(name[len("nks_sweep"):len("nks_sweep") + 3]))
        out["steps"] = np.int32(steps)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main()
