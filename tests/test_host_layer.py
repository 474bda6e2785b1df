"""The C++ host layer (include/cffc_euler2d.hpp): deck parsing, block
building and the case-file export run on the CPU; the GPU tests drive the
same decks through the device and compare with the C restatement (oracle)
on the exported blocks.

The driver tests/cpp/host_driver.cc is compiled here against the built
libcffc_e2d.so."""
import os
import subprocess
import sys

import numpy as np
import pytest

from cffc_b200 import capi, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cffc_b200")
R_AIR = 8.314511 / (28.9640 * 0.001)  # R_UNIVERSAL / (MOLE_WT_AIR * MILLI)

DECK = """# periodic box, 2 x 2 blocks of 16 x 16 cells
Time_Integration_Type =
Explicit_Predictor_Corrector
Reconstruction_Type =
Least_Squares
Limiter_Type =
Venkatakrishnan
Flux_Function_Type =
Roe
ICs_Type =
Uniform
Grid_Type =
Periodic_Box
Box_Width =
2.0
Box_Height =
1.0
Number_of_Cells_Idir =
32
Number_of_Cells_Jdir =
32
Number_of_Blocks_Idir =
2
Number_of_Blocks_Jdir =
2
Number_of_Ghost_Cells =
2
# keywords of the reference outside this path are skipped
Number_of_Initial_Mesh_Refinements =
0
   Mach_Number =
0.5
Pressure =
101.325
Temperature =
288.16
CFL_Number =
0.5
Maximum_Number_of_Time_Steps =
{steps}
GPU_Precision =
{precision}
Execute
"""


def write_deck(path, steps=10, precision="FP64_Exact", text=DECK):
    with open(path, "w") as f:
        f.write(text.format(steps=steps, precision=precision))
    return str(path)


def expected_blocks():
    """The same grid and freestream built in Python: Periodic_Box spans
    [-W/2, W/2] x [-H/2, H/2]; rho = p / (R T), u = M a."""
    p, T, M = 101.325 * 1000.0, 288.16, 0.5
    rho = p / (R_AIR * T)
    a = np.sqrt(1.4 * p / rho)
    u = M * a * np.cos(2.0 * np.pi * 0.0 / 360.0)

    def nodes(I, J):
        return -0.5 * 2.0 + 2.0 * I / 32.0, -0.5 * 1.0 + 1.0 * J / 32.0

    def W_fn(x, y, b):
        return np.stack([np.full_like(x, rho), np.full_like(x, u), np.full_like(x, 0.0), np.full_like(x, p)])

    bs = cases.structured(2, 2, 16, 16, nodes, True, True, W_fn=W_fn)
    return bs, (rho, u, p)


def test_deck_parses_and_builds_the_blocks(driver, tmp_path):
    deck = write_deck(tmp_path / "box.in")
    case = str(tmp_path / "box.case")
    out = subprocess.run([driver, "parse", deck, case], capture_output=True, text=True, check=True).stdout.split()
    assert out[0] == "ok" and int(out[1]) == 1  # Number_of_Initial_Mesh_Refinements
    got = cases.read_case(case)
    want, (rho, u, p) = expected_blocks()
    assert float(out[2]) == rho and float(out[3]) == u and float(out[4]) == p
    for f in ("neighbour", "bc_w", "bc_e", "bc_s", "bc_n", "node_x", "node_y", "W"):
        assert np.array_equal(getattr(got, f), getattr(want, f)), f
    assert got.scheme.n_stage == 2 and got.scheme.limiter == cases.LIMITER_VENKATAKRISHNAN
    assert got.scheme.cfl == 0.5 and got.periodic == 1


def test_invalid_entry_reports_its_line(driver, tmp_path):
    bad = DECK.replace("CFL_Number =\n0.5", "CFL_Number =\n-1.0")
    deck = write_deck(tmp_path / "bad.in", text=bad)
    r = subprocess.run([driver, "parse", deck, str(tmp_path / "x.case")], capture_output=True, text=True)
    assert r.returncode == 3
    line = int(r.stdout.split()[-1])
    assert open(deck).read().split("\n")[line - 1].strip() == "-1.0"


def test_unsupported_scheme_is_rejected(driver, tmp_path):
    bad = DECK.replace("Flux_Function_Type =\nRoe", "Flux_Function_Type =\nAUSM_plus_up")
    deck = write_deck(tmp_path / "bad2.in", text=bad)
    r = subprocess.run([driver, "parse", deck, str(tmp_path / "x.case")], capture_output=True, text=True)
    assert r.returncode == 3


@pytest.mark.parametrize("name,code", [("Godunov", 1), ("Roe", 2), ("Rusanov", 3), ("HLLE", 4), ("Linde", 5),
                                       ("HLLC", 6), ("VanLeer", 8), ("AUSM", 9), ("AUSM+", 10)])
def test_flux_function_keywords(driver, tmp_path, name, code):
    """The Flux_Function_Type names of Euler2DInput.cc:1850-1872 select the
    reference's i_Flux_Function codes."""
    text = DECK.replace("Flux_Function_Type =\nRoe", "Flux_Function_Type =\n" + name)
    deck = write_deck(tmp_path / "f.in", text=text)
    case = str(tmp_path / "f.case")
    subprocess.run([driver, "parse", deck, case], check=True, capture_output=True)
    assert cases.read_case(case).scheme.flux == code


@pytest.mark.gpu
def test_deck_run_matches_oracle_bitwise(driver, tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import e2d_oracle
    deck = write_deck(tmp_path / "run.in", steps=20)
    case, state = str(tmp_path / "run.case"), str(tmp_path / "run.bin")
    subprocess.run([driver, "run", deck, case, state], check=True, capture_output=True)
    bs = cases.read_case(case)
    W = np.fromfile(state).reshape(bs.cell_shape())
    o = e2d_oracle.Oracle(bs)
    o.set_state()
    rc, _ = o.rk_steps(20)
    assert rc == 0
    Wo, _ = o.get_state()
    assert np.array_equal(bs.interior(W), bs.interior(Wo))


@pytest.mark.gpu
def test_single_block_residual_and_cfl(driver, tmp_path):
    """dUdt_Residual_Evaluation on one block (ghosts from the multi-block
    exchange) equals that block's part of the multi-block residual; CFL
    returns the block's minimum step."""
    deck = write_deck(tmp_path / "r.in", steps=0)
    out = str(tmp_path / "r.bin")
    subprocess.run([driver, "residual1", deck, out], check=True, capture_output=True)
    bs, _ = expected_blocks()
    n = 4 * bs.NCj * bs.NCi
    raw = np.fromfile(out)
    per = 2 * n + bs.NCj * bs.NCi + 2
    assert raw.size == per * bs.nblk
    for b in range(bs.nblk):
        rec = raw[b * per:(b + 1) * per]
        single, multi = rec[:n], rec[n:2 * n]
        dt = rec[2 * n:2 * n + bs.NCj * bs.NCi].reshape(bs.NCj, bs.NCi)
        assert np.array_equal(single, multi)
        assert rec[-2] == np.min(dt[2:-2, 2:-2]) and rec[-2] > 0
        d = single.reshape(4, bs.NCj, bs.NCi)[0, 2:-2, 2:-2]
        assert rec[-1] == np.sqrt(np.sum(d * d))  or np.isclose(rec[-1], np.sqrt(np.sum(d * d)), rtol=1e-14)


@pytest.mark.gpu
def test_solver_entry_point_writes_output(tmp_path):
    lib = capi.load_library()
    text = DECK + ""
    deck = write_deck(tmp_path / "s.in", steps=5)
    outname = str(tmp_path / "s.dat")  # the keyword's value + ".dat", as the reference names it
    with open(deck) as f:
        body = f.read().replace("Execute", "Output_File_Name =\n%s\nExecute" % outname[:-4])
    with open(deck, "w") as f:
        f.write(body)
    lib.e2d_solver_run.argtypes = [capi.C.c_char_p, capi.C.c_int]
    assert lib.e2d_solver_run(deck.encode(), 1) == 0
    rows = [l for l in open(outname) if l and l[0] in "-0123456789"]
    assert len(rows) == 32 * 32
    vals = np.array([[float(x) for x in r.split()] for r in rows])
    assert np.all(vals[:, 2] > 0) and np.all(vals[:, 5] > 0)


@pytest.mark.parametrize("lines,want", [
    ("", (0, 0, 0)),
    ("GMRES_Block_Preconditioner =\nILUK\nGMRES_ILUK_Level_of_Fill =\n4\n", (1, 4, 0)),
    ("GMRES_Block_Preconditioner =\nDiagonal\n", (0, 0, 0)),
    ("GMRES_Block_Preconditioner =\nAnything\nJacobian_Order =\nSource_Terms_Only\n", (1, 0, 1)),
    ("Jacobian_Order =\nFirst_Order_Inviscid_HLLE\n", (0, 0, 0)),
    ("Jacobian_Order =\nSomething_Unknown\n", (0, 0, 0)),
])
def test_block_preconditioner_keywords(driver, tmp_path, lines, want):
    """GMRES_Block_Preconditioner, GMRES_ILUK_Level_of_Fill and Jacobian_Order
    as NKS_Input_Parameters parses them (NKSInput2D.h:523-560): "Diagonal" is
    block Jacobi, any other value ILU(k); an unknown Jacobian order is
    first-order HLLE."""
    deck = write_deck(tmp_path / "p.in", text=DECK.replace("Execute", lines + "Execute"))
    out = subprocess.run([driver, "parse", deck, str(tmp_path / "p.case")], capture_output=True, text=True,
                         check=True).stdout.split()
    assert tuple(int(x) for x in out[5:8]) == want


@pytest.mark.parametrize("value", ["First_Order_Inviscid_Roe", "First_Order_Inviscid_AUSM_plus_up",
                                   "Second_Order_Diamond_Path_with_HLLE"])
def test_jacobian_orders_without_euler2d_specialization_are_rejected(driver, tmp_path, value):
    deck = write_deck(tmp_path / "j.in", text=DECK.replace("Execute", "Jacobian_Order =\n%s\nExecute" % value))
    r = subprocess.run([driver, "parse", deck, str(tmp_path / "j.case")], capture_output=True, text=True)
    assert r.returncode == 3


@pytest.mark.parametrize("lines,ok", [
    ("GMRES_Overlap =\n0\n", True), ("GMRES_Overlap =\n1\n", False),
    ("NKS_Finite_Time_Step =\nON\n", True), ("NKS_Finite_Time_Step =\nOFF\n", False),
    ("GMRES_Normalization =\nON\n", True), ("GMRES_Normalization =\n0\n", False),
])
def test_nks_options_outside_the_built_solver_are_rejected(driver, tmp_path, lines, ok):
    """Schwarz overlap, fixed-CFL Newton steps and unnormalized GMRES are not
    built: a deck asking for them is rejected instead of silently run with the
    reference's defaults."""
    deck = write_deck(tmp_path / "o.in", text=DECK.replace("Execute", lines + "Execute"))
    r = subprocess.run([driver, "parse", deck, str(tmp_path / "o.case")], capture_output=True, text=True)
    assert (r.returncode == 0) == ok
