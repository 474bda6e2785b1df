"""Block-set builders for the Euler2D path: geometry, topology, boundary data
and initial states of multi-block structured grids, in the array layout of
``include/cffc_e2d.h``.

A :class:`BlockSet` holds what the reference keeps in ``Euler2D_Quad_Block``
and ``Grid2D_Quad_Block_HO`` (src_2D/Euler2D/Euler2DQuad.h:140-599,
src_2D/Grid/HO_Grid2DQuad.h:277-305): nodes including ghost nodes, the
per-edge BC type arrays ``BCtypeW/E/S/N``, the reference states ``WoW/E/S/N``
and the primitive state ``W`` of every cell, plus the same-resolution
neighbour table the reference keeps in its quadtree
(src_2D/AMR/QuadTree.cc:363).

The named workloads follow the benchmark configurations of this path:

* :func:`periodic_box_bumps` — unit square, 4x4 blocks of 32x32 cells,
  periodic, rho = p = 1, u = 0.5 plus 8 seeded Gaussian bumps in rho and p;
* :func:`curvilinear_mach2` — [0,4]x[0,1], 32x8 blocks of 64x64 cells made
  curvilinear by seeded sinusoidal node displacement, Mach-2 freestream with
  a seeded 5% density perturbation, periodic;
* :func:`channel` — small walled channels exercising every supported BC.

Seeds use numpy's PCG64 generator; the draw order is documented per builder.
"""
from __future__ import annotations

import dataclasses
import os
import struct

import numpy as np

# Reference BC codes (src_2D/CFD/CFD.h:270-351).
BC_NONE = 0
BC_CONSTANT_EXTRAPOLATION = 4001
BC_PERIODIC = 6000
BC_REFLECTION = 7001
BC_CHARACTERISTIC = 8001
BC_FIXED = 11000

LIMITER_ONE = -1
LIMITER_ZERO = 0
LIMITER_BARTH_JESPERSEN = 8
LIMITER_VENKATAKRISHNAN = 9
# i_Time_Integration codes of the explicit schemes (CFD.h:651-659)
TIME_EXPLICIT_EULER = 0
TIME_PREDICTOR_CORRECTOR = 3
TIME_OPTIMAL_SMOOTHING = 7
TIME_RUNGE_KUTTA = 8
# i_Flux_Function codes (CFD.h:768-778)
FLUX_GODUNOV = 1
FLUX_ROE = 2
FLUX_RUSANOV = 3
FLUX_HLLE = 4
FLUX_LINDE = 5
FLUX_HLLC = 6
FLUX_VANLEER = 8
FLUX_AUSM = 9
FLUX_AUSMPLUS = 10

GAMMA_AIR = 1.40
NG = 2

# neighbour slots: W, E, S, N, SW, SE, NW, NE
_NEIGH_OFFSETS = [(-1, 0), (1, 0), (0, -1), (0, 1), (-1, -1), (1, -1), (-1, 1), (1, 1)]


@dataclasses.dataclass
class Scheme:
    """The subset of ``Euler2D_Input_Parameters`` the path reads."""

    limiter: int = LIMITER_VENKATAKRISHNAN
    flux: int = FLUX_ROE
    n_stage: int = 2
    local_dt: int = 0
    precision: int = 0
    cfl: float = 0.5
    gamma: float = GAMMA_AIR
    time_integration: int = 0   # i_Time_Integration (TIME_* below)
    rs_epsilon: float = 0.0     # Residual_Smoothing_Epsilon (> 0: on)
    rs_iterations: int = 2      # Residual_Smoothing_Gauss_Seidel_Iterations
    freeze_limiter: int = 0     # Freeze_Limiter
    freeze_level: float = 0.0   # Freeze_Limiter_Residual_Level


@dataclasses.dataclass
class BlockSet:
    nci: int
    ncj: int
    neighbour: np.ndarray  # (nblk, 8) int32
    bc_w: np.ndarray  # (nblk, NCj) int32
    bc_e: np.ndarray
    bc_s: np.ndarray  # (nblk, NCi) int32
    bc_n: np.ndarray
    node_x: np.ndarray  # (nblk, NNj, NNi) float64
    node_y: np.ndarray
    wo_w: np.ndarray  # (nblk, 4, NCj) float64
    wo_e: np.ndarray
    wo_s: np.ndarray  # (nblk, 4, NCi) float64
    wo_n: np.ndarray
    W: np.ndarray  # (nblk, 4, NCj, NCi) float64
    scheme: Scheme = dataclasses.field(default_factory=Scheme)
    name: str = ""
    ng: int = NG
    nbi: int = 0          # structured block layout (0: not a structured layout)
    nbj: int = 0
    periodic: int = 0     # 1: periodic in both directions (periodic-box wiring)

    @property
    def nblk(self) -> int:
        return int(self.neighbour.shape[0])

    @property
    def NCi(self) -> int:
        return self.nci + 2 * self.ng

    @property
    def NCj(self) -> int:
        return self.ncj + 2 * self.ng

    @property
    def n_interior(self) -> int:
        return self.nblk * self.nci * self.ncj

    def cell_shape(self):
        return (self.nblk, 4, self.NCj, self.NCi)

    def interior(self, a: np.ndarray) -> np.ndarray:
        """View of the interior cells of a cell array (..., NCj, NCi)."""
        g = self.ng
        return a[..., g:g + self.ncj, g:g + self.nci]

    def contiguous(self) -> "BlockSet":
        for f in dataclasses.fields(self):
            v = getattr(self, f.name)
            if isinstance(v, np.ndarray):
                dt = np.int32 if v.dtype.kind in "iu" else np.float64
                setattr(self, f.name, np.ascontiguousarray(v, dtype=dt))
        return self


def U_of_W(W: np.ndarray, gamma: float = GAMMA_AIR) -> np.ndarray:
    """Conserved state from primitive (Euler2D_pState::U, Euler2DState.h:1748)."""
    gm1i = 1.0 / (gamma - 1.0)
    d, u, v, p = W[:, 0], W[:, 1], W[:, 2], W[:, 3]
    return np.stack([d, d * u, d * v, p * gm1i + 0.5 * d * (u * u + v * v)], axis=1)


def structured(nbi, nbj, nci, ncj, node_fn, periodic_i=False, periodic_j=False,
               bc=None, wo=None, W_fn=None, scheme=None, name="") -> BlockSet:
    """Blocks of nci x ncj cells on an nbi x nbj structured layout.

    node_fn(I, J) maps global node indices (ghost nodes included, so I and J
    run from -NG to nb*nc + NG) to coordinates.  Block b = bj*nbi + bi.
    bc = dict(W=, E=, S=, N=) gives the BC code of each physical domain edge
    (ignored across periodic directions); wo = dict of primitive reference
    states (4-tuples) per edge.  W_fn(x, y) gives the initial primitive
    state at cell centres (arrays of shape (4, ...)).
    """
    bc = dict(bc or {})
    wo = dict(wo or {})
    # Periodic in both directions is the reference's GRID_PERIODIC_BOX: its
    # root blocks are wired across the box edges only when there are several
    # blocks in both directions (Find_Neighbours_of_Root_Solution_Blocks,
    # src_2D/AMR/QuadTree.cc:363), and a direction with a single block gets
    # BC_PERIODIC on its two edges instead, BC_NONE otherwise
    # (src_2D/Grid/HO_Grid2DQuadMultiBlock.h:1299-1330).  A box of 2 x 1
    # blocks is therefore not wrapped in i at all, as in the reference.
    box = periodic_i and periodic_j
    if box:
        per_i = BC_PERIODIC if nbi == 1 else BC_NONE
        per_j = BC_PERIODIC if nbj == 1 else BC_NONE
        bc = dict(W=per_i, E=per_i, S=per_j, N=per_j)
        periodic_i = periodic_j = nbi > 1 and nbj > 1
    nblk = nbi * nbj
    NCi, NCj = nci + 2 * NG, ncj + 2 * NG
    NNi, NNj = NCi + 1, NCj + 1
    neighbour = np.full((nblk, 8), -1, np.int32)
    bc_w = np.zeros((nblk, NCj), np.int32)
    bc_e = np.zeros((nblk, NCj), np.int32)
    bc_s = np.zeros((nblk, NCi), np.int32)
    bc_n = np.zeros((nblk, NCi), np.int32)
    node_x = np.zeros((nblk, NNj, NNi))
    node_y = np.zeros((nblk, NNj, NNi))
    wo_w = np.zeros((nblk, 4, NCj))
    wo_e = np.zeros((nblk, 4, NCj))
    wo_s = np.zeros((nblk, 4, NCi))
    wo_n = np.zeros((nblk, 4, NCi))
    W = np.zeros((nblk, 4, NCj, NCi))
    for bj in range(nbj):
        for bi in range(nbi):
            b = bj * nbi + bi
            for k, (di, dj) in enumerate(_NEIGH_OFFSETS):
                ni, nj = bi + di, bj + dj
                if periodic_i:
                    ni %= nbi
                if periodic_j:
                    nj %= nbj
                if 0 <= ni < nbi and 0 <= nj < nbj:
                    neighbour[b, k] = nj * nbi + ni
            I = bi * nci + np.arange(NNi) - NG
            J = bj * ncj + np.arange(NNj) - NG
            II, JJ = np.meshgrid(I, J)
            x, y = node_fn(II.astype(np.float64), JJ.astype(np.float64))
            node_x[b], node_y[b] = x, y
            if not periodic_i and bi == 0:
                bc_w[b] = bc.get("W", BC_NONE)
                wo_w[b] = np.asarray(wo.get("W", (1.0, 0.0, 0.0, 1.0)))[:, None]
            if not periodic_i and bi == nbi - 1:
                bc_e[b] = bc.get("E", BC_NONE)
                wo_e[b] = np.asarray(wo.get("E", (1.0, 0.0, 0.0, 1.0)))[:, None]
            if not periodic_j and bj == 0:
                bc_s[b] = bc.get("S", BC_NONE)
                wo_s[b] = np.asarray(wo.get("S", (1.0, 0.0, 0.0, 1.0)))[:, None]
            if not periodic_j and bj == nbj - 1:
                bc_n[b] = bc.get("N", BC_NONE)
                wo_n[b] = np.asarray(wo.get("N", (1.0, 0.0, 0.0, 1.0)))[:, None]
            if W_fn is not None:
                xc = 0.25 * (x[:-1, :-1] + x[:-1, 1:] + x[1:, 1:] + x[1:, :-1])
                yc = 0.25 * (y[:-1, :-1] + y[:-1, 1:] + y[1:, 1:] + y[1:, :-1])
                W[b] = W_fn(xc, yc, b)
    return BlockSet(nci, ncj, neighbour, bc_w, bc_e, bc_s, bc_n, node_x, node_y,
                    wo_w, wo_e, wo_s, wo_n, W, scheme or Scheme(), name, NG, nbi, nbj,
                    int(box)).contiguous()


def periodic_box_bumps(nb=4, nc=32, n_bumps=8, seed=20261203, scheme=None, nbj=None) -> BlockSet:
    """Unit square, nb x nbj blocks (nbj defaults to nb) of nc x nc cells, periodic; rho = p = 1,
    u = 0.5, v = 0 plus n_bumps Gaussian bumps added to rho and p.
    Draw order (PCG64(seed)): for each bump, amplitude U(0, 0.1), width
    U(0.03, 0.1), centre x U(0, 1), centre y U(0, 1).  Distances are taken to
    the nearest periodic image so the field is smooth across the box edges."""
    rng = np.random.Generator(np.random.PCG64(seed))
    bumps = [(rng.uniform(0, 0.1), rng.uniform(0.03, 0.1), rng.uniform(0, 1), rng.uniform(0, 1))
             for _ in range(n_bumps)]
    nbj = nb if nbj is None else nbj
    hx, hy = 1.0 / (nb * nc), 1.0 / (nbj * nc)

    def nodes(I, J):
        return I * hx, J * hy

    def W_fn(x, y, b):
        g = np.zeros_like(x)
        for amp, w, cx, cy in bumps:
            dx = (x - cx + 0.5) % 1.0 - 0.5
            dy = (y - cy + 0.5) % 1.0 - 0.5
            g += amp * np.exp(-(dx * dx + dy * dy) / (w * w))
        return np.stack([1.0 + g, np.full_like(x, 0.5), np.zeros_like(x), 1.0 + g])

    return structured(nb, nbj, nc, nc, nodes, True, True, W_fn=W_fn,
                      scheme=scheme or Scheme(cfl=0.5, n_stage=2),
                      name=f"periodic_box_{nb}x{nbj}x{nc}^2")


def curvilinear_mach2(nbi=32, nbj=8, nc=64, seed=20261204, scheme=None,
                      amplitude=0.2) -> BlockSet:
    """[0,4]x[0,1] split into nbi x nbj blocks of nc x nc cells, made
    curvilinear by displacing every node by amplitude*h*(1/3)*sum of three
    sine modes per direction; periodic in both directions (integer
    wavenumbers keep the displacement periodic).  Mach-2 freestream along x
    with rho = 1 + 0.05*N(0,1) per cell, p = 1.
    Draw order (PCG64(seed)): for x then y displacement, three modes each of
    (kx in 1..4, ky in 1..4, phase U(0, 2pi)); then one N(0,1) per cell of
    the whole block set in block order, rows of i (ghost cells included)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Lx, Ly = 4.0, 1.0
    nx, ny = nbi * nc, nbj * nc
    hx, hy = Lx / nx, Ly / ny
    modes = [[(int(rng.integers(1, 5)), int(rng.integers(1, 5)), rng.uniform(0, 2 * np.pi))
              for _ in range(3)] for _ in range(2)]

    def nodes(I, J):
        x0, y0 = I * hx, J * hy
        dx = sum(np.sin(2 * np.pi * (kx * x0 / Lx + ky * y0 / Ly) + ph) for kx, ky, ph in modes[0])
        dy = sum(np.sin(2 * np.pi * (kx * x0 / Lx + ky * y0 / Ly) + ph) for kx, ky, ph in modes[1])
        return x0 + amplitude * hx / 3.0 * dx, y0 + amplitude * hy / 3.0 * dy

    NCi, NCj = nc + 2 * NG, nc + 2 * NG
    noise = rng.standard_normal((nbi * nbj, NCj, NCi))
    a = np.sqrt(GAMMA_AIR)

    def W_fn(x, y, b):
        return np.stack([1.0 + 0.05 * noise[b], np.full_like(x, 2.0 * a), np.zeros_like(x),
                         np.ones_like(x)])

    return structured(nbi, nbj, nc, nc, nodes, True, True, W_fn=W_fn,
                      scheme=scheme or Scheme(cfl=0.5, n_stage=2),
                      name=f"curvilinear_mach2_{nbi}x{nbj}x{nc}^2")


def channel(nbi=2, nbj=2, nci=8, ncj=6, bc=None, seed=7, mach=0.5, scheme=None,
            skew=0.15) -> BlockSet:
    """Small skewed channel [0,2]x[0,1] with physical boundaries on all
    sides, for boundary-condition parity cases.  Default BCs: W fixed inflow,
    E constant extrapolation, S/N reflection.  Initial state: freestream at
    `mach` plus a seeded smooth perturbation (PCG64(seed): 4 amplitudes
    U(-0.05, 0.05) then 4 phases U(0, 2pi))."""
    rng = np.random.Generator(np.random.PCG64(seed))
    amps = rng.uniform(-0.05, 0.05, 4)
    ph = rng.uniform(0, 2 * np.pi, 4)
    nx, ny = nbi * nci, nbj * ncj
    hx, hy = 2.0 / nx, 1.0 / ny
    a = np.sqrt(GAMMA_AIR)
    free = (1.0, mach * a, 0.0, 1.0)
    bc = bc or dict(W=BC_FIXED, E=BC_CONSTANT_EXTRAPOLATION, S=BC_REFLECTION, N=BC_REFLECTION)
    wo = dict(W=free, E=free, S=free, N=free)

    def nodes(I, J):
        x0, y0 = I * hx, J * hy
        return x0 + skew * hx * np.sin(np.pi * y0) * np.cos(1.3 * x0), \
            y0 + skew * hy * np.sin(2.1 * x0) * np.sin(np.pi * y0)

    def W_fn(x, y, b):
        d = 1.0 + amps[0] * np.sin(3 * x + ph[0]) * np.cos(2 * y + ph[1])
        u = mach * a * (1.0 + amps[1] * np.cos(2 * x + ph[2]))
        v = 0.1 * amps[2] * np.sin(4 * y + ph[3])
        p = 1.0 + amps[3] * np.cos(3 * y + 2 * x)
        return np.stack([d, u, v, p])

    return structured(nbi, nbj, nci, ncj, nodes, False, False, bc=bc, wo=wo, W_fn=W_fn,
                      scheme=scheme or Scheme(cfl=0.5, n_stage=2, local_dt=0),
                      name=f"channel_{nbi}x{nbj}x{nci}x{ncj}")


def bump_channel(nbi=12, nbj=4, nci=64, ncj=32, h=0.1, mach=0.5, bc=None, scheme=None,
                 stretch=0.0) -> BlockSet:
    """Channel [-1.5,1.5]x[0,1] with a bump y = h*sin^2(pi*(x+0.5)) on the
    lower wall for |x| <= 0.5; nbi x nbj blocks of nci x ncj cells.  Nodes:
    x uniform, y = y_w(x) + eta*(1 - y_w(x)), eta = J/(nbj*ncj) (optionally
    clustered to the wall by `stretch`); ghost nodes continue the same map.
    Freestream rho = p = 1 at `mach`.  Default BCs: characteristic inflow /
    outflow (W, E) with the freestream as reference state, reflecting walls
    (S, N).  Steady-state scheme: local time stepping."""
    nx, ny = nbi * nci, nbj * ncj
    a = np.sqrt(GAMMA_AIR)
    free = (1.0, mach * a, 0.0, 1.0)
    bc = bc or dict(W=BC_CHARACTERISTIC, E=BC_CHARACTERISTIC, S=BC_REFLECTION, N=BC_REFLECTION)

    def wall(x):
        return np.where(np.abs(x) <= 0.5, h * np.sin(np.pi * (x + 0.5)) ** 2, 0.0)

    def nodes(I, J):
        x = -1.5 + 3.0 * I / nx
        eta = J / ny
        if stretch:
            eta = np.sinh(stretch * eta) / np.sinh(stretch)
        yw = wall(x)
        return x, yw + eta * (1.0 - yw)

    def W_fn(x, y, b):
        return np.stack([np.full_like(x, free[0]), np.full_like(x, free[1]),
                         np.full_like(x, free[2]), np.full_like(x, free[3])])

    return structured(nbi, nbj, nci, ncj, nodes, False, False, bc=bc,
                      wo=dict(W=free, E=free, S=free, N=free), W_fn=W_fn,
                      scheme=scheme or Scheme(cfl=1.0, n_stage=2, local_dt=1),
                      name=f"bump_channel_{nbi}x{nbj}x{nci}x{ncj}")


# ---------------------------------------------------------------------------
# Case-file serialisation (the format read by the reference harness; the
# layout is documented in the harness source).
_MAGIC = 0x43443245


def write_case(path: str, bs: BlockSet, W: np.ndarray | None = None) -> None:
    sc = bs.scheme
    W = bs.W if W is None else W
    with open(path, "wb") as f:
        f.write(struct.pack("<2i", _MAGIC, 2))
        f.write(struct.pack("<4i", bs.nblk, bs.nci, bs.ncj, bs.ng))
        f.write(struct.pack("<8i", sc.limiter, sc.flux, sc.n_stage, sc.local_dt, 1,
                            bs.nbi, bs.nbj, bs.periodic))
        f.write(struct.pack("<4d", sc.cfl, sc.rs_epsilon, sc.freeze_level, 0.0))
        f.write(struct.pack("<4i", sc.time_integration, sc.rs_iterations, sc.freeze_limiter, 0))
        for b in range(bs.nblk):
            f.write(bs.neighbour[b].astype("<i4").tobytes())
            for a in (bs.bc_w, bs.bc_e, bs.bc_s, bs.bc_n):
                f.write(a[b].astype("<i4").tobytes())
            f.write(bs.node_x[b].astype("<f8").tobytes())
            f.write(bs.node_y[b].astype("<f8").tobytes())
            for a in (bs.wo_w, bs.wo_e, bs.wo_s, bs.wo_n):
                f.write(a[b].astype("<f8").tobytes())
            f.write(np.ascontiguousarray(W[b]).astype("<f8").tobytes())


def read_case(path: str) -> BlockSet:
    """Reads a case file written by write_case (or by the C++ host layer's
    Write_Case_File) back into a BlockSet."""
    buf = open(path, "rb").read()
    magic, version = struct.unpack_from("<2i", buf, 0)
    if magic != _MAGIC or version not in (1, 2):
        raise ValueError(f"{path}: not a case file")
    nblk, nci, ncj, ng = struct.unpack_from("<4i", buf, 8)
    limiter, flux, n_stage, local_dt, _, nbi, nbj, periodic = struct.unpack_from("<8i", buf, 24)
    cfl, rs_eps, fz_level, _ = struct.unpack_from("<4d", buf, 56)
    tint, rs_it, fz = struct.unpack_from("<3i", buf, 88) if version == 2 else (0, 2, 0)
    NCi, NCj = nci + 2 * ng, ncj + 2 * ng
    NNi, NNj = NCi + 1, NCj + 1
    off = 104 if version == 2 else 88
    arrays = {k: [] for k in ("neighbour", "bc_w", "bc_e", "bc_s", "bc_n", "node_x", "node_y",
                              "wo_w", "wo_e", "wo_s", "wo_n", "W")}

    def take(dtype, shape):
        nonlocal off
        n = int(np.prod(shape))
        a = np.frombuffer(buf, dtype=dtype, count=n, offset=off).reshape(shape)
        off += n * np.dtype(dtype).itemsize
        return a.copy()

    for _ in range(nblk):
        arrays["neighbour"].append(take("<i4", (8,)))
        for k, n in (("bc_w", NCj), ("bc_e", NCj), ("bc_s", NCi), ("bc_n", NCi)):
            arrays[k].append(take("<i4", (n,)))
        arrays["node_x"].append(take("<f8", (NNj, NNi)))
        arrays["node_y"].append(take("<f8", (NNj, NNi)))
        for k, n in (("wo_w", NCj), ("wo_e", NCj), ("wo_s", NCi), ("wo_n", NCi)):
            arrays[k].append(take("<f8", (4, n)))
        arrays["W"].append(take("<f8", (4, NCj, NCi)))
    a = {k: np.stack(v) for k, v in arrays.items()}
    scheme = Scheme(limiter=limiter, flux=flux, n_stage=n_stage, local_dt=local_dt, cfl=cfl,
                    time_integration=tint, rs_epsilon=rs_eps, rs_iterations=rs_it, freeze_limiter=fz,
                    freeze_level=fz_level)
    return BlockSet(nci, ncj, a["neighbour"], a["bc_w"], a["bc_e"], a["bc_s"], a["bc_n"], a["node_x"],
                    a["node_y"], a["wo_w"], a["wo_e"], a["wo_s"], a["wo_n"], a["W"], scheme,
                    os.path.basename(path), ng, nbi, nbj, periodic).contiguous()


# block layouts of the batched sweep: 8 to 96 blocks of 32 x 32 cells
LAYOUTS_8_96 = ((4, 2), (6, 2), (8, 2), (6, 3), (8, 3), (12, 2), (8, 4), (12, 4), (16, 4), (12, 6), (16, 6))


def bump_family(n_cases: int, seed: int = 20261205, mach=(1.35, 1.6), height=(0.02, 0.045),
                layouts=((4, 2), (6, 2), (8, 2), (6, 3), (8, 3), (12, 2), (8, 4), (12, 4)), nc: int = 32,
                precision: int = 0) -> list:
    """A sweep of steady supersonic bump-channel cases for batched solves:
    per case (PCG64(seed), in this order) Mach ~ U(mach), bump height ~
    U(height) and a block layout drawn from `layouts` (nbi x nbj blocks of
    nc x nc cells: 8 to 48 blocks).  First order (limiter zero), local time
    stepping: the configuration the reference's block-Jacobi Newton-Krylov
    drives to a 1e-10 residual drop."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for k in range(n_cases):
        m = rng.uniform(*mach)
        h = rng.uniform(*height)
        nbi, nbj = layouts[int(rng.integers(len(layouts)))]
        bs = bump_channel(nbi=nbi, nbj=nbj, nci=nc, ncj=nc, mach=m, h=h,
                          scheme=Scheme(limiter=LIMITER_ZERO, local_dt=1, precision=precision))
        bs.name = f"bump_m{m:.3f}_h{h:.4f}_{nbi}x{nbj}"
        out.append(bs)
    return out
