// e2d_march.cuh — the column-marching stage kernel of the fast FP64 and FP32
// paths: the same residual / explicit stage / Frechet product as
// stage_kernel (e2d_stage.cuh), restating the same reference routines
//   Linear_Reconstruction_LeastSquares   src_2D/Euler2D/Euler2DQuadSingleBlock.cc:3678-4087
//   Euler2D_Quad_Block::dUdt_Residual_Evaluation   src_2D/Euler2D/Euler2DQuad.cc:814-1227
//   Euler2D_Quad_Block::dUdt_Multistage_Explicit   src_2D/Euler2D/Euler2DQuad.cc:1235-1727
//   Update_Solution_Multistage_Explicit   src_2D/Euler2D/Euler2DQuadSingleBlock.cc:5300-5507
// but organised for the hardware:
//
// * Work: a block is cut into column strips of MI = 32 interior cells, a
//   strip into chunks of ch rows (ch <= 8, chosen per block shape by the
//   handle's autotuner; the last chunk of a strip takes a remainder that fits
//   in 8 rows).  With 8 warps a chunk of 7 rows reconstructs its 7 rows and
//   their 2 edge columns in one round, its 15 face rows in two and updates in
//   one.  The launch is persistent: CTA k takes
//   a contiguous range of the (block, strip, chunk) list, so every SM gets the
//   same number of chunks to within one, and marches up its strips.
// * Reuse along j: the one-cell reconstruction ring and the bottom j-face row
//   a chunk needs were computed by the chunk below; they are carried in
//   shared memory, so each cell is reconstructed once (plus the 2 ring columns
//   of its strip) and each face evaluated once.
// * Staging: the chunk's window of primitive state (36 x 12 cells, 4
//   variables), centroids and nodes arrives through three TMA tensor copies
//   issued by one thread and completing on an mbarrier.  With two staging
//   buffers (E2D_MARCH_NBUF 2) the next chunk's copies are issued before the
//   current chunk is computed; with one, after the chunk's faces, and the
//   other CTA on the SM covers the copy latency.
// * Faces: an i-face and a j-face item differ only in their cells, edge and
//   destination and share one flux evaluation; a chunk that reaches no block
//   edge with a face-setting boundary condition (reflection, characteristic:
//   a mask of sides per block) evaluates its faces without the BC codes.
// * Geometry is not recomputed per stage: centroids, the least-squares
//   inverse of each cell's stencil, 1/area and the CFL lengths were computed
//   once per handle (e2d_march_args.h); face normals and lengths come from
//   the staged nodes with one reciprocal square root per face.
//
// The exact build (no E2D_FAST, compiled without FMA contraction) restates
// the reference's arithmetic instead: the least-squares sums averaged over
// the stencil and divided by the determinant, the limiter over the face-point
// values, IEEE division and square root, the Roe flux of e2d_device.cuh, and
// each face's flux times its length divided by the area in the reference's
// order (so the faces keep flux and length apart).  Its per-handle geometry
// holds the quantities the reference computes from the grid alone, in its
// order (e2d_march_args.h), and its results equal stage_kernel's bit for bit.
//
// Used when the block set allows it (even nci, no degenerate edges), for
// every flux function (the Roe flux in an instance of its own);
// stage_kernel covers the other block sets.
#pragma once
#include "e2d_march_args.h"
#include "e2d_tc.cuh"

namespace e2d {
namespace E2D_NS {
namespace mk {

#ifndef E2D_MARCH_COLS
#define E2D_MARCH_COLS 32
#endif
#ifndef E2D_MARCH_THREADS
#define E2D_MARCH_THREADS 256
#endif
constexpr int MI = E2D_MARCH_COLS, MJ = 8, CH = 7;  // interior columns; rows of a chunk (at most; default)
constexpr int WI = MI + 4, WJ = MJ + 4, NWI = MI + 6;  // staged window (cells, node columns)
constexpr int RCI = MI + 2, RCJ = MJ + 2;          // reconstruction slots (cols, rows j0+1..j0+10)
#ifndef E2D_MARCH_NBUF
#define E2D_MARCH_NBUF 2
#endif
constexpr int THREADS = E2D_MARCH_THREADS, NWARP = THREADS / 32;
#ifdef E2D_MARCH_MINCTAS
constexpr int MIN_CTAS = E2D_MARCH_MINCTAS;
#else
constexpr int MIN_CTAS = 65536 / (128 * THREADS);                     // CTAs per SM at 128 registers
#endif
constexpr int NBUF = E2D_MARCH_NBUF;  // staging buffers: 2 = the next chunk's copies overlap this chunk
#ifndef E2D_MARCH_UPD
#define E2D_MARCH_UPD 0
#endif
// E2D_MARCH_UPD 1: the explicit stages' update inputs of a chunk (base state,
// stage-1 residual, the area plane and the CFL geometry) arrive in shared memory by TMA
// while the chunk's faces are evaluated, instead of as global loads in the
// update (whose latency every warp meets at once after the phase barrier)
constexpr bool UPD = E2D_MARCH_UPD;
constexpr uint32_t WAIT_ITERS = 1u << 24;          // bounded mbarrier wait (about a second)
constexpr int ST_TIMEOUT = 2;                      // status code: a staging wait ran out

// geometry planes of the window: centroid x, y and the least-squares
// inverse K0, K1, K2 (planes G_XC .. G_K2 of the per-handle geometry)
constexpr int TG = G_K2 + 1;
struct Tile {
  double W[4][WJ][WI];   // primitive state, rows j0 .. j0+11, cols i0 .. i0+35
  double G[TG][WJ][WI];  // centroids, least-squares inverse
  double N[2][WJ][NWI];  // nodes, cols i0 .. i0+37
};
constexpr uint32_t TILE_BYTES = sizeof(double) * ((4 + TG) * WJ * WI + 2 * WJ * NWI);
static_assert(sizeof(Tile) == TILE_BYTES && TILE_BYTES % 128 == 0, "tile packing");
static_assert((4 * WJ * WI * 8) % 128 == 0 && ((4 + TG) * WJ * WI * 8) % 128 == 0, "TMA destinations 128-byte aligned");
static_assert(THREADS >= MJ * MI, "one thread per update cell");
static_assert(MI % 2 == 0 && (MI * 8) % 16 == 0, "strip origins on 16-byte boundaries");

// Reconstructions and j-face fluxes live in rings indexed by the array row
// (row mod RR): a chunk reads the top reconstruction row and the bottom j-face
// row the chunk below it left there.  Live at once: the reconstruction rows
// j0+1 .. j0+h+2 of the chunk being evaluated (its own and the two carried
// up), at most RCJ; the j-face rows j0+2 .. j0+h+2 of a chunk between its
// faces and its update, at most MJ + 1 (the update of chunk c-1 runs before
// chunk c's faces overwrite any of its rows).
constexpr int RR = RCJ;
static_assert(RR >= RCJ && RR >= MJ + 1, "ring holds the live rows");

// Update inputs of a chunk's cells (rows j0+2 .., columns i0+2 ..): the base
// conserved state, the residual RK stage 2 adds to, and geometry planes
// G_RA .. G_VJY (plane G_RA, 1/A or in the exact build A, alone without the
// fused CFL step).
struct UpdIn {
  double U[4][MJ][MI];
  double R[4][MJ][MI];
  double G[GEOM_NF - G_RA][MJ][MI];
};
static_assert(sizeof(double) * 4 * MJ * MI % 128 == 0, "update buffers 128-byte aligned");

struct Smem {
  Tile in[NBUF];
#if E2D_MARCH_UPD
  UpdIn up;
#endif
  RT px[RR][4][RCI], py[RR][4][RCI];    // phi * gradient of the reconstructed cells
  double Fi[MJ][4][MI + 1];             // i-face flux x length, faces I-1/2, I = i0+2 .. i0+34
  double Fj[RR][4][MI];                 // j-face flux x length, face row J (face J-1/2)
#ifndef E2D_FAST
  double li[MJ][MI + 1], lj[RR][MI];    // exact build: face lengths (Fi, Fj hold the bare fluxes)
#endif
  double red[4][NWARP];
  uint64_t full[2];
  uint64_t fullu;  // the update inputs
  int failed;
};

// neighbour k of the canonical stencil order
__device__ constexpr int KDI[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
__device__ constexpr int KDJ[8] = {-1, -1, -1, 0, 0, 1, 1, 1};

__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(bar)), "r"(bytes)
               : "memory");
}
// 3D tiled tensor copy global -> this CTA's shared memory (no multicast).
__device__ __forceinline__ void tma3(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(tc::smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(tc::smem_addr(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

struct Chunk {
  int b, i0, j0, c, h;  // block, strip origin (interior column), chunk origin (interior row), chunk index, rows
  int r0;               // ring slot of the chunk's first reconstruction row (array row j0+1)
};
__device__ __forceinline__ Chunk decode(const MarchArgs& m, long long g) {
  Chunk k;
  const long long strip = g / m.cps;
  k.c = int(g - strip * m.cps);
  k.b = int(strip / m.strips);
  k.i0 = int(strip - (long long)k.b * m.strips) * MI;
  k.j0 = k.c * m.ch;
  k.h = k.c == m.cps - 1 ? min(MJ, m.a.B.ncj - k.j0) : m.ch;
  k.r0 = (k.j0 + 1) % RR;
  return k;
}

__device__ __forceinline__ PState<RT> wwin(const Tile& T, int wj, int wi) {
  PState<RT> w;
  w.d = RT(T.W[0][wj][wi]); w.u = RT(T.W[1][wj][wi]); w.v = RT(T.W[2][wj][wi]); w.p = RT(T.W[3][wj][wi]);
  return w;
}

// Ring slot of the reconstruction of chunk slot sl (array row j0+1+sl) and
// of j-face slot sl (face row j0+2+sl); r0 + sl < 2 RR (r0 < RR, sl <= RCJ - 1).
__device__ __forceinline__ int rslot(const Chunk& k, int sl) {
  const int r = k.r0 + sl;
  return r >= RR ? r - RR : r;
}
__device__ __forceinline__ int fslot(const Chunk& k, int sl) { return rslot(k, sl + 1); }

// Limited linear state of reconstructed cell (slot sl, column c; window
// (c+1, sl+1)) at the face point (fx, fy).
__device__ __forceinline__ PState<RT> fstate(const Smem& s, const Tile& T, const Chunk& k, int sl, int c, double fx,
                                             double fy) {
  const RT dx = RT(fx - T.G[0][sl + 1][c + 1]), dy = RT(fy - T.G[1][sl + 1][c + 1]);
  PState<RT> w = wwin(T, sl + 1, c + 1);
  const int rs = rslot(k, sl);
  w.d = w.d + s.px[rs][0][c] * dx + s.py[rs][0][c] * dy;
  w.u = w.u + s.px[rs][1][c] * dx + s.py[rs][1][c] * dy;
  w.v = w.v + s.px[rs][2][c] * dx + s.py[rs][2][c] * dy;
  w.p = w.p + s.px[rs][3][c] * dx + s.py[rs][3][c] * dy;
  return w;
}

// The per-cell input of a reconstruction from global memory: its stencil
// mask (loaded before the staging wait, so its latency overlaps it; the
// least-squares inverse arrives with the window).
struct ReconIn {
  unsigned msk;
};
__device__ __forceinline__ ReconIn recon_in(const MarchArgs& m, const Chunk& k, int sl, int c, size_t plane) {
  const Blocks& B = m.a.B;
  ReconIn r{0u};
  const int I = k.i0 + 1 + c, J = k.j0 + 1 + sl;
  if (I > B.nci + 2 || J > B.ncj + 2) return r;
  r.msk = m.mask[size_t(k.b) * plane + size_t(J) * B.NCi + I];
  return r;
}

// Least-squares gradients and limiter of the cell in slot sl, column c.
// frozen: the case's limiters are frozen (Freeze_Limiter): phi is the stored
// one.  With B.dWdx set the gradients and limiter are exported as well.
__device__ __forceinline__ void recon_cell(const MarchArgs& m, Smem& s, const Tile& T, const Chunk& k, int sl, int c,
                                           const ReconIn& in, bool frozen) {
  const Blocks& B = m.a.B;
  const int I = k.i0 + 1 + c, J = k.j0 + 1 + sl;
  if (I > B.nci + 2 || J > B.ncj + 2) return;  // beyond the block's ring: never read
  const unsigned msk = in.msk;
  if (msk == 0) {
#pragma unroll
    for (int v = 0; v < 4; ++v) { s.px[rslot(k, sl)][v][c] = RT(0); s.py[rslot(k, sl)][v][c] = RT(0); }
    if (B.dWdx)
      for (int v = 0; v < 4; ++v) {
        const size_t o = cell_var(B, k.b, v, J, I);
        B.dWdx[o] = 0.0; B.dWdy[o] = 0.0; B.phi[o] = 0.0;
      }
    return;
  }
  const int wi = c + 1, wj = sl + 1;
  // fast builds: the least-squares inverse; exact build: the averaged sums
  // DxDx, DxDy, DyDy of the stencil
  const RT K0 = RT(T.G[G_K0][wj][wi]), K1 = RT(T.G[G_K1][wj][wi]), K2 = RT(T.G[G_K2][wj][wi]);
  const double xc0 = T.G[0][wj][wi], yc0 = T.G[1][wj][wi];
  RT w0[4], Sx[4], Sy[4], mn[4], mx[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    w0[v] = RT(T.W[v][wj][wi]);
    Sx[v] = RT(0); Sy[v] = RT(0); mn[v] = w0[v]; mx[v] = w0[v];
  }
  // the full eight-point stencil (every cell away from a boundary condition)
  // as straight-line code, so its shared-memory loads can be issued together;
  // reduced stencils through the mask
  auto add = [&](int q) {
    const int ni = wi + KDI[q], nj = wj + KDJ[q];
    const RT dx = RT(T.G[0][nj][ni] - xc0), dy = RT(T.G[1][nj][ni] - yc0);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const RT w = RT(T.W[v][nj][ni]);
      const RT du = w - w0[v];
      Sx[v] += du * dx;
      Sy[v] += du * dy;
      mn[v] = dmin(mn[v], w);
      mx[v] = dmax(mx[v], w);
    }
  };
  if (msk == 0xFFu) {
#pragma unroll
    for (int q = 0; q < 8; ++q) add(q);
  } else {
#pragma unroll 1
    for (int q = 0; q < 8; ++q)
      if (msk & (1u << q)) add(q);
  }
  // face midpoints E, W, N, S of the cell, relative to its centroid
  const double x00 = T.N[0][wj][wi], y00 = T.N[1][wj][wi], x10 = T.N[0][wj][wi + 1], y10 = T.N[1][wj][wi + 1];
  const double x01 = T.N[0][wj + 1][wi], y01 = T.N[1][wj + 1][wi];
  const double x11 = T.N[0][wj + 1][wi + 1], y11 = T.N[1][wj + 1][wi + 1];
  const RT ofx[4] = {RT(HALF * (x10 + x11) - xc0), RT(HALF * (x00 + x01) - xc0), RT(HALF * (x01 + x11) - xc0),
                     RT(HALF * (x00 + x10) - xc0)};
  const RT ofy[4] = {RT(HALF * (y10 + y11) - yc0), RT(HALF * (y00 + y01) - yc0), RT(HALF * (y01 + y11) - yc0),
                     RT(HALF * (y00 + y10) - yc0)};
  const int rs = rslot(k, sl);
#ifdef E2D_FAST
  if (!frozen && !B.freeze && !B.dWdx && B.limiter == E2D_LIMITER_VENKATAKRISHNAN) {
    // the common case (uniform): Venkatakrishnan, no freezing, no export
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const RT gx = Sx[v] * K0 + Sy[v] * K1;
      const RT gy = Sx[v] * K1 + Sy[v] * K2;
      RT dq[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) dq[q] = gx * ofx[q] + gy * ofy[q];
      const RT phi = fm::limiter_diff_k<E2D_LIMITER_VENKATAKRISHNAN>(dq, mn[v] - w0[v], mx[v] - w0[v]);
      s.px[rs][v][c] = phi * gx;
      s.py[rs][v][c] = phi * gy;
    }
    return;
  }
#else
  // the reference's sums are averages over the stencil's n points (x / 8 and
  // x * 0.125 round alike: both are the correctly rounded x / 8)
  const int np = __popc(msk);
  if (np == 8) {
#pragma unroll
    for (int v = 0; v < 4; ++v) { Sx[v] = Sx[v] * 0.125; Sy[v] = Sy[v] * 0.125; }
  } else {
    const double dn = double(np);
#pragma unroll
    for (int v = 0; v < 4; ++v) { Sx[v] = Sx[v] / dn; Sy[v] = Sy[v] / dn; }
  }
  const double det = K0 * K2 - K1 * K1;
#endif
#pragma unroll
  for (int v = 0; v < 4; ++v) {
#ifdef E2D_FAST
    const RT gx = Sx[v] * K0 + Sy[v] * K1;
    const RT gy = Sx[v] * K1 + Sy[v] * K2;
    RT dq[4];  // unlimited change from the centroid to each face point
#pragma unroll
    for (int q = 0; q < 4; ++q) dq[q] = gx * ofx[q] + gy * ofy[q];
#else
    const double gx = (Sx[v] * K2 - Sy[v] * K1) / det;
    const double gy = (Sy[v] * K0 - Sx[v] * K1) / det;
    double uq[4];  // unlimited state at each face point
#pragma unroll
    for (int q = 0; q < 4; ++q) uq[q] = w0[v] + gx * ofx[q] + gy * ofy[q];
#endif
    RT phi;
    if (frozen) {
      phi = RT(B.phi_keep[cell_var(B, k.b, v, J, I)]);
    } else {
#ifdef E2D_FAST
      phi = fm::limiter_diff<RT>(B.limiter, dq, mn[v] - w0[v], mx[v] - w0[v]);
#else
      phi = limiter(B.limiter, uq, w0[v], mn[v], mx[v]);
#endif
      if (B.freeze) B.phi_keep[cell_var(B, k.b, v, J, I)] = double(phi);
    }
    s.px[rs][v][c] = phi * gx;
    s.py[rs][v][c] = phi * gy;
    if (B.dWdx) {
      const size_t o = cell_var(B, k.b, v, J, I);
      B.dWdx[o] = gx; B.dWdy[o] = gy; B.phi[o] = phi;
    }
  }
}

// Face normal, length and midpoint of the edge a -> c (outward normal of the
// cell on the left of a -> c: (dy, -dx) / |d|, d = a - c).
struct FaceGeo {
  double nx, ny, l, mx, my;
};
__device__ __forceinline__ FaceGeo face_geo(double ax, double ay, double cx, double cy) {
  FaceGeo f;
  const double dx = ax - cx, dy = ay - cy;
  const double q = dx * dx + dy * dy;
#ifdef E2D_FAST
  const double rn = fm::rsqrt(q);
  f.l = fm::sqrt_from_rsqrt(q, rn);
  f.nx = dy * rn;
  f.ny = -dx * rn;
#else
  f.l = sqrt(q);
  f.nx = dy / f.l;
  f.ny = -dx / f.l;
#endif
  f.mx = HALF * (cx + ax);
  f.my = HALF * (cy + ay);
  return f;
}

// Face item t of chunk k.  Items [0, ni) are the i-faces I-1/2 of rows
// r = t / (MI+1) (I = i0+2+q, J = j0+2+r), the rest the j-faces J-1/2 of
// slots sl in [sf_lo, h] (J = j0+2+sl, I = i0+2+q).  Both kinds share one
// flux evaluation; only the cells, the edge and the destination differ.  BC:
// the chunk has faces on a block edge whose boundary condition sets the face
// state (otherwise the BC codes are not read).
template <bool BC, bool ROE>
__device__ __forceinline__ void face(const MarchArgs& m, Smem& s, const Tile& T, const Chunk& k, int t, int ni,
                                     int sf_lo) {
  const Blocks& B = m.a.B;
  int ls, lc, rs, rc;  // reconstructed cells on the left / right: slot, column
  int aj, ai, cj, ci;  // window row and node column of the edge's ends a -> c
  double* out;         // flux x length, variable v at out[v * vs]
  int vs;
#ifndef E2D_FAST
  double* lout;        // exact build: the face length (out holds the bare flux)
#endif
  int bcl = E2D_BC_NONE, bcr = E2D_BC_NONE;  // face-setting BC on the left (W, S) / right (E, N) edge
  const double *wol = nullptr, *wor = nullptr;
  int wlen = 0, widx = 0;
  if (t < ni) {
    const int r = t / (MI + 1), q = t - r * (MI + 1);
    const int I = k.i0 + 2 + q, J = k.j0 + 2 + r;
    if (I > B.nci + 2 || J > B.ncj + 1) return;
    // left cell (I-1, J): slot r+1, column q; right cell (I, J): column q+1;
    // nodes (I, J+1) -> (I, J)
    ls = r + 1; lc = q; rs = r + 1; rc = q + 1;
    aj = r + 3; ai = q + 2; cj = r + 2; ci = q + 2;
    out = &s.Fi[r][0][q];
    vs = MI + 1;
#ifndef E2D_FAST
    lout = &s.li[r][q];
#endif
    if (BC) {  // BC codes matter at the block's west and east faces only
      if (I == NG) bcl = B.bcw[size_t(k.b) * B.NCj + J];
      if (I == B.nci + NG) bcr = B.bce[size_t(k.b) * B.NCj + J];
      wol = B.wow; wor = B.woe; wlen = B.NCj; widx = J;
    }
  } else {
    const int u = t - ni, sl = sf_lo + u / MI, q = u % MI;
    const int I = k.i0 + 2 + q, J = k.j0 + 2 + sl;
    if (I > B.nci + 1 || J > B.ncj + 2) return;
    // lower cell (I, J-1): slot sl, column q+1; upper cell (I, J): slot
    // sl+1; nodes (I, J) -> (I+1, J)
    ls = sl; lc = q + 1; rs = sl + 1; rc = q + 1;
    aj = sl + 2; ai = q + 2; cj = sl + 2; ci = q + 3;
    out = &s.Fj[fslot(k, sl)][0][q];
    vs = MI;
#ifndef E2D_FAST
    lout = &s.lj[fslot(k, sl)][q];
#endif
    if (BC) {
      if (J == NG) bcl = B.bcs[size_t(k.b) * B.NCi + I];
      if (J == B.ncj + NG) bcr = B.bcn[size_t(k.b) * B.NCi + I];
      wol = B.wos; wor = B.won; wlen = B.NCi; widx = I;
    }
  }
  const FaceGeo f = face_geo(T.N[0][aj][ai], T.N[1][aj][ai], T.N[0][cj][ci], T.N[1][cj][ci]);
  const RT g = RT(B.g), gm1 = RT(B.gm1), gm1i = RT(B.gm1i);
  PState<RT> wl, wr;
  if (BC && face_bc(bcl)) {
    wr = fstate(s, T, k, rs, rc, f.mx, f.my);
    wl = (bcl == E2D_BC_REFLECTION) ? reflect(wr, RT(-f.nx), RT(-f.ny))
                                    : bc_char_pressure(wr, load_wo(wol, k.b, wlen, widx), RT(-f.nx), RT(-f.ny), g, gm1i);
  } else if (BC && face_bc(bcr)) {
    wl = fstate(s, T, k, ls, lc, f.mx, f.my);
    wr = (bcr == E2D_BC_REFLECTION) ? reflect(wl, RT(f.nx), RT(f.ny))
                                    : bc_char_pressure(wl, load_wo(wor, k.b, wlen, widx), RT(f.nx), RT(f.ny), g, gm1i);
  } else {
    wl = fstate(s, T, k, ls, lc, f.mx, f.my);
    wr = fstate(s, T, k, rs, rc, f.mx, f.my);
  }
  const CState<RT> F = face_flux<ROE>(B.flux, wl, wr, RT(f.nx), RT(f.ny), g, gm1, gm1i);
#ifdef E2D_FAST
  out[0] = double(F.d) * f.l;
  out[vs] = double(F.mx) * f.l;
  out[2 * vs] = double(F.my) * f.l;
  out[3 * vs] = double(F.E) * f.l;
#else
  out[0] = F.d;
  out[vs] = F.mx;
  out[2 * vs] = F.my;
  out[3 * vs] = F.E;
  *lout = f.l;
#endif
}

// Contributions of the CTA's cells to the next step's CFL minimum and
// residual norms of case cs, added into the step history.
__device__ __forceinline__ void flush_next(const StageArgs& a, Smem& s, int cs, double dt_next, double n1, double n2,
                                           double nmax) {
  const int tid = threadIdx.x;
  for (int o = 16; o > 0; o >>= 1) {
    dt_next = dmin(dt_next, __shfl_xor_sync(0xffffffffu, dt_next, o));
    n1 += __shfl_xor_sync(0xffffffffu, n1, o);
    n2 += __shfl_xor_sync(0xffffffffu, n2, o);
    nmax = dmax(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
  }
  if ((tid & 31) == 0) {
    s.red[0][tid >> 5] = dt_next; s.red[1][tid >> 5] = n1; s.red[2][tid >> 5] = n2; s.red[3][tid >> 5] = nmax;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < NWARP; ++w) {
      dt_next = dmin(dt_next, s.red[0][w]); n1 += s.red[1][w]; n2 += s.red[2][w]; nmax = dmax(nmax, s.red[3][w]);
    }
    double* next = const_cast<double*>(a.hist) + 4 * ((*a.step + 1) * a.B.ncase + cs);
    atomicMin(reinterpret_cast<unsigned long long*>(next), (unsigned long long)__double_as_longlong(dt_next));
    atomicAdd(next + 1, n1);
    atomicAdd(next + 2, n2);
    atomicMax(reinterpret_cast<unsigned long long*>(next + 3), (unsigned long long)__double_as_longlong(nmax));
  }
  __syncthreads();
}

// Flux divergence and update of cell (row r, column q) of chunk k (case cs):
// dUdt from the chunk's face fluxes, then per MODE the residual, the Frechet
// product or the explicit update with its positivity back-off and, fused, the
// cell's CFL step and density-residual contributions to the next step.
// Non-positive density, total energy or specific internal energy (the
// reference's test U.d <= 0 || U.E <= 0 || U.e() <= 0, with e <= 0 taken as
// E d - (mx^2 + my^2) / 2 <= 0 for d > 0: no division).
__device__ __forceinline__ double e_times_d2(const CState<double>& u) {
  return u.E * u.d - 0.5 * (u.mx * u.mx + u.my * u.my);
}
__device__ __forceinline__ bool not_positive(const CState<double>& u) {
#ifdef E2D_FAST
  return u.d <= 0.0 || u.E <= 0.0 || e_times_d2(u) <= 0.0;
#else
  return u.d <= 0.0 || u.E <= 0.0 || e_of_U(u) <= 0.0;
#endif
}
__device__ __forceinline__ bool positive(const CState<double>& u) {
#ifdef E2D_FAST
  return u.d > 0.0 && u.E > 0.0 && e_times_d2(u) > 0.0;
#else
  return u.d > 0.0 && u.E > 0.0 && e_of_U(u) > 0.0;
#endif
}

// dtg: the case's global time step of this explicit step (modes 1, 2 with
// global time stepping).
// up: the chunk's update inputs in shared memory (null: global loads).
// PLAIN: the common explicit stage (up set, global time step, no RK4 slot
// combination, no residual-only stage), with those tests compiled out.
template <int MODE, bool FUSE, bool PLAIN>
__device__ __forceinline__ void update_cell(const MarchArgs& m, const Smem& s, const Chunk& k, int cs, int r, int q,
                                            size_t plane, double dtg, const UpdIn* up, double& dt_next, double& n1,
                                            double& n2, double& nmax) {
  const StageArgs& a = m.a;
  const Blocks& B = a.B;
  const int I = k.i0 + NG + q, J = k.j0 + NG + r;
  if (I > B.nci + 1 || J > B.ncj + 1) return;
  const double g = B.g, gm1 = B.gm1;
  // offsets of the cell: in its block's plane, in the scalar arrays, and of
  // variable 0 in the [nblk][4][NCj][NCi] arrays (variable v: + v * plane)
  const size_t off = size_t(J) * B.NCi + I;
  const size_t c = size_t(k.b) * plane + off;
  const size_t c0 = size_t(k.b) * 4 * plane + off;
  const double* gp = m.geom + size_t(k.b) * GEOM_NF * plane + off;
  const bool su = PLAIN || up != nullptr;  // update inputs in shared memory
  const bool ldt = !PLAIN && B.local_dt;
  // plane G_RA: 1 / A (fast builds), A (exact build)
  const double gA = su ? up->G[0][r][q] : gp[G_RA * plane];
  double kk = 1.0;
  if (MODE == 1 || MODE == 2) kk = B.cfl * (ldt ? B.dt[c] : dtg);
#ifdef E2D_FAST
  const double kA = kk * gA;
#endif
  const int fs = fslot(k, r), fn = fslot(k, r + 1);
  double res[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    double d = 0.0;
    if (MODE == 2) {
      const size_t qv = c0 + v * plane;
      d = su ? up->R[v][r][q] : a.res_out[qv];
      if (!PLAIN && a.acc1) d = d + 2.0 * a.acc1[qv] + 2.0 * a.acc2[qv];
    }
#ifdef E2D_FAST
    d += s.Fi[r][v][q] * kA;
    d -= s.Fi[r][v][q + 1] * kA;
    d += s.Fj[fs][v][q] * kA;
    d -= s.Fj[fn][v][q] * kA;
#else
    // faces W, E, S, N: (k F) l / A each, in the reference's order
    if (MODE == 1 || MODE == 2) {
      d += kk * s.Fi[r][v][q] * s.li[r][q] / gA;
      d -= kk * s.Fi[r][v][q + 1] * s.li[r][q + 1] / gA;
      d += kk * s.Fj[fs][v][q] * s.lj[fs][q] / gA;
      d -= kk * s.Fj[fn][v][q] * s.lj[fn][q] / gA;
    } else {
      d += s.Fi[r][v][q] * s.li[r][q] / gA;
      d -= s.Fi[r][v][q + 1] * s.li[r][q + 1] / gA;
      d += s.Fj[fs][v][q] * s.lj[fs][q] / gA;
      d -= s.Fj[fn][v][q] * s.lj[fn][q] / gA;
    }
#endif
    res[v] = d;
  }
  if (MODE == 0) {
#pragma unroll
    for (int v = 0; v < 4; ++v) B.dUdt[c0 + v * plane] = res[v];
  } else if (MODE == 3) {
    // Frechet derivative (GMRES2D.h:445-488):
    // V = (normalizeR(R) - b)/eps - normalizeUtoR(z * (1/dt))
    const double eps = a.nks_eps[cs];
    const double rdt = 1.0 / B.dt[c];
    const size_t qv = c * 4;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double val = (res[v] / a.normR[v] - a.nks_b[qv + v]) / eps;
      val -= (a.nks_z[qv + v] * rdt) * a.normU[v] / a.normR[v];
      a.nks_v[qv + v] = val;
    }
  } else if (!PLAIN && a.no_update) {
#pragma unroll
    for (int v = 0; v < 4; ++v) a.res_out[c0 + v * plane] = res[v];
  } else {
    // Update_Solution_Multistage_Explicit: U = Uo + omega*dUdt
    CState<double> uo;
    if (su) {
      uo.d = up->U[0][r][q]; uo.mx = up->U[1][r][q]; uo.my = up->U[2][r][q]; uo.E = up->U[3][r][q];
    } else {
      uo.d = a.Ubase[c0]; uo.mx = a.Ubase[c0 + plane];
      uo.my = a.Ubase[c0 + 2 * plane]; uo.E = a.Ubase[c0 + 3 * plane];
    }
    const double omega = a.omega;
    CState<double> u;
    u.d = uo.d + omega * res[0]; u.mx = uo.mx + omega * res[1];
    u.my = uo.my + omega * res[2]; u.E = uo.E + omega * res[3];
    if (not_positive(u)) {
      if (!ldt) {
        set_status(B.status, ST_NEGATIVE, int(c));
      } else {
        double rrf = 1.0, dtc = B.dt[c];
        for (int nr = 1; nr <= 10; ++nr) {
          rrf = HALF * rrf;
          dtc = rrf * dtc;
#pragma unroll
          for (int v = 0; v < 4; ++v) res[v] = rrf * res[v];
          u.d = uo.d + omega * res[0]; u.mx = uo.mx + omega * res[1];
          u.my = uo.my + omega * res[2]; u.E = uo.E + omega * res[3];
          if (positive(u)) break;
        }
        B.dt[c] = dtc;
        if (not_positive(u)) set_status(B.status, ST_NEGATIVE, int(c));
      }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) a.res_out[c0 + v * plane] = res[v];
#ifdef E2D_FAST
    // W(U) (fm::W_of_U) with its reciprocal density kept for the CFL step
    const double rd = fm::rcp(u.d);
    PState<double> w;
    w.d = u.d; w.u = u.mx * rd; w.v = u.my * rd;
    w.p = gm1 * (u.E - 0.5 * (u.mx * u.mx + u.my * u.my) * rd);
#else
    const PState<double> w = W_of_U(u, gm1);
#endif
    a.Uout[c0] = u.d; a.Uout[c0 + plane] = u.mx; a.Uout[c0 + 2 * plane] = u.my; a.Uout[c0 + 3 * plane] = u.E;
    a.Wout[c0] = w.d; a.Wout[c0 + plane] = w.u; a.Wout[c0 + 2 * plane] = w.v; a.Wout[c0 + 3 * plane] = w.p;
    if (FUSE) {
      // CFL of the updated cell (Euler2DQuadSingleBlock.cc:3019-3080)
      auto geo = [&](int f) { return su ? up->G[f - G_RA][r][q] : gp[f * plane]; };
#ifdef E2D_FAST
      const double v_i = w.u * geo(G_VIX) + w.v * geo(G_VIY);
      const double v_j = w.u * geo(G_VJX) + w.v * geo(G_VJY);
      const double c2 = g * w.p * rd;
      const double snd = fm::sqrt_from_rsqrt(c2, fm::rsqrt(c2));
      const double ti = geo(G_DI) * fm::rcp(snd + fabs(v_i));
      const double tj = geo(G_DJ) * fm::rcp(snd + fabs(v_j));
#else
      // v_i = v.(n_E - n_W)/2, v_j = v.(n_N - n_S)/2; d_i / (a + |v_i|)
      const double v_i = HALF * (w.u * geo(G_VIX) + w.v * geo(G_VIY));
      const double v_j = HALF * (w.u * geo(G_VJX) + w.v * geo(G_VJY));
      const double snd = a_of(w, g);
      const double ti = geo(G_DI) / (snd + fabs(v_i));
      const double tj = geo(G_DJ) / (snd + fabs(v_j));
#endif
      const double dtc = dmin(ti, tj);
      if (ldt) B.dt[c] = dtc;
      dt_next = dmin(dt_next, dtc);
      n1 += fabs(res[0]);
      n2 += res[0] * res[0];
      nmax = dmax(nmax, fabs(res[0]));
    }
  }
}

// Schedule of a CTA over its chunks c = g0 .. g1-1: per chunk one phase that
// reconstructs chunk c and updates chunk c-1 (whose face fluxes are complete),
// then one phase that evaluates chunk c's faces; the last chunk's update runs
// after the loop.  Two CTA barriers a chunk (and the staging wait).
// ROE: the kernel instance of the Roe flux; the other instance dispatches
// over the remaining flux functions (face_flux), so neither carries the
// other's registers.
template <int MODE, bool FUSE, bool ROE>
__global__ void __launch_bounds__(THREADS, MIN_CTAS) march_kernel(const __grid_constant__ MarchArgs m) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // TMA destinations want 128-byte alignment: align the base by hand
  const uint32_t base = tc::smem_addr(smem_raw);
  Smem& s = *reinterpret_cast<Smem*>(smem_raw + ((128u - (base & 127u)) & 127u));
  const StageArgs& a = m.a;
  const Blocks& B = a.B;
  const int tid = threadIdx.x;
  const long long g0 = m.nchunk * blockIdx.x / gridDim.x, g1 = m.nchunk * (blockIdx.x + 1) / gridDim.x;
  if (tid == 0) {
    s.failed = *(volatile int*)B.status;
    tc::mbar_init(&s.full[0], 1);
    tc::mbar_init(&s.full[1], 1);
    tc::mbar_init(&s.fullu, 1);
  }
  __syncthreads();
  if (s.failed || g0 >= g1) return;  // an earlier kernel failed: stop marching (uniform)
  const size_t plane = size_t(B.NCi) * B.NCj;

  auto issue = [&](long long gg, int buf) {
    const Chunk k = decode(m, gg);
    uint64_t* bar = &s.full[buf];
    expect_tx(bar, TILE_BYTES);
    tma3(&s.in[buf].W[0][0][0], &m.tmW, bar, k.i0, k.j0, 4 * k.b);
    tma3(&s.in[buf].G[0][0][0], &m.tmG, bar, k.i0, k.j0, GEOM_NF * k.b);
    tma3(&s.in[buf].N[0][0][0], &m.tmN, bar, k.i0, k.j0, 2 * k.b);
  };
  if (tid == 0) issue(g0, 0);
  // update inputs by TMA (explicit stages whose arrays have tensor maps)
  const bool upd = UPD && (MODE == 1 || MODE == 2) && m.upd;
#if E2D_MARCH_UPD
  const UpdIn* upp = upd ? &s.up : nullptr;
#else
  const UpdIn* upp = nullptr;
#endif
  auto issue_upd = [&](const Chunk& k) {
#if E2D_MARCH_UPD
    constexpr uint32_t PLANE_BYTES = sizeof(double) * MJ * MI;
    const uint32_t bytes = PLANE_BYTES * (4 + (MODE == 2 ? 4 : 0) + (FUSE ? GEOM_NF - G_RA : 1));
    expect_tx(&s.fullu, bytes);
    tma3(&s.up.U[0][0][0], &m.tmU, &s.fullu, k.i0 + NG, k.j0 + NG, 4 * k.b);
    if (MODE == 2) tma3(&s.up.R[0][0][0], &m.tmR, &s.fullu, k.i0 + NG, k.j0 + NG, 4 * k.b);
    tma3(&s.up.G[0][0][0], FUSE ? &m.tmGF : &m.tmGA, &s.fullu, k.i0 + NG, k.j0 + NG, GEOM_NF * k.b + G_RA);
#endif
  };
  int upd_issued = 0, upd_waited = 0;  // update-input copies issued / consumed
  // the common explicit stage: update inputs in shared memory, global time
  // step, no RK4 slot combination, no residual-only stage (uniform)
  const bool plain = upp != nullptr && !a.acc1 && !a.no_update && !B.local_dt;

  // the L2 prefetch share of this thread (fixed over the chunks): row pf_r
  // of the chunk, field pf_f (0-3 U, 4 1/A, 5-6 CFL lengths), column pf_c
  constexpr int PER_ROW = MI / 16;
  const int pf_r = tid / (11 * PER_ROW), pf_f = (tid % (11 * PER_ROW)) / PER_ROW;
  const int pf_c = 16 * (tid % PER_ROW);
  // the global time step of case cs for this explicit step
  auto step_dt = [&](int cs) {
    return (MODE == 1 || MODE == 2) && !B.local_dt ? a.hist[4 * ((*a.step) * B.ncase + cs)] : 0.0;
  };

  double dt_next = 1000000.0, n1 = 0.0, n2 = 0.0, nmax = 0.0;  // fused next-step CFL / norms
  int cur_case = -1;  // case the fused contributions belong to
  Chunk pk{};         // chunk whose update is pending (faces done)
  int pcase = -1;     // its case, -1: none pending
  int it = 0;
  for (long long gg = g0; gg < g1; ++gg, ++it) {
    const int buf = NBUF == 2 ? (it & 1) : 0;
    const uint32_t par = NBUF == 2 ? (uint32_t(it >> 1) & 1u) : (uint32_t(it) & 1u);
    const Chunk k = decode(m, gg);
    if (NBUF == 2 && tid == 0 && gg + 1 < g1) {
      tc::fence_async_smem();  // the other buffer's generic reads come before its overwrite
      issue(gg + 1, buf ^ 1);
    }
    // per-block facts of the chunk (uniform), loaded ahead of the staging wait
    const int cs = case_id(B, k.b);
    const bool on = !B.case_active || B.case_active[cs];  // a finished case of a batch: skipped (uniform)
    const bool frozen = B.freeze && B.freeze[cs];
    const unsigned sides = m.bcside[k.b];
    const bool pro = (gg == g0) || (k.c == 0);  // start of a strip: no rows below in the rings
    const int s_lo = pro ? 0 : 2, nrow = k.h + 2 - s_lo;  // reconstruction slots [s_lo, h+2)
    // this chunk's update cells' own inputs into L2 (its update runs one
    // chunk later): every 16th cell of a row per field
    if (MODE != 0 && MODE != 3 && !upd) {
      const int J = k.j0 + NG + pf_r, I = k.i0 + NG + pf_c;
      if (pf_r < k.h && J <= B.ncj + 1 && I <= B.nci + 1) {
        const size_t off = size_t(J) * B.NCi + I;
        if (pf_f < 4) {
          const size_t q = (size_t(k.b) * 4 + pf_f) * plane + off;
          prefetch_l2(a.Ubase + q);
          if (MODE == 2) prefetch_l2(a.res_out + q);
        } else if (pf_f == 4 || FUSE) {
          prefetch_l2(m.geom + (size_t(k.b) * GEOM_NF + (pf_f == 4 ? G_RA : G_DI + pf_f - 5)) * plane + off);
        }
      }
    }
    // this thread's first reconstruction cell: its inputs, ahead of the wait
    ReconIn rin{0u};
    if (tid < nrow * RCI) rin = recon_in(m, k, s_lo + tid / RCI, tid % RCI, plane);
    bool ok = tc::mbar_wait(&s.full[buf], par, WAIT_ITERS);
    if (upd && pcase >= 0) ok = tc::mbar_wait(&s.fullu, uint32_t(upd_waited) & 1u, WAIT_ITERS) && ok;
    if (__syncthreads_or(!ok)) {
      // a staging copy did not complete in time: record it, let the copies
      // in flight land (bounded), and stop
      if (tid == 0) {
        set_status(B.status, ST_TIMEOUT, int(gg));
        tc::mbar_wait(&s.full[buf], par, WAIT_ITERS);
        if (NBUF == 2 && gg + 1 < g1) tc::mbar_wait(&s.full[buf ^ 1], uint32_t((it + 1) >> 1) & 1u, WAIT_ITERS);
        if (upd_issued > upd_waited) tc::mbar_wait(&s.fullu, uint32_t(upd_waited) & 1u, WAIT_ITERS);
      }
      return;
    }
    if (upd && pcase >= 0) ++upd_waited;
    if (FUSE && pcase >= 0 && pcase != cur_case) {
      if (cur_case >= 0) flush_next(a, s, cur_case, dt_next, n1, n2, nmax);
      cur_case = pcase;
      dt_next = 1000000.0; n1 = 0.0; n2 = 0.0; nmax = 0.0;
    }
    const Tile& T = s.in[buf];

    // ---- reconstruction of chunk gg, update of the pending chunk -------------
    {
      // the update items start on a warp boundary: no warp runs both kinds
      const int nrec = on ? nrow * RCI : 0, nupd = pcase >= 0 ? pk.h * MI : 0;
      const int nrec_w = (nrec + 31) & ~31;
      const double dtg = pcase >= 0 ? step_dt(pcase) : 0.0;
      for (int t = tid; t < nrec_w + nupd; t += THREADS) {
        if (t < nrec) {
          const int sl = s_lo + t / RCI, c = t % RCI;
          recon_cell(m, s, T, k, sl, c, t == tid ? rin : recon_in(m, k, sl, c, plane), frozen);
        } else if (t >= nrec_w) {
          const int u = t - nrec_w;
          if (plain)
            update_cell<MODE, FUSE, true>(m, s, pk, pcase, u / MI, u % MI, plane, dtg, upp, dt_next, n1, n2, nmax);
          else
            update_cell<MODE, FUSE, false>(m, s, pk, pcase, u / MI, u % MI, plane, dtg, upp, dt_next, n1, n2, nmax);
        }
      }
    }
    __syncthreads();
    pcase = -1;
    // this chunk's update inputs, now that the pending update has read the
    // buffer; they land while the faces are evaluated
    if (upd && on && tid == 0) {
      tc::fence_async_smem();
      issue_upd(k);
    }
    if (upd && on) ++upd_issued;

    // ---- faces of chunk gg: i-faces (h rows of MI+1), j-faces (slots [sf_lo, h]) ---
    if (on) {
      const int h = k.h, sf_lo = pro ? 0 : 1, ni = h * (MI + 1), nj = (h + 1 - sf_lo) * MI;
      // does the chunk reach a block edge whose boundary condition sets the
      // face state?  (uniform; most chunks do not, and skip the BC codes)
      const bool bc = ((sides & 1u) && k.i0 == 0) || ((sides & 2u) && k.i0 + MI >= B.nci) ||
                      ((sides & 4u) && k.c == 0) || ((sides & 8u) && k.c == m.cps - 1);
      if (bc) {
        for (int t = tid; t < ni + nj; t += THREADS) face<true, ROE>(m, s, T, k, t, ni, sf_lo);
      } else {
        for (int t = tid; t < ni + nj; t += THREADS) face<false, ROE>(m, s, T, k, t, ni, sf_lo);
      }
      pk = k;
      pcase = cs;
    }
    __syncthreads();
    if (NBUF == 1 && tid == 0 && gg + 1 < g1) {
      tc::fence_async_smem();  // this chunk's generic reads come before the overwrite
      issue(gg + 1, 0);
    }
  }
  // the last chunk's update
  if (pcase >= 0) {
    if (FUSE && pcase != cur_case) {
      if (cur_case >= 0) flush_next(a, s, cur_case, dt_next, n1, n2, nmax);
      cur_case = pcase;
      dt_next = 1000000.0; n1 = 0.0; n2 = 0.0; nmax = 0.0;
    }
    if (upd) {
      const bool ok = tc::mbar_wait(&s.fullu, uint32_t(upd_waited) & 1u, WAIT_ITERS);
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          set_status(B.status, ST_TIMEOUT, int(g1));
          tc::mbar_wait(&s.fullu, uint32_t(upd_waited) & 1u, WAIT_ITERS);
        }
        return;
      }
      ++upd_waited;
    }
    const double dtg = step_dt(pcase);
    for (int t = tid; t < pk.h * MI; t += THREADS) {
      if (plain)
        update_cell<MODE, FUSE, true>(m, s, pk, pcase, t / MI, t % MI, plane, dtg, upp, dt_next, n1, n2, nmax);
      else
        update_cell<MODE, FUSE, false>(m, s, pk, pcase, t / MI, t % MI, plane, dtg, upp, dt_next, n1, n2, nmax);
    }
  }
  if (FUSE && cur_case >= 0) flush_next(a, s, cur_case, dt_next, n1, n2, nmax);
}

}  // namespace mk

size_t march_smem_bytes() { return sizeof(mk::Smem) + 128; }

template <int MODE, bool FUSE, bool ROE>
cudaError_t march_one(const MarchArgs& m, int grid, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(mk::march_kernel<MODE, FUSE, ROE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(march_smem_bytes()));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  mk::march_kernel<MODE, FUSE, ROE><<<grid, mk::THREADS, march_smem_bytes(), st>>>(m);
  return cudaGetLastError();
}
// grid: CTAs of the persistent launch (the caller sizes it to the SMs)
template <bool ROE>
cudaError_t launch_march_flux(const MarchArgs& m, int grid, cudaStream_t st) {
  switch (m.a.mode * 2 + (m.a.fuse_next ? 1 : 0)) {
    case 0: return march_one<0, false, ROE>(m, grid, st);
    case 2: return march_one<1, false, ROE>(m, grid, st);
    case 3: return march_one<1, true, ROE>(m, grid, st);
    case 4: return march_one<2, false, ROE>(m, grid, st);
    case 5: return march_one<2, true, ROE>(m, grid, st);
    case 6: return march_one<3, false, ROE>(m, grid, st);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t launch_march(const MarchArgs& m, int grid, cudaStream_t st) {
  return m.a.B.flux == E2D_FLUX_ROE ? launch_march_flux<true>(m, grid, st) : launch_march_flux<false>(m, grid, st);
}
int march_ctas_per_sm() {
  int n = 0;
  if (cudaFuncSetAttribute(mk::march_kernel<1, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(march_smem_bytes())) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mk::march_kernel<1, false, true>, mk::THREADS,
                                                    march_smem_bytes()) != cudaSuccess)
    return 0;
  return n;
}
int march_strip_cols() { return mk::MI; }
int march_chunk_rows() { return mk::CH; }
int march_max_rows() { return mk::MJ; }
int march_window_rows() { return mk::WJ; }
// chunks per strip of ncj rows: ch rows each, a remainder that fits joining
// the last full chunk (at most MJ rows)
int march_chunks(int ncj, int ch) {
  const int n = ncj / ch, r = ncj % ch;
  if (r == 0 || (n > 0 && ch + r <= mk::MJ)) return n;
  return n + 1;
}

}  // namespace E2D_NS
}  // namespace e2d

#if !defined(E2D_FP32)
// ---- per-handle geometry of the marching kernel ------------------------------
// (the FP32 build shares the fast FP64 build's; the exact build computes its
// own planes with the reference's arithmetic)
namespace e2d {
namespace E2D_NS {
namespace mk {

__device__ __forceinline__ void cell_geo(const Blocks& B, int b, int I, int J, double& xc, double& yc, double& A) {
#ifdef E2D_FAST
  fm::quad_centroid(B.X[node_ix(B, b, J, I)], B.Y[node_ix(B, b, J, I)], B.X[node_ix(B, b, J, I + 1)],
                    B.Y[node_ix(B, b, J, I + 1)], B.X[node_ix(B, b, J + 1, I + 1)], B.Y[node_ix(B, b, J + 1, I + 1)],
                    B.X[node_ix(B, b, J + 1, I)], B.Y[node_ix(B, b, J + 1, I)], xc, yc, A);
#else
  quad_centroid(B.X[node_ix(B, b, J, I)], B.Y[node_ix(B, b, J, I)], B.X[node_ix(B, b, J, I + 1)],
                B.Y[node_ix(B, b, J, I + 1)], B.X[node_ix(B, b, J + 1, I + 1)], B.Y[node_ix(B, b, J + 1, I + 1)],
                B.X[node_ix(B, b, J + 1, I)], B.Y[node_ix(B, b, J + 1, I)], xc, yc, A);
#endif
}
__device__ __forceinline__ double node_len(const Blocks& B, int b, int ai, int aj, int ci, int cj) {
  const double dx = B.X[node_ix(B, b, aj, ai)] - B.X[node_ix(B, b, cj, ci)];
  const double dy = B.Y[node_ix(B, b, aj, ai)] - B.Y[node_ix(B, b, cj, ci)];
  const double q = dx * dx + dy * dy;
#ifdef E2D_FAST
  return fm::sqrt_from_rsqrt(q, fm::rsqrt(q));
#else
  return sqrt(q);
#endif
}

// One thread per cell (ghosts included): centroid; for ring cells the
// stencil mask and least-squares inverse; for interior cells 1/A and the CFL
// lengths; and the degenerate-edge test (an edge no longer than 1e-9 of its
// cell's perimeter takes the reference's ihat normal, which the marching
// kernel does not restate: *degenerate is set and the stage kernel is used).
__global__ void geometry_kernel(Blocks B, double* geom, unsigned char* mask, int* degenerate) {
  const long long plane = (long long)B.NCi * B.NCj;
  const long long n = plane * B.nblk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int b = int(t / plane);
    const long long r = t - b * plane;
    const int J = int(r / B.NCi), I = int(r - (long long)J * B.NCi);
    double* gp = geom + size_t(b) * GEOM_NF * plane + r;
    double xc, yc, A;
    cell_geo(B, b, I, J, xc, yc, A);
    gp[G_XC * plane] = xc;
    gp[G_YC * plane] = yc;
    for (int f = G_K0; f < GEOM_NF; ++f) gp[f * plane] = 0.0;
    mask[t] = 0;
    const bool ring = I >= 1 && I <= B.nci + 2 && J >= 1 && J <= B.ncj + 2;
    if (!ring) continue;
    const double lE = node_len(B, b, I + 1, J, I + 1, J + 1), lN = node_len(B, b, I, J + 1, I + 1, J + 1);
    const double lW = node_len(B, b, I, J, I, J + 1), lS = node_len(B, b, I, J, I + 1, J);
    const double per = lE + lN + lW + lS;
    if (!(lE > NANO * per && lN > NANO * per && lW > NANO * per && lS > NANO * per)) atomicOr(degenerate, 1);
    int di[8], dj[8];
    const int np = lsq_stencil(B, b, I, J, di, dj);
    unsigned m = 0;
    double DxDx = 0, DxDy = 0, DyDy = 0;
    for (int k = 0; k < np; ++k) {
      int q = (dj[k] + 1) * 3 + (di[k] + 1);
      if (q > 4) --q;
      m |= 1u << q;
    }
    for (int q = 0; q < 8; ++q) {
      if (!(m & (1u << q))) continue;
      double xn, yn, An;
      cell_geo(B, b, I + KDI[q], J + KDJ[q], xn, yn, An);
      const double dx = xn - xc, dy = yn - yc;
      DxDx += dx * dx; DxDy += dx * dy; DyDy += dy * dy;
    }
    mask[t] = (unsigned char)m;
    if (m) {
#ifdef E2D_FAST
      const double rdet = fm::rcp(DxDx * DyDy - DxDy * DxDy);
      gp[G_K0 * plane] = DyDy * rdet;
      gp[G_K1 * plane] = -DxDy * rdet;
      gp[G_K2 * plane] = DxDx * rdet;
#else
      // the sums averaged over the stencil's points, as the reference
      // divides them (Euler2DQuadSingleBlock.cc:4010-4019)
      const double dn = double(__popc(m));
      gp[G_K0 * plane] = DxDx / dn;
      gp[G_K1 * plane] = DxDy / dn;
      gp[G_K2 * plane] = DyDy / dn;
#endif
    }
    if (I >= NG && I <= B.nci + 1 && J >= NG && J <= B.ncj + 1) {
#ifdef E2D_FAST
      gp[G_RA * plane] = fm::rcp(A);
      gp[G_DI * plane] = 2.0 * A * fm::rcp(lE + lW);
      gp[G_DJ * plane] = 2.0 * A * fm::rcp(lN + lS);
#else
      gp[G_RA * plane] = A;
      gp[G_DI * plane] = 2.0 * (A / (lE + lW));
      gp[G_DJ * plane] = 2.0 * (A / (lN + lS));
#endif
      // outward unit normals nfaceE/W/N/S of the cell (edges a -> c:
      // (dy, -dx) / |d|, d = a - c)
      auto nrm = [&](int ai, int aj, int ci, int cj, double& nx, double& ny) {
        const double dx = B.X[node_ix(B, b, aj, ai)] - B.X[node_ix(B, b, cj, ci)];
        const double dy = B.Y[node_ix(B, b, aj, ai)] - B.Y[node_ix(B, b, cj, ci)];
#ifdef E2D_FAST
        const double rn = fm::rsqrt(dx * dx + dy * dy);
        nx = dy * rn;
        ny = -dx * rn;
#else
        const double n = sqrt(dx * dx + dy * dy);
        nx = dy / n;
        ny = -dx / n;
#endif
      };
      double eX, eY, wX, wY, nX, nY, sX, sY;
      nrm(I + 1, J + 1, I + 1, J, eX, eY);
      nrm(I, J, I, J + 1, wX, wY);
      nrm(I, J + 1, I + 1, J + 1, nX, nY);
      nrm(I + 1, J, I, J, sX, sY);
#ifdef E2D_FAST
      gp[G_VIX * plane] = HALF * (eX - wX);
      gp[G_VIY * plane] = HALF * (eY - wY);
      gp[G_VJX * plane] = HALF * (nX - sX);
      gp[G_VJY * plane] = HALF * (nY - sY);
#else
      // the differences alone: the stage halves their dot product with v
      gp[G_VIX * plane] = eX - wX;
      gp[G_VIY * plane] = eY - wY;
      gp[G_VJX * plane] = nX - sX;
      gp[G_VJY * plane] = nY - sY;
#endif
    }
  }
}

// Per block a bit per side (1 W, 2 E, 4 S, 8 N): at least one of the
// side's edge cells has a boundary condition that sets the face state
// (reflection, characteristic).  One warp per block.
__global__ void bc_side_kernel(Blocks B, unsigned char* side) {
  const int b = blockIdx.x;
  unsigned m = 0;
  for (int J = threadIdx.x; J < B.NCj; J += 32) {
    if (face_bc(B.bcw[size_t(b) * B.NCj + J])) m |= 1u;
    if (face_bc(B.bce[size_t(b) * B.NCj + J])) m |= 2u;
  }
  for (int I = threadIdx.x; I < B.NCi; I += 32) {
    if (face_bc(B.bcs[size_t(b) * B.NCi + I])) m |= 4u;
    if (face_bc(B.bcn[size_t(b) * B.NCi + I])) m |= 8u;
  }
  m = __reduce_or_sync(0xffffffffu, m);
  if (threadIdx.x == 0) side[b] = (unsigned char)m;
}

// Nodes [nblk][NNj][NNi] -> [nblk][2][NNj][NNp] (X, Y; rows padded to NNp).
__global__ void pad_nodes_kernel(Blocks B, int NNp, double* out) {
  const long long plane = (long long)B.NNi * B.NNj;
  const long long n = plane * B.nblk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int b = int(t / plane);
    const long long r = t - b * plane;
    const int j = int(r / B.NNi), i = int(r - (long long)j * B.NNi);
    double* o = out + size_t(b) * 2 * B.NNj * NNp + size_t(j) * NNp + i;
    o[0] = B.X[t];
    o[size_t(B.NNj) * NNp] = B.Y[t];
  }
}

}  // namespace mk

cudaError_t launch_geometry(const Blocks& B, double* geom, unsigned char* mask, unsigned char* bcside, int* degenerate,
                            int NNp, double* nodes_pad, cudaStream_t st) {
  mk::geometry_kernel<<<1024, 256, 0, st>>>(B, geom, mask, degenerate);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  mk::bc_side_kernel<<<B.nblk, 32, 0, st>>>(B, bcside);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  mk::pad_nodes_kernel<<<1024, 256, 0, st>>>(B, NNp, nodes_pad);
  return cudaGetLastError();
}

}  // namespace E2D_NS
}  // namespace e2d
#endif
