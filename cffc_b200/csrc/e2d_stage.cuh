// e2d_stage.cuh — the fused residual / explicit-stage kernel.
//
// One CTA per TI x TJ tile of interior cells of one block.  The CTA stages the
// tile's primitive state with its two-cell halo and the tile's nodes in
// shared memory, computes cell centroids, the least-squares gradients and
// limiter of every cell that touches a tile face, the Roe flux of every face
// of the tile exactly once, and then, per interior cell, the flux divergence
// and (for an RK stage) the solution update — one pass over HBM per stage.
//
// It restates, fused:
//   Linear_Reconstruction_LeastSquares   src_2D/Euler2D/Euler2DQuadSingleBlock.cc:3678-4087
//   Euler2D_Quad_Block::dUdt_Residual_Evaluation   src_2D/Euler2D/Euler2DQuad.cc:814-1227
//   Euler2D_Quad_Block::dUdt_Multistage_Explicit   src_2D/Euler2D/Euler2DQuad.cc:1235-1727
//   Update_Solution_Multistage_Explicit   src_2D/Euler2D/Euler2DQuadSingleBlock.cc:5300-5507
// with each cell's residual accumulated in the reference's loop order
// (west + , east - , south + , north -).
//
// This header is compiled three times: with -fmad=false (namespace
// e2d::exact, bit-identical to the FP64 reference), with contraction on
// (namespace e2d::fast), and with the reconstruction and flux in FP32
// (namespace e2d::f32, E2D_FP32: the staged state, gradients, limiter, face
// states and Roe flux are float; geometry, the flux divergence, the RK update,
// the CFL step and the norms stay FP64).  E2D_NS names the namespace.
#pragma once
#include "e2d_device.cuh"

#ifndef E2D_NS
#error "E2D_NS must name the kernel namespace"
#endif

// The fast path (E2D_FAST) replaces IEEE division and square root by the
// Newton-refined reciprocal / reciprocal square root of e2d_fastmath.cuh and
// uses the division-lean flux, gradient and limiter forms; it is tuned for
// two CTAs per SM.
#ifdef E2D_FAST
#include "e2d_fastmath.cuh"
#ifndef E2D_MIN_CTAS
#define E2D_MIN_CTAS 2
#endif
#ifndef E2D_THREADS
#define E2D_THREADS 320  // measured: +5% over 256 (the face phase fits two rounds)
#endif
#define E2D_QC fm::quad_centroid
#else
#ifndef E2D_MIN_CTAS
#define E2D_MIN_CTAS 1
#endif
#define E2D_QC quad_centroid
#endif
// Threads per CTA: at least one per tile cell; more balance the face and
// reconstruction phases (which have more work items than cells).
#ifndef E2D_THREADS
#define E2D_THREADS 256
#endif

namespace e2d {
namespace E2D_NS {

#ifdef E2D_FP32
using RT = float;   // reconstruction and flux arithmetic
#else
using RT = double;
#endif

#ifndef E2D_TI
#define E2D_TI 32
#endif
#ifndef E2D_TJ
#define E2D_TJ 8
#endif
constexpr int TI = E2D_TI, TJ = E2D_TJ;  // interior cells per tile
constexpr int HI = TI + 4, HJ = TJ + 4; // W tile with 2-cell halo
constexpr int NI = TI + 5, NJ = TJ + 5; // nodes of the halo tile
constexpr int RI = TI + 2, RJ = TJ + 2; // cells reconstructed (tile + 1 ring)
constexpr int NTHREADS = E2D_THREADS;
static_assert(NTHREADS >= TI * TJ && NTHREADS % 32 == 0, "one thread per tile cell at least");

struct Smem {
  RT W[4][HJ][HI];
  double X[NJ][NI], Y[NJ][NI];
  double xc[HJ][HI], yc[HJ][HI];
  RT px[4][RJ][RI], py[4][RJ][RI];   // phi^dWdx, phi^dWdy
  RT Fi[4][TJ][TI + 1], Fj[4][TJ + 1][TI];  // face fluxes
  double li[TJ][TI + 1], lj[TJ + 1][TI];    // face lengths
};

__device__ __forceinline__ bool face_bc(int bc) {
  return bc == E2D_BC_REFLECTION || bc == E2D_BC_CHARACTERISTIC;
}

// Outward normal of the edge a->c with the reference's degenerate-edge test
// (l > NANO * perimeter of the owning cell, else ihat).
__device__ __forceinline__ void edge_normal(double ax, double ay, double cx, double cy, double l,
                                            double perim, double& nx, double& ny) {
  if (l > NANO * perim) {
    const double dx = ax - cx, dy = ay - cy;
#ifdef E2D_FAST
    const double rn = fm::rsqrt(dx * dx + dy * dy);
    nx = dy * rn;
    ny = -dx * rn;
#else
    const double n = sqrt(dx * dx + dy * dy);
    nx = (ay - cy) / n;
    ny = -(ax - cx) / n;
#endif
  } else {
    nx = 1.0; ny = 0.0;
  }
}
__device__ __forceinline__ double edge_len(double ax, double ay, double cx, double cy) {
  const double dx = ax - cx, dy = ay - cy;
#ifdef E2D_FAST
  const double q = dx * dx + dy * dy;
  return fm::sqrt_from_rsqrt(q, fm::rsqrt(q));
#else
  return sqrt(dx * dx + dy * dy);
#endif
}

// Perimeter of halo cell (hi, hj) in the reference's order lE + lN + lW + lS.
__device__ __forceinline__ double cell_perimeter(const Smem& s, int hi, int hj) {
  const double lE = edge_len(s.X[hj][hi + 1], s.Y[hj][hi + 1], s.X[hj + 1][hi + 1], s.Y[hj + 1][hi + 1]);
  const double lN = edge_len(s.X[hj + 1][hi], s.Y[hj + 1][hi], s.X[hj + 1][hi + 1], s.Y[hj + 1][hi + 1]);
  const double lW = edge_len(s.X[hj][hi], s.Y[hj][hi], s.X[hj + 1][hi], s.Y[hj + 1][hi]);
  const double lS = edge_len(s.X[hj][hi], s.Y[hj][hi], s.X[hj][hi + 1], s.Y[hj][hi + 1]);
  return lE + lN + lW + lS;
}
// A cheap upper bound of the perimeter (sum of |dx|+|dy| of the edges): when
// l exceeds NANO times it, the exact test passes too.
__device__ __forceinline__ double perimeter_bound(const Smem& s, int hi, int hj) {
  const double x0 = s.X[hj][hi], y0 = s.Y[hj][hi], x1 = s.X[hj][hi + 1], y1 = s.Y[hj][hi + 1];
  const double x2 = s.X[hj + 1][hi + 1], y2 = s.Y[hj + 1][hi + 1], x3 = s.X[hj + 1][hi], y3 = s.Y[hj + 1][hi];
  return 2.0 * (fabs(x1 - x0) + fabs(y1 - y0) + fabs(x2 - x1) + fabs(y2 - y1) + fabs(x3 - x2) +
                fabs(y3 - y2) + fabs(x0 - x3) + fabs(y0 - y3));
}
__device__ __forceinline__ double perim_for_test(const Smem& s, int hi, int hj, double l) {
  const double pb = perimeter_bound(s, hi, hj);
  return (l > NANO * pb) ? 0.0 : cell_perimeter(s, hi, hj);
}

// Least-squares stencil (Euler2DQuadSingleBlock.cc:3692-3990) of array cell
// (I, J).  Writes offsets (di, dj) relative to the cell in the reference's
// order; returns n_pts.  (Measured: this indexed form runs ~11% faster on
// B200 than an unrolled bit-mask form of the same stencils.)
__device__ __forceinline__ int lsq_stencil(const Blocks& B, int b, int I, int J, int* di, int* dj) {
  const int ICl = NG, ICu = B.nci + NG - 1, JCl = NG, JCu = B.ncj + NG - 1;
  int n = 0;
#define P(a, c) (di[n] = (a), dj[n] = (c), ++n)
#define FULL8 P(-1,-1); P(0,-1); P(1,-1); P(-1,0); P(1,0); P(-1,1); P(0,1); P(1,1)
#define EXTRAP(t) ((t) == E2D_BC_PERIODIC || (t) == E2D_BC_CONSTANT_EXTRAPOLATION || (t) == 4002 || (t) == E2D_BC_CHARACTERISTIC)
  if (I == ICl - NG || I == ICu + NG || J == JCl - NG || J == JCu + NG) return 0;
  const bool westG = (I == ICl - NG + 1), eastG = (I == ICu + NG - 1);
  const bool southG = (J == JCl - NG + 1), northG = (J == JCu + NG - 1);
  if (!(westG || eastG || southG || northG)) { FULL8; return n; }
  const int bw = B.bcw[size_t(b) * B.NCj + J], be = B.bce[size_t(b) * B.NCj + J];
  const int bs = B.bcs[size_t(b) * B.NCi + I], bn = B.bcn[size_t(b) * B.NCi + I];
  if (westG && bw != E2D_BC_NONE) {
    if (southG || northG) return 0;
    if (EXTRAP(bw)) {
      if (J == JCl) { P(-1,0); P(1,0); P(-1,1); P(0,1); P(1,1); }
      else if (J == JCu) { P(-1,-1); P(0,-1); P(1,-1); P(-1,0); P(1,0); }
      else { FULL8; }
    } else {
      if (J == JCl) { P(1,0); P(0,1); P(1,1); }
      else if (J == JCu) { P(0,-1); P(1,-1); P(1,0); }
      else { P(0,-1); P(1,-1); P(1,0); P(0,1); P(1,1); }
    }
  } else if (eastG && be != E2D_BC_NONE) {
    if (southG || northG) return 0;
    if (EXTRAP(be)) {
      if (J == JCl) { P(-1,0); P(1,0); P(-1,1); P(0,1); P(1,1); }
      else if (J == JCu) { P(-1,-1); P(0,-1); P(1,-1); P(-1,0); P(1,0); }
      else { FULL8; }
    } else {
      if (J == JCl) { P(-1,0); P(-1,1); P(0,1); }
      else if (J == JCu) { P(-1,-1); P(0,-1); P(-1,0); }
      else { P(-1,-1); P(0,-1); P(-1,0); P(-1,1); P(0,1); }
    }
  } else if (southG && bs != E2D_BC_NONE) {
    if (westG || eastG) return 0;
    if (EXTRAP(bs)) {
      if (I == ICl) { P(0,-1); P(1,-1); P(1,0); P(0,1); P(1,1); }
      else if (I == ICu) { P(-1,-1); P(0,-1); P(-1,0); P(-1,1); P(0,1); }
      else { FULL8; }
    } else {
      if (I == ICl) { P(1,0); P(0,1); P(1,1); }
      else if (I == ICu) { P(-1,0); P(-1,1); P(0,1); }
      else { P(-1,0); P(1,0); P(-1,1); P(0,1); P(1,1); }
    }
  } else if (northG && bn != E2D_BC_NONE) {
    if (westG || eastG) return 0;
    if (EXTRAP(bn)) {
      if (I == ICl) { P(0,-1); P(1,-1); P(1,0); P(0,1); P(1,1); }
      else if (I == ICu) { P(-1,-1); P(0,-1); P(-1,0); P(-1,1); P(0,1); }
      else { FULL8; }
    } else {
      if (I == ICl) { P(0,-1); P(1,-1); P(1,0); }
      else if (I == ICu) { P(-1,-1); P(0,-1); P(-1,0); }
      else { P(-1,-1); P(0,-1); P(1,-1); P(-1,0); P(1,0); }
    }
  } else {
    FULL8;
  }
#undef P
#undef FULL8
#undef EXTRAP
  return n;
}

// Limited linear face state of halo cell (hi, hj) (recon index hi-1, hj-1)
// at face point (fx, fy): W + (phi^dWdx)*dx + (phi^dWdy)*dy.
__device__ __forceinline__ PState<RT> face_state(const Smem& s, int hi, int hj, double fx, double fy) {
  const RT dx = RT(fx - s.xc[hj][hi]), dy = RT(fy - s.yc[hj][hi]);
  PState<RT> w;
  w.d = s.W[0][hj][hi] + s.px[0][hj - 1][hi - 1] * dx + s.py[0][hj - 1][hi - 1] * dy;
  w.u = s.W[1][hj][hi] + s.px[1][hj - 1][hi - 1] * dx + s.py[1][hj - 1][hi - 1] * dy;
  w.v = s.W[2][hj][hi] + s.px[2][hj - 1][hi - 1] * dx + s.py[2][hj - 1][hi - 1] * dy;
  w.p = s.W[3][hj][hi] + s.px[3][hj - 1][hi - 1] * dx + s.py[3][hj - 1][hi - 1] * dy;
  return w;
}

constexpr double MILLION_D = 1000000.0;

// CFL time step of halo cell (hi, hj) (Euler2DQuadSingleBlock.cc:3038-3048):
// dt = min(d_i / (a + |v_i|), d_j / (a + |v_j|)), d = 2A / (l + l'),
// v_i = v.(n_E - n_W)/2, v_j = v.(n_N - n_S)/2, normals with the cell's own
// degenerate-edge test.
__device__ __forceinline__ double cell_dt(const Smem& s, int hi, int hj, double A, double lE, double lW,
                                          double lN, double lS, const PState<double>& w, double g) {
  const double per = lE + lN + lW + lS;
  double nEx, nEy, nWx, nWy, nNx, nNy, nSx, nSy;
  edge_normal(s.X[hj + 1][hi + 1], s.Y[hj + 1][hi + 1], s.X[hj][hi + 1], s.Y[hj][hi + 1], lE, per, nEx, nEy);
  edge_normal(s.X[hj][hi], s.Y[hj][hi], s.X[hj + 1][hi], s.Y[hj + 1][hi], lW, per, nWx, nWy);
  edge_normal(s.X[hj + 1][hi], s.Y[hj + 1][hi], s.X[hj + 1][hi + 1], s.Y[hj + 1][hi + 1], lN, per, nNx, nNy);
  edge_normal(s.X[hj][hi + 1], s.Y[hj][hi + 1], s.X[hj][hi], s.Y[hj][hi], lS, per, nSx, nSy);
  const double v_i = HALF * (w.u * (nEx - nWx) + w.v * (nEy - nWy));
  const double v_j = HALF * (w.u * (nNx - nSx) + w.v * (nNy - nSy));
#ifdef E2D_FAST
  const double c2 = g * w.p * fm::rcp(w.d);
  const double a = fm::sqrt_from_rsqrt(c2, fm::rsqrt(c2));
  const double d_i = 2.0 * A * fm::rcp(lE + lW), d_j = 2.0 * A * fm::rcp(lN + lS);
  const double ti = d_i * fm::rcp(a + fabs(v_i)), tj = d_j * fm::rcp(a + fabs(v_j));
#else
  const double a = a_of(w, g);
  const double d_i = 2.0 * (A / (lE + lW)), d_j = 2.0 * (A / (lN + lS));
  const double ti = d_i / (a + fabs(v_i)), tj = d_j / (a + fabs(v_j));
#endif
  return dmin(ti, tj);
}

__device__ __forceinline__ PState<RT> load_wo(const double* wo, int b, int len, int k) {
  const double* p = wo + size_t(b) * 4 * len;
  PState<RT> w;
  w.d = RT(p[k]); w.u = RT(p[len + k]); w.v = RT(p[2 * len + k]); w.p = RT(p[3 * len + k]);
  return w;
}

// Flux and limiter of the reconstruction type: the division-lean FP64 forms
// on the fast path, the reference's forms otherwise (FP32 included).
// ROE: the kernel instance of the Roe flux; the other instance dispatches
// over the remaining flux functions, so neither carries the other's registers.
template <bool ROE>
__device__ __forceinline__ CState<RT> face_flux(int kind, const PState<RT>& wl, const PState<RT>& wr, RT nx, RT ny,
                                                RT g, RT gm1, RT gm1i) {
  if (!ROE) return flux_n(kind, wl, wr, nx, ny, g, gm1, gm1i);
#if defined(E2D_FAST)
  return fm::flux_roe_n<RT>(wl, wr, nx, ny, g, gm1, gm1i);
#else
  return flux_roe_n(wl, wr, nx, ny, g, gm1, gm1i);
#endif
}
__device__ __forceinline__ RT cell_limiter(int kind, const RT* uq, RT u0, RT umin, RT umax) {
#if defined(E2D_FAST)
  return fm::limiter<RT>(kind, uq, u0, umin, umax);
#else
  return limiter(kind, uq, u0, umin, umax);
#endif
}

template <int MODE, bool FUSE, bool ROE>
__global__ void __launch_bounds__(NTHREADS, E2D_MIN_CTAS) stage_kernel(StageArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& s = *reinterpret_cast<Smem*>(smem_raw);
  const Blocks& B = a.B;
  const int tid = threadIdx.x;
  const int tiles = a.tiles_i * a.tiles_j;
  const int b = blockIdx.x / tiles;
  const int t = blockIdx.x % tiles;
  const int i0 = (t % a.tiles_i) * TI;   // interior index of the tile's first cell
  const int j0 = (t / a.tiles_i) * TJ;   // == array index of the halo origin
  __shared__ int failed, frozen;
  if (tid == 0) {
    failed = *(volatile int*)B.status;
    frozen = B.freeze ? B.freeze[case_id(B, b)] : 0;
  }
  __syncthreads();
  if (failed) return;  // an earlier kernel failed: stop marching (uniform per CTA)
  const int cs = case_id(B, b);  // the block's case: its slot of the step history
  if (B.case_active && !B.case_active[cs]) return;  // a finished case of a batch (uniform per CTA)
  const double* dtmin_p = a.hist ? a.hist + 4 * ((*a.step) * B.ncase + cs) : nullptr;
  const double g = B.g, gm1 = B.gm1, gm1i = B.gm1i;

  // ---- stage W and nodes (halo tile) --------------------------------------
  for (int q = tid; q < 4 * HJ * HI; q += NTHREADS) {
    const int v = q / (HJ * HI), r = q % (HJ * HI), hj = r / HI, hi = r % HI;
    const int I = i0 + hi, J = j0 + hj;
    s.W[v][hj][hi] = RT((I < B.NCi && J < B.NCj) ? a.Win[cell_var(B, b, v, J, I)] : 0.0);
  }
  for (int q = tid; q < NJ * NI; q += NTHREADS) {
    const int nj = q / NI, ni = q % NI, I = i0 + ni, J = j0 + nj;
    const bool in = I < B.NNi && J < B.NNj;
    s.X[nj][ni] = in ? B.X[node_ix(B, b, J, I)] : 0.0;
    s.Y[nj][ni] = in ? B.Y[node_ix(B, b, J, I)] : 0.0;
  }
  __syncthreads();

  // ---- centroids of the halo tile ------------------------------------------
  for (int q = tid; q < HJ * HI; q += NTHREADS) {
    const int hj = q / HI, hi = q % HI;
    double xc, yc, area;
    E2D_QC(s.X[hj][hi], s.Y[hj][hi], s.X[hj][hi + 1], s.Y[hj][hi + 1], s.X[hj + 1][hi + 1],
                  s.Y[hj + 1][hi + 1], s.X[hj + 1][hi], s.Y[hj + 1][hi], xc, yc, area);
    s.xc[hj][hi] = xc;
    s.yc[hj][hi] = yc;
  }
  __syncthreads();

  // ---- least-squares gradients and limiter of the ring-1 region -----------
  const int nci_t = min(TI, B.nci - i0), ncj_t = min(TJ, B.ncj - j0);
  for (int q = tid; q < RJ * RI; q += NTHREADS) {
    const int rj = q / RI, ri = q % RI;
    const int hi = ri + 1, hj = rj + 1;
    const int I = i0 + hi, J = j0 + hj;
    if (ri > nci_t + 1 || rj > ncj_t + 1) continue;
    int di[8], dj[8];
    const int n = lsq_stencil(B, b, I, J, di, dj);
    if (n == 0) {
      for (int v = 0; v < 4; ++v) { s.px[v][rj][ri] = RT(0); s.py[v][rj][ri] = RT(0); }
      if (B.dWdx)
        for (int v = 0; v < 4; ++v) {
          const size_t o = cell_var(B, b, v, J, I);
          B.dWdx[o] = 0.0; B.dWdy[o] = 0.0; B.phi[o] = 0.0;
        }
      continue;
    }
    RT DUDx[4] = {0, 0, 0, 0}, DUDy[4] = {0, 0, 0, 0}, DxDx = 0, DxDy = 0, DyDy = 0;
    const double xc0 = s.xc[hj][hi], yc0 = s.yc[hj][hi];
    for (int k = 0; k < n; ++k) {
      const RT dx = RT(s.xc[hj + dj[k]][hi + di[k]] - xc0);
      const RT dy = RT(s.yc[hj + dj[k]][hi + di[k]] - yc0);
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const RT DU = s.W[v][hj + dj[k]][hi + di[k]] - s.W[v][hj][hi];
        DUDx[v] += DU * dx;
        DUDy[v] += DU * dy;
      }
      DxDx += dx * dx; DxDy += dx * dy; DyDy += dy * dy;
    }
#if defined(E2D_FP32)
    const RT rdet = RT(1) / (DxDx * DyDy - DxDy * DxDy);
#elif defined(E2D_FAST)
    // the 1/n averaging cancels in the gradient
    const double rdet = fm::rcp(DxDx * DyDy - DxDy * DxDy);
#else
    const double dn = double(n);
#pragma unroll
    for (int v = 0; v < 4; ++v) { DUDx[v] = DUDx[v] / dn; DUDy[v] = DUDy[v] / dn; }
    DxDx = DxDx / dn; DxDy = DxDy / dn; DyDy = DyDy / dn;
    const double det = DxDx * DyDy - DxDy * DxDy;
#endif
    // face midpoints E, W, N, S of the cell
    const double fx[4] = {HALF * (s.X[hj][hi + 1] + s.X[hj + 1][hi + 1]), HALF * (s.X[hj][hi] + s.X[hj + 1][hi]),
                          HALF * (s.X[hj + 1][hi] + s.X[hj + 1][hi + 1]), HALF * (s.X[hj][hi] + s.X[hj][hi + 1])};
    const double fy[4] = {HALF * (s.Y[hj][hi + 1] + s.Y[hj + 1][hi + 1]), HALF * (s.Y[hj][hi] + s.Y[hj + 1][hi]),
                          HALF * (s.Y[hj + 1][hi] + s.Y[hj + 1][hi + 1]), HALF * (s.Y[hj][hi] + s.Y[hj][hi + 1])};
    RT ofx[4], ofy[4];
#pragma unroll
    for (int q2 = 0; q2 < 4; ++q2) { ofx[q2] = RT(fx[q2] - xc0); ofy[q2] = RT(fy[q2] - yc0); }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
#if defined(E2D_FAST) || defined(E2D_FP32)
      const RT gx = (DUDx[v] * DyDy - DUDy[v] * DxDy) * rdet;
      const RT gy = (DUDy[v] * DxDx - DUDx[v] * DxDy) * rdet;
#else
      const double gx = (DUDx[v] * DyDy - DUDy[v] * DxDy) / det;
      const double gy = (DUDy[v] * DxDx - DUDx[v] * DxDy) / det;
#endif
      const RT u0 = s.W[v][hj][hi];
      RT umin = u0, umax = u0;
      for (int k = 0; k < n; ++k) {
        const RT w = s.W[v][hj + dj[k]][hi + di[k]];
        umin = dmin(umin, w);
        umax = dmax(umax, w);
      }
      RT uq[4];
#pragma unroll
      for (int q2 = 0; q2 < 4; ++q2) uq[q2] = u0 + gx * ofx[q2] + gy * ofy[q2];
      RT phi;
      if (frozen) {  // Freeze_Limiter: the limiter of the last reconstruction before freezing
        phi = RT(B.phi_keep[cell_var(B, b, v, J, I)]);
      } else {
        phi = cell_limiter(B.limiter, uq, u0, umin, umax);
        if (B.freeze) B.phi_keep[cell_var(B, b, v, J, I)] = double(phi);
      }
      s.px[v][rj][ri] = phi * gx;
      s.py[v][rj][ri] = phi * gy;
      if (B.dWdx) {
        const size_t o = cell_var(B, b, v, J, I);
        B.dWdx[o] = gx; B.dWdy[o] = gy; B.phi[o] = phi;
      }
    }
  }
  __syncthreads();

  // ---- face fluxes -----------------------------------------------------------
  const int ICl = NG, ICu = B.nci + NG - 1, JCl = NG, JCu = B.ncj + NG - 1;
  const int nfi = (TI + 1) * TJ, nfj = TI * (TJ + 1);
  for (int q = tid; q < nfi + nfj; q += NTHREADS) {
    PState<RT> wl, wr;
    double nx, ny, l;
    int fi, fj;
    bool is_i = q < nfi;
    if (is_i) {
      fj = q / (TI + 1); fi = q % (TI + 1);
      if (fi > nci_t || fj >= ncj_t) continue;
      // face between halo cells (fi+1, fj+2) and (fi+2, fj+2): east face of the left cell
      const int hl = fi + 1, hj = fj + 2, I = i0 + hl, J = j0 + hj;
      const double ax = s.X[hj + 1][hl + 1], ay = s.Y[hj + 1][hl + 1];  // node (I+1, J+1)
      const double cx = s.X[hj][hl + 1], cy = s.Y[hj][hl + 1];          // node (I+1, J)
      l = edge_len(cx, cy, ax, ay);
      edge_normal(ax, ay, cx, cy, l, perim_for_test(s, hl, hj, l), nx, ny);
      const double mx = HALF * (cx + ax), my = HALF * (cy + ay);
      const int bw = B.bcw[size_t(b) * B.NCj + J], be = B.bce[size_t(b) * B.NCj + J];
      if (I == ICl - 1 && face_bc(bw)) {
        wr = face_state(s, hl + 1, hj, mx, my);
        // nfaceW(ICl, J) with the right cell's perimeter
        double wx, wy;
        edge_normal(cx, cy, ax, ay, l, perim_for_test(s, hl + 1, hj, l), wx, wy);
        wl = (bw == E2D_BC_REFLECTION) ? reflect(wr, RT(wx), RT(wy))
                                       : bc_char_pressure(wr, load_wo(B.wow, b, B.NCj, J), RT(wx), RT(wy), RT(g), RT(gm1i));
      } else if (I == ICu && face_bc(be)) {
        wl = face_state(s, hl, hj, mx, my);
        wr = (be == E2D_BC_REFLECTION) ? reflect(wl, RT(nx), RT(ny))
                                       : bc_char_pressure(wl, load_wo(B.woe, b, B.NCj, J), RT(nx), RT(ny), RT(g), RT(gm1i));
      } else {
        wl = face_state(s, hl, hj, mx, my);
        wr = face_state(s, hl + 1, hj, mx, my);
      }
    } else {
      const int q2 = q - nfi;
      fj = q2 / TI; fi = q2 % TI;
      if (fi >= nci_t || fj > ncj_t) continue;
      // face between halo cells (fi+2, fj+1) and (fi+2, fj+2): north face of the lower cell
      const int hi = fi + 2, hl = fj + 1, I = i0 + hi, J = j0 + hl;
      const double ax = s.X[hl + 1][hi], ay = s.Y[hl + 1][hi];          // node (I, J+1)
      const double cx = s.X[hl + 1][hi + 1], cy = s.Y[hl + 1][hi + 1];  // node (I+1, J+1)
      l = edge_len(ax, ay, cx, cy);
      edge_normal(ax, ay, cx, cy, l, perim_for_test(s, hi, hl, l), nx, ny);
      const double mx = HALF * (ax + cx), my = HALF * (ay + cy);
      const int bs = B.bcs[size_t(b) * B.NCi + I], bn = B.bcn[size_t(b) * B.NCi + I];
      if (J == JCl - 1 && face_bc(bs)) {
        wr = face_state(s, hi, hl + 1, mx, my);
        double sx, sy;  // nfaceS(I, JCl): edge (I+1,J+1)->(I,J+1) of the upper cell
        edge_normal(cx, cy, ax, ay, l, perim_for_test(s, hi, hl + 1, l), sx, sy);
        wl = (bs == E2D_BC_REFLECTION) ? reflect(wr, RT(sx), RT(sy))
                                       : bc_char_pressure(wr, load_wo(B.wos, b, B.NCi, I), RT(sx), RT(sy), RT(g), RT(gm1i));
      } else if (J == JCu && face_bc(bn)) {
        wl = face_state(s, hi, hl, mx, my);
        wr = (bn == E2D_BC_REFLECTION) ? reflect(wl, RT(nx), RT(ny))
                                       : bc_char_pressure(wl, load_wo(B.won, b, B.NCi, I), RT(nx), RT(ny), RT(g), RT(gm1i));
      } else {
        wl = face_state(s, hi, hl, mx, my);
        wr = face_state(s, hi, hl + 1, mx, my);
      }
    }
    const CState<RT> F = face_flux<ROE>(B.flux, wl, wr, RT(nx), RT(ny), RT(g), RT(gm1), RT(gm1i));
    if (is_i) {
      s.Fi[0][fj][fi] = F.d; s.Fi[1][fj][fi] = F.mx; s.Fi[2][fj][fi] = F.my; s.Fi[3][fj][fi] = F.E;
      s.li[fj][fi] = l;
    } else {
      s.Fj[0][fj][fi] = F.d; s.Fj[1][fj][fi] = F.mx; s.Fj[2][fj][fi] = F.my; s.Fj[3][fj][fi] = F.E;
      s.lj[fj][fi] = l;
    }
  }
  __syncthreads();

  // ---- flux divergence and update, one interior cell per thread -------------
  const int ti = tid % TI, tj = tid / TI;
  const bool active = tid < TI * TJ && ti < nci_t && tj < ncj_t;
  const int hi = ti + 2, hj = tj + 2, I = i0 + hi, J = j0 + hj;
  // contributions of this cell to the next step's CFL minimum and residual norms
  double dt_next = MILLION_D, n1 = 0.0, n2 = 0.0, nmax = 0.0;
  if (active) {
    double xc, yc, A;
    E2D_QC(s.X[hj][hi], s.Y[hj][hi], s.X[hj][hi + 1], s.Y[hj][hi + 1], s.X[hj + 1][hi + 1],
           s.Y[hj + 1][hi + 1], s.X[hj + 1][hi], s.Y[hj + 1][hi], xc, yc, A);
    const double lW = s.li[tj][ti], lE = s.li[tj][ti + 1], lS = s.lj[tj][ti], lN = s.lj[tj + 1][ti];
#ifdef E2D_FAST
    const double rA = fm::rcp(A);
#endif
    const size_t c = cell_sc(B, b, J, I);
    double k = 1.0;
    if (MODE == 1 || MODE == 2) k = B.cfl * (B.local_dt ? B.dt[c] : *dtmin_p);
    double res[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      double d = 0.0;
      if (MODE == 2) {
        const size_t q = cell_var(B, b, v, J, I);
        d = a.res_out[q];
        if (a.acc1) d = d + 2.0 * a.acc1[q] + 2.0 * a.acc2[q];
      }
      if (MODE == 1 || MODE == 2) {
#ifdef E2D_FAST
        d += k * s.Fi[v][tj][ti] * lW * rA;
        d -= k * s.Fi[v][tj][ti + 1] * lE * rA;
        d += k * s.Fj[v][tj][ti] * lS * rA;
        d -= k * s.Fj[v][tj + 1][ti] * lN * rA;
#else
        d += k * s.Fi[v][tj][ti] * lW / A;
        d -= k * s.Fi[v][tj][ti + 1] * lE / A;
        d += k * s.Fj[v][tj][ti] * lS / A;
        d -= k * s.Fj[v][tj + 1][ti] * lN / A;
#endif
      } else {
#ifdef E2D_FAST
        d += s.Fi[v][tj][ti] * lW * rA;
        d -= s.Fi[v][tj][ti + 1] * lE * rA;
        d += s.Fj[v][tj][ti] * lS * rA;
        d -= s.Fj[v][tj + 1][ti] * lN * rA;
#else
        d += s.Fi[v][tj][ti] * lW / A;
        d -= s.Fi[v][tj][ti + 1] * lE / A;
        d += s.Fj[v][tj][ti] * lS / A;
        d -= s.Fj[v][tj + 1][ti] * lN / A;
#endif
      }
      res[v] = d;
    }
    if (MODE == 0) {
#pragma unroll
      for (int v = 0; v < 4; ++v) B.dUdt[cell_var(B, b, v, J, I)] = res[v];
    } else if (MODE == 3) {
      // Frechet derivative: calculate_Matrix_Free (GMRES2D.h:445-488),
      // V = (normalizeR(R) - b)/eps - normalizeUtoR(z * (1/dt))
      const double eps = a.nks_eps[cs];  // the case's epsilon
      const double rdt = 1.0 / B.dt[c];
      const size_t q = c * 4;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        double val = (res[v] / a.normR[v] - a.nks_b[q + v]) / eps;
        val -= (a.nks_z[q + v] * rdt) * a.normU[v] / a.normR[v];
        a.nks_v[q + v] = val;
      }
    } else if (a.no_update) {
      // the stage's residual only: residual smoothing and the update follow
#pragma unroll
      for (int v = 0; v < 4; ++v) a.res_out[cell_var(B, b, v, J, I)] = res[v];
    } else {
      // Update_Solution_Multistage_Explicit: U = Uo + omega*dUdt
      CState<double> uo;
      uo.d = a.Ubase[cell_var(B, b, 0, J, I)]; uo.mx = a.Ubase[cell_var(B, b, 1, J, I)];
      uo.my = a.Ubase[cell_var(B, b, 2, J, I)]; uo.E = a.Ubase[cell_var(B, b, 3, J, I)];
      const double omega = a.omega;
      CState<double> u;
      u.d = uo.d + omega * res[0]; u.mx = uo.mx + omega * res[1];
      u.my = uo.my + omega * res[2]; u.E = uo.E + omega * res[3];
      if (u.d <= 0.0 || u.E <= 0.0 || e_of_U(u) <= 0.0) {
        if (!B.local_dt) {
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
            if (u.d > 0.0 && u.E > 0.0 && e_of_U(u) > 0.0) break;
          }
          B.dt[c] = dtc;
          if (u.d <= 0.0 || u.E <= 0.0 || e_of_U(u) <= 0.0) set_status(B.status, ST_NEGATIVE, int(c));
        }
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) a.res_out[cell_var(B, b, v, J, I)] = res[v];
#ifdef E2D_FAST
      const PState<double> w = fm::W_of_U(u, gm1);
#else
      const PState<double> w = W_of_U(u, gm1);
#endif
      a.Uout[cell_var(B, b, 0, J, I)] = u.d; a.Uout[cell_var(B, b, 1, J, I)] = u.mx;
      a.Uout[cell_var(B, b, 2, J, I)] = u.my; a.Uout[cell_var(B, b, 3, J, I)] = u.E;
      a.Wout[cell_var(B, b, 0, J, I)] = w.d; a.Wout[cell_var(B, b, 1, J, I)] = w.u;
      a.Wout[cell_var(B, b, 2, J, I)] = w.v; a.Wout[cell_var(B, b, 3, J, I)] = w.p;
      if (FUSE) {
        // CFL of the updated cell (Euler2DQuadSingleBlock.cc:3019-3080) and its
        // density residual, for the next explicit step.
        dt_next = cell_dt(s, hi, hj, A, lE, lW, lN, lS, w, g);
        if (B.local_dt) B.dt[c] = dt_next;
        n1 = fabs(res[0]);
        n2 = res[0] * res[0];
        nmax = n1;
      }
    }
  }
  if (FUSE) {
    // CTA reduction, then one atomic per quantity into the next step's slot
    __shared__ double red[4][NTHREADS / 32];
    for (int o = 16; o > 0; o >>= 1) {
      dt_next = dmin(dt_next, __shfl_xor_sync(0xffffffffu, dt_next, o));
      n1 += __shfl_xor_sync(0xffffffffu, n1, o);
      n2 += __shfl_xor_sync(0xffffffffu, n2, o);
      nmax = dmax(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
    }
    if ((tid & 31) == 0) {
      red[0][tid >> 5] = dt_next; red[1][tid >> 5] = n1; red[2][tid >> 5] = n2; red[3][tid >> 5] = nmax;
    }
    __syncthreads();
    if (tid == 0) {
      for (int w2 = 1; w2 < NTHREADS / 32; ++w2) {
        dt_next = dmin(dt_next, red[0][w2]); n1 += red[1][w2]; n2 += red[2][w2]; nmax = dmax(nmax, red[3][w2]);
      }
      double* next = const_cast<double*>(a.hist) + 4 * ((*a.step + 1) * B.ncase + cs);
      atomicMin(reinterpret_cast<unsigned long long*>(next), (unsigned long long)__double_as_longlong(dt_next));
      atomicAdd(next + 1, n1);
      atomicAdd(next + 2, n2);
      atomicMax(reinterpret_cast<unsigned long long*>(next + 3), (unsigned long long)__double_as_longlong(nmax));
    }
  }
}

}  // namespace E2D_NS
}  // namespace e2d

namespace e2d {
namespace E2D_NS {
size_t stage_smem_bytes() { return sizeof(Smem); }
template <int MODE, bool FUSE, bool ROE>
cudaError_t launch_one(const StageArgs& a, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<MODE, FUSE, ROE>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(sizeof(Smem)));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const int grid = a.B.nblk * a.tiles_i * a.tiles_j;
  stage_kernel<MODE, FUSE, ROE><<<grid, NTHREADS, sizeof(Smem), st>>>(a);
  return cudaGetLastError();
}
template <bool ROE>
cudaError_t launch_flux(const StageArgs& a, cudaStream_t st) {
  switch (a.mode * 2 + (a.fuse_next ? 1 : 0)) {
    case 0: return launch_one<0, false, ROE>(a, st);
    case 2: return launch_one<1, false, ROE>(a, st);
    case 3: return launch_one<1, true, ROE>(a, st);
    case 4: return launch_one<2, false, ROE>(a, st);
    case 5: return launch_one<2, true, ROE>(a, st);
    case 6: return launch_one<3, false, ROE>(a, st);
    default: return cudaErrorInvalidValue;
  }
}
cudaError_t launch_stage(const StageArgs& a, cudaStream_t st) {
  return a.B.flux == E2D_FLUX_ROE ? launch_flux<true>(a, st) : launch_flux<false>(a, st);
}
int tile_i() { return TI; }
int tile_j() { return TJ; }
}  // namespace E2D_NS
}  // namespace e2d
