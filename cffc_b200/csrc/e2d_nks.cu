// e2d_nks.cu — pseudo-transient Newton-Krylov steady solver on the device:
// the Newton loop of Internal_Newton_Krylov_Schwarz_Solver
// (NewtonKrylovSchwarz2D/NKS2D.h:412-1258), right-preconditioned restarted
// matrix-free GMRES (NewtonKrylovSchwarz2D/GMRES2D.h:790-1544), the block
// Jacobi preconditioner on the first-order HLLE Jacobian
// (NewtonKrylovSchwarz2D/Block_Preconditioner2D.h:352-584) and the Euler2D
// Newton_Update with positivity back-off (Euler2D/Euler2DQuadNKS.h:23-92).
//
// Batches.  A handle may hold several independent cases (e2d_create_batch).
// Every case runs its own Newton loop and GMRES — own norms, CFL, epsilon,
// Hessenberg matrix, Givens rotations and stopping decisions — while the
// device work of all cases still iterating runs in the same launches, in
// lockstep: all cases start GMRES together, a case that meets its tolerance
// drops out (its blocks are skipped through the per-case active mask) and
// the restarted cases go on together.  Reductions are per block, then per
// case in block order, so a case gives the same bits in a batch as alone.
//
// Layout.  Krylov vectors are the reference's per-block GMRES vectors laid
// end to end: [nblk][NCj][NCi][4] doubles (GMRES_Block::index,
// GMRES2D.h:84), ghost entries held at zero.  The preconditioner keeps one
// 4x4 inverse per cell, row-major [nblk][NCj][NCi][16] (identity on ghost
// cells, as Create_Preconditioner leaves them).  Per-case scalars are
// [ncase] arrays; the Hessenberg column of iteration j is [j+2][ncase].
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <vector>

#include "e2d_geom.cuh"
#include "e2d_handle.h"

using namespace e2d;

namespace {

constexpr int VT = 256;           // threads of the vector kernels
constexpr int VGRID = 148 * 4;    // CTAs of the grid-stride kernels
constexpr double RHO_STD = 1.225;       // Euler2D_W_STDATM.d
constexpr double P_STD = 101325.0;      // Euler2D_W_STDATM.p

enum Final { FIN_SUM = 0, FIN_SQRT = 1, FIN_EPS = 2 };

__device__ __forceinline__ bool case_on(const Blocks& B, int c) { return !B.case_active || B.case_active[c]; }

// CTA sum of v (fixed order: warp shuffles, then the warps in order).
__device__ double cta_sum(double v) {
  __shared__ double red[VT / 32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < VT / 32; ++w) s += red[w];
  return s;  // valid in thread 0
}

// Reductions: each block's entries are split into `ch` chunks, one CTA per
// chunk; the CTA writes its partial sum to partial[block * ch + chunk], and
// the last CTA of a case to arrive (per-case counter) sums the case's
// partials in block and chunk order — a fixed order, whichever CTA is last —
// and writes out[c] = f(sum): the sum, its square root, or eps0 / sqrt
// (calculate_epsilon, GMRES2D.h:1628-1640).
__device__ void partial_done(double s, double* partial, int slot, const Blocks& B, int c, int ch, unsigned* counter,
                             double* out, int fin, double eps0) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partial[slot] = s;
    __threadfence();
    const int b0 = B.case_start ? B.case_start[c] : 0, b1 = B.case_start ? B.case_start[c + 1] : B.nblk;
    const unsigned n = unsigned((b1 - b0) * ch);
    last = atomicAdd(&counter[c], 1u) == n - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x >= 32) return;
  __threadfence();
  const int b0 = B.case_start ? B.case_start[c] : 0, b1 = B.case_start ? B.case_start[c + 1] : B.nblk;
  // each lane sums partials lane, lane + 32, ... in that order; the loads of
  // eight of them are issued together (from L2, where the other CTAs'
  // fenced writes are), then added one after another
  double t = 0.0;
  const int q1 = b1 * ch;
  for (int q = b0 * ch + threadIdx.x; q < q1; q += 32 * 8) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = q + 32 * u < q1 ? __ldcg(partial + q + 32 * u) : 0.0;
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (q + 32 * u < q1) t += v[u];
  }
  for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  if (threadIdx.x == 0) {
    out[c] = fin == FIN_SUM ? t : (fin == FIN_SQRT ? sqrt(t) : eps0 / sqrt(t));
    counter[c] = 0u;
  }
}

// out[case] = f(sum of a*b over the case); grid = nblk * ch CTAs, nper2
// double2 entries per block.
__global__ void __launch_bounds__(VT) blk_dot_kernel(const double* __restrict__ a, const double* __restrict__ bv,
                                                     int nper2, int ch, double* partial, unsigned* counter,
                                                     double* out, int fin, double eps0, Blocks B) {
  const int blk = blockIdx.x / ch, part = blockIdx.x % ch;
  const int c = case_id(B, blk);
  if (!case_on(B, c)) return;  // uniform per CTA
  const int len = (nper2 + ch - 1) / ch, q0 = part * len, q1 = min(nper2, q0 + len);
  const double2* a2 = reinterpret_cast<const double2*>(a) + size_t(blk) * nper2;
  const double2* b2 = reinterpret_cast<const double2*>(bv) + size_t(blk) * nper2;
  double s = 0.0;
  for (int q = q0 + threadIdx.x; q < q1; q += VT) {
    const double2 x = a2[q], y = b2[q];
    s += x.x * y.x;
    s += x.y * y.y;
  }
  s = cta_sum(s);
  partial_done(s, partial, blockIdx.x, B, c, ch, counter, out, fin, eps0);
}

// One modified Gram-Schmidt update fused with the next reduction: y -=
// coef[case] * x (the axpy of axpy_kernel, element for element), then
// out[case] = f(sum of y * b) with b the next Krylov vector, or y itself
// when b is null (the norm that closes the step) -- the same products in
// the same order as blk_dot_kernel over the updated y, so the results are
// those of the separate axpy and dot kernels, with one pass over y instead
// of two.  Grid as blk_dot_kernel.
__global__ void __launch_bounds__(VT) axpy_dot_kernel(double* __restrict__ y, const double* __restrict__ x,
                                                      const double* coef, const double* bv, int nper2, int ch,
                                                      double* partial, unsigned* counter, double* out, int fin,
                                                      Blocks B) {
  const int blk = blockIdx.x / ch, part = blockIdx.x % ch;
  const int c = case_id(B, blk);
  if (!case_on(B, c)) return;  // uniform per CTA
  const int len = (nper2 + ch - 1) / ch, q0 = part * len, q1 = min(nper2, q0 + len);
  double2* y2 = reinterpret_cast<double2*>(y) + size_t(blk) * nper2;
  const double2* x2 = reinterpret_cast<const double2*>(x) + size_t(blk) * nper2;
  const double2* b2 = bv ? reinterpret_cast<const double2*>(bv) + size_t(blk) * nper2 : nullptr;
  const double alpha = -1.0 * coef[c];
  double s = 0.0;
  for (int q = q0 + threadIdx.x; q < q1; q += VT) {
    double2 v = y2[q];
    const double2 u = x2[q];
    v.x = v.x + alpha * u.x;
    v.y = v.y + alpha * u.y;
    y2[q] = v;
    const double2 w = b2 ? b2[q] : v;
    s += v.x * w.x;
    s += v.y * w.y;
  }
  s = cta_sum(s);
  partial_done(s, partial, blockIdx.x, B, c, ch, counter, out, fin, 0.0);
}

// y += alpha * x, alpha = sign * coef[case] (device, per case) or alpha_h.
__global__ void __launch_bounds__(VT) axpy_kernel(double* __restrict__ y, const double* __restrict__ x, long long n2,
                                                  int nper2, const double* coef, double sign, double alpha_h, Blocks B) {
  double2* y2 = reinterpret_cast<double2*>(y);
  const double2* x2 = reinterpret_cast<const double2*>(x);
  for (long long q = blockIdx.x * (long long)VT + threadIdx.x; q < n2; q += (long long)gridDim.x * VT) {
    const int c = case_id(B, int(q / nper2));
    if (!case_on(B, c)) continue;
    const double alpha = coef ? sign * coef[c] : alpha_h;
    double2 v = y2[q];
    const double2 u = x2[q];
    v.x = v.x + alpha * u.x;
    v.y = v.y + alpha * u.y;
    y2[q] = v;
  }
}

// y *= sign / s[case] (dscal by ONE/H or -ONE/beta, GMRES2D.h:1080, :1246).
__global__ void __launch_bounds__(VT) scale_kernel(double* __restrict__ y, long long n2, int nper2, const double* s,
                                                   double sign, Blocks B) {
  double2* y2 = reinterpret_cast<double2*>(y);
  for (long long q = blockIdx.x * (long long)VT + threadIdx.x; q < n2; q += (long long)gridDim.x * VT) {
    const int c = case_id(B, int(q / nper2));
    if (!case_on(B, c)) continue;
    const double f = sign / s[c];
    double2 v = y2[q];
    v.x = f * v.x;
    v.y = f * v.y;
    y2[q] = v;
  }
}

// x = x + s_0 Z_0 + ... + s_{k-1} Z_{k-1} per case, in the reference's daxpy
// order (GMRES2D.h:1300-1304); k = kcount[case] (0: x unchanged).
__global__ void __launch_bounds__(VT) update_x_kernel(double* __restrict__ x, const double* __restrict__ Z, long long n,
                                                      int nper, const double* __restrict__ s, const int* kcount,
                                                      int m, Blocks B) {
  for (long long q = blockIdx.x * (long long)VT + threadIdx.x; q < n; q += (long long)gridDim.x * VT) {
    const int c = case_id(B, int(q / nper));
    const int k = kcount[c];
    if (k == 0) continue;
    double v = x[q];
    for (int j = 0; j < k; ++j) v = v + s[size_t(c) * m + j] * Z[size_t(j) * n + q];
    x[q] = v;
  }
}

// z = Minv v per cell, and eps[case] = eps0 / ||z|| over the case; grid =
// nblk * ch CTAs, each a chunk of a block's cells.
// vscale (null: none): v is first divided in place by vscale[case] (the
// dscal by ONE/H that closes the previous Arnoldi step, GMRES2D.h:1246,
// done here instead of in its own pass: the same product f * v).
__global__ void __launch_bounds__(VT) precon_apply_kernel(const double* __restrict__ Minv, double* __restrict__ v,
                                                          double* __restrict__ z, int cells_per_block, int ch,
                                                          double* partial, unsigned* counter, double* eps_out,
                                                          double eps0, const double* vscale, Blocks B) {
  const int blk = blockIdx.x / ch, part = blockIdx.x % ch;
  const int cs = case_id(B, blk);
  if (!case_on(B, cs)) return;
  const int len = (cells_per_block + ch - 1) / ch, r0 = part * len, r1 = min(cells_per_block, r0 + len);
  const double f = vscale ? 1.0 / vscale[cs] : 1.0;
  double s = 0.0;
  for (int r = r0 + threadIdx.x; r < r1; r += VT) {
    const size_t c = size_t(blk) * cells_per_block + r;
    double2* v2 = reinterpret_cast<double2*>(v + 4 * c);
    double2 va = v2[0], vb = v2[1];
    if (vscale) {
      va.x = f * va.x; va.y = f * va.y; vb.x = f * vb.x; vb.y = f * vb.y;
      v2[0] = va;
      v2[1] = vb;
    }
    const double* M = Minv + 16 * c;
    double o[4];
#pragma unroll
    for (int row = 0; row < 4; ++row) {
      double t = 0.0;
      t = t + va.x * M[4 * row + 0];
      t = t + va.y * M[4 * row + 1];
      t = t + vb.x * M[4 * row + 2];
      t = t + vb.y * M[4 * row + 3];
      o[row] = t;
      s += t * t;
    }
    double2* z2 = reinterpret_cast<double2*>(z + 4 * c);
    z2[0] = make_double2(o[0], o[1]);
    z2[1] = make_double2(o[2], o[3]);
  }
  s = cta_sum(s);
  partial_done(s, partial, blockIdx.x, B, cs, ch, counter, eps_out, FIN_EPS, eps0);
}

struct Norm4 {
  double u[4], r[4];
};

// U = Uo + (eps * dir) * normU on every cell, ghosts included, and W = W(U)
// (calculate_perturbed_residual, GMRES2D.h:388-409).
__global__ void __launch_bounds__(VT) perturb_kernel(Blocks B, const double* __restrict__ Uo,
                                                     const double* __restrict__ dir, const double* eps_case, Norm4 nm) {
  const long long ncell = (long long)B.nblk * B.NCj * B.NCi;
  const int per = B.NCj * B.NCi;
  for (long long c = blockIdx.x * (long long)VT + threadIdx.x; c < ncell; c += (long long)gridDim.x * VT) {
    const int b = int(c / per), r = int(c % per);
    const int cs = case_id(B, b);
    if (!case_on(B, cs)) continue;
    const double eps = eps_case[cs];
    const int j = r / B.NCi, i = r % B.NCi;
    double uv[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) uv[v] = Uo[cell_var(B, b, v, j, i)] + (eps * dir[4 * c + v]) * nm.u[v];
    CState<double> u;
    u.d = uv[0]; u.mx = uv[1]; u.my = uv[2]; u.E = uv[3];
    stU(B, b, i, j, u);
    stW(B, b, i, j, W_of_U(u, B.gm1));
  }
}

// b = normalizeR(dUdt) on interior cells (GMRES_Block::Initialize, GMRES2D.h:374-380).
__global__ void __launch_bounds__(VT) load_b_kernel(Blocks B, double* __restrict__ bvec, Norm4 nm) {
  const long long n = (long long)B.nblk * B.nci * B.ncj;
  const int per = B.nci * B.ncj;
  for (long long q = blockIdx.x * (long long)VT + threadIdx.x; q < n; q += (long long)gridDim.x * VT) {
    const int b = int(q / per), r = int(q % per);
    if (!case_on(B, case_id(B, b))) continue;
    const int i = NG + r % B.nci, j = NG + r / B.nci;
    const size_t c = cell_sc(B, b, j, i);
#pragma unroll
    for (int v = 0; v < 4; ++v) bvec[4 * c + v] = B.dUdt[cell_var(B, b, v, j, i)] / nm.r[v];
  }
}

// Time step of the Newton step: the CFL-limited local step scaled by the
// case's finite-time-step CFL, or the case's minimum times it (NKS2D.h:913-930).
__global__ void __launch_bounds__(VT) set_dt_kernel(Blocks B, const double* slots, const double* cfl_case) {
  const long long n = (long long)B.nblk * B.nci * B.ncj;
  const int per = B.nci * B.ncj;
  for (long long q = blockIdx.x * (long long)VT + threadIdx.x; q < n; q += (long long)gridDim.x * VT) {
    const int b = int(q / per), r = int(q % per);
    const int cs = case_id(B, b);
    if (!case_on(B, cs)) continue;
    const int i = NG + r % B.nci, j = NG + r / B.nci;
    const size_t c = cell_sc(B, b, j, i);
    const double cfl = cfl_case[cs];
    B.dt[c] = B.local_dt ? B.dt[c] * cfl : slots[4 * cs] * cfl;
  }
}

// Newton_Update (Euler2DQuadNKS.h:23-92): U = Uo + relax * x * normU on
// interior cells, halving the update up to ten times while the density,
// total energy or internal energy is not positive; W = W(U).
__global__ void __launch_bounds__(VT) newton_update_kernel(Blocks B, const double* __restrict__ Uo,
                                                           const double* __restrict__ x, Norm4 nm, double relax) {
  const long long n = (long long)B.nblk * B.nci * B.ncj;
  const int per = B.nci * B.ncj;
  for (long long q = blockIdx.x * (long long)VT + threadIdx.x; q < n; q += (long long)gridDim.x * VT) {
    const int b = int(q / per), r = int(q % per);
    if (!case_on(B, case_id(B, b))) continue;
    const int i = NG + r % B.nci, j = NG + r / B.nci;
    const size_t c = cell_sc(B, b, j, i);
    double uo[4], du[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      uo[v] = Uo[cell_var(B, b, v, j, i)];
      du[v] = x[4 * c + v] * nm.u[v];  // GMRES.deltaU = denormalizeU(x)
    }
    CState<double> u;
    u.d = uo[0] + relax * du[0]; u.mx = uo[1] + relax * du[1];
    u.my = uo[2] + relax * du[2]; u.E = uo[3] + relax * du[3];
    if (u.d <= 0.0 || e_of_U(u) <= 0.0 || u.E <= 0.0) {
      double f = 1.0;
      for (int k = 1; k <= 10; ++k) {
        f = HALF * f;
        u.d = uo[0] + du[0] * f; u.mx = uo[1] + du[1] * f;
        u.my = uo[2] + du[2] * f; u.E = uo[3] + du[3] * f;
        if (u.d > 0.0 && u.E > 0.0 && e_of_U(u) > 0.0) break;
      }
      if (u.d <= 0.0 || e_of_U(u) <= 0.0) set_status(B.status, ST_NEGATIVE, int(c));
    }
    stU(B, b, i, j, u);
    stW(B, b, i, j, W_of_U(u, B.gm1));
  }
}

// ---- block Jacobi preconditioner ------------------------------------------

__device__ __forceinline__ PState<double> rotate(const PState<double>& w, double nx, double ny) {
  PState<double> r;
  r.d = w.d;
  r.u = w.u * nx + w.v * ny;
  r.v = -w.u * ny + w.v * nx;
  r.p = w.p;
  return r;
}

// HLLE_wavespeeds (Euler2D/Euler2DState.cc:3199-3230): (lambda-, lambda+)
// of the rotated Riemann problem.
__device__ void hlle_wavespeeds(const PState<double>& wl0, const PState<double>& wr0, double nx, double ny,
                                double g, double gm1, double& lm, double& lp) {
  const PState<double> wl = rotate(wl0, nx, ny), wr = rotate(wr0, nx, ny);
  const double hl = h_of(wl, g, gm1), hr = h_of(wr, g, gm1);
  const double sdl = sqrt(wl.d), sdr = sqrt(wr.d);
  PState<double> wa;
  wa.d = sdl * sdr;
  wa.u = (sdl * wl.u + sdr * wr.u) / (sdl + sdr);
  wa.v = (sdl * wl.v + sdr * wr.v) / (sdl + sdr);
  const double ha = (sdl * hl + sdr * hr) / (sdl + sdr);
  const double aa2 = gm1 * (ha - HALF * (sqr(wa.u) + sqr(wa.v)));
  wa.p = wa.d * aa2 / g;
  lm = dmin(wl.u - a_of(wl, g), wa.u - a_of(wa, g));
  lp = dmax(wr.u + a_of(wr, g), wa.u + a_of(wa, g));
  lm = dmin(lm, 0.0);
  lp = dmax(lp, 0.0);
}

// Euler2D_pState::dFdU (Euler2D/Euler2DState.h:1792-1806) of a rotated state.
__device__ void dfdu(const PState<double>& w, double g, double gm1, double gm1i, double m[4][4]) {
  const double ux = w.u, uy = w.v;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) m[r][c] = 0.0;
  m[0][1] = 1.0;
  m[1][0] = HALF * (sqr(ux) * (g - 3.0) + sqr(uy) * gm1);
  m[1][1] = -(ux * (g - 3.0));
  m[1][2] = -(uy * gm1);
  m[1][3] = gm1;
  m[2][0] = -(ux * uy);
  m[2][1] = uy;
  m[2][2] = ux;
  m[3][0] = HALF * gm1i * ux * (w.d * (2.0 + g * g - 3.0 * g) * (sqr(ux) + sqr(uy)) - 2.0 * w.p * g) / w.d;
  m[3][1] = HALF * gm1i * (sqr(ux) * w.d * (5.0 * g - 3.0 - 2.0 * g * g) + sqr(uy) * w.d * gm1 + 2.0 * w.p * g) / w.d;
  m[3][2] = -(ux * uy * gm1);
  m[3][3] = g * ux;
}

// One face's block l * AI * (beta dFdU(Rotate(Wc, n)) + gamma I) * A
// (First_Order_Inviscid_Jacobian_HLLE, Block_Preconditioner2D.h:491-584),
// accumulated into acc.
__device__ void face_jacobian(const PState<double>& wc, const PState<double>& wn, double nx, double ny, double l,
                              double g, double gm1, double gm1i, double acc[4][4]) {
  double lm, lp;
  hlle_wavespeeds(wn, wc, nx, ny, g, gm1, lm, lp);
  const double gam = (lm * lp) / (lp - lm);
  const double bet = -lm / (lp - lm);
  double d[4][4];
  dfdu(rotate(wc, nx, ny), g, gm1, gm1i, d);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
#pragma unroll
    for (int c = 0; c < 4; ++c) d[r][c] = bet * d[r][c];
    d[r][r] = d[r][r] + gam;
  }
  // rotation matrices: A = identity with A(1,1)=c, A(1,2)=s, A(2,1)=-s,
  // A(2,2)=c; AI is its transpose (Rotation_Matrix, Block_Preconditioner2D.h:862)
  double Am[4][4] = {{1, 0, 0, 0}, {0, nx, ny, 0}, {0, -ny, nx, 0}, {0, 0, 0, 1}};
  double AI[4][4] = {{1, 0, 0, 0}, {0, nx, -ny, 0}, {0, ny, nx, 0}, {0, 0, 0, 1}};
  double t[4][4], u[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) t[r][c] = l * AI[r][c];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) s += t[r][k] * d[k][c];
      u[r][c] = s;
    }
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 4; ++k) s += u[r][k] * Am[k][c];
      acc[r][c] += s;
    }
}

// In-place inverse of a 4x4 matrix by LU with partial pivoting (the
// LAPACK dgetrf/dgetri pair BPKIT's LP_INVERSE calls).  Returns false on a
// zero pivot.
__device__ bool invert4(double a[4][4]) {
  int piv[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int p = k;
    double best = fabs(a[k][k]);
#pragma unroll
    for (int r = k + 1; r < 4; ++r)
      if (fabs(a[r][k]) > best) { best = fabs(a[r][k]); p = r; }
    piv[k] = p;
    if (best == 0.0) return false;
    // row interchange written with static indices only (keeps a[][] in registers)
#pragma unroll
    for (int r = k + 1; r < 4; ++r)
      if (r == p) {
#pragma unroll
        for (int c = 0; c < 4; ++c) { const double t = a[k][c]; a[k][c] = a[r][c]; a[r][c] = t; }
      }
    const double rp = 1.0 / a[k][k];
#pragma unroll
    for (int r = k + 1; r < 4; ++r) {
      a[r][k] *= rp;
#pragma unroll
      for (int c = k + 1; c < 4; ++c) a[r][c] -= a[r][k] * a[k][c];
    }
  }
  // inverse of U in place (upper triangle)
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    a[j][j] = 1.0 / a[j][j];
    const double ajj = -a[j][j];
#pragma unroll
    for (int r = 0; r < j; ++r) {
      double s = 0.0;
#pragma unroll
      for (int k = r; k < j; ++k) s += a[r][k] * a[k][j];
      a[r][j] = s;
    }
#pragma unroll
    for (int r = 0; r < j; ++r) a[r][j] *= ajj;
  }
  // solve inv(A) * L = inv(U) for inv(A), columns from the right
  double w[4];
#pragma unroll
  for (int j = 2; j >= 0; --j) {
#pragma unroll
    for (int r = j + 1; r < 4; ++r) { w[r] = a[r][j]; a[r][j] = 0.0; }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      double s = a[r][j];
#pragma unroll
      for (int k = j + 1; k < 4; ++k) s -= a[r][k] * w[k];
      a[r][j] = s;
    }
  }
  // undo the row interchanges as column interchanges
#pragma unroll
  for (int j = 2; j >= 0; --j) {
    const int p = piv[j];
#pragma unroll
    for (int c = j + 1; c < 4; ++c)
      if (c == p) {
#pragma unroll
        for (int r = 0; r < 4; ++r) { const double t = a[r][j]; a[r][j] = a[r][c]; a[r][c] = t; }
      }
  }
  return true;
}

// normalize_Preconditioner_dFdU (Euler2D/Euler2DQuadNKS.h:115-137)
__device__ __forceinline__ void normalize_block(double m[4][4], double ao) {
  const double ia = 1.0 / ao, ia2 = 1.0 / (ao * ao), ia3 = 1.0 / (ao * ao * ao);
  m[0][0] *= ia; m[0][3] *= ao;
  m[1][0] *= ia2; m[1][1] *= ia; m[1][2] *= ia;
  m[2][0] *= ia2; m[2][1] *= ia; m[2][2] *= ia;
  m[3][0] *= ia3; m[3][1] *= ia2; m[3][2] *= ia2; m[3][3] *= ia;
}

// Diagonal block of the approximate Jacobian for each interior cell,
// normalized (normalize_Preconditioner_dFdU, Euler2DQuadNKS.h:115-137) and
// inverted: CENTER = -I / dt + (J_N + J_S + J_E + J_W) / A.
// order E2D_JACOBIAN_SOURCE_TERMS_ONLY keeps -I / dt alone.
__global__ void __launch_bounds__(128) precon_build_kernel(Blocks B, double* __restrict__ Minv, double ao, int order) {
  const long long n = (long long)B.nblk * B.nci * B.ncj;
  const int per = B.nci * B.ncj;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int b = int(q / per), r = int(q % per);
    if (B.case_active && !B.case_active[case_id(B, b)]) continue;
    const int i = NG + r % B.nci, j = NG + r / B.nci;
    const size_t c = cell_sc(B, b, j, i);
    const PState<double> wc = ldW(B, b, i, j);
    double acc[4][4];
#pragma unroll
    for (int rr = 0; rr < 4; ++rr)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) acc[rr][cc] = 0.0;
    double nx, ny;
    if (order == E2D_JACOBIAN_FIRST_ORDER_HLLE) {
    // N: the north face of the cell below, pointing into this cell
    nfaceN(B, b, i, j - 1, nx, ny);
    face_jacobian(wc, ldW(B, b, i, j - 1), nx, ny, glen(B, b, i, j, i + 1, j), B.g, B.gm1, B.gm1i, acc);
    nfaceS(B, b, i, j + 1, nx, ny);
    face_jacobian(wc, ldW(B, b, i, j + 1), nx, ny, glen(B, b, i, j + 1, i + 1, j + 1), B.g, B.gm1, B.gm1i, acc);
    nfaceE(B, b, i - 1, j, nx, ny);
    face_jacobian(wc, ldW(B, b, i - 1, j), nx, ny, glen(B, b, i, j, i, j + 1), B.g, B.gm1, B.gm1i, acc);
    nfaceW(B, b, i + 1, j, nx, ny);
    face_jacobian(wc, ldW(B, b, i + 1, j), nx, ny, glen(B, b, i + 1, j, i + 1, j + 1), B.g, B.gm1, B.gm1i, acc);
    }
    double xc, yc, A;
    quad_centroid(nodeX(B, b, i, j), nodeY(B, b, i, j), nodeX(B, b, i + 1, j), nodeY(B, b, i + 1, j),
                  nodeX(B, b, i + 1, j + 1), nodeY(B, b, i + 1, j + 1), nodeX(B, b, i, j + 1),
                  nodeY(B, b, i, j + 1), xc, yc, A);
    const double lhs = 1.0 / B.dt[c];
    double m[4][4];
#pragma unroll
    for (int rr = 0; rr < 4; ++rr)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc)
        m[rr][cc] = order == E2D_JACOBIAN_FIRST_ORDER_HLLE ? (rr == cc ? -lhs : 0.0) + acc[rr][cc] / A
                                                            : (rr == cc ? -lhs : 0.0);
    normalize_block(m, ao);
    if (!invert4(m)) set_status(B.status, 3, int(c));
    double* o = Minv + 16 * c;
#pragma unroll
    for (int rr = 0; rr < 4; ++rr)
#pragma unroll
      for (int cc = 0; cc < 4; ++cc) o[4 * rr + cc] = m[rr][cc];
  }
}

__global__ void identity_blocks_kernel(double* Minv, long long ncell) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < 16 * ncell;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = int(q % 16);
    Minv[q] = (e / 4 == e % 4) ? 1.0 : 0.0;
  }
}

#include "e2d_ilu.cuh"

// ---- GMRES bookkeeping on the device ----------------------------------------
// Per case: the rotated Hessenberg columns, Givens rotations and right-hand
// side of the least-squares problem (GMRES2D.h:761-783, 1250-1304), the
// residual at the cycle's start and the current relative residual, the
// iteration count and the stop state.  The host only launches the Arnoldi
// steps; it reads the number of cases still iterating a few steps behind and
// the per-case results once per restart cycle.
enum GmresFlag { GF_MET = 1, GF_FAILED = 2, GF_RESTARTED = 4, GF_DONE = 8 };

struct GmresDev {
  int m, ncase;                    // m: the buffers' cycle length (array strides)
  const int* cfg;                  // device: [0] cycle length of this solve (<= m), [1] iteration cap
  double *H, *cs, *sn, *sv;        // [C][m][m+1], [C][m], [C][m], [C][m+1]
  double *resid0, *relres, *tol;   // [C]
  int *iters, *flags, *jstop;      // [C]
  int* its;                        // iterations of this GMRES solve (all cases in lockstep)
  int* err;                        // first error (E2D_ERR_*), 0 = none
  int* progress;                   // host-mapped [m]: cases still iterating after step j
};

__device__ void gm_error(const GmresDev& G, int code) { atomicCAS(G.err, 0, code); }

// Start of a restart cycle: the cases not yet done iterate (active mask),
// their right-hand side is (beta, 0, ..., 0) with beta = ||V0|| (nrm), and
// the first cycle records beta as the solve's initial residual.
__global__ void gmres_cycle_start_kernel(GmresDev G, const double* nrm, int* active, int first) {
  for (int c = threadIdx.x; c < G.ncase; c += blockDim.x) {
    const bool on = !(G.flags[c] & GF_DONE);
    active[c] = on ? 1 : 0;
    if (!on) continue;
    const double beta = nrm[c];
    if (!(beta > 0.0) || !isfinite(beta)) gm_error(G, E2D_ERR_GMRES);
    double* sv = G.sv + size_t(c) * (G.m + 1);
    sv[0] = beta;
    for (int q = 1; q <= G.cfg[0]; ++q) sv[q] = 0.0;
    if (first) G.resid0[c] = beta;
    G.flags[c] = 0;
    G.jstop[c] = -1;
  }
}

// The multi-block cycle activity: cases not yet done (before the restart's
// J x + b product).
__global__ void gmres_cycle_active_kernel(GmresDev G, int* active) {
  for (int c = threadIdx.x; c < G.ncase; c += blockDim.x) active[c] = (G.flags[c] & GF_DONE) ? 0 : 1;
}

__device__ __forceinline__ void apply_rot(double& dx, double& dy, double cs, double sn) {
  const double t = cs * dx + sn * dy;
  dy = -sn * dx + cs * dy;
  dx = t;
}

// End of Arnoldi step j: per iterating case, the Hessenberg column (hcol,
// [j+2][ncase]) takes the previous rotations, a new rotation zeroes its
// subdiagonal, the right-hand side rotates with it, and the stop test
// (tolerance met, iteration cap, end of the cycle) runs.  One CTA.
__global__ void gmres_givens_kernel(GmresDev G, const double* hcol, int* active, int j) {
  __shared__ int its, count;
  if (threadIdx.x == 0) {
    its = ++*G.its;
    count = 0;
  }
  __syncthreads();
  const int m = G.m, C = G.ncase, mc = G.cfg[0], cap = G.cfg[1];
  for (int c = threadIdx.x; c < C; c += blockDim.x) {
    if (!active[c]) continue;
    double* Hj = G.H + (size_t(c) * m + j) * (m + 1);
    double* cs = G.cs + size_t(c) * m;
    double* sn = G.sn + size_t(c) * m;
    double* sv = G.sv + size_t(c) * (m + 1);
    // the previous rotations, entry k with entry k+1 in order; the entry
    // being rotated is carried in a register and the column, cosines and
    // sines (read-only here) are loaded independently of that chain
    double a = __ldg(hcol + c);
#pragma unroll 4
    for (int k = 0; k < j; ++k) {
      double b = __ldg(hcol + size_t(k + 1) * C + c);
      apply_rot(a, b, __ldg(cs + k), __ldg(sn + k));
      Hj[k] = a;
      a = b;
    }
    const double hlast = __ldg(hcol + size_t(j + 1) * C + c);
    if (!isfinite(hlast)) gm_error(G, E2D_ERR_NAN);
    Hj[j] = a;
    Hj[j + 1] = hlast;
    // generate_rotation (GMRES2D.h:761-775)
    const double dx = Hj[j], dy = Hj[j + 1];
    double cj, sj;
    if (dy == 0.0) {
      cj = 1.0; sj = 0.0;
    } else if (fabs(dy) > fabs(dx)) {
      const double t = dx / dy;
      sj = 1.0 / sqrt(1.0 + t * t);
      cj = t * sj;
    } else {
      const double t = dy / dx;
      cj = 1.0 / sqrt(1.0 + t * t);
      sj = t * cj;
    }
    cs[j] = cj; sn[j] = sj;
    apply_rot(Hj[j], Hj[j + 1], cj, sj);
    apply_rot(sv[j], sv[j + 1], cj, sj);
    const double rr = fabs(sv[j + 1]) / G.resid0[c];
    G.relres[c] = rr;
    int f = 0;
    if (rr <= G.tol[c]) f = GF_MET;
    else if (its >= cap) f = GF_FAILED;
    else if (j >= mc - 1) f = GF_RESTARTED;
    if (f) {
      G.flags[c] = f;
      G.jstop[c] = j;
      G.iters[c] = its;
      active[c] = 0;
    } else {
      atomicAdd(&count, 1);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    *(volatile int*)(G.progress + j) = count;
    __threadfence_system();
  }
}

// End of a cycle: back substitution of the triangular system of every case
// that iterated in it (GMRES2D.h:1290-1299), its coefficients for the
// x update, and the cases that met the tolerance or the cap are done.
__global__ void gmres_backsub_kernel(GmresDev G, double* svals, int* kcount) {
  const int m = G.m;
  for (int c = threadIdx.x; c < G.ncase; c += blockDim.x) {
    kcount[c] = 0;
    const int f = G.flags[c];
    if (f & GF_DONE) continue;
    const int jj0 = G.jstop[c];
    if (jj0 < 0) continue;
    double* sv = G.sv + size_t(c) * (m + 1);
    const double* H = G.H + size_t(c) * m * (m + 1);
    for (int jj = jj0; jj >= 0; --jj) {
      sv[jj] /= H[size_t(jj) * (m + 1) + jj];
      for (int k = jj - 1; k >= 0; --k) sv[k] -= H[size_t(jj) * (m + 1) + k] * sv[jj];
    }
    for (int q = 0; q <= jj0; ++q) svals[size_t(c) * m + q] = sv[q];
    kcount[c] = jj0 + 1;
    if (f & (GF_MET | GF_FAILED)) G.flags[c] = f | GF_DONE;
  }
}

}  // namespace

struct e2d_nks_state {
  int m = 0;                 // restart length the buffers are sized for
  int ncase = 0;
  long long n = 0;           // vector length (4 * cells, ghosts included)
  int nper4 = 0;             // vector entries per block
  double* Uo = nullptr;      // [nblk][4][NCj][NCi]
  double* Minv = nullptr;    // [cells][16]
  IluPattern ilu_pat;        // ILU(k) pattern and schedules (host copy)
  IluDev ilu{};              // device copies, values and inverted diagonals
  int ilu_level = -1;        // level the ILU arrays are built for (-1: none)
  size_t ilu_smem = 0;       // dynamic shared memory of the apply (0: D.work)
  size_t ilu_factor_smem = 0; // dynamic shared memory of the factorization
  std::vector<void*> ilu_allocs;
  double* bvec = nullptr;
  double* x = nullptr;
  double* V = nullptr;       // (m + 1) * n
  double* Z = nullptr;       // m * n
  double* partial = nullptr; // [nblk * ch]
  unsigned* counter = nullptr; // [ncase] arrivals of the reduction CTAs
  int ch_vec = 1, ch_cell = 1; // CTAs per block of the vector / per-cell reductions
  std::vector<cudaGraphExec_t> graphs;  // Arnoldi step j, captured on its second use
  std::vector<int> graph_uses;
  double graph_eps0 = -1.0;
  int graph_ilu = -2;        // preconditioner the graphs were captured with:
                             // the ILU level of fill, -1 block Jacobi
  double* eps = nullptr;     // [ncase]
  double* nrm = nullptr;     // [ncase]
  double* hcol = nullptr;    // [m + 2][ncase]
  double* svals = nullptr;   // [ncase][m]
  int* kcount = nullptr;     // [ncase]
  double* cflv = nullptr;    // [ncase]
  int* active = nullptr;     // [ncase]
  double* slots = nullptr;   // [ncase][4]: CFL minimum and residual norms
  int* step0 = nullptr;
  double* host = nullptr;    // pinned staging
  size_t host_n = 0;
  // device-side GMRES bookkeeping; progress is host memory mapped into the
  // device, step_done the events of the Arnoldi steps in flight
  GmresDev gd{};
  int* progress_host = nullptr;
  int* gcfg = nullptr;       // GmresDev::cfg
  std::vector<cudaEvent_t> step_done;
  std::vector<void*> allocs;
};

namespace e2d_host {

void nks_free(e2d_handle* h) {
  if (!h->nks) return;
  for (auto g : h->nks->graphs)
    if (g) cudaGraphExecDestroy(g);
  for (auto ev : h->nks->step_done)
    if (ev) cudaEventDestroy(ev);
  if (h->nks->progress_host) cudaFreeHost(h->nks->progress_host);
  for (void* p : h->nks->allocs) cudaFree(p);
  for (void* p : h->nks->ilu_allocs) cudaFree(p);
  if (h->nks->host) cudaFreeHost(h->nks->host);
  delete h->nks;
  h->nks = nullptr;
}

}  // namespace e2d_host

namespace {

using namespace e2d_host;

void drop_graphs(e2d_nks_state* s);

}  // namespace

void e2d_host::nks_drop_graphs(e2d_handle* h) {
  if (h->nks) drop_graphs(h->nks);
}

namespace {

// Destroys the captured Arnoldi-step graphs: they hold the preconditioner's
// device pointers and launch shapes by value, so they must go before any of
// those arrays is freed or resized.
void drop_graphs(e2d_nks_state* s) {
  for (auto& g : s->graphs)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  std::fill(s->graph_uses.begin(), s->graph_uses.end(), 0);
  s->graph_ilu = -2;
}

template <class T> int nalloc(e2d_nks_state* s, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, sizeof(T) * (n ? n : 1)) != cudaSuccess) return E2D_ERR_NOMEM;
  s->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return 0;
}

int nks_setup(e2d_handle* h, int m) {
  if (h->nks && h->nks->m >= m) return 0;
  nks_free(h);
  e2d_nks_state* s = new e2d_nks_state;
  h->nks = s;
  const int C = h->B.ncase;
  s->m = m;
  s->ncase = C;
  s->n = 4 * (long long)h->ncell;
  s->nper4 = 4 * h->B.NCi * h->B.NCj;
  const size_t n = size_t(s->n);
  int rc;
  if ((rc = nalloc(s, &s->Uo, n)) || (rc = nalloc(s, &s->Minv, 16 * h->ncell)) || (rc = nalloc(s, &s->bvec, n)) ||
      (rc = nalloc(s, &s->x, n)) || (rc = nalloc(s, &s->V, (m + 1) * n)) || (rc = nalloc(s, &s->Z, m * n)) ||
      (rc = nalloc(s, &s->partial, size_t(h->B.nblk) * 16)) || (rc = nalloc(s, &s->counter, C)) ||
      (rc = nalloc(s, &s->eps, C)) || (rc = nalloc(s, &s->nrm, C)) ||
      (rc = nalloc(s, &s->hcol, size_t(m + 2) * C)) || (rc = nalloc(s, &s->svals, size_t(m) * C)) ||
      (rc = nalloc(s, &s->kcount, C)) || (rc = nalloc(s, &s->cflv, C)) || (rc = nalloc(s, &s->active, C)) ||
      (rc = nalloc(s, &s->slots, 4 * size_t(C))) || (rc = nalloc(s, &s->step0, 1))) {
    nks_free(h);
    return rc;
  }
  s->host_n = std::max(std::max(size_t(m + 2) * C, size_t(m + 1) * C + C), 5 * size_t(C)) + 8;
  if (cudaMallocHost(&s->host, sizeof(double) * s->host_n) != cudaSuccess) {
    nks_free(h);
    return E2D_ERR_NOMEM;
  }
  GmresDev& G = s->gd;
  G.m = m;
  G.ncase = C;
  if ((rc = nalloc(s, &G.H, size_t(C) * m * (m + 1))) || (rc = nalloc(s, &G.cs, size_t(C) * m)) ||
      (rc = nalloc(s, &G.sn, size_t(C) * m)) || (rc = nalloc(s, &G.sv, size_t(C) * (m + 1))) ||
      (rc = nalloc(s, &G.resid0, C)) || (rc = nalloc(s, &G.relres, C)) || (rc = nalloc(s, &G.tol, C)) ||
      (rc = nalloc(s, &G.iters, C)) || (rc = nalloc(s, &G.flags, C)) || (rc = nalloc(s, &G.jstop, C)) ||
      (rc = nalloc(s, &G.its, 1)) || (rc = nalloc(s, &G.err, 1)) || (rc = nalloc(s, &s->gcfg, 2))) {
    nks_free(h);
    return rc;
  }
  if (cudaHostAlloc(&s->progress_host, sizeof(int) * m, cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(reinterpret_cast<void**>(&G.progress), s->progress_host, 0) != cudaSuccess) {
    nks_free(h);
    return E2D_ERR_NOMEM;
  }
  G.cfg = s->gcfg;
  s->step_done.assign(m, nullptr);
  for (auto& ev : s->step_done)
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      nks_free(h);
      return E2D_ERR_CUDA;
    }
  E2D_CK(cudaMemsetAsync(s->V, 0, sizeof(double) * (m + 1) * n, h->stream));
  E2D_CK(cudaMemsetAsync(s->Z, 0, sizeof(double) * m * n, h->stream));
  E2D_CK(cudaMemsetAsync(s->bvec, 0, sizeof(double) * n, h->stream));
  E2D_CK(cudaMemsetAsync(s->step0, 0, sizeof(int), h->stream));
  E2D_CK(cudaMemsetAsync(s->counter, 0, sizeof(unsigned) * C, h->stream));
  // enough CTAs per block for small block counts (about 512 double2 / 512
  // cells per CTA), at most 16
  s->ch_vec = std::max(1, std::min(16, s->nper4 / 2 / 512));
  s->graphs.assign(m, nullptr);
  s->graph_uses.assign(m, 0);
  s->ch_cell = std::max(1, std::min(16, h->B.NCi * h->B.NCj / 512));
  identity_blocks_kernel<<<VGRID, VT, 0, h->stream>>>(s->Minv, (long long)h->ncell);
  E2D_CK(cudaGetLastError());
  return 0;
}

int grid_for(long long n) {
  long long g = (n + VT - 1) / VT;
  if (g > VGRID) g = VGRID;
  return int(g < 1 ? 1 : g);
}

// ILU(k) pattern, schedules and value arrays for the handle's block shape,
// built once per level of fill.
int ilu_setup(e2d_handle* h, int level) {
  e2d_nks_state* s = h->nks;
  if (s->ilu_level == level) return 0;
  drop_graphs(s);  // they reference the arrays freed next
  for (void* p : s->ilu_allocs) cudaFree(p);
  s->ilu_allocs.clear();
  s->ilu_level = -1;
  IluPattern& P = s->ilu_pat;
  if (!ilu_pattern(h->B.nci, h->B.ncj, level, P)) return E2D_ERR_NOMEM;
  IluDev& D = s->ilu;
  D = IluDev{};
  D.nrow = P.nrow; D.nnz = P.nnz; D.nflev = P.nflev; D.nblev = P.nblev; D.maxrow = P.maxrow;
  D.maxops = P.maxops;
  auto up = [&](const void* src, size_t bytes, void** dst) -> int {
    void* q = nullptr;
    if (cudaMalloc(&q, bytes ? bytes : 1) != cudaSuccess) return E2D_ERR_NOMEM;
    s->ilu_allocs.push_back(q);
    if (src && bytes && cudaMemcpy(q, src, bytes, cudaMemcpyHostToDevice) != cudaSuccess) return E2D_ERR_CUDA;
    *dst = q;
    return 0;
  };
  const int nblk = h->B.nblk;
  int rc;
  void *a0, *a1, *a2, *a3, *a4, *a5, *a6, *a7, *a8, *a9, *d0, *d1, *x0, *x1, *v0, *v1;
  if ((rc = up(P.row_ptr.data(), sizeof(int) * P.row_ptr.size(), &a0)) ||
      (rc = up(P.nlow.data(), sizeof(int) * P.nlow.size(), &a1)) ||
      (rc = up(P.col.data(), sizeof(int) * P.col.size(), &a2)) ||
      (rc = up(P.fop_ptr.data(), sizeof(int) * P.fop_ptr.size(), &a3)) ||
      (rc = up(P.fop.data(), sizeof(int2) * P.fop.size(), &a4)) ||
      (rc = up(P.flev_ptr.data(), sizeof(int) * P.flev_ptr.size(), &a5)) ||
      (rc = up(P.flev_rows.data(), sizeof(int) * P.flev_rows.size(), &a6)) ||
      (rc = up(P.blev_ptr.data(), sizeof(int) * P.blev_ptr.size(), &a7)) ||
      (rc = up(P.blev_rows.data(), sizeof(int) * P.blev_rows.size(), &a8)) ||
      (rc = up(P.apos.data(), sizeof(int) * P.apos.size(), &a9)) ||
      (rc = up(P.fdesc.data(), sizeof(int4) * P.fdesc.size(), &d0)) ||
      (rc = up(P.bdesc.data(), sizeof(int4) * P.bdesc.size(), &d1)) ||
      (rc = up(P.xdesc.data(), sizeof(int4) * P.xdesc.size(), &x0)) ||
      (rc = up(P.xops.data(), sizeof(int2) * P.xops.size(), &x1)) ||
      (rc = up(nullptr, sizeof(double) * 16 * size_t(P.nnz) * nblk, &v0)) ||
      (rc = up(nullptr, sizeof(double) * 16 * size_t(P.nrow) * nblk, &v1)))
    return rc;
  D.row_ptr = static_cast<int*>(a0); D.nlow = static_cast<int*>(a1); D.col = static_cast<int*>(a2);
  D.fop_ptr = static_cast<int*>(a3); D.fop = static_cast<int2*>(a4);
  D.flev_ptr = static_cast<int*>(a5); D.flev_rows = static_cast<int*>(a6);
  D.blev_ptr = static_cast<int*>(a7); D.blev_rows = static_cast<int*>(a8); D.apos = static_cast<int*>(a9);
  D.fdesc = static_cast<int4*>(d0); D.bdesc = static_cast<int4*>(d1);
  D.xdesc = static_cast<int4*>(x0); D.xops = static_cast<int2*>(x1);
  D.vals = static_cast<double*>(v0); D.dinv = static_cast<double*>(v1);
  // a block's vector in shared memory when it fits, else a global work array
  const size_t smem = sizeof(double) * 4 * size_t(P.nrow) + sizeof(int4) * 2 * size_t(P.nrow) +
                      sizeof(int) * size_t(P.nflev + P.nblev + 2);
  int dev = 0, optin = 0;
  E2D_CK(cudaGetDevice(&dev));
  E2D_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  if (smem <= size_t(optin)) {
    E2D_CK(cudaFuncSetAttribute(ilu_apply_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    s->ilu_smem = smem;
  } else {
    void* w;
    if ((rc = up(nullptr, sizeof(double) * 4 * size_t(P.nrow) * nblk, &w))) return rc;
    D.work = static_cast<double*>(w);
    s->ilu_smem = 0;
  }
  // one row (blocks, columns, work list) per 16-thread group
  s->ilu_factor_smem = ilu_factor_smem_bytes(P);
  cudaFuncAttributes fa{};
  E2D_CK(cudaFuncGetAttributes(&fa, ilu_factor_kernel));  // its static shared memory counts too
  if (s->ilu_factor_smem + fa.sharedSizeBytes > size_t(optin)) return E2D_ERR_ARG;
  E2D_CK(cudaFuncSetAttribute(ilu_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(s->ilu_factor_smem)));
  s->ilu_level = level;
  return 0;
}

bool use_ilu(const e2d_nks_params& p) { return p.block_preconditioner == E2D_PRECON_BLOCK_ILUK; }

// The preconditioner at the current state and dt (Update_Jacobian_and_Preconditioner).
int precon_build(e2d_handle* h, const e2d_nks_params& p, double ao, const Blocks& B) {
  e2d_nks_state* s = h->nks;
  const long long nint = (long long)h->B.nblk * h->B.nci * h->B.ncj;
  if (use_ilu(p)) {
    int rc;
    if ((rc = ilu_setup(h, p.ilu_level_of_fill))) return rc;
    E2D_CK(cudaMemsetAsync(s->ilu.vals, 0, sizeof(double) * 16 * size_t(s->ilu.nnz) * h->B.nblk, h->stream));
    ilu_assemble_kernel<<<grid_for(nint) * 2, 128, 0, h->stream>>>(B, s->ilu, ao,
                                                                   p.jacobian_order == E2D_JACOBIAN_FIRST_ORDER_HLLE);
    E2D_CK(cudaGetLastError());
    ilu_factor_kernel<<<h->B.nblk, ILU_THREADS, s->ilu_factor_smem, h->stream>>>(B, s->ilu);
    E2D_CK(cudaGetLastError());
    return 0;
  }
  precon_build_kernel<<<grid_for(nint) * 2, 128, 0, h->stream>>>(B, s->Minv, ao, p.jacobian_order);
  E2D_CK(cudaGetLastError());
  return 0;
}

// The per-case active mask the kernels see (and the stage kernel through
// Blocks::case_active).
int set_active(e2d_handle* h, const std::vector<int>& on) {
  e2d_nks_state* s = h->nks;
  int* hb = reinterpret_cast<int*>(s->host);
  E2D_CK(cudaStreamSynchronize(h->stream));  // the staging buffer is free
  for (int c = 0; c < s->ncase; ++c) hb[c] = on[c];
  E2D_CK(cudaMemcpyAsync(s->active, hb, sizeof(int) * s->ncase, cudaMemcpyHostToDevice, h->stream));
  E2D_CK(cudaStreamSynchronize(h->stream));
  return 0;
}

Blocks act(e2d_handle* h) {
  Blocks B = h->B;
  B.case_active = h->nks->active;
  return B;
}

// Stage kernel in Frechet mode: v = (R(U)/normR - b)/eps - (z/dt) normU/normR.
cudaError_t launch_frechet(e2d_handle* h, const double* z, double* v, const Norm4& nm) {
  StageArgs a{};
  a.B = act(h);
  a.mode = 3;
  a.fuse_next = 0;
  a.hist = nullptr;
  a.step = h->step;
  a.Win = h->B.W;
  a.Ubase = h->B.U;
  a.Wout = h->B.W;
  a.Uout = h->B.U;
  a.nks_b = h->nks->bvec;
  a.nks_z = z;
  a.nks_v = v;
  a.nks_eps = h->nks->eps;
  for (int k = 0; k < 4; ++k) { a.normU[k] = nm.u[k]; a.normR[k] = nm.r[k]; }
  return launch_stage_args(h, a);
}

// Perturbed residual + Frechet product: U = Uo + eps*dir (all cells), ghost
// exchange and BCs, residual, v = J dir (GMRES2D.h:1106-1221).
int matvec(e2d_handle* h, const double* dir, double* v, const Norm4& nm) {
  e2d_nks_state* s = h->nks;
  perturb_kernel<<<grid_for((long long)h->ncell), VT, 0, h->stream>>>(act(h), s->Uo, dir, s->eps, nm);
  E2D_CK(cudaGetLastError());
  E2D_CK(ghost_fill_for(h, 0));
  E2D_CK(launch_frechet(h, dir, v, nm));
  return 0;
}

// out[c] = f(dot(a, b) over case c) for the active cases.
int dot(e2d_handle* h, const double* a, const double* b, double* out, int fin, double eps0 = 0.0) {
  e2d_nks_state* s = h->nks;
  const Blocks B = act(h);
  blk_dot_kernel<<<h->B.nblk * s->ch_vec, VT, 0, h->stream>>>(a, b, s->nper4 / 2, s->ch_vec, s->partial, s->counter,
                                                               out, fin, eps0, B);
  E2D_CK(cudaGetLastError());
  return 0;
}

// y -= coef[case] * x, then out[case] = f(dot(y, b)) (b null: dot(y, y)).
int axpy_dot(e2d_handle* h, double* y, const double* x, const double* coef, const double* b, double* out, int fin) {
  e2d_nks_state* s = h->nks;
  axpy_dot_kernel<<<h->B.nblk * s->ch_vec, VT, 0, h->stream>>>(y, x, coef, b, s->nper4 / 2, s->ch_vec, s->partial,
                                                               s->counter, out, fin, act(h));
  E2D_CK(cudaGetLastError());
  return 0;
}

int axpy(e2d_handle* h, double* y, const double* x, const double* coef, double sign, double alpha) {
  e2d_nks_state* s = h->nks;
  axpy_kernel<<<VGRID, VT, 0, h->stream>>>(y, x, s->n / 2, s->nper4 / 2, coef, sign, alpha, act(h));
  E2D_CK(cudaGetLastError());
  return 0;
}

int scale(e2d_handle* h, double* y, const double* sdev, double sign) {
  e2d_nks_state* s = h->nks;
  scale_kernel<<<VGRID, VT, 0, h->stream>>>(y, s->n / 2, s->nper4 / 2, sdev, sign, act(h));
  E2D_CK(cudaGetLastError());
  return 0;
}

int fetch(e2d_handle* h, const double* dev, size_t count, double* out) {
  E2D_CK(cudaMemcpyAsync(h->nks->host, dev, sizeof(double) * count, cudaMemcpyDeviceToHost, h->stream));
  E2D_CK(cudaStreamSynchronize(h->stream));
  memcpy(out, h->nks->host, sizeof(double) * count);
  return 0;
}

// z = M^-1 v with the ILU factors, every active block.
int ilu_apply(e2d_handle* h, const double* v, double* z) {
  e2d_nks_state* s = h->nks;
  if (s->ilu_smem)
    ilu_apply_kernel<true><<<h->B.nblk, ILU_APPLY_THREADS, s->ilu_smem, h->stream>>>(act(h), s->ilu, v, z);
  else
    ilu_apply_kernel<false><<<h->B.nblk, ILU_APPLY_THREADS, 0, h->stream>>>(act(h), s->ilu, v, z);
  E2D_CK(cudaGetLastError());
  return 0;
}

// One Arnoldi step j of GMRES (GMRES2D.h:1020-1250): z_j = M^-1 v_j with
// eps = eps0 / ||z_j||, v_{j+1} = J z_j, modified Gram-Schmidt against
// v_0..v_j into the Hessenberg column, ||v_{j+1}||, v_{j+1} /= it.  Only
// enqueues device work (it is captured into a graph per j).
int arnoldi_step(e2d_handle* h, int j, double eps0, const Norm4& nm, bool ilu) {
  e2d_nks_state* s = h->nks;
  const int C = s->ncase;
  const long long n = s->n;
  int rc;
  double* Vj = s->V + size_t(j) * n;
  double* Vn = s->V + size_t(j + 1) * n;
  double* Zj = s->Z + size_t(j) * n;
  if (ilu) {
    if ((rc = ilu_apply(h, Vj, Zj))) return rc;
    if ((rc = dot(h, Zj, Zj, s->eps, FIN_EPS, eps0))) return rc;
  } else {
    // v_j = w_j / h(j, j-1) for j > 0 (the previous step's closing scale,
    // deferred into this pass; h(j, j-1) is still in the column buffer)
    precon_apply_kernel<<<h->B.nblk * s->ch_cell, VT, 0, h->stream>>>(
        s->Minv, Vj, Zj, h->B.NCi * h->B.NCj, s->ch_cell, s->partial, s->counter, s->eps, eps0,
        j > 0 ? s->hcol + size_t(j) * C : nullptr, act(h));
    E2D_CK(cudaGetLastError());
  }
  if ((rc = matvec(h, Zj, Vn, nm))) return rc;
  // modified Gram-Schmidt (GMRES2D.h:1224-1240): h_k = (w, v_k), w -= h_k
  // v_k for k = 0..j, then ||w||; each update runs fused with the next dot
  double* hn = s->hcol + size_t(j + 1) * C;
  if ((rc = dot(h, Vn, s->V, s->hcol, FIN_SUM))) return rc;
  for (int k = 0; k <= j; ++k) {
    const double* hk = s->hcol + size_t(k) * C;
    const bool last = k == j;
    if ((rc = axpy_dot(h, Vn, s->V + size_t(k) * n, hk, last ? nullptr : s->V + size_t(k + 1) * n,
                       last ? hn : s->hcol + size_t(k + 1) * C, last ? FIN_SQRT : FIN_SUM)))
      return rc;
  }
  // v_{j+1} = w / ||w||: here for ILU(k); the block-Jacobi apply of the next
  // step does it in its own pass (a step that ends the cycle leaves the
  // last vector unscaled, which nothing reads)
  if (ilu && (rc = scale(h, Vn, hn, 1.0))) return rc;
  gmres_givens_kernel<<<1, VT, 0, h->stream>>>(s->gd, s->hcol, s->active, j);
  E2D_CK(cudaGetLastError());
  return 0;
}

// Arnoldi step j through a CUDA graph: the first use of a j runs eagerly,
// the second captures the step, later uses replay it (one launch instead of
// about 2j + 8).  Every pointer the step reads is fixed for the life of the
// work arrays; the per-case active mask and scalars are read from device
// memory at run time.
int run_arnoldi(e2d_handle* h, int j, double eps0, const Norm4& nm, bool ilu) {
  e2d_nks_state* s = h->nks;
  const int key = ilu ? s->ilu_level : -1;
  if (s->graph_eps0 != eps0 || s->graph_ilu != key) {
    drop_graphs(s);
    s->graph_eps0 = eps0;
    s->graph_ilu = key;
  }
  if (s->graphs[j]) {
    E2D_CK(cudaGraphLaunch(s->graphs[j], h->stream));
    return 0;
  }
  if (s->graph_uses[j]++ == 0) return arnoldi_step(h, j, eps0, nm, ilu);
  cudaGraph_t g = nullptr;
  E2D_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  const int rc = arnoldi_step(h, j, eps0, nm, ilu);
  const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return rc ? rc : E2D_ERR_CUDA;
  }
  const cudaError_t e2 = cudaGraphInstantiate(&s->graphs[j], g, 0);
  cudaGraphDestroy(g);
  if (e2 != cudaSuccess) { s->graphs[j] = nullptr; return E2D_ERR_CUDA; }
  E2D_CK(cudaGraphLaunch(s->graphs[j], h->stream));
  return 0;
}

struct GmresCase {
  double resid0 = 0, relres = 0;
  int iters = 0;
  bool restarted = false, failed = false, met = false;
};

// Steps launched ahead of the one whose progress the host reads.
constexpr int GMRES_LOOKAHEAD = 2;

// GMRES_RightPrecon_MatrixFree::solve (GMRES2D.h:790-1544) with the default
// options (first-order Frechet derivative, no GMRES check), for every case
// with on[c] set, in lockstep.  The rotations, the stop test and the back
// substitution run on the device (gmres_*_kernel); the host launches the
// Arnoldi steps of a cycle one after another and stops launching when the
// step GMRES_LOOKAHEAD behind reports no case still iterating (the steps
// already launched run with every case masked off).  One synchronisation per
// cycle reads the cases' results.
int gmres(e2d_handle* h, const e2d_nks_params& p, const std::vector<double>& tol, const std::vector<int>& on,
          const Norm4& nm, std::vector<GmresCase>& G) {
  e2d_nks_state* s = h->nks;
  const int m = p.gmres_restart, C = s->ncase;
  const long long n = s->n;
  const size_t nb = sizeof(double) * size_t(n);
  int rc;
  const GmresDev D = s->gd;
  G.assign(C, GmresCase());
  // per-case tolerance and start state: the cases not iterating are done
  double* ht = s->host;
  int* hf = reinterpret_cast<int*>(s->host + C);
  E2D_CK(cudaStreamSynchronize(h->stream));  // the staging buffer is free
  for (int c = 0; c < C; ++c) {
    ht[c] = tol[c];
    hf[c] = on[c] ? 0 : GF_DONE;
  }
  hf[C] = m;  // cycle length and iteration cap of this solve
  hf[C + 1] = p.max_gmres;
  E2D_CK(cudaMemcpyAsync(s->gcfg, hf + C, sizeof(int) * 2, cudaMemcpyHostToDevice, h->stream));
  E2D_CK(cudaMemcpyAsync(D.tol, ht, sizeof(double) * C, cudaMemcpyHostToDevice, h->stream));
  E2D_CK(cudaMemcpyAsync(D.flags, hf, sizeof(int) * C, cudaMemcpyHostToDevice, h->stream));
  E2D_CK(cudaMemsetAsync(D.its, 0, sizeof(int), h->stream));
  E2D_CK(cudaMemsetAsync(D.err, 0, sizeof(int), h->stream));
  E2D_CK(cudaMemsetAsync(s->x, 0, nb, h->stream));
  // V(0) = b (the Initialize'd V(0) is zero; daxpy adds b)
  E2D_CK(cudaMemcpyAsync(s->V, s->bvec, nb, cudaMemcpyDeviceToDevice, h->stream));
  std::vector<double> res(3 * size_t(C));
  std::vector<int> ires(3 * size_t(C) + 1);
  bool first = true;
  for (;;) {
    gmres_cycle_active_kernel<<<1, VT, 0, h->stream>>>(D, s->active);
    E2D_CK(cudaGetLastError());
    if (!first) {
      // V(0) = J x + b with eps = eps0 / ||x|| (GMRES2D.h:838-1000)
      if ((rc = dot(h, s->x, s->x, s->eps, FIN_EPS, p.epsilon0))) return rc;
      if ((rc = matvec(h, s->x, s->V, nm))) return rc;
      if ((rc = axpy(h, s->V, s->bvec, nullptr, 0.0, 1.0))) return rc;
    }
    if ((rc = dot(h, s->V, s->V, s->nrm, FIN_SQRT))) return rc;
    if ((rc = scale(h, s->V, s->nrm, -1.0))) return rc;
    gmres_cycle_start_kernel<<<1, VT, 0, h->stream>>>(D, s->nrm, s->active, first ? 1 : 0);
    E2D_CK(cudaGetLastError());
    for (int q = 0; q < m; ++q) s->progress_host[q] = -1;
    for (int j = 0; j < m; ++j) {
      if ((rc = run_arnoldi(h, j, p.epsilon0, nm, use_ilu(p)))) return rc;
      E2D_CK(cudaEventRecord(s->step_done[j], h->stream));
      const int k = j - GMRES_LOOKAHEAD;
      if (k < 0) continue;
      E2D_CK(cudaEventSynchronize(s->step_done[k]));
      if (*(volatile int*)(s->progress_host + k) == 0) break;  // no case iterates after step k
    }
    // back substitution and x += sum s_k Z_k per case (GMRES2D.h:1290-1304)
    gmres_backsub_kernel<<<1, VT, 0, h->stream>>>(D, s->svals, s->kcount);
    E2D_CK(cudaGetLastError());
    update_x_kernel<<<VGRID, VT, 0, h->stream>>>(s->x, s->Z, n, s->nper4, s->svals, s->kcount, m, h->B);
    E2D_CK(cudaGetLastError());
    double* hr = s->host;
    int* hi = reinterpret_cast<int*>(s->host + 3 * size_t(C));
    E2D_CK(cudaMemcpyAsync(hr, D.resid0, sizeof(double) * C, cudaMemcpyDeviceToHost, h->stream));
    E2D_CK(cudaMemcpyAsync(hr + C, D.relres, sizeof(double) * C, cudaMemcpyDeviceToHost, h->stream));
    E2D_CK(cudaMemcpyAsync(hi, D.iters, sizeof(int) * C, cudaMemcpyDeviceToHost, h->stream));
    E2D_CK(cudaMemcpyAsync(hi + C, D.flags, sizeof(int) * C, cudaMemcpyDeviceToHost, h->stream));
    E2D_CK(cudaMemcpyAsync(hi + 2 * C, D.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    E2D_CK(cudaStreamSynchronize(h->stream));
    if (hi[2 * C]) return hi[2 * C];
    bool more = false;
    for (int c = 0; c < C; ++c) {
      if (!on[c]) continue;
      GmresCase& g = G[c];
      const int f = hi[C + c];
      g.resid0 = hr[c];
      g.relres = hr[C + c];
      g.iters = hi[c];
      if (f & GF_RESTARTED) g.restarted = true;
      if (f & GF_MET) g.met = true;
      if (f & GF_FAILED) g.failed = true;
      if (!(f & GF_DONE)) more = true;
    }
    if (!more) break;
    first = false;
  }
  return 0;
}

}  // namespace

static int nks_run(e2d_handle* h, const e2d_nks_params* p, e2d_nks_step* hist, int* n_steps);

static bool params_ok(const e2d_nks_params& p) {
  return (p.block_preconditioner == E2D_PRECON_BLOCK_JACOBI || p.block_preconditioner == E2D_PRECON_BLOCK_ILUK) &&
         p.ilu_level_of_fill >= 0 && p.ilu_level_of_fill <= 16 &&
         (p.jacobian_order == E2D_JACOBIAN_FIRST_ORDER_HLLE || p.jacobian_order == E2D_JACOBIAN_SOURCE_TERMS_ONLY);
}

// The Newton-Krylov solve starts with the limiters unfrozen and never
// freezes them (Evaluate_Limiters, NKS2D.h:90; its freezing code is
// disabled): the solve runs without the freezing machinery.
extern "C" int e2d_nks(e2d_handle* h, const e2d_nks_params* p, e2d_nks_step* hist, int* n_steps) {
  if (!h) return nks_run(h, p, hist, n_steps);
  if (!h->subs.empty()) return p ? composite_nks(h, p, hist, n_steps) : E2D_ERR_ARG;
  if (h->freeze && cudaMemset(h->freeze, 0, sizeof(int) * h->B.ncase) != cudaSuccess) return E2D_ERR_CUDA;
  const int* saved = h->B.freeze;
  h->B.freeze = nullptr;
  const int rc = nks_run(h, p, hist, n_steps);
  h->B.freeze = saved;
  return rc;
}

static int nks_run(e2d_handle* h, const e2d_nks_params* p, e2d_nks_step* hist, int* n_steps) {
  if (!h || !p || p->max_newton < 0 || p->gmres_restart < 1 || p->gmres_restart > 500 || p->max_gmres < 1 ||
      !(p->epsilon0 > 0.0) || !(p->cfl0 > 0.0) || !(p->gmres_tol_initial > 0.0) || !(p->gmres_tol_final > 0.0) ||
      !(p->min_ratio > 0.0) || !params_ok(*p)) {
    if (n_steps) *n_steps = 0;
    return E2D_ERR_ARG;
  }
  const int C = h->B.ncase;
  if (n_steps)
    for (int c = 0; c < C; ++c) n_steps[c] = 0;
  if (cudaSetDevice(h->device) != cudaSuccess) return E2D_ERR_CUDA;
  int rc;
  if ((rc = nks_setup(h, p->gmres_restart))) return rc;
  e2d_nks_state* s = h->nks;
  Blocks& B = h->B;
  const long long nint = (long long)B.nblk * B.nci * B.ncj;
  // normalisation by the standard atmosphere (GMRES_Block::set_normalize_values,
  // Euler2DQuadNKS.h:148-166)
  const double ao = sqrt(h->sc.gamma * P_STD / RHO_STD);
  const double rho = RHO_STD;
  Norm4 nm;
  nm.u[0] = rho; nm.u[1] = rho * ao; nm.u[2] = rho * ao; nm.u[3] = rho * ao * ao;
  nm.r[0] = rho * ao; nm.r[1] = rho * ao * ao; nm.r[2] = rho * ao * ao; nm.r[3] = rho * ao * ao * ao;
  // GMRES forcing: tol = min(0.9, tol_i * ratio^(log(f/i)/log(max(L, 1e-18))))
  const double L = p->overall_tol > 1e-18 ? p->overall_tol : 1e-18;
  const double forcing = log(p->gmres_tol_final / p->gmres_tol_initial) / log(L);
  std::vector<int> on(C, 1), cnt(C, 0);
  std::vector<double> l2_first(C, -1.0), ratio(C, 1.0), cfl(C, 0.0), tol(C, 0.0), slots(4 * size_t(C));
  std::vector<e2d_nks_step> cur(C);
  std::vector<GmresCase> G;
  auto record = [&](int c) {
    if (hist) hist[size_t(c) * p->max_newton + cnt[c]] = cur[c];
    ++cnt[c];
  };
  auto finish = [&](int code) {
    if (n_steps)
      for (int c = 0; c < C; ++c) n_steps[c] = cnt[c];
    B.case_active = nullptr;
    return code;
  };
  // the caller's state: exchange and BCs first (as before the solver call)
  E2D_CK(launch_ghost_fill(B, h->stream));
  for (int newton = 1; newton <= p->max_newton; ++newton) {
    if ((rc = set_active(h, on))) return finish(rc);
    // residual and its density norms (NKS2D.h:552-593)
    B.case_active = s->active;
    const cudaError_t e0 = launch_stage_any(h, 0, 0);
    B.case_active = nullptr;
    E2D_CK(e0);
    E2D_CK(launch_slot_init(s->slots, s->step0, 0, C, h->stream));
    E2D_CK(launch_norms(B, h->part, s->slots, s->step0, h->stream));
    if ((rc = fetch(h, s->slots, 4 * size_t(C), slots.data()))) return finish(rc);
    if ((rc = check_status(h))) return finish(rc);
    bool any = false;
    for (int c = 0; c < C; ++c) {
      if (!on[c]) continue;
      const double l2 = slots[4 * c + 2];
      if (!std::isfinite(l2)) return finish(E2D_ERR_NAN);
      if (l2_first[c] <= 0.0)
        l2_first[c] = (p->l2_reference && p->l2_reference[c] > 0.0) ? p->l2_reference[c] : l2;
      ratio[c] = l2 / l2_first[c];
      cur[c] = e2d_nks_step{};
      cur[c].l1 = slots[4 * c + 1]; cur[c].l2 = l2; cur[c].lmax = slots[4 * c + 3]; cur[c].ratio = ratio[c];
      if (!(ratio[c] > p->overall_tol)) {
        record(c);  // converged: the loop's stop test (NKS2D.h:902)
        on[c] = 0;
        continue;
      }
      any = true;
      // SER finite time step (Finite_Time_Step, NKS2D.h:1316-1340)
      const double cr = (p->cfl_reference && p->cfl_reference[c] > 0.0) ? l2 / p->cfl_reference[c] : ratio[c];
      cfl[c] = cr > p->min_ratio ? p->cfl0 * pow(std::max(1.0, 1.0 / cr), 1.0) : p->cfl0 / p->min_ratio;
      cur[c].cfl = cfl[c];
      tol[c] = std::min(0.9, p->gmres_tol_initial * pow(ratio[c], forcing));
    }
    if (!any) break;
    if ((rc = set_active(h, on))) return finish(rc);
    double* hc = s->host;
    for (int c = 0; c < C; ++c) hc[c] = cfl[c];
    E2D_CK(cudaMemcpyAsync(s->cflv, hc, sizeof(double) * C, cudaMemcpyHostToDevice, h->stream));
    E2D_CK(launch_slot_init(s->slots, s->step0, 0, C, h->stream));
    E2D_CK(launch_cfl(B, s->slots, s->step0, h->stream));
    set_dt_kernel<<<grid_for(nint), VT, 0, h->stream>>>(act(h), s->slots, s->cflv);
    E2D_CK(cudaGetLastError());
    // Uo = U (ghosts included) and the preconditioner at Uo
    E2D_CK(cudaMemcpyAsync(s->Uo, B.U, sizeof(double) * 4 * h->ncell, cudaMemcpyDeviceToDevice, h->stream));
    if ((rc = precon_build(h, *p, ao, act(h)))) return finish(rc);
    load_b_kernel<<<grid_for(nint), VT, 0, h->stream>>>(act(h), s->bvec, nm);
    E2D_CK(cudaGetLastError());
    if ((rc = gmres(h, *p, tol, on, nm, G))) return finish(rc);
    for (int c = 0; c < C; ++c) {
      if (!on[c]) continue;
      cur[c].gmres_resid0 = G[c].resid0; cur[c].gmres_relres = G[c].relres; cur[c].gmres_iters = G[c].iters;
      cur[c].gmres_restarts = G[c].restarted ? 1 : 0; cur[c].gmres_failed = G[c].failed ? 1 : 0;
      record(c);
    }
    // U = Uo + x for the cases still stepping, exchange and BCs (NKS2D.h:1058-1090)
    if ((rc = set_active(h, on))) return finish(rc);
    newton_update_kernel<<<grid_for(nint), VT, 0, h->stream>>>(act(h), s->Uo, s->x, nm, 1.0);
    E2D_CK(cudaGetLastError());
    E2D_CK(launch_ghost_fill(B, h->stream));
    if ((rc = check_status(h))) return finish(rc);
  }
  E2D_CK(cudaStreamSynchronize(h->stream));
  return finish(0);
}

// The Newton step's preconditioner alone (parity checks and callers that run
// their own Krylov solver): dt as the Newton loop sets it, the block
// preconditioner at the current state, z = M^-1 v.  Ghost rows are identity
// rows, as in the reference's block matrix: ghost entries pass through.
extern "C" int e2d_block_precon_apply(e2d_handle* h, const e2d_nks_params* p, double cfl, const double* v,
                                      double* z) {
  if (!h || !h->subs.empty() || !p || !v || !z || !(cfl > 0.0) || !params_ok(*p) || p->gmres_restart < 1 ||
      p->gmres_restart > 500)
    return E2D_ERR_ARG;
  if (cudaSetDevice(h->device) != cudaSuccess) return E2D_ERR_CUDA;
  int rc;
  if ((rc = nks_setup(h, p->gmres_restart))) return rc;
  e2d_nks_state* s = h->nks;
  Blocks& B = h->B;
  const int C = B.ncase;
  const long long nint = (long long)B.nblk * B.nci * B.ncj;
  const double ao = sqrt(h->sc.gamma * P_STD / RHO_STD);
  if ((rc = set_active(h, std::vector<int>(C, 1)))) return rc;
  E2D_CK(launch_ghost_fill(B, h->stream));
  for (int c = 0; c < C; ++c) s->host[c] = cfl;
  E2D_CK(cudaMemcpyAsync(s->cflv, s->host, sizeof(double) * C, cudaMemcpyHostToDevice, h->stream));
  E2D_CK(launch_slot_init(s->slots, s->step0, 0, C, h->stream));
  E2D_CK(launch_cfl(B, s->slots, s->step0, h->stream));
  set_dt_kernel<<<grid_for(nint), VT, 0, h->stream>>>(act(h), s->slots, s->cflv);
  E2D_CK(cudaGetLastError());
  if ((rc = precon_build(h, *p, ao, act(h)))) return rc;
  const size_t nb = sizeof(double) * size_t(s->n);
  E2D_CK(cudaMemcpyAsync(s->V, v, nb, cudaMemcpyHostToDevice, h->stream));
  if (use_ilu(*p)) {
    E2D_CK(cudaMemcpyAsync(s->Z, s->V, nb, cudaMemcpyDeviceToDevice, h->stream));
    if ((rc = ilu_apply(h, s->V, s->Z))) return rc;
  } else {
    precon_apply_kernel<<<B.nblk * s->ch_cell, VT, 0, h->stream>>>(s->Minv, s->V, s->Z, B.NCi * B.NCj, s->ch_cell,
                                                                   s->partial, s->counter, s->eps, 1.0, nullptr,
                                                                   act(h));
    E2D_CK(cudaGetLastError());
  }
  E2D_CK(cudaMemcpyAsync(z, s->Z, nb, cudaMemcpyDeviceToHost, h->stream));
  E2D_CK(cudaStreamSynchronize(h->stream));
  // the Krylov buffers start clean for the next solve
  E2D_CK(cudaMemsetAsync(s->V, 0, nb, h->stream));
  E2D_CK(cudaMemsetAsync(s->Z, 0, nb, h->stream));
  return check_status(h);
}

// The level-of-fill pattern the ILU(k) preconditioner uses for blocks of
// nci x ncj cells (host work only, no device needed): interior rows in cell
// order, columns ascending.  row_ptr gets nci*ncj + 1 offsets, col up to
// cap column indices; *nnz the pattern's size (col untouched when it
// exceeds cap); levels (may be NULL) the forward and backward level counts.
extern "C" int e2d_ilu_pattern(int32_t nci, int32_t ncj, int32_t level, int32_t* row_ptr, int32_t* col,
                               int32_t cap, int32_t* nnz, int32_t* levels) {
  if (nci < 1 || ncj < 1 || level < 0 || level > 16 || !row_ptr || !nnz || cap < 0 ||
      (long long)nci * ncj > (1 << 22))
    return E2D_ERR_ARG;
  IluPattern P;
  if (!ilu_pattern(nci, ncj, level, P)) return E2D_ERR_NOMEM;
  std::copy(P.row_ptr.begin(), P.row_ptr.end(), row_ptr);
  *nnz = P.nnz;
  if (col && P.nnz <= cap) std::copy(P.col.begin(), P.col.end(), col);
  if (levels) { levels[0] = P.nflev; levels[1] = P.nblev; }
  return 0;
}
