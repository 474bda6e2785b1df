// e2d_smooth.cuh — the explicit-stage pieces that run between the residual
// and the update when implicit residual smoothing is on, and the limiter
// freezing switch.  Included by e2d_capi.cu (compiled without contraction:
// FP64 in the reference's rounding order).
//
//   residual_smoothing_kernel  Residual_Smoothing (Euler2DQuadSingleBlock.cc:4521-4563)
//   stage_update_kernel        Update_Solution_Multistage_Explicit
//                              (Euler2DQuadSingleBlock.cc:5300-5430)
//   freeze_check_kernel        the limiter-freezing test of the explicit loop
//                              (Euler2DQuadSolvers.cc:794-803)
#pragma once
#include "e2d_device.cuh"

namespace e2d {

constexpr int SMOOTH_THREADS = 128;

// Gauss-Seidel smoothing of one block's stage residual R (slot 0), one CTA
// per block.  The reference smooths the cells one away from the block edges,
// ICl+1..ICu-1 x JCl+1..JCu-1, in lexicographic order (j outer, i inner),
// iters sweeps of
//   S(i,j) = (R(i,j) + eps*(S(i,j-1) + S(i-1,j) + S(i+1,j) + S(i,j+1))) / (1 + 4 eps)
// on a scratch copy S whose entries outside that region stay zero (the
// reference's second residual slot there, never written on this path), and
// then R = S on the region.  A cell reads its south and west neighbours from
// the current sweep and its east and north neighbours from the previous one,
// so every anti-diagonal i+j = const updates at once: the sweep runs
// diagonal by diagonal with a barrier between them and gives the
// lexicographic result bit for bit.  S lives in shared memory (dynamic,
// [4][ny+2][nx+2]) or, when SHARED is false, in the global scratch of the
// block (same layout).
template <bool SHARED>
__global__ void __launch_bounds__(SMOOTH_THREADS) residual_smoothing_kernel(Blocks B, double* R, double* scratch,
                                                                           double eps, int iters) {
  extern __shared__ __align__(16) double smem_s[];
  const int b = blockIdx.x;
  const int nx = B.nci - 2, ny = B.ncj - 2;
  if (nx <= 0 || ny <= 0) return;
  const int sx = nx + 2, sy = ny + 2, sv = sx * sy;
  double* S = SHARED ? smem_s : scratch + size_t(b) * 4 * sv;
  const int i0 = NG, j0 = NG;  // S(0, 0) is cell (ICl, JCl)
  for (int q = threadIdx.x; q < 4 * sv; q += blockDim.x) {
    const int v = q / sv, r = q % sv, jj = r / sx, ii = r % sx;
    const bool region = ii >= 1 && ii <= nx && jj >= 1 && jj <= ny;
    S[q] = region ? R[cell_var(B, b, v, j0 + jj, i0 + ii)] : 0.0;
  }
  __syncthreads();
  const double den = 1.0 + 4.0 * eps;
  for (int n = 0; n < iters; ++n) {
    for (int d = 0; d <= nx + ny - 2; ++d) {
      const int ylo = d - (nx - 1) > 0 ? d - (nx - 1) : 0, yhi = d < ny - 1 ? d : ny - 1;
      for (int k = threadIdx.x; k < 4 * (yhi - ylo + 1); k += blockDim.x) {
        const int v = k & 3, y = ylo + (k >> 2), x = d - y;
        const int jj = y + 1, ii = x + 1;
        double* Sv = S + v * sv;
        const double r = R[cell_var(B, b, v, j0 + jj, i0 + ii)];
        Sv[jj * sx + ii] =
            (r + eps * (Sv[(jj - 1) * sx + ii] + Sv[jj * sx + ii - 1] + Sv[jj * sx + ii + 1] + Sv[(jj + 1) * sx + ii])) /
            den;
      }
      __syncthreads();
    }
  }
  for (int q = threadIdx.x; q < 4 * sv; q += blockDim.x) {
    const int v = q / sv, r = q % sv, jj = r / sx, ii = r % sx;
    if (ii >= 1 && ii <= nx && jj >= 1 && jj <= ny) R[cell_var(B, b, v, j0 + jj, i0 + ii)] = S[q];
  }
}

// U = Ubase + omega*R on every interior cell, with the reference's handling
// of a non-physical result (global time step: the cell's index goes to the
// status word; local time step: up to ten halvings of the cell's step and
// residual), then W = W(U).  R keeps the (possibly halved) residual.
__global__ void stage_update_kernel(Blocks B, const double* Ubase, double* R, double omega, double* Wout,
                                    double* Uout) {
  const long long per = (long long)B.nci * B.ncj, n = per * B.nblk;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const int b = int(q / per), r = int(q % per);
    const int I = NG + r % B.nci, J = NG + r / B.nci;
    if (B.case_active && !B.case_active[case_id(B, b)]) continue;
    const size_t c = cell_sc(B, b, J, I);
    size_t o[4];
    double res[4];
    CState<double> uo;
    for (int v = 0; v < 4; ++v) { o[v] = cell_var(B, b, v, J, I); res[v] = R[o[v]]; }
    uo.d = Ubase[o[0]]; uo.mx = Ubase[o[1]]; uo.my = Ubase[o[2]]; uo.E = Ubase[o[3]];
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
          for (int v = 0; v < 4; ++v) res[v] = rrf * res[v];
          u.d = uo.d + omega * res[0]; u.mx = uo.mx + omega * res[1];
          u.my = uo.my + omega * res[2]; u.E = uo.E + omega * res[3];
          if (u.d > 0.0 && u.E > 0.0 && e_of_U(u) > 0.0) break;
        }
        B.dt[c] = dtc;
        if (u.d <= 0.0 || u.E <= 0.0 || e_of_U(u) <= 0.0) set_status(B.status, ST_NEGATIVE, int(c));
      }
    }
    for (int v = 0; v < 4; ++v) R[o[v]] = res[v];
    const PState<double> w = W_of_U(u, B.gm1);
    Uout[o[0]] = u.d; Uout[o[1]] = u.mx; Uout[o[2]] = u.my; Uout[o[3]] = u.E;
    Wout[o[0]] = w.d; Wout[o[1]] = w.u; Wout[o[2]] = w.v; Wout[o[3]] = w.p;
  }
}

// At the head of each explicit step but the first of a run: freeze the
// limiters of every case whose residual L2 norm (this step's history slot)
// is at or below the level.  Once frozen they stay frozen.
__global__ void freeze_check_kernel(const double* hist, const int* step, int ncase, double level, int* freeze,
                                    int* first) {
  if (threadIdx.x != 0) return;
  if (!*first)
    for (int c = 0; c < ncase; ++c)
      if (!freeze[c] && hist[4 * ((*step) * ncase + c) + 2] <= level) freeze[c] = 1;
  *first = 0;
}

}  // namespace e2d
