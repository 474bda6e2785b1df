// e2d_aux.cuh — ghost fill, time step and residual-norm kernels.
//
//   ghost_fill_kernel   same-resolution exchange between blocks
//                       (Send_All_Messages, src_2D/AMR/AdaptiveBlock2D_MessagePassing.h:7883;
//                        LoadSendBuffer/UnloadReceiveBuffer, src_2D/Euler2D/Euler2DQuad.h:1570-1650)
//                       followed by BCs (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:2354-2995)
//   cfl_kernel          CFL (Euler2DQuadSingleBlock.cc:3019-3080) + the global minimum
//                       (CFFC_Minimum_MPI, Euler2DQuadSolvers.cc:657-660)
//   norm kernels        L1/L2/Max_Norm_Residual (Euler2DQuadSingleBlock.cc:3111-3167,
//                       Euler2DQuadMultiBlock.cc:1017-1190)
// Compiled in the exact (no-FMA) translation unit only.
#pragma once
#include "e2d_device.cuh"
#include "e2d_geom.cuh"

#include <algorithm>

namespace e2d {

constexpr int AUX_THREADS = 256;
// most threads of a ghost-fill CTA; two such CTAs fit an SM (at most 56
// registers a thread), so a launch over 256 blocks runs in one wave
constexpr int GHOST_THREADS = 576;
constexpr double MILLION = 1000000.0;

// One edge-cell of the W or E (vertical) boundary: side 0 = W, 1 = E.
__device__ void bc_vertical(const Blocks& B, int b, int j, int side) {
  const int ICl = NG, ICu = B.nci + NG - 1;
  const int bc = side == 0 ? B.bcw[size_t(b) * B.NCj + j] : B.bce[size_t(b) * B.NCj + j];
  const int in = side == 0 ? ICl : ICu;           // first interior column
  const int dir = side == 0 ? -1 : 1;             // towards the ghosts
  const double* wo = side == 0 ? B.wow : B.woe;
  switch (bc) {
    case E2D_BC_NONE: break;
    case E2D_BC_FIXED:
      for (int g = 1; g <= NG; ++g) ghost_set(B, b, in + dir * g, j, wo_at(wo, b, B.NCj, j));
      break;
    case E2D_BC_REFLECTION: {
      double nx, ny;
      if (side == 0) nfaceW(B, b, ICl, j, nx, ny); else nfaceE(B, b, ICu, j, nx, ny);
      for (int g = 1; g <= NG; ++g)
        ghost_set(B, b, in + dir * g, j, reflect(ldW(B, b, in - dir * (g - 1), j), nx, ny));
      break;
    }
    case E2D_BC_PERIODIC:
      for (int g = 1; g <= NG; ++g)
        ghost_copy(B, b, in + dir * g, j, side == 0 ? ICu - g + 1 : ICl + g - 1, j);
      break;
    case E2D_BC_CHARACTERISTIC: {
      double nx, ny;
      if (side == 0) nfaceW(B, b, ICl, j, nx, ny); else nfaceE(B, b, ICu, j, nx, ny);
      ghost_set(B, b, in + dir, j, bc_char_pressure(ldW(B, b, in, j), wo_at(wo, b, B.NCj, j), nx, ny, B.g, B.gm1i));
      for (int g = 2; g <= NG; ++g) ghost_copy(B, b, in + dir * g, j, in + dir, j);
      break;
    }
    default:  // BC_CONSTANT_EXTRAPOLATION (and the reference's default)
      for (int g = 1; g <= NG; ++g) ghost_copy(B, b, in + dir * g, j, in, j);
      break;
  }
}

// One edge-cell of the S or N (horizontal) boundary: side 0 = S, 1 = N.
__device__ void bc_horizontal(const Blocks& B, int b, int i, int side) {
  const int JCl = NG, JCu = B.ncj + NG - 1;
  const int bc = side == 0 ? B.bcs[size_t(b) * B.NCi + i] : B.bcn[size_t(b) * B.NCi + i];
  const int in = side == 0 ? JCl : JCu;
  const int dir = side == 0 ? -1 : 1;
  const double* wo = side == 0 ? B.wos : B.won;
  switch (bc) {
    case E2D_BC_NONE: break;
    case E2D_BC_FIXED:
      for (int g = 1; g <= NG; ++g) ghost_set(B, b, i, in + dir * g, wo_at(wo, b, B.NCi, i));
      break;
    case E2D_BC_REFLECTION: {
      double nx, ny;
      if (side == 0) nfaceS(B, b, i, JCl, nx, ny); else nfaceN(B, b, i, JCu, nx, ny);
      for (int g = 1; g <= NG; ++g)
        ghost_set(B, b, i, in + dir * g, reflect(ldW(B, b, i, in - dir * (g - 1)), nx, ny));
      break;
    }
    case E2D_BC_PERIODIC:
      for (int g = 1; g <= NG; ++g)
        ghost_copy(B, b, i, in + dir * g, i, side == 0 ? JCu - g + 1 : JCl + g - 1);
      break;
    case E2D_BC_CHARACTERISTIC: {
      double nx, ny;
      if (side == 0) nfaceS(B, b, i, JCl, nx, ny); else nfaceN(B, b, i, JCu, nx, ny);
      ghost_set(B, b, i, in + dir, bc_char_pressure(ldW(B, b, i, in), wo_at(wo, b, B.NCi, i), nx, ny, B.g, B.gm1i));
      for (int g = 2; g <= NG; ++g) ghost_copy(B, b, i, in + dir * g, i, in + dir);
      break;
    }
    default:
      for (int g = 1; g <= NG; ++g) ghost_copy(B, b, i, in + dir * g, i, in);
      break;
  }
}

// One CTA per block: exchange, then W/E BCs, then S/N BCs (the reference's
// order; the S/N pass also fills the corner ghosts).  The status word, the
// 8 neighbours and the block's BC codes are read together up front; a block
// whose edges all have code BC_NONE (every edge exchanged) stops after the
// exchange.
__global__ void __launch_bounds__(GHOST_THREADS, 2) ghost_fill_kernel(Blocks B) {
  const int b = blockIdx.x;
  const int ICl = NG, ICu = B.nci + NG - 1, JCl = NG, JCu = B.ncj + NG - 1;
  __shared__ int failed, nb[8];
  if (threadIdx.x == 0) failed = *(volatile int*)B.status;
  if (threadIdx.x < 8) nb[threadIdx.x] = B.neigh[b * 8 + threadIdx.x];
  int bc_here = 0;
  for (int q = threadIdx.x; q < 2 * (B.NCj + B.NCi); q += blockDim.x) {
    const int code = q < B.NCj           ? B.bcw[size_t(b) * B.NCj + q]
                     : q < 2 * B.NCj     ? B.bce[size_t(b) * B.NCj + q - B.NCj]
                     : q < 2 * B.NCj + B.NCi ? B.bcs[size_t(b) * B.NCi + q - 2 * B.NCj]
                                         : B.bcn[size_t(b) * B.NCi + q - 2 * B.NCj - B.NCi];
    bc_here |= code != E2D_BC_NONE;
  }
  const bool any_bc = __syncthreads_or(bc_here);
  if (failed) return;  // uniform per CTA
  // exchange: edges (2 layers) and corners (2x2) from the 8 neighbours
  const int ne = NG * B.ncj, nn = NG * B.nci, nc = NG * NG;
  const int total = 2 * ne + 2 * nn + 4 * nc;
  for (int q = threadIdx.x; q < total; q += blockDim.x) {
    int k, r = q;
    if (r < 2 * ne) { k = r / ne; r %= ne; }
    else if ((r -= 2 * ne) < 2 * nn) { k = 2 + r / nn; r %= nn; }
    else { r -= 2 * nn; k = 4 + r / nc; r %= nc; }
    const int s = nb[k];
    if (s < 0) continue;
    int i, j, di, dj;
    const bool wi = (k == 0 || k == 4 || k == 6), ei = (k == 1 || k == 5 || k == 7);
    const bool sj = (k == 2 || k == 4 || k == 5), nj = (k == 3 || k == 6 || k == 7);
    int ri, rj;  // position inside the ghost patch
    if (k < 2) { ri = r % NG; rj = r / NG; }
    else if (k < 4) { ri = r % B.nci; rj = r / B.nci; }
    else { ri = r % NG; rj = r / NG; }
    if (wi) { i = ICl - NG + ri; di = (ICu + 1) - ICl; }
    else if (ei) { i = ICu + 1 + ri; di = ICl - (ICu + 1); }
    else { i = ICl + ri; di = 0; }
    if (sj) { j = JCl - NG + rj; dj = (JCu + 1) - JCl; }
    else if (nj) { j = JCu + 1 + rj; dj = JCl - (JCu + 1); }
    else { j = JCl + rj; dj = 0; }
    const CState<double> u = ldU(B, s, i + di, j + dj);
    stU(B, b, i, j, u);
    stW(B, b, i, j, W_of_U(u, B.gm1));
  }
  if (!any_bc) return;  // uniform: no boundary condition to apply
  __syncthreads();
  const bool s_none_w = B.bcs[size_t(b) * B.NCi + ICl - 1] == E2D_BC_NONE;
  const bool n_none_w = B.bcn[size_t(b) * B.NCi + ICl - 1] == E2D_BC_NONE;
  const bool s_none_e = B.bcs[size_t(b) * B.NCi + ICu + 1] == E2D_BC_NONE;
  const bool n_none_e = B.bcn[size_t(b) * B.NCi + ICu + 1] == E2D_BC_NONE;
  for (int j = threadIdx.x; j < B.NCj; j += blockDim.x) {
    const bool mid = (j >= JCl && j <= JCu);
    if (mid || (j < JCl && s_none_w) || (j > JCu && n_none_w)) bc_vertical(B, b, j, 0);
    if (mid || (j < JCl && s_none_e) || (j > JCu && n_none_e)) bc_vertical(B, b, j, 1);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < B.NCi; i += blockDim.x) {
    bc_horizontal(B, b, i, 0);
    bc_horizontal(B, b, i, 1);
  }
}

// Positive doubles order like their int64 bit patterns.
__device__ __forceinline__ void atomic_min_pos(double* addr, double v) {
  atomicMin(reinterpret_cast<unsigned long long*>(addr), __double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_pos(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), __double_as_longlong(v));
}

// Local time step of every interior cell and the minimum of each case (into
// its slot of the step history).  One CTA per block.
__global__ void __launch_bounds__(AUX_THREADS) cfl_kernel(Blocks B, double* hist, const int* step) {
  __shared__ double red[AUX_THREADS / 32];
  const int b = blockIdx.x;
  double* dtmin = hist + 4 * ((*step) * B.ncase + case_id(B, b));
  const int per = B.nci * B.ncj;
  double m = MILLION;
  for (int r = threadIdx.x; r < per; r += blockDim.x) {
    const int i = NG + r % B.nci, j = NG + r / B.nci;
    double xc, yc, A;
    quad_centroid(nodeX(B, b, i, j), nodeY(B, b, i, j), nodeX(B, b, i + 1, j), nodeY(B, b, i + 1, j),
                  nodeX(B, b, i + 1, j + 1), nodeY(B, b, i + 1, j + 1), nodeX(B, b, i, j + 1),
                  nodeY(B, b, i, j + 1), xc, yc, A);
    const double lE = glen(B, b, i + 1, j, i + 1, j + 1), lW = glen(B, b, i, j, i, j + 1);
    const double lN = glen(B, b, i, j + 1, i + 1, j + 1), lS = glen(B, b, i, j, i + 1, j);
    const double per_c = lE + lN + lW + lS;
    double nEx, nEy, nWx, nWy, nNx, nNy, nSx, nSy;
    gnormal(B, b, i + 1, j + 1, i + 1, j, lE, per_c, nEx, nEy);
    gnormal(B, b, i, j, i, j + 1, lW, per_c, nWx, nWy);
    gnormal(B, b, i, j + 1, i + 1, j + 1, lN, per_c, nNx, nNy);
    gnormal(B, b, i + 1, j, i, j, lS, per_c, nSx, nSy);
    const PState<double> w = ldW(B, b, i, j);
    const double d_i = 2.0 * (A / (lE + lW));
    const double d_j = 2.0 * (A / (lN + lS));
    const double v_i = HALF * (w.u * (nEx - nWx) + w.v * (nEy - nWy));
    const double v_j = HALF * (w.u * (nNx - nSx) + w.v * (nNy - nSy));
    const double a = a_of(w, B.g);
    const double dt = dmin(d_i / (a + fabs(v_i)), d_j / (a + fabs(v_j)));
    if (B.local_dt) B.dt[cell_sc(B, b, j, i)] = dt;
    m = dmin(m, dt);
  }
  for (int o = 16; o > 0; o >>= 1) m = dmin(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < AUX_THREADS / 32 ? red[threadIdx.x] : MILLION;
    for (int o = 16; o > 0; o >>= 1) m = dmin(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) atomic_min_pos(dtmin, m);
  }
}

// Per-block sums of |r|, r^2 and max |r| of the density residual.
__global__ void __launch_bounds__(AUX_THREADS) norm_partial_kernel(Blocks B, double* part) {
  __shared__ double red[3][AUX_THREADS / 32];
  const int b = blockIdx.x;
  double s1 = 0, s2 = 0, mx = 0;
  for (int r = threadIdx.x; r < B.nci * B.ncj; r += blockDim.x) {
    const int i = NG + r % B.nci, j = NG + r / B.nci;
    const double v = B.dUdt[cell_var(B, b, 0, j, i)];
    s1 += fabs(v);
    s2 += v * v;
    mx = dmax(mx, fabs(v));
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    mx = dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = s1; red[1][threadIdx.x >> 5] = s2; red[2][threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s1 = 0; s2 = 0; mx = 0;
    for (int w = 0; w < AUX_THREADS / 32; ++w) { s1 += red[0][w]; s2 += red[1][w]; mx = dmax(mx, red[2][w]); }
    part[3 * b] = s1; part[3 * b + 1] = s2; part[3 * b + 2] = mx;
  }
}

// Combines the per-block partials in block order as the multi-block norms
// and the solver loop do; out = (L1, L2, Max) of each case.
// One warp per case: lane l sums the case's blocks l, l+32, ...; the lanes
// are then combined.
__global__ void norm_final_kernel(Blocks B, const double* part, double* hist, const int* step) {
  if (threadIdx.x >= 32) return;
  const int c = blockIdx.x;
  const int b0 = B.case_start ? B.case_start[c] : 0, b1 = B.case_start ? B.case_start[c + 1] : B.nblk;
  double l1 = 0, l2 = 0, mx = 0;
  for (int b = b0 + threadIdx.x; b < b1; b += 32) {
    l1 += part[3 * b];
    l2 += sqr(sqrt(part[3 * b + 1]));
    mx = dmax(mx, part[3 * b + 2]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    l1 += __shfl_xor_sync(0xffffffffu, l1, o);
    l2 += __shfl_xor_sync(0xffffffffu, l2, o);
    mx = dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if (threadIdx.x == 0) {
    double* out = hist + 4 * ((*step) * B.ncase + c) + 1;
    out[0] = l1;
    out[1] = sqrt(sqr(sqrt(l2)));
    out[2] = mx;
  }
}

__global__ void fill_kernel(double* p, long long n, double v) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    p[q] = v;
}

// Explicit-step bookkeeping: the step index lives on the device so that one
// captured step graph replays for every step.
// Slot of step *step + offset: dt = MILLION (min-reduced), norms = 0 (summed).
__global__ void slot_init_kernel(double* hist, const int* step, int offset, int ncase) {
  for (int c = threadIdx.x; c < ncase; c += blockDim.x) {
    double* h = hist + 4 * ((*step + offset) * ncase + c);
    h[0] = MILLION; h[1] = 0.0; h[2] = 0.0; h[3] = 0.0;
  }
}
// End of a step: the fused epilogue summed r^2 into the next slots' L2 entries.
__global__ void step_end_kernel(double* hist, int* step, int fused, int ncase) {
  if (fused)
    for (int c = threadIdx.x; c < ncase; c += blockDim.x) {
      double* h = hist + 4 * ((*step + 1) * ncase + c);
      h[2] = sqrt(h[2]);
    }
  __syncthreads();
  if (threadIdx.x == 0) *step += 1;
}

cudaError_t launch_ghost_fill(const Blocks& B, cudaStream_t st) {
  // one thread per exchanged ghost cell where the block allows (the exchange
  // is a single round of independent loads), at least one CTA of AUX_THREADS
  const int cells = 2 * NG * (B.nci + B.ncj) + 4 * NG * NG;
  const int threads = std::min(GHOST_THREADS, std::max(AUX_THREADS, (cells + 31) / 32 * 32));
  ghost_fill_kernel<<<B.nblk, threads, 0, st>>>(B);
  return cudaGetLastError();
}

cudaError_t launch_cfl(const Blocks& B, double* hist, const int* step, cudaStream_t st) {
  cfl_kernel<<<B.nblk, AUX_THREADS, 0, st>>>(B, hist, step);
  return cudaGetLastError();
}

cudaError_t launch_norms(const Blocks& B, double* part, double* hist, const int* step, cudaStream_t st) {
  norm_partial_kernel<<<B.nblk, AUX_THREADS, 0, st>>>(B, part);
  norm_final_kernel<<<B.ncase, 32, 0, st>>>(B, part, hist, step);
  return cudaGetLastError();
}

cudaError_t launch_slot_init(double* hist, const int* step, int offset, int ncase, cudaStream_t st) {
  slot_init_kernel<<<1, 128, 0, st>>>(hist, step, offset, ncase);
  return cudaGetLastError();
}
cudaError_t launch_step_end(double* hist, int* step, int fused, int ncase, cudaStream_t st) {
  step_end_kernel<<<1, 128, 0, st>>>(hist, step, fused, ncase);
  return cudaGetLastError();
}
cudaError_t launch_fill(double* p, long long n, double v, cudaStream_t st) {
  int grid = int((n + 255) / 256);
  if (grid > 1184) grid = 1184;
  if (grid < 1) grid = 1;
  fill_kernel<<<grid, 256, 0, st>>>(p, n, v);
  return cudaGetLastError();
}

}  // namespace e2d
