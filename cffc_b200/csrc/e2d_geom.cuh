// e2d_geom.cuh — cell-state loads/stores and grid geometry of the reference
// Grid2DQuad accessors (face lengths lfaceX, unit normals nfaceX, perimeter),
// evaluated from the node arrays, for the ghost-fill, CFL and NKS kernels.
// Compiled in no-FMA translation units only.
#pragma once
#include "e2d_device.cuh"

namespace e2d {

__device__ __forceinline__ PState<double> ldW(const Blocks& B, int b, int i, int j) {
  PState<double> w;
  w.d = B.W[cell_var(B, b, 0, j, i)]; w.u = B.W[cell_var(B, b, 1, j, i)];
  w.v = B.W[cell_var(B, b, 2, j, i)]; w.p = B.W[cell_var(B, b, 3, j, i)];
  return w;
}
__device__ __forceinline__ CState<double> ldU(const Blocks& B, int b, int i, int j) {
  CState<double> u;
  u.d = B.U[cell_var(B, b, 0, j, i)]; u.mx = B.U[cell_var(B, b, 1, j, i)];
  u.my = B.U[cell_var(B, b, 2, j, i)]; u.E = B.U[cell_var(B, b, 3, j, i)];
  return u;
}
__device__ __forceinline__ void stW(const Blocks& B, int b, int i, int j, const PState<double>& w) {
  B.W[cell_var(B, b, 0, j, i)] = w.d; B.W[cell_var(B, b, 1, j, i)] = w.u;
  B.W[cell_var(B, b, 2, j, i)] = w.v; B.W[cell_var(B, b, 3, j, i)] = w.p;
}
__device__ __forceinline__ void stU(const Blocks& B, int b, int i, int j, const CState<double>& u) {
  B.U[cell_var(B, b, 0, j, i)] = u.d; B.U[cell_var(B, b, 1, j, i)] = u.mx;
  B.U[cell_var(B, b, 2, j, i)] = u.my; B.U[cell_var(B, b, 3, j, i)] = u.E;
}
__device__ __forceinline__ double nodeX(const Blocks& B, int b, int i, int j) { return B.X[node_ix(B, b, j, i)]; }
__device__ __forceinline__ double nodeY(const Blocks& B, int b, int i, int j) { return B.Y[node_ix(B, b, j, i)]; }

__device__ __forceinline__ double glen(const Blocks& B, int b, int ai, int aj, int ci, int cj) {
  const double dx = nodeX(B, b, ai, aj) - nodeX(B, b, ci, cj), dy = nodeY(B, b, ai, aj) - nodeY(B, b, ci, cj);
  return sqrt(dx * dx + dy * dy);
}
// Cell perimeter lE + lN + lW + lS.
__device__ __forceinline__ double gperim(const Blocks& B, int b, int i, int j) {
  return glen(B, b, i + 1, j, i + 1, j + 1) + glen(B, b, i, j + 1, i + 1, j + 1) + glen(B, b, i, j, i, j + 1) +
         glen(B, b, i, j, i + 1, j);
}
// Normal of edge a->c: (a.y - c.y, -(a.x - c.x)) / |a - c|, degenerate -> ihat.
__device__ __forceinline__ void gnormal(const Blocks& B, int b, int ai, int aj, int ci, int cj, double l,
                                        double per, double& nx, double& ny) {
  if (l > NANO * per) {
    const double ax = nodeX(B, b, ai, aj), ay = nodeY(B, b, ai, aj);
    const double cx = nodeX(B, b, ci, cj), cy = nodeY(B, b, ci, cj);
    const double dx = ax - cx, dy = ay - cy;
    const double n = sqrt(dx * dx + dy * dy);
    nx = (ay - cy) / n;
    ny = -(ax - cx) / n;
  } else {
    nx = 1.0; ny = 0.0;
  }
}
// nfaceW/E/S/N(i, j) of the reference grid.
__device__ __forceinline__ void nfaceW(const Blocks& B, int b, int i, int j, double& nx, double& ny) {
  gnormal(B, b, i, j, i, j + 1, glen(B, b, i, j, i, j + 1), gperim(B, b, i, j), nx, ny);
}
__device__ __forceinline__ void nfaceE(const Blocks& B, int b, int i, int j, double& nx, double& ny) {
  gnormal(B, b, i + 1, j + 1, i + 1, j, glen(B, b, i + 1, j, i + 1, j + 1), gperim(B, b, i, j), nx, ny);
}
__device__ __forceinline__ void nfaceS(const Blocks& B, int b, int i, int j, double& nx, double& ny) {
  gnormal(B, b, i + 1, j, i, j, glen(B, b, i, j, i + 1, j), gperim(B, b, i, j), nx, ny);
}
__device__ __forceinline__ void nfaceN(const Blocks& B, int b, int i, int j, double& nx, double& ny) {
  gnormal(B, b, i, j + 1, i + 1, j + 1, glen(B, b, i, j + 1, i + 1, j + 1), gperim(B, b, i, j), nx, ny);
}

__device__ __forceinline__ PState<double> wo_at(const double* wo, int b, int len, int k) {
  const double* p = wo + size_t(b) * 4 * len;
  PState<double> w;
  w.d = p[k]; w.u = p[len + k]; w.v = p[2 * len + k]; w.p = p[3 * len + k];
  return w;
}

__device__ __forceinline__ void ghost_set(const Blocks& B, int b, int i, int j, const PState<double>& w) {
  stW(B, b, i, j, w);
  stU(B, b, i, j, U_of_W(w, B.gm1i));
}
__device__ __forceinline__ void ghost_copy(const Blocks& B, int b, int id, int jd, int is, int js) {
  stW(B, b, id, jd, ldW(B, b, is, js));
  stU(B, b, id, jd, ldU(B, b, is, js));
}

}  // namespace e2d
