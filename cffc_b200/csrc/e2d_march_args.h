// e2d_march_args.h — arguments of the column-marching stage kernel
// (e2d_march.cuh) and the layout of the per-cell geometry it streams.
//
// Geometry (computed once per handle from the nodes): an array
// [nblk][GEOM_NF][NCj][NCi] of doubles holding, per cell, in the fast
// builds' arithmetic
//   0, 1  centroid xc, yc                         (every cell, ghosts included)
//   2..4  least-squares inverse K0, K1, K2         (ring cells: the interior and
//         one ghost layer); the gradient of a variable is
//         (Sx K0 + Sy K1, Sx K1 + Sy K2) with Sx, Sy the sums of dW dx, dW dy
//         over the cell's stencil
//   5     1 / area                                 (interior cells)
//   6, 7  2 A / (lE + lW), 2 A / (lN + lS)          (interior cells, CFL step)
//   8..11 (n_E - n_W) / 2 and (n_N - n_S) / 2, x then y, with the cell's own
//         outward unit normals                      (interior cells, CFL step)
// and, for the exact build (a second array of the same layout), the
// quantities the reference derives from the grid alone, in its arithmetic:
// planes 2..4 the averaged sums DxDx / n, DxDy / n, DyDy / n of the stencil,
// plane 5 the area A, planes 6, 7 2 (A / (lE + lW)) and 2 (A / (lN + lS)),
// planes 8..11 the normal differences n_E - n_W and n_N - n_S (not halved);
// and a byte per cell naming the stencil's neighbours: bit k set when
// neighbour k of (-1,-1) (0,-1) (1,-1) (-1,0) (1,0) (-1,1) (0,1) (1,1)
// belongs to the least-squares stencil (the reference's stencils are all
// subsets of these eight, listed in this order).  The nodes are kept a second
// time with rows padded to an even length, [nblk][2][NNj][NNp] (X then Y),
// so that a tensor map can describe them (row strides must be multiples of
// 16 bytes).
#pragma once
#include <cuda.h>

#include "e2d_device.cuh"

namespace e2d {

constexpr int GEOM_NF = 12;
enum GeomField { G_XC = 0, G_YC, G_K0, G_K1, G_K2, G_RA, G_DI, G_DJ, G_VIX, G_VIY, G_VJX, G_VJY };

struct MarchArgs {
  StageArgs a;
  CUtensorMap tmW;   // the stage's input primitive state, as [4 nblk][NCj][NCi]
  CUtensorMap tmG;   // the geometry, as [GEOM_NF nblk][NCj][NCi]
  CUtensorMap tmN;   // padded nodes, as [2 nblk][NNj][NNp]
  // update inputs of the explicit stages (builds with E2D_MARCH_UPD), boxes
  // of 32 columns x 8 rows: the base conserved state and the residual of
  // RK stage 1 as [4 nblk][NCj][NCi], geometry plane G_RA alone and planes
  // G_RA .. G_VJY, as [GEOM_NF nblk][NCj][NCi]
  CUtensorMap tmU, tmR, tmGA, tmGF;
  int upd;           // 1: the update inputs of this launch arrive through these maps
  const double* geom;
  const unsigned char* mask;
  const unsigned char* bcside;  // per block: sides with face-setting boundary conditions (bits W E S N)
  int strips;        // column strips per block
  int ch;            // rows of a chunk (the last chunk of a strip may hold up to 8)
  int cps;           // chunks per strip
  long long nchunk;  // strips * cps * nblk
};

}  // namespace e2d
