// Exact FP64 kernels: compiled with -fmad=false so that every expression
// rounds as the reference's x86-64 code does (no fused multiply-add).
// Also holds the ghost-fill, time-step and norm kernels, which every
// precision path shares.
#define E2D_NS exact
// marching kernel: one staging buffer and the update inputs by TMA, as in
// the fast builds
#define E2D_MARCH_NBUF 1
#define E2D_MARCH_UPD 1
#include "e2d_stage.cuh"
#include "e2d_aux.cuh"
#include "e2d_march.cuh"
