// Mixed-precision stage kernel: reconstruction (least-squares gradients,
// limiter, face states) and the Roe flux in FP32; geometry, flux divergence,
// RK accumulation, CFL and residual norms in FP64.  Built with FMA
// contraction and the approximate FP32 division / square root
// (-prec-div=false -prec-sqrt=false affect only float operations).
#define E2D_NS f32
#define E2D_FAST 1
#define E2D_FP32 1
// marching kernel: one staging buffer and the update inputs by TMA, as in
// the FP64 build (1M-cell set: 146 / 157 us against 151 / 173 with two
// buffers and global update inputs)
#define E2D_MARCH_NBUF 1
#define E2D_MARCH_UPD 1
#include "e2d_stage.cuh"
#include "e2d_march.cuh"
