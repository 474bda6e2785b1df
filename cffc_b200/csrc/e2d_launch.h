// Host-side declarations of the kernel launchers (one set per precision path).
#pragma once
#include <cuda_runtime.h>

#include "e2d_device.cuh"
#include "e2d_march_args.h"

namespace e2d {
namespace exact {
cudaError_t launch_stage(const StageArgs& a, cudaStream_t st);
size_t stage_smem_bytes();
int tile_i();
int tile_j();
// column-marching stage kernel in the reference's arithmetic and its geometry
cudaError_t launch_march(const MarchArgs& m, int grid, cudaStream_t st);
int march_ctas_per_sm();
cudaError_t launch_geometry(const Blocks& B, double* geom, unsigned char* mask, unsigned char* bcside, int* degenerate,
                            int NNp, double* nodes_pad, cudaStream_t st);
}  // namespace exact
namespace fast {
cudaError_t launch_stage(const StageArgs& a, cudaStream_t st);
size_t stage_smem_bytes();
int tile_i();
int tile_j();
// column-marching stage kernel (e2d_march.cuh) and its per-handle geometry
cudaError_t launch_march(const MarchArgs& m, int grid, cudaStream_t st);
int march_ctas_per_sm();
int march_strip_cols();
int march_chunk_rows();
int march_max_rows();
int march_window_rows();
int march_chunks(int ncj, int ch);
cudaError_t launch_geometry(const Blocks& B, double* geom, unsigned char* mask, unsigned char* bcside, int* degenerate,
                            int NNp, double* nodes_pad, cudaStream_t st);
}  // namespace fast
namespace f32 {
cudaError_t launch_stage(const StageArgs& a, cudaStream_t st);
size_t stage_smem_bytes();
int tile_i();
int tile_j();
cudaError_t launch_march(const MarchArgs& m, int grid, cudaStream_t st);
int march_ctas_per_sm();
}  // namespace f32

// The stage kernel of a precision (E2D_PREC_*): launch and tile shape.
inline cudaError_t launch_stage_prec(int precision, const StageArgs& a, cudaStream_t st) {
  if (precision == E2D_PREC_FP64_EXACT) return exact::launch_stage(a, st);
  if (precision == E2D_PREC_FP32) return f32::launch_stage(a, st);
  return fast::launch_stage(a, st);
}
inline void stage_tile(int precision, int* ti, int* tj) {
  if (precision == E2D_PREC_FP64_EXACT) { *ti = exact::tile_i(); *tj = exact::tile_j(); }
  else if (precision == E2D_PREC_FP32) { *ti = f32::tile_i(); *tj = f32::tile_j(); }
  else { *ti = fast::tile_i(); *tj = fast::tile_j(); }
}
cudaError_t launch_ghost_fill(const Blocks& B, cudaStream_t st);
cudaError_t launch_cfl(const Blocks& B, double* hist, const int* step, cudaStream_t st);
cudaError_t launch_norms(const Blocks& B, double* part, double* hist, const int* step, cudaStream_t st);
cudaError_t launch_slot_init(double* hist, const int* step, int offset, int ncase, cudaStream_t st);
cudaError_t launch_step_end(double* hist, int* step, int fused, int ncase, cudaStream_t st);
cudaError_t launch_fill(double* p, long long n, double v, cudaStream_t st);
}  // namespace e2d
