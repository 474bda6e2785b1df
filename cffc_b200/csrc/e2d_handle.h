// e2d_handle.h — the library's handle (internal; the C ABI sees it as an
// opaque pointer) and the host helpers the translation units share.
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "../../include/cffc_e2d.h"
#include "e2d_launch.h"

struct e2d_nks_state;  // NKS work arrays (e2d_nks.cu)

struct e2d_handle {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream the work is enqueued on
  cudaStream_t own_stream = nullptr;  // the handle's own stream
  e2d_scheme sc{};
  e2d::Blocks B{};
  size_t ncell = 0, nnode = 0;
  // device allocations (owned)
  std::vector<void*> allocs;
  double* hist = nullptr;  // [hist_cap][4]
  int hist_cap = 0;
  int* step = nullptr;     // device step counter
  double* part = nullptr;  // [nblk][3] norm partials
  bool recon_out = false;  // dWdx/dWdy/phi arrays allocated
  // third stage state (schemes of three or more stages) and the second and
  // third residual slots of RK4 (dUdt[i][j][1..2] of the reference)
  double *W3 = nullptr, *U3 = nullptr, *R1 = nullptr, *R2 = nullptr;
  // limiter freezing: per-case frozen flags and the "first step of the run"
  // flag (device); residual smoothing: global scratch when a block's
  // smoothing region does not fit in shared memory
  int *freeze = nullptr, *first = nullptr;
  double* smooth_scratch = nullptr;
  size_t smooth_smem = 0;
  // column-marching stage kernel: per-cell geometry (the fast builds' and
  // the exact build's), padded nodes, tensor maps of the stage inputs (W, W2,
  // W3), the geometry and the nodes, and the persistent grid size
  bool march = false;
  double* geom = nullptr;
  double* geomx = nullptr;
  CUtensorMap tmGx, tmGAx, tmGFx;  // the exact build's geometry: window, update inputs
  unsigned char* gmask = nullptr;
  unsigned char* bcside = nullptr;  // per block: sides with face-setting BCs (marching kernel)
  // A batch whose cases have different block shapes holds no blocks of its
  // own: one uniform sub-batch per shape, every call dispatched to them.
  // Per case (in the order given): its sub-batch and index there, and the
  // offsets of its arrays in the callers' concatenated host arrays (cell
  // arrays of 4 variables, scalar per-cell arrays).
  std::vector<e2d_handle*> subs;
  std::vector<int> sub_of, local_of;
  std::vector<size_t> off4, size4, off1, size1;
  CUtensorMap tmU[2], tmR, tmGA, tmGF;  // marching kernel update inputs: U and U2, dUdt, geometry
  bool upd_ok = false;
  double* nodes_pad = nullptr;
  CUtensorMap tmW[3], tmG, tmN;
  int march_grid = 0;
  int march_rows = 7;  // rows of a chunk
  double tune_us = 0.0;  // the autotuner's time of one explicit stage with the chosen kernel
  bool march_ok = false;  // geometry and tensor maps set up
  // the autotuner's choice per precision (E2D_PREC_FP64, E2D_PREC_FP32,
  // E2D_PREC_FP64_EXACT)
  bool sel_march[3] = {false, false, false};
  int sel_rows[3] = {7, 7, 7};
  double sel_us[3] = {0.0, 0.0, 0.0};
  // captured explicit step
  cudaGraphExec_t step_graph = nullptr;
  e2d_nks_state* nks = nullptr;
};

#define E2D_CK(call)                                                           \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      fprintf(stderr, "cffc_e2d: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
      return E2D_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)

namespace e2d_host {

template <class T> int dalloc(e2d_handle* h, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, sizeof(T) * (n ? n : 1)) != cudaSuccess) return E2D_ERR_NOMEM;
  h->allocs.push_back(q);
  *p = static_cast<T*>(q);
  return 0;
}

int check_status(e2d_handle* h);
cudaError_t launch_stage_any(e2d_handle* h, int mode, int fuse_next);
cudaError_t launch_stage_args(e2d_handle* h, e2d::StageArgs& a);
// Newton-Krylov over the sub-batches of a mixed-shape batch (e2d_nks).
int composite_nks(e2d_handle* h, const e2d_nks_params* p, e2d_nks_step* hist, int* n_steps);
cudaError_t ghost_fill_for(e2d_handle* h, int mode);
int ensure_hist(e2d_handle* h, int n);
void nks_free(e2d_handle* h);
void nks_drop_graphs(e2d_handle* h);

}  // namespace e2d_host
