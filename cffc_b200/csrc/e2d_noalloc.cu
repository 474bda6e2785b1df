// e2d_noalloc.cu — residual norms of a caller-owned device residual with no
// device allocation at all.
//
// Some callers cannot allocate device memory when they need the norms: a host
// code that must not let cudaMalloc/cudaFree stall or synchronise the device
// in the middle of its time loop, a plugin loaded into a process whose own
// allocator owns the whole device-memory budget, or a code that forbids any
// allocation after start-up.  For them this entry point does the same
// per-block reduction as e2d_norms with its scratch in a fixed, file-scope
// device array instead of memory from cudaMalloc.
//
// The scratch array holds three doubles per block (the per-block sum of |r|,
// sum of r^2 and max |r|); it is sized for E2D_NORMS_STATIC_MAX_BLOCKS blocks
// (96 KiB) and, like any __device__ variable, occupies that much memory on
// every GPU that loads the library until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/cffc_e2d.h"
#include "e2d_device.cuh"

namespace {

constexpr int kThreads = 256;

// The shared scratch: every call writes the slots [0, 3*nblk) before reading
// them, so no slot needs clearing between calls.  Calls that overlap on the
// GPU (two streams, or two host threads) use the same slots and race.
static __device__ __align__(256) double g_norm_scratch[3 * E2D_NORMS_STATIC_MAX_BLOCKS];

// Device address of g_norm_scratch per device (the symbol's name in host code
// is a host-side stand-in, not a device address).
constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_mutex;

int scratch_for_current_device(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return E2D_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_norm_scratch) != cudaSuccess || !p) return E2D_ERR_CUDA;
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return 0;
}

// Per-block sums of |r|, r^2 and max |r| of the density residual r over the
// block's interior cells (L1/L2/Max_Norm_Residual of one block,
// src_2D/Euler2D/Euler2DQuadSingleBlock.cc:3111-3167).
__global__ void __launch_bounds__(kThreads) static_norm_partial(const double* dUdt, int nci, int ncj,
                                                                double* part) {
  __shared__ double red[3][kThreads / 32];
  const int b = blockIdx.x;
  const int NCi = nci + 2 * e2d::NG, NCj = ncj + 2 * e2d::NG;
  const double* r0 = dUdt + size_t(b) * 4 * NCi * NCj;  // variable 0 (density) of block b
  double s1 = 0, s2 = 0, mx = 0;
  for (int q = threadIdx.x; q < nci * ncj; q += blockDim.x) {
    const int i = e2d::NG + q % nci, j = e2d::NG + q / nci;
    const double v = r0[size_t(j) * NCi + i];
    s1 += fabs(v);
    s2 += v * v;
    mx = e2d::dmax(mx, fabs(v));
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    mx = e2d::dmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = s1; red[1][threadIdx.x >> 5] = s2; red[2][threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s1 = 0; s2 = 0; mx = 0;
    for (int w = 0; w < kThreads / 32; ++w) { s1 += red[0][w]; s2 += red[1][w]; mx = e2d::dmax(mx, red[2][w]); }
    part[3 * b] = s1; part[3 * b + 1] = s2; part[3 * b + 2] = mx;
  }
}

// Block partials combined in block order as the multi-block norms and the
// solver loop do (Euler2DQuadMultiBlock.cc:1017-1190, Euler2DQuadSolvers.cc:687-696).
__global__ void static_norm_final(int nblk, const double* part, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double l1 = 0, l2 = 0, mx = 0;
  for (int b = 0; b < nblk; ++b) {
    l1 += part[3 * b];
    const double s = sqrt(part[3 * b + 1]);
    l2 += s * s;
    mx = e2d::dmax(mx, part[3 * b + 2]);
  }
  const double r = sqrt(l2);
  out[0] = l1;
  out[1] = sqrt(r * r);
  out[2] = mx;
}

}  // namespace

extern "C" int e2d_residual_norms_static(const double* dUdt, int32_t nblk, int32_t nci, int32_t ncj,
                                         double* out, void* stream) {
  if (!dUdt || !out || nblk < 1 || nci < 1 || ncj < 1) return E2D_ERR_ARG;
  if (nblk > E2D_NORMS_STATIC_MAX_BLOCKS) return E2D_ERR_ARG;
  double* scratch = nullptr;
  const int rc = scratch_for_current_device(&scratch);
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  static_norm_partial<<<nblk, kThreads, 0, st>>>(dUdt, nci, ncj, scratch);
  static_norm_final<<<1, 32, 0, st>>>(nblk, scratch, out);
  return cudaGetLastError() == cudaSuccess ? 0 : E2D_ERR_CUDA;
}
