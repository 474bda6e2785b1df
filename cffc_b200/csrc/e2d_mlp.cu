// e2d_mlp.cu — the learned warm start's network on the tensor cores: a
// per-cell MLP (16 input features -> 128 -> 128 -> 16 outputs, tanh hidden
// layers) whose forward pass (inference) and forward + backward pass
// (training) are hand-written tcgen05 kernels: BF16 operands staged in
// shared memory, FP32 accumulators in TMEM, one CTA of 128 threads per tile
// of 128 cells, every matrix product an M = 128 UMMA.
//
// Training products per tile (cells c, hidden h, outputs o, features f):
//   forward   D1 = X W1^T, H1 = tanh(D1 + b1); D2 = H1 W2^T, H2 = tanh(..);
//             Y = H2 W3^T + b3
//   backward  dY = 2 (Y - T) / n  (the four used outputs)
//             dW3^T = H2^T dY      (M = h, K = c)     dH2 = dY W3      (M = c)
//             dZ2 = dH2 (1 - H2^2); dW2 = dZ2^T H1  (M = o, K = c)
//             dH1 = dZ2 W2; dZ1 = dH1 (1 - H1^2);   dW1 = dZ1^T X   (M = h, K = c)
// Weight gradients of all tiles are summed with FP32 atomics.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/cffc_e2d.h"
#include "e2d_tc.cuh"

using namespace e2d;

namespace {

constexpr uint32_t WAIT_ITERS = 1u << 22;  // bounded mbarrier waits (about a second)

// ---------------------------------------------------------------------------
// Self-test of the building blocks: D[128 x N] = A[128 x K] B[N x K]^T.
__global__ void __launch_bounds__(128) tc_selftest_kernel(const uint16_t* A, const uint16_t* Bm, float* D, int N,
                                                          int K, uint32_t ncols, int* err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t taddr;
  uint8_t* As = sm;
  uint8_t* Bs = sm + 128 * K * 2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int idx = tid; idx < 128 * K; idx += 128)
    *reinterpret_cast<uint16_t*>(As + tc::kmaj_off(idx / K, idx % K, K)) = A[idx];
  for (int idx = tid; idx < N * K; idx += 128)
    *reinterpret_cast<uint16_t*>(Bs + tc::kmaj_off(idx / K, idx % K, K)) = Bm[idx];
  if (tid == 0) tc::mbar_init(&bar, 1);
  if (warp == 0) tc::tmem_alloc(&taddr, ncols);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t t0 = taddr;
  if (tid == 0) {
    const uint32_t id = tc::idesc_bf16(128, N);
    for (int t = 0; t < K / 16; ++t)
      tc::mma_bf16(t0, tc::smem_desc(tc::smem_addr(As) + 256 * t, 128, K * 16),
                   tc::smem_desc(tc::smem_addr(Bs) + 256 * t, 128, K * 16), id, t > 0);
    tc::mma_commit(&bar);
  }
  __syncwarp();
  // warp-uniform outcome: the TMEM loads below are .sync.aligned
  const bool ok = __all_sync(0xffffffffu, tc::mbar_wait(&bar, 0, WAIT_ITERS));
  tc::fence_after_sync();
  if (!ok) {
    if (lane == 0) atomicExch(err, 1);
  } else {
    const int row = 32 * warp + lane;
    for (int col = 0; col < N; col += 16) {
      float v[16];
      tc::tmem_ld16(t0 + (uint32_t(32 * warp) << 16) + uint32_t(col), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) D[size_t(row) * N + col + q] = v[q];
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(t0, ncols);
}

}  // namespace

extern "C" int e2d_tc_selftest(const uint16_t* A, const uint16_t* B, float* D, int N, int K) {
  if (!A || !B || !D || N < 16 || N > 256 || N % 16 || K < 16 || K > 128 || K % 16) return E2D_ERR_ARG;
  uint16_t *dA = nullptr, *dB = nullptr;
  float* dD = nullptr;
  int* derr = nullptr;
  int rc = 0;
  const size_t smem = size_t(128) * K * 2 + size_t(N) * K * 2;
  uint32_t ncols = 32;
  while (ncols < uint32_t(N)) ncols <<= 1;
  if (cudaMalloc(&dA, 2 * 128 * K) || cudaMalloc(&dB, 2 * size_t(N) * K) || cudaMalloc(&dD, 4 * 128 * size_t(N)) ||
      cudaMalloc(&derr, sizeof(int))) {
    rc = E2D_ERR_NOMEM;
  } else if (cudaMemcpy(dA, A, 2 * 128 * K, cudaMemcpyHostToDevice) ||
             cudaMemcpy(dB, B, 2 * size_t(N) * K, cudaMemcpyHostToDevice) || cudaMemset(derr, 0, sizeof(int)) ||
             cudaFuncSetAttribute(tc_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) {
    rc = E2D_ERR_CUDA;
  } else {
    tc_selftest_kernel<<<1, 128, smem>>>(dA, dB, dD, N, K, ncols, derr);
    int herr = 0;
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost) ||
        cudaMemcpy(D, dD, 4 * 128 * size_t(N), cudaMemcpyDeviceToHost))
      rc = E2D_ERR_CUDA;
    else if (herr)
      rc = E2D_ERR_CUDA;
  }
  cudaFree(dA); cudaFree(dB); cudaFree(dD); cudaFree(derr);
  return rc;
}
