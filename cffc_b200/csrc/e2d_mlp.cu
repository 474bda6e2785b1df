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
// Each CTA accumulates its tiles' weight gradients in TMEM (FP32) and
// writes them to its own slot; the slots are summed in CTA order, so
// training is deterministic.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/cffc_e2d.h"
#include <cuda_bf16.h>

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

// ===========================================================================
// The warm-start network.
namespace {

constexpr int MF = 16;    // input features
constexpr int MH = 128;   // hidden units (both layers)
constexpr int MO = 16;    // outputs computed (the first MO_USED are trained)
constexpr int MO_USED = 4;
constexpr int TILE = 128; // cells per tile (the UMMA M)
constexpr int NPARAM = MH * MF + MH + MH * MH + MH + MO * MH + MO;
// offsets of the flat parameter vector
constexpr int P_W1 = 0, P_B1 = P_W1 + MH * MF, P_W2 = P_B1 + MH, P_B2 = P_W2 + MH * MH, P_W3 = P_B2 + MH,
              P_B3 = P_W3 + MO * MH;

// BF16 copies of the weights the products read, laid out row-major:
// W1 [MH][MF], W2 [MH][MH], W3 [MO][MH], and the transposes W2T [MH][MH],
// W3T [MH][MO] for the backward products.
struct MlpDev {
  const uint16_t *w1, *w2, *w3, *w2t, *w3t;
  const float* p;  // FP32 parameters (biases read from here)
};

// Shared memory (bytes).  Every operand tile in the canonical K-major layout.
struct MlpSmem {
  uint8_t X[TILE * MF * 2];    // [cells][MF]        A of F1
  uint8_t XT[MF * TILE * 2];   // [MF][cells]        B of dW1 (train)
  uint8_t W1[MH * MF * 2];     // [MH][MF]           B of F1
  uint8_t W3[MO * MH * 2];     // [MO][MH]           B of F3
  uint8_t W3T[MH * MO * 2];    // [MH][MO]           B of dH2 (train)
  uint8_t dY[TILE * MO * 2];   // [cells][MO]        A of dH2 (train)
  uint8_t dYT[MO * TILE * 2];  // [MO][cells]        B of dW3^T (train)
  uint8_t W23[MH * MH * 2];    // W2 (B of F2), then W2T (B of dH1, train)
  uint8_t P[TILE * MH * 2];    // H1 [cells][MH] (A of F2), then dZ2 [cells][MH] (A of dH1)
  uint8_t Q[TILE * MH * 2];    // H2 [cells][MH] (A of F3), then dZ2T [MH][cells] (A of dW2)
  uint8_t R[MH * TILE * 2];    // H1T [MH][cells] (B of dW2, train)
  uint8_t S[MH * TILE * 2];    // H2T [MH][cells] (A of dW3^T), then dZ1T (A of dW1) (train)
  float b1[MH], b2[MH], b3[MO];
  float gb1[4][MH], gb2[4][MH], gb3[4][MO];  // per-warp bias gradients (train)
  double lw[4];                                // per-warp loss sums
};

__device__ __forceinline__ uint16_t f2bf(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}
__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float(uint32_t(b) << 16); }
__device__ __forceinline__ void st_bf(uint8_t* base, uint32_t off, float v) {
  *reinterpret_cast<uint16_t*>(base + off) = f2bf(v);
}
__device__ __forceinline__ float ld_bf(const uint8_t* base, uint32_t off) {
  return bf2f(*reinterpret_cast<const uint16_t*>(base + off));
}

// Global BF16 [rows][K] row-major -> shared canonical tile.
__device__ void stage_rows(uint8_t* dst, const uint16_t* src, int rows, int K) {
  for (int idx = threadIdx.x; idx < rows * K; idx += TILE)
    *reinterpret_cast<uint16_t*>(dst + tc::kmaj_off(idx / K, idx % K, K)) = src[idx];
}

// One product D (+)= A B^T over K (multiple of 16), issued by thread 0.
__device__ __forceinline__ void issue(uint32_t d, const uint8_t* A, const uint8_t* Bm, int K, int N, bool acc) {
  const uint32_t id = tc::idesc_bf16(128, N);
  const uint32_t a0 = tc::smem_addr(A), b0 = tc::smem_addr(Bm);
  for (int t = 0; t < K / 16; ++t)
    tc::mma_bf16(d, tc::smem_desc(a0 + 256 * t, 128, K * 16), tc::smem_desc(b0 + 256 * t, 128, K * 16), id,
                 (acc || t > 0) ? 1u : 0u);
}

// Commit (thread 0) and bounded wait of every thread; warp-uniform result.
__device__ __forceinline__ bool complete(uint64_t* bar, uint32_t& phase) {
  if (threadIdx.x == 0) tc::mma_commit(bar);
  __syncwarp();
  const bool ok = __all_sync(0xffffffffu, tc::mbar_wait(bar, phase, WAIT_ITERS));
  phase ^= 1u;
  tc::fence_after_sync();
  return ok;
}

__device__ __forceinline__ void cta_sync_async() {
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

__device__ __forceinline__ float warp_sum(float v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// TMEM columns: forward D1, D3 and backward dH2 share [0,128) (each is read
// out before the next is written), D2 / dH1 [128,256); training
// accumulators dW3^T [256,272), dW1 [272,288), dW2 [384,512).  Inference
// allocates 256 columns, training 512.
constexpr uint32_t C_D1 = 0, C_D2 = 128, C_D3 = 0, C_GW3 = 256, C_GW1 = 272, C_GW2 = 384;

// Persistent kernel over tiles of 128 cells.  TRAIN = false: Y = f(X) for the
// rows of the tiles.  TRAIN = true: the gradient of
// loss = sum over rows and the four outputs of (y - t)^2 / n_total,
// accumulated in TMEM over the CTA's tiles and written to the CTA's slot of
// grad (and of loss).
template <bool TRAIN>
__global__ void __launch_bounds__(TILE, 1) mlp_kernel(MlpDev w, const float* __restrict__ X,
                                                      const float* __restrict__ T, int n, float inv_n,
                                                      float* __restrict__ Y, float* grad, double* loss, int* err) {
  extern __shared__ __align__(1024) uint8_t smraw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(smraw);
  __shared__ uint64_t bar;
  __shared__ uint32_t taddr;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = TRAIN ? 512u : 256u;
  const int ntiles = (n + TILE - 1) / TILE;
  // constant operands: W1, W3 (W3T), biases
  stage_rows(s.W1, w.w1, MH, MF);
  stage_rows(s.W3, w.w3, MO, MH);
  if (TRAIN) stage_rows(s.W3T, w.w3t, MH, MO);
  for (int k = tid; k < MH; k += TILE) {
    s.b1[k] = w.p[P_B1 + k];
    s.b2[k] = w.p[P_B2 + k];
    for (int q = 0; q < 4; ++q) { s.gb1[q][k] = 0.0f; s.gb2[q][k] = 0.0f; }
  }
  if (tid < MO) {
    s.b3[tid] = w.p[P_B3 + tid];
    for (int q = 0; q < 4; ++q) s.gb3[q][tid] = 0.0f;
  }
  if (tid == 0) tc::mbar_init(&bar, 1);
  if (warp == 0) tc::tmem_alloc(&taddr, ncols);
  cta_sync_async();
  const uint32_t tm = taddr;
  const uint32_t lane_base = uint32_t(32 * warp) << 16;  // this warp's TMEM lanes
  uint32_t phase = 0;
  bool ok = true;
  bool first = true;
  double lsum = 0.0;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int row = tile * TILE + tid;  // this thread's cell (row of the tile)
    const bool valid = row < n;
    // ---- stage X (and XT), W2 -------------------------------------------
    {
      const float* xr = X + size_t(row) * MF;
#pragma unroll
      for (int f = 0; f < MF; ++f) {
        const float v = valid ? xr[f] : 0.0f;
        st_bf(s.X, tc::kmaj_off(tid, f, MF), v);
        if (TRAIN) st_bf(s.XT, tc::kmaj_off(f, tid, TILE), v);
      }
    }
    stage_rows(s.W23, w.w2, MH, MH);
    cta_sync_async();
    // ---- F1: D1 = X W1^T; H1 = tanh(D1 + b1) ------------------------------
    if (tid == 0) issue(tm + C_D1, s.X, s.W1, MF, MH, false);
    if (!(ok = complete(&bar, phase))) break;
    for (int c0 = 0; c0 < MH; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tm + lane_base + C_D1 + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float h = tanhf(v[q] + s.b1[c0 + q]);
        st_bf(s.P, tc::kmaj_off(tid, c0 + q, MH), h);
        if (TRAIN) st_bf(s.R, tc::kmaj_off(c0 + q, tid, TILE), h);
      }
    }
    cta_sync_async();
    // ---- F2: D2 = H1 W2^T; H2 = tanh(D2 + b2) -----------------------------
    if (tid == 0) issue(tm + C_D2, s.P, s.W23, MH, MH, false);
    if (!(ok = complete(&bar, phase))) break;
    for (int c0 = 0; c0 < MH; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tm + lane_base + C_D2 + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float h = tanhf(v[q] + s.b2[c0 + q]);
        st_bf(s.Q, tc::kmaj_off(tid, c0 + q, MH), h);
        if (TRAIN) st_bf(s.S, tc::kmaj_off(c0 + q, tid, TILE), h);
      }
    }
    cta_sync_async();
    // ---- F3: Y = H2 W3^T + b3 ---------------------------------------------
    if (tid == 0) issue(tm + C_D3, s.Q, s.W3, MH, MO, false);
    if (!(ok = complete(&bar, phase))) break;
    float y[16];
    tc::tmem_ld16(tm + lane_base + C_D3, y);
#pragma unroll
    for (int q = 0; q < 16; ++q) y[q] += s.b3[q];
    if (!TRAIN) {
      if (valid)
#pragma unroll
        for (int q = 0; q < MO_USED; ++q) Y[size_t(row) * MO_USED + q] = y[q];
      __syncthreads();
      continue;
    }
    // ---- backward: dY, loss, b3 gradient; W2T into W23 --------------------
    float dy[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      float d = 0.0f;
      if (q < MO_USED && valid) {
        const float e = y[q] - T[size_t(row) * MO_USED + q];
        lsum += double(e) * double(e);
        d = 2.0f * e * inv_n;
      }
      dy[q] = d;
      st_bf(s.dY, tc::kmaj_off(tid, q, MO), d);
      st_bf(s.dYT, tc::kmaj_off(q, tid, TILE), d);
    }
#pragma unroll
    for (int q = 0; q < MO_USED; ++q) {
      const float t = warp_sum(dy[q]);
      if (lane == 0) s.gb3[warp][q] += t;
    }
    stage_rows(s.W23, w.w2t, MH, MH);
    cta_sync_async();
    // ---- B1: dW3^T += H2^T dY; dH2 = dY W3 --------------------------------
    if (tid == 0) {
      issue(tm + C_GW3, s.S, s.dYT, TILE, MO, !first);
      issue(tm + C_D1, s.dY, s.W3T, MO, MH, false);
    }
    if (!(ok = complete(&bar, phase))) break;
    for (int c0 = 0; c0 < MH; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tm + lane_base + C_D1 + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float h2 = ld_bf(s.Q, tc::kmaj_off(tid, c0 + q, MH));
        const float dz = valid ? v[q] * (1.0f - h2 * h2) : 0.0f;
        st_bf(s.P, tc::kmaj_off(tid, c0 + q, MH), dz);  // dZ2 (H1 is no longer read)
        const float t = warp_sum(dz);
        if (lane == 0) s.gb2[warp][c0 + q] += t;
      }
    }
    __syncthreads();  // H2 in Q is read no more: dZ2T overwrites it
    for (int c = 0; c < MH; ++c)
      *reinterpret_cast<uint16_t*>(s.Q + tc::kmaj_off(c, tid, TILE)) =
          *reinterpret_cast<const uint16_t*>(s.P + tc::kmaj_off(tid, c, MH));
    cta_sync_async();
    // ---- B2: dW2 += dZ2^T H1; dH1 = dZ2 W2 --------------------------------
    if (tid == 0) {
      issue(tm + C_GW2, s.Q, s.R, TILE, MH, !first);
      issue(tm + C_D2, s.P, s.W23, MH, MH, false);
    }
    if (!(ok = complete(&bar, phase))) break;
    for (int c0 = 0; c0 < MH; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tm + lane_base + C_D2 + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float h1 = ld_bf(s.R, tc::kmaj_off(c0 + q, tid, TILE));
        const float dz = valid ? v[q] * (1.0f - h1 * h1) : 0.0f;
        st_bf(s.S, tc::kmaj_off(c0 + q, tid, TILE), dz);  // dZ1T (H2T was consumed by B1)
        const float t = warp_sum(dz);
        if (lane == 0) s.gb1[warp][c0 + q] += t;
      }
    }
    cta_sync_async();
    // ---- B3: dW1 += dZ1^T X ------------------------------------------------
    if (tid == 0) issue(tm + C_GW1, s.S, s.XT, TILE, MF, !first);
    if (!(ok = complete(&bar, phase))) break;
    first = false;
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else if (TRAIN && !first) {
    // the CTA's accumulated gradients into its own slot of grad (summed
    // over the CTAs in CTA order by mlp_reduce_kernel: training is
    // deterministic); TMEM lane = output row
    float* gs = grad + size_t(blockIdx.x) * NPARAM;
    const int r = tid;
    float v[16];
    tc::tmem_ld16(tm + lane_base + C_GW3, v);  // dW3^T: row h, columns o
#pragma unroll
    for (int q = 0; q < MO; ++q) gs[P_W3 + q * MH + r] = q < MO_USED ? v[q] : 0.0f;
    tc::tmem_ld16(tm + lane_base + C_GW1, v);  // dW1: row h, columns f
#pragma unroll
    for (int q = 0; q < MF; ++q) gs[P_W1 + r * MF + q] = v[q];
    for (int c0 = 0; c0 < MH; c0 += 16) {       // dW2: row o, columns h
      tc::tmem_ld16(tm + lane_base + C_GW2 + c0, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) gs[P_W2 + r * MH + c0 + q] = v[q];
    }
    __syncthreads();
    gs[P_B1 + r] = ((s.gb1[0][r] + s.gb1[1][r]) + s.gb1[2][r]) + s.gb1[3][r];
    gs[P_B2 + r] = ((s.gb2[0][r] + s.gb2[1][r]) + s.gb2[2][r]) + s.gb2[3][r];
    if (r < MO) gs[P_B3 + r] = r < MO_USED ? ((s.gb3[0][r] + s.gb3[1][r]) + s.gb3[2][r]) + s.gb3[3][r] : 0.0f;
  }
  if (TRAIN && ok) {
    double sum = lsum;
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) s.lw[warp] = sum;
    __syncthreads();
    if (tid == 0) loss[blockIdx.x] = ((s.lw[0] + s.lw[1]) + s.lw[2]) + s.lw[3];
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tm, ncols);
}

// BF16 copies (and transposes) of the FP32 parameters.
__global__ void mlp_cast_kernel(const float* __restrict__ p, uint16_t* w1, uint16_t* w2, uint16_t* w3,
                                uint16_t* w2t, uint16_t* w3t) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < MH * MH; q += gridDim.x * blockDim.x) {
    const int r = q / MH, c = q % MH;
    w2[q] = f2bf(p[P_W2 + q]);
    w2t[c * MH + r] = f2bf(p[P_W2 + q]);
    if (q < MH * MF) w1[q] = f2bf(p[P_W1 + q]);
    if (q < MO * MH) {
      const int o = q / MH, h = q % MH;
      w3[q] = f2bf(p[P_W3 + q]);
      w3t[h * MO + o] = f2bf(p[P_W3 + q]);
    }
  }
}

// Adam (Kingma & Ba, 2015): m = b1 m + (1-b1) g; v = b2 v + (1-b2) g^2;
// p -= lr * (m / (1-b1^t)) / (sqrt(v / (1-b2^t)) + eps).
__global__ void adam_kernel(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
  }
}

// grad[q] = sum over the CTAs' slots in CTA order; loss likewise.
__global__ void mlp_reduce_kernel(const float* __restrict__ parts, int nparts, float* __restrict__ grad,
                                  const double* lparts, double* loss) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < NPARAM; q += gridDim.x * blockDim.x) {
    float t = 0.0f;
    for (int c = 0; c < nparts; ++c) t += parts[size_t(c) * NPARAM + q];
    grad[q] = t;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double t = 0.0;
    for (int c = 0; c < nparts; ++c) t += lparts[c];
    *loss = t;
  }
}

}  // namespace

struct e2d_mlp {
  int device = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  float* gpart = nullptr;     // [sms][NPARAM] per-CTA gradient slots
  double* lpart = nullptr;    // [sms] per-CTA loss sums
  uint16_t *w1 = nullptr, *w2 = nullptr, *w3 = nullptr, *w2t = nullptr, *w3t = nullptr;
  double* loss = nullptr;
  int* err = nullptr;
  int adam_t = 0;
  int sms = 148;
};

namespace {

int mlp_refresh(e2d_mlp* mm, cudaStream_t st) {
  mlp_cast_kernel<<<64, 256, 0, st>>>(mm->p, mm->w1, mm->w2, mm->w3, mm->w2t, mm->w3t);
  return cudaGetLastError() == cudaSuccess ? 0 : E2D_ERR_CUDA;
}

MlpDev dev_of(const e2d_mlp* mm) { return MlpDev{mm->w1, mm->w2, mm->w3, mm->w2t, mm->w3t, mm->p}; }

template <bool TRAIN>
int mlp_launch(e2d_mlp* mm, const float* X, const float* T, int n, float* Y, cudaStream_t st) {
  static bool configured = false;
  const size_t smem = sizeof(MlpSmem);
  if (!configured) {
    if (cudaFuncSetAttribute(mlp_kernel<TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) !=
        cudaSuccess)
      return E2D_ERR_CUDA;
    configured = true;
  }
  const int ntiles = (n + TILE - 1) / TILE;
  const int grid = ntiles < mm->sms ? ntiles : mm->sms;  // persistent: one CTA per SM
  mlp_kernel<TRAIN><<<grid, TILE, smem, st>>>(dev_of(mm), X, T, n, 1.0f / float(n), Y, mm->gpart, mm->lpart,
                                               mm->err);
  if (cudaGetLastError() != cudaSuccess) return E2D_ERR_CUDA;
  if (TRAIN) {
    mlp_reduce_kernel<<<(NPARAM + 255) / 256, 256, 0, st>>>(mm->gpart, grid, mm->g, mm->lpart, mm->loss);
    if (cudaGetLastError() != cudaSuccess) return E2D_ERR_CUDA;
  }
  return 0;
}

int mlp_check(e2d_mlp* mm, cudaStream_t st) {
  int e = 0;
  if (cudaMemcpyAsync(&e, mm->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return E2D_ERR_CUDA;
  return e ? E2D_ERR_CUDA : 0;
}

// PCG32 (O'Neill, 2014) for the initial weights.
struct Pcg {
  uint64_t s, inc;
  uint32_t next() {
    const uint64_t old = s;
    s = old * 6364136223846793005ULL + inc;
    const uint32_t x = uint32_t(((old >> 18u) ^ old) >> 27u), r = uint32_t(old >> 59u);
    return (x >> r) | (x << ((32 - r) & 31));
  }
  double uniform() { return (next() + 0.5) / 4294967296.0; }
};

}  // namespace

extern "C" {

e2d_mlp* e2d_mlp_create(uint64_t seed, int* err) {
  if (err) *err = 0;
  e2d_mlp* mm = new e2d_mlp;
  cudaGetDevice(&mm->device);
  cudaDeviceGetAttribute(&mm->sms, cudaDevAttrMultiProcessorCount, mm->device);
  bool bad = cudaMalloc(&mm->p, 4 * NPARAM) || cudaMalloc(&mm->g, 4 * NPARAM) || cudaMalloc(&mm->m, 4 * NPARAM) ||
             cudaMalloc(&mm->v, 4 * NPARAM) || cudaMalloc(&mm->w1, 2 * MH * MF) || cudaMalloc(&mm->w2, 2 * MH * MH) ||
             cudaMalloc(&mm->w3, 2 * MO * MH) || cudaMalloc(&mm->w2t, 2 * MH * MH) ||
             cudaMalloc(&mm->w3t, 2 * MO * MH) || cudaMalloc(&mm->loss, sizeof(double)) ||
             cudaMalloc(&mm->gpart, 4 * size_t(NPARAM) * mm->sms) || cudaMalloc(&mm->lpart, sizeof(double) * mm->sms) ||
             cudaMalloc(&mm->err, sizeof(int));
  if (bad) {
    if (err) *err = E2D_ERR_NOMEM;
    e2d_mlp_destroy(mm);
    return nullptr;
  }
  // Glorot-uniform weights, zero biases
  std::vector<float> h(NPARAM, 0.0f);
  Pcg rng{seed * 2 + 1, (seed << 1) | 1};
  auto fill = [&](int off, int rows, int cols) {
    const double a = std::sqrt(6.0 / double(rows + cols));
    for (int q = 0; q < rows * cols; ++q) h[off + q] = float((2.0 * rng.uniform() - 1.0) * a);
  };
  fill(P_W1, MH, MF);
  fill(P_W2, MH, MH);
  fill(P_W3, MO, MH);
  if (cudaMemcpy(mm->p, h.data(), 4 * NPARAM, cudaMemcpyHostToDevice) || cudaMemset(mm->m, 0, 4 * NPARAM) ||
      cudaMemset(mm->v, 0, 4 * NPARAM) || cudaMemset(mm->err, 0, sizeof(int)) || mlp_refresh(mm, 0) ||
      cudaDeviceSynchronize()) {
    if (err) *err = E2D_ERR_CUDA;
    e2d_mlp_destroy(mm);
    return nullptr;
  }
  return mm;
}

void e2d_mlp_destroy(e2d_mlp* mm) {
  if (!mm) return;
  for (void* q : {(void*)mm->gpart, (void*)mm->lpart, (void*)mm->p, (void*)mm->g, (void*)mm->m, (void*)mm->v, (void*)mm->w1, (void*)mm->w2,
                  (void*)mm->w3, (void*)mm->w2t, (void*)mm->w3t, (void*)mm->loss, (void*)mm->err})
    if (q) cudaFree(q);
  delete mm;
}

int e2d_mlp_nparams(void) { return NPARAM; }

int e2d_mlp_params(e2d_mlp* mm, float* out, const float* in) {
  if (!mm) return E2D_ERR_ARG;
  if (in) {
    if (cudaMemcpy(mm->p, in, 4 * NPARAM, cudaMemcpyHostToDevice) != cudaSuccess) return E2D_ERR_CUDA;
    if (mlp_refresh(mm, 0) || cudaDeviceSynchronize() != cudaSuccess) return E2D_ERR_CUDA;
  }
  if (out && cudaMemcpy(out, mm->p, 4 * NPARAM, cudaMemcpyDeviceToHost) != cudaSuccess) return E2D_ERR_CUDA;
  return 0;
}

int e2d_mlp_forward(e2d_mlp* mm, const float* X, int n, float* Y, void* stream) {
  if (!mm || !X || !Y || n < 1) return E2D_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = mlp_launch<false>(mm, X, nullptr, n, Y, st);
  return rc ? rc : mlp_check(mm, st);
}

int e2d_mlp_gradient(e2d_mlp* mm, const float* X, const float* T, int n, float* grad, double* loss, void* stream) {
  if (!mm || !X || !T || n < 1) return E2D_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = mlp_launch<true>(mm, X, T, n, nullptr, st);
  if (rc || (rc = mlp_check(mm, st))) return rc;
  if (grad && cudaMemcpy(grad, mm->g, 4 * NPARAM, cudaMemcpyDeviceToHost) != cudaSuccess) return E2D_ERR_CUDA;
  if (loss) {
    double l = 0.0;
    if (cudaMemcpy(&l, mm->loss, sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) return E2D_ERR_CUDA;
    *loss = l / double(n);
  }
  return 0;
}

int e2d_mlp_train(e2d_mlp* mm, const float* X, const float* T, int n, int steps, float lr, float* loss_hist,
                  void* stream) {
  if (!mm || !X || !T || n < 1 || steps < 0 || !(lr > 0.0f)) return E2D_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int k = 0; k < steps; ++k) {
    double l = 0.0;
    int rc = e2d_mlp_gradient(mm, X, T, n, nullptr, loss_hist ? &l : nullptr, stream);
    if (rc) return rc;
    if (loss_hist) loss_hist[k] = float(l);
    ++mm->adam_t;
    const float c1 = 1.0f - powf(b1, float(mm->adam_t)), c2 = 1.0f - powf(b2, float(mm->adam_t));
    adam_kernel<<<64, 256, 0, st>>>(mm->p, mm->g, mm->m, mm->v, NPARAM, lr, b1, b2, eps, c1, c2);
    if (cudaGetLastError() != cudaSuccess || mlp_refresh(mm, st)) return E2D_ERR_CUDA;
  }
  return cudaStreamSynchronize(st) == cudaSuccess ? 0 : E2D_ERR_CUDA;
}

}  // extern "C"
