// e2d_mlp_deep.cu — the deep warm-start network on the tensor cores: 5 input
// features (padded to 16), four hidden layers of 256 units with GELU (tanh
// form), 4 outputs (padded to 16).  The network runs layer by layer over a
// batch of rows, a layer's activations in HBM between kernels:
//
//   dense_kernel<FWD_GELU>   Z = A W^T + b (FP32, kept for the backward pass),
//                            H = bf16(gelu(Z))
//   dense_kernel<FWD_LINEAR> Y = A W^T + b                       (output layer)
//   dense_kernel<BWD_GELU>   dZp = bf16((dZ W) * gelu'(Zp))      (W^T staged)
//   dw_kernel                dW = dZ^T A over a CTA's rows -> its slot; the
//                            slots are summed in CTA order (deterministic)
//
// Every product is one elected thread issuing tcgen05.mma of BF16 operands
// in shared memory (canonical K-major layout, e2d_tc.cuh) into an FP32 TMEM
// accumulator, committed to an mbarrier that the CTA waits on with a bounded
// spin; a wait that runs out sets the error word and the kernel returns
// after freeing its TMEM.  One CTA of 128 threads per SM, persistent over
// tiles of 128 rows (a row is a TMEM lane, a thread its epilogue).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/cffc_e2d.h"
#include "e2d_tc.cuh"

using namespace e2d;

namespace {

constexpr int DF = 16, DH = 256, DO = 16, DO_USED = 4, DNL = 4;  // features, width, outputs (padded), hidden layers
constexpr int NLAYER = DNL + 1;
constexpr int TILE = 128;          // rows per tile (UMMA M), threads per CTA
constexpr int RC = 64;             // rows per chunk of the weight-gradient product
constexpr uint32_t WAIT_ITERS = 1u << 22;

__host__ __device__ constexpr int layer_in(int l) { return l == 0 ? DF : DH; }
__host__ __device__ constexpr int layer_out(int l) { return l == DNL ? DO : DH; }
// flat parameter vector: W_l [out][in] then b_l [out], layers 0..4
__host__ __device__ constexpr int w_off(int l) {
  return l == 0 ? 0 : w_off(l - 1) + layer_out(l - 1) * layer_in(l - 1) + layer_out(l - 1);
}
__host__ __device__ constexpr int b_off(int l) { return w_off(l) + layer_out(l) * layer_in(l); }
constexpr int NPARAM = w_off(NLAYER);

enum Epi { FWD_GELU = 0, FWD_LINEAR = 1, BWD_GELU = 2 };

__device__ __forceinline__ uint16_t f2bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float bf2f(uint16_t b) { return __uint_as_float(uint32_t(b) << 16); }

// GELU, tanh form, and its derivative.
__device__ __forceinline__ float gelu(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  return 0.5f * z * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_prime(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  const float t = tanhf(u);
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * 0.7978845608028654f * (1.0f + 0.134145f * z * z);
}

// Row-major BF16 [rows][K] (global) -> canonical K-major tile (shared), 16
// bytes (8 values of one row) at a time; rows at or past `valid` are zero.
__device__ void stage_tile(uint8_t* dst, const uint16_t* src, int rows, int K, int valid) {
  const int per_row = K / 8;
  for (int q = threadIdx.x; q < rows * per_row; q += TILE) {
    const int r = q / per_row, c = (q % per_row) * 8;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (r < valid) v = *reinterpret_cast<const uint4*>(src + size_t(r) * K + c);
    *reinterpret_cast<uint4*>(dst + tc::kmaj_off(r, c, K)) = v;
  }
}

__device__ __forceinline__ void cta_sync_async() {
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
}

// Commit (thread 0) and bounded wait of every thread; CTA-uniform result.
__device__ __forceinline__ bool complete(uint64_t* bar, uint32_t& phase) {
  if (threadIdx.x == 0) tc::mma_commit(bar);
  __syncwarp();
  const bool ok = tc::mbar_wait(bar, phase, WAIT_ITERS);
  phase ^= 1u;
  tc::fence_after_sync();
  return __syncthreads_and(ok) != 0;
}

__host__ __device__ inline uint32_t tmem_cols(int n) {
  uint32_t c = 32;
  while (c < uint32_t(n)) c <<= 1;
  return c;
}

// D[tile rows][N] = A[tile rows][K] B[N][K]^T with the epilogue EPI; B stays
// in shared memory for all of the CTA's tiles.  K and N: multiples of 16, at
// most 256.
template <int EPI>
__global__ void __launch_bounds__(TILE, 1) dense_kernel(const uint16_t* __restrict__ A, int K,
                                                        const uint16_t* __restrict__ Bw, int N,
                                                        const float* __restrict__ bias, int n,
                                                        float* __restrict__ Zout, uint16_t* __restrict__ Hout,
                                                        const float* __restrict__ Zp, float* __restrict__ Yout,
                                                        int* err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t taddr;
  uint8_t* Bs = sm;                      // [N][K]
  uint8_t* As = sm + size_t(N) * K * 2;  // [TILE][K]
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ncols = tmem_cols(N);
  stage_tile(Bs, Bw, N, K, N);
  if (tid == 0) tc::mbar_init(&bar, 1);
  if (warp == 0) tc::tmem_alloc(&taddr, ncols);
  cta_sync_async();
  const uint32_t tm = taddr;
  const uint32_t lane_base = uint32_t(32 * warp) << 16;
  const uint32_t id = tc::idesc_bf16(TILE, N);
  uint32_t phase = 0;
  const int ntiles = (n + TILE - 1) / TILE;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r0 = tile * TILE;
    stage_tile(As, A + size_t(r0) * K, TILE, K, n - r0);
    cta_sync_async();
    if (tid == 0) {
      const uint32_t a0 = tc::smem_addr(As), b0 = tc::smem_addr(Bs);
      for (int t = 0; t < K / 16; ++t)
        tc::mma_bf16(tm, tc::smem_desc(a0 + 256 * t, 128, K * 16), tc::smem_desc(b0 + 256 * t, 128, K * 16), id,
                     t > 0 ? 1u : 0u);
    }
    if (!complete(&bar, phase)) {
      if (tid == 0) atomicExch(err, 1);
      break;
    }
    const int row = r0 + tid;
    const bool valid = row < n;
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      tc::tmem_ld16(tm + lane_base + uint32_t(c0), v);
      if (!valid) continue;
      if (EPI == FWD_GELU || EPI == FWD_LINEAR) {
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] += bias[c0 + q];
      }
      if (EPI == FWD_LINEAR) {
        float4* y = reinterpret_cast<float4*>(Yout + size_t(row) * N + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q) y[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        continue;
      }
      if (EPI == FWD_GELU) {
        float4* z = reinterpret_cast<float4*>(Zout + size_t(row) * N + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q) z[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
#pragma unroll
        for (int q = 0; q < 16; ++q) v[q] = gelu(v[q]);
      } else {  // BWD_GELU
        const float4* zp = reinterpret_cast<const float4*>(Zp + size_t(row) * N + c0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 z = zp[q];
          v[4 * q] *= gelu_prime(z.x); v[4 * q + 1] *= gelu_prime(z.y);
          v[4 * q + 2] *= gelu_prime(z.z); v[4 * q + 3] *= gelu_prime(z.w);
        }
      }
      uint32_t pk[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) pk[q] = uint32_t(f2bf(v[2 * q])) | (uint32_t(f2bf(v[2 * q + 1])) << 16);
      uint4* h = reinterpret_cast<uint4*>(Hout + size_t(row) * N + c0);
      h[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
      h[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tm, ncols);
}

// Row-major BF16 [rows][F] (global) -> the transposed canonical tile
// [F][RC] (shared; K = rows): element (f, r) at kmaj_off(f, r, RC).
__device__ void stage_transposed(uint8_t* dst, const uint16_t* src, int rows, int F, int valid) {
  const int per_row = F / 8;
  for (int q = threadIdx.x; q < rows * per_row; q += TILE) {
    const int r = q / per_row, f0 = (q % per_row) * 8;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (r < valid) v = *reinterpret_cast<const uint4*>(src + size_t(r) * F + f0);
    const uint16_t* e = reinterpret_cast<const uint16_t*>(&v);
#pragma unroll
    for (int k = 0; k < 8; ++k) *reinterpret_cast<uint16_t*>(dst + tc::kmaj_off(f0 + k, r, RC)) = e[k];
  }
}

// slot[blockIdx][256][N2] = P^T Q over the CTA's rows [r0, r1): P [n][256],
// Q [n][N2] row-major BF16, N2 16 or 256; the two 128-row halves of P^T
// accumulate in TMEM columns [0, N2) and [N2, 2 N2).
__global__ void __launch_bounds__(TILE, 1) dw_kernel(const uint16_t* __restrict__ P, const uint16_t* __restrict__ Q,
                                                     int N2, int n, int rows_per_cta, float* __restrict__ slots,
                                                     int* err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t taddr;
  uint8_t* Ps = sm;                      // [256][RC]
  uint8_t* Qs = sm + size_t(DH) * RC * 2;  // [N2][RC]
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t ncols = tmem_cols(2 * N2);
  if (tid == 0) tc::mbar_init(&bar, 1);
  if (warp == 0) tc::tmem_alloc(&taddr, ncols);
  cta_sync_async();
  const uint32_t tm = taddr;
  const uint32_t lane_base = uint32_t(32 * warp) << 16;
  const uint32_t id = tc::idesc_bf16(TILE, N2);
  const int r0 = blockIdx.x * rows_per_cta, r1 = min(n, r0 + rows_per_cta);
  uint32_t phase = 0;
  bool ok = true, any = false;
  for (int c = r0; c < r1 && ok; c += RC) {
    stage_transposed(Ps, P + size_t(c) * DH, RC, DH, r1 - c);
    stage_transposed(Qs, Q + size_t(c) * N2, RC, N2, r1 - c);
    cta_sync_async();
    if (tid == 0) {
      const uint32_t p0 = tc::smem_addr(Ps), q0 = tc::smem_addr(Qs);
      for (int h = 0; h < 2; ++h)
        for (int t = 0; t < RC / 16; ++t)
          tc::mma_bf16(tm + uint32_t(h * N2), tc::smem_desc(p0 + h * (TILE * RC * 2) + 256 * t, 128, RC * 16),
                       tc::smem_desc(q0 + 256 * t, 128, RC * 16), id, (any || t > 0) ? 1u : 0u);
    }
    any = true;
    ok = complete(&bar, phase);
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    float* out = slots + size_t(blockIdx.x) * DH * N2;
    for (int h = 0; h < 2; ++h) {
      const int f = h * TILE + tid;
      for (int c0 = 0; c0 < N2; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tm + lane_base + uint32_t(h * N2 + c0), v);
#pragma unroll
        for (int q = 0; q < 16; ++q) out[size_t(f) * N2 + c0 + q] = any ? v[q] : 0.0f;
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tm, ncols);
}

// The CTAs' slots summed in CTA order into the gradient of W_l: slot layout
// [256][N2]; transpose = the slots hold W_l^T (the output layer).
__global__ void dw_reduce_kernel(const float* __restrict__ slots, int nslot, int N2, float* __restrict__ g,
                                 int woff, int transpose) {
  const int total = DH * N2;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
    float t = 0.0f;
    for (int c = 0; c < nslot; ++c) t += slots[size_t(c) * total + q];
    const int f = q / N2, k = q % N2;
    if (transpose) {
      g[woff + k * DH + f] = k < DO_USED ? t : 0.0f;  // W5 [16][256]: rows past the used outputs stay 0
    } else {
      g[woff + q] = t;
    }
  }
}

// Column sums of D [n][F] (BF16) over rows: per-CTA partials, then in order.
__global__ void colsum_kernel(const uint16_t* __restrict__ D, int n, int F, int rows_per_cta, float* part) {
  const int c = threadIdx.x;
  if (c >= F) return;
  const int r0 = blockIdx.x * rows_per_cta, r1 = min(n, r0 + rows_per_cta);
  float t = 0.0f;
  for (int r = r0; r < r1; ++r) t += bf2f(D[size_t(r) * F + c]);
  part[size_t(blockIdx.x) * F + c] = t;
}
__global__ void colsum_reduce_kernel(const float* part, int nslot, int F, float* g, int boff, int used) {
  const int c = threadIdx.x;
  if (c >= F) return;
  float t = 0.0f;
  for (int k = 0; k < nslot; ++k) t += part[size_t(k) * F + c];
  g[boff + c] = c < used ? t : 0.0f;
}

// dY = bf16(2 (y - t) / n) on the used outputs (0 elsewhere) and per-CTA
// loss partials sum (y - t)^2.
__global__ void loss_kernel(const float* __restrict__ Y, const float* __restrict__ T, int n, float inv_n,
                            uint16_t* __restrict__ dY, double* lpart) {
  __shared__ double red[8];
  double s = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    for (int q = 0; q < DO; ++q) {
      float d = 0.0f;
      if (q < DO_USED) {
        const float e = Y[size_t(r) * DO + q] - T[size_t(r) * DO_USED + q];
        s += double(e) * double(e);
        d = 2.0f * e * inv_n;
      }
      dY[size_t(r) * DO + q] = f2bf(d);
    }
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < int(blockDim.x / 32); ++w) t += red[w];
    lpart[blockIdx.x] = t;
  }
}

// Rows idx[k] (or k when idx is null) of X [*][16] -> BF16 [n][16]; of T
// [*][4] -> [n][4].
__global__ void gather_kernel(const float* __restrict__ X, const float* __restrict__ T, const int* __restrict__ idx,
                              int n, uint16_t* __restrict__ Xb, float* __restrict__ Tb) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n * DF; q += gridDim.x * blockDim.x) {
    const int r = q / DF, f = q % DF;
    const int s = idx ? idx[r] : r;
    Xb[q] = f2bf(X[size_t(s) * DF + f]);
    if (T && f < DO_USED) Tb[size_t(r) * DO_USED + f] = T[size_t(s) * DO_USED + f];
  }
}

// Y [n][16] -> the used outputs [n][4].
__global__ void take_outputs_kernel(const float* __restrict__ Y, int n, float* __restrict__ out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n * DO_USED; q += gridDim.x * blockDim.x)
    out[q] = Y[size_t(q / DO_USED) * DO + q % DO_USED];
}

// BF16 copies of the weights, row-major [out][in], and their transposes [in][out].
__global__ void cast_kernel(const float* __restrict__ p, uint16_t* wb, uint16_t* wt) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < NPARAM; q += gridDim.x * blockDim.x) {
    int l = 0;
    while (l < NLAYER - 1 && q >= w_off(l + 1)) ++l;
    const int rel = q - w_off(l), nw = layer_out(l) * layer_in(l);
    if (rel >= nw) continue;  // a bias
    const int o = rel / layer_in(l), i = rel % layer_in(l);
    const uint16_t b = f2bf(p[q]);
    wb[q] = b;
    wt[w_off(l) + i * layer_out(l) + o] = b;
  }
}

// Adam (Kingma & Ba, 2015).
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

// The network and its work arrays (rows: the capacity of one pass).
struct e2d_mlp_deep {
  int device = 0, sms = 148, cap = 0, adam_t = 0;
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  uint16_t *wb = nullptr, *wt = nullptr;       // BF16 weights and transposes (param offsets)
  uint16_t* xb = nullptr;                      // [cap][16]
  uint16_t* act[DNL] = {};                     // H_1..H_4 [cap][256]
  float* z[DNL] = {};                          // Z_1..Z_4 [cap][256]
  float* y = nullptr;                          // [cap][16]
  float* tb = nullptr;                         // [cap][4]
  uint16_t* dy = nullptr;                      // [cap][16]
  uint16_t* dz[2] = {};                        // [cap][256] ping-pong deltas
  float* slots = nullptr;                      // [sms][256][256]
  float* bpart = nullptr;                      // [sms][256]
  double* lpart = nullptr;                     // [sms]
  int* idx = nullptr;                          // [cap] minibatch rows
  int* err = nullptr;
  std::vector<void*> ws;                       // work arrays (rebuilt on growth)
};

namespace {

template <class T> bool dalloc(std::vector<void*>& v, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, sizeof(T) * (n ? n : 1)) != cudaSuccess) return false;
  v.push_back(q);
  *p = static_cast<T*>(q);
  return true;
}

void free_ws(e2d_mlp_deep* d) {
  for (void* q : d->ws) cudaFree(q);
  d->ws.clear();
  d->cap = 0;
}

int ensure_cap(e2d_mlp_deep* d, int rows) {
  if (rows <= d->cap) return 0;
  free_ws(d);
  const size_t c = size_t(rows);
  bool ok = dalloc(d->ws, &d->xb, c * DF) && dalloc(d->ws, &d->y, c * DO) && dalloc(d->ws, &d->tb, c * DO_USED) &&
            dalloc(d->ws, &d->dy, c * DO) && dalloc(d->ws, &d->dz[0], c * DH) && dalloc(d->ws, &d->dz[1], c * DH) &&
            dalloc(d->ws, &d->idx, c);
  for (int l = 0; l < DNL && ok; ++l) ok = dalloc(d->ws, &d->act[l], c * DH) && dalloc(d->ws, &d->z[l], c * DH);
  if (!ok) {
    free_ws(d);
    return E2D_ERR_NOMEM;
  }
  d->cap = rows;
  return 0;
}

size_t dense_smem(int K, int N) { return size_t(N) * K * 2 + size_t(TILE) * K * 2; }
// The weight-gradient product holds up to 512 TMEM columns: a request above
// half the SM's shared memory keeps it to one CTA per SM, so no CTA waits in
// tcgen05.alloc for another's columns.
size_t dw_smem(int N2) {
  const size_t need = size_t(DH) * RC * 2 + size_t(N2) * RC * 2;
  return need < 120 * 1024 ? 120 * 1024 : need;
}

template <int EPI>
int dense(e2d_mlp_deep* d, const uint16_t* A, int K, const uint16_t* Bw, int N, const float* bias, int n, float* Z,
          uint16_t* H, const float* Zp, float* Y, cudaStream_t st) {
  const size_t smem = dense_smem(K, N);
  if (cudaFuncSetAttribute(dense_kernel<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return E2D_ERR_CUDA;
  const int ntiles = (n + TILE - 1) / TILE;
  dense_kernel<EPI><<<ntiles < d->sms ? ntiles : d->sms, TILE, smem, st>>>(A, K, Bw, N, bias, n, Z, H, Zp, Y,
                                                                           d->err);
  return cudaGetLastError() == cudaSuccess ? 0 : E2D_ERR_CUDA;
}

// Forward pass over n rows already in d->xb: activations, pre-activations
// and the outputs d->y.
int forward_rows(e2d_mlp_deep* d, int n, cudaStream_t st) {
  int rc;
  const uint16_t* a = d->xb;
  for (int l = 0; l < DNL; ++l) {
    if ((rc = dense<FWD_GELU>(d, a, layer_in(l), d->wb + w_off(l), DH, d->p + b_off(l), n, d->z[l], d->act[l],
                              nullptr, nullptr, st)))
      return rc;
    a = d->act[l];
  }
  return dense<FWD_LINEAR>(d, a, DH, d->wb + w_off(DNL), DO, d->p + b_off(DNL), n, nullptr, nullptr, nullptr, d->y,
                           st);
}

int weight_grad(e2d_mlp_deep* d, const uint16_t* P, const uint16_t* Q, int N2, int n, int woff, int transpose,
                cudaStream_t st) {
  const size_t smem = dw_smem(N2);
  if (cudaFuncSetAttribute(dw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
    return E2D_ERR_CUDA;
  int rows = (n + d->sms - 1) / d->sms;
  rows = ((rows + RC - 1) / RC) * RC;
  const int grid = (n + rows - 1) / rows;
  dw_kernel<<<grid, TILE, smem, st>>>(P, Q, N2, n, rows, d->slots, d->err);
  dw_reduce_kernel<<<64, 256, 0, st>>>(d->slots, grid, N2, d->g, woff, transpose);
  return cudaGetLastError() == cudaSuccess ? 0 : E2D_ERR_CUDA;
}

int bias_grad(e2d_mlp_deep* d, const uint16_t* D, int F, int n, int boff, int used, cudaStream_t st) {
  const int rows = (n + d->sms - 1) / d->sms;
  const int grid = (n + rows - 1) / rows;
  colsum_kernel<<<grid, 256, 0, st>>>(D, n, F, rows, d->bpart);
  colsum_reduce_kernel<<<1, 256, 0, st>>>(d->bpart, grid, F, d->g, boff, used);
  return cudaGetLastError() == cudaSuccess ? 0 : E2D_ERR_CUDA;
}

// Gradient of loss = sum over rows and the used outputs of (y - t)^2 / n
// for the n rows in d->xb / d->tb, into d->g; the loss sum into *lsum.
int gradient_rows(e2d_mlp_deep* d, int n, double* lsum, cudaStream_t st) {
  int rc;
  if ((rc = forward_rows(d, n, st))) return rc;
  const int lgrid = d->sms;
  loss_kernel<<<lgrid, 256, 0, st>>>(d->y, d->tb, n, 1.0f / float(n), d->dy, d->lpart);
  if (cudaGetLastError() != cudaSuccess) return E2D_ERR_CUDA;
  // output layer: dW5^T = H4^T dY (transposed into W5), db5 = column sums of dY
  if ((rc = weight_grad(d, d->act[DNL - 1], d->dy, DO, n, w_off(DNL), 1, st)) ||
      (rc = bias_grad(d, d->dy, DO, n, b_off(DNL), DO_USED, st)))
    return rc;
  // dZ4 = (dY W5) * gelu'(Z4): A = dY [n][16], B = W5^T [256][16]
  if ((rc = dense<BWD_GELU>(d, d->dy, DO, d->wt + w_off(DNL), DH, nullptr, n, nullptr, d->dz[0], d->z[DNL - 1],
                            nullptr, st)))
    return rc;
  int cur = 0;
  for (int l = DNL - 1; l >= 0; --l) {
    const uint16_t* dz = d->dz[cur];
    const uint16_t* ain = l == 0 ? d->xb : d->act[l - 1];
    // dW_l = dZ^T A_in [256][in], db_l = column sums of dZ
    if ((rc = weight_grad(d, dz, ain, layer_in(l), n, w_off(l), 0, st)) ||
        (rc = bias_grad(d, dz, DH, n, b_off(l), DH, st)))
      return rc;
    if (l == 0) break;
    // dZ_{l-1} = (dZ_l W_l) * gelu'(Z_{l-1}): B = W_l^T [256 in][256 out]
    if ((rc = dense<BWD_GELU>(d, dz, DH, d->wt + w_off(l), DH, nullptr, n, nullptr, d->dz[cur ^ 1], d->z[l - 1],
                              nullptr, st)))
      return rc;
    cur ^= 1;
  }
  if (lsum) {
    std::vector<double> lp(lgrid);
    if (cudaMemcpyAsync(lp.data(), d->lpart, sizeof(double) * lgrid, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      return E2D_ERR_CUDA;
    double t = 0.0;
    for (double x : lp) t += x;
    *lsum = t;
  }
  return 0;
}

int check_err(e2d_mlp_deep* d, cudaStream_t st) {
  int e = 0;
  if (cudaMemcpyAsync(&e, d->err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return E2D_ERR_CUDA;
  return e ? E2D_ERR_CUDA : 0;
}

int refresh(e2d_mlp_deep* d, cudaStream_t st) {
  cast_kernel<<<256, 256, 0, st>>>(d->p, d->wb, d->wt);
  return cudaGetLastError() == cudaSuccess ? 0 : E2D_ERR_CUDA;
}

}  // namespace

extern "C" {

e2d_mlp_deep* e2d_mlp_deep_create(uint64_t seed, int* err) {
  if (err) *err = 0;
  e2d_mlp_deep* d = new e2d_mlp_deep;
  cudaGetDevice(&d->device);
  cudaDeviceGetAttribute(&d->sms, cudaDevAttrMultiProcessorCount, d->device);
  std::vector<void*> fixed;
  bool ok = cudaMalloc(&d->p, 4 * size_t(NPARAM)) == cudaSuccess && cudaMalloc(&d->g, 4 * size_t(NPARAM)) == cudaSuccess &&
            cudaMalloc(&d->m, 4 * size_t(NPARAM)) == cudaSuccess && cudaMalloc(&d->v, 4 * size_t(NPARAM)) == cudaSuccess &&
            cudaMalloc(&d->wb, 2 * size_t(NPARAM)) == cudaSuccess && cudaMalloc(&d->wt, 2 * size_t(NPARAM)) == cudaSuccess &&
            cudaMalloc(&d->slots, 4 * size_t(d->sms) * DH * DH) == cudaSuccess &&
            cudaMalloc(&d->bpart, 4 * size_t(d->sms) * DH) == cudaSuccess &&
            cudaMalloc(&d->lpart, sizeof(double) * d->sms) == cudaSuccess &&
            cudaMalloc(&d->err, sizeof(int)) == cudaSuccess;
  if (!ok) {
    if (err) *err = E2D_ERR_NOMEM;
    e2d_mlp_deep_destroy(d);
    return nullptr;
  }
  // Glorot-uniform weights, zero biases
  std::vector<float> h(NPARAM, 0.0f);
  Pcg rng{seed * 2 + 1, (seed << 1) | 1};
  for (int l = 0; l < NLAYER; ++l) {
    const int fan_in = l == 0 ? 5 : layer_in(l), fan_out = l == DNL ? DO_USED : layer_out(l);
    const double a = std::sqrt(6.0 / double(fan_in + fan_out));
    for (int o = 0; o < layer_out(l); ++o)
      for (int i = 0; i < layer_in(l); ++i) {
        const double u = (2.0 * rng.uniform() - 1.0) * a;
        // inputs past the 5 features and outputs past the 4 used ones start at zero
        const bool live = (l > 0 || i < 5) && (l < DNL || o < DO_USED);
        h[w_off(l) + o * layer_in(l) + i] = live ? float(u) : 0.0f;
      }
  }
  if (cudaMemcpy(d->p, h.data(), 4 * size_t(NPARAM), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(d->m, 0, 4 * size_t(NPARAM)) != cudaSuccess || cudaMemset(d->v, 0, 4 * size_t(NPARAM)) != cudaSuccess ||
      cudaMemset(d->g, 0, 4 * size_t(NPARAM)) != cudaSuccess || cudaMemset(d->wt, 0, 2 * size_t(NPARAM)) != cudaSuccess ||
      cudaMemset(d->err, 0, sizeof(int)) != cudaSuccess || refresh(d, 0) || cudaDeviceSynchronize() != cudaSuccess) {
    if (err) *err = E2D_ERR_CUDA;
    e2d_mlp_deep_destroy(d);
    return nullptr;
  }
  return d;
}

void e2d_mlp_deep_destroy(e2d_mlp_deep* d) {
  if (!d) return;
  free_ws(d);
  for (void* q : {(void*)d->p, (void*)d->g, (void*)d->m, (void*)d->v, (void*)d->wb, (void*)d->wt, (void*)d->slots,
                  (void*)d->bpart, (void*)d->lpart, (void*)d->err})
    if (q) cudaFree(q);
  delete d;
}

int e2d_mlp_deep_nparams(void) { return NPARAM; }

int e2d_mlp_deep_params(e2d_mlp_deep* d, float* out, const float* in) {
  if (!d) return E2D_ERR_ARG;
  if (in) {
    if (cudaMemcpy(d->p, in, 4 * size_t(NPARAM), cudaMemcpyHostToDevice) != cudaSuccess) return E2D_ERR_CUDA;
    if (refresh(d, 0) || cudaDeviceSynchronize() != cudaSuccess) return E2D_ERR_CUDA;
  }
  if (out && cudaMemcpy(out, d->p, 4 * size_t(NPARAM), cudaMemcpyDeviceToHost) != cudaSuccess) return E2D_ERR_CUDA;
  return 0;
}

int e2d_mlp_deep_forward(e2d_mlp_deep* d, const float* X, int n, float* Y, void* stream) {
  if (!d || !X || !Y || n < 1) return E2D_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int chunk = n < 65536 ? n : 65536;
  int rc;
  if ((rc = ensure_cap(d, chunk))) return rc;
  for (int r0 = 0; r0 < n; r0 += chunk) {
    const int m = n - r0 < chunk ? n - r0 : chunk;
    gather_kernel<<<256, 256, 0, st>>>(X + size_t(r0) * DF, nullptr, nullptr, m, d->xb, nullptr);
    if (cudaGetLastError() != cudaSuccess) return E2D_ERR_CUDA;
    if ((rc = forward_rows(d, m, st))) return rc;
    take_outputs_kernel<<<256, 256, 0, st>>>(d->y, m, Y + size_t(r0) * DO_USED);
    if (cudaGetLastError() != cudaSuccess) return E2D_ERR_CUDA;
  }
  return check_err(d, st);
}

int e2d_mlp_deep_gradient(e2d_mlp_deep* d, const float* X, const float* T, int n, float* grad, double* loss,
                          void* stream) {
  if (!d || !X || !T || n < 1) return E2D_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc;
  if ((rc = ensure_cap(d, n))) return rc;
  gather_kernel<<<256, 256, 0, st>>>(X, T, nullptr, n, d->xb, d->tb);
  if (cudaGetLastError() != cudaSuccess) return E2D_ERR_CUDA;
  double l = 0.0;
  if ((rc = gradient_rows(d, n, &l, st)) || (rc = check_err(d, st))) return rc;
  if (grad && cudaMemcpy(grad, d->g, 4 * size_t(NPARAM), cudaMemcpyDeviceToHost) != cudaSuccess) return E2D_ERR_CUDA;
  if (loss) *loss = l / double(n);
  return 0;
}

int e2d_mlp_deep_train(e2d_mlp_deep* d, const float* X, const float* T, int n, int steps, int batch, float lr,
                       uint64_t seed, float* loss_hist, void* stream) {
  if (!d || !X || !T || n < 1 || steps < 0 || batch < 1 || !(lr > 0.0f)) return E2D_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int b = batch < n ? batch : n;
  int rc;
  if ((rc = ensure_cap(d, b))) return rc;
  Pcg rng{seed * 2 + 1, (seed << 1) | 1};
  std::vector<int> perm(n), hidx(b);
  for (int q = 0; q < n; ++q) perm[q] = q;
  int pos = n;  // reshuffle at the first step
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int k = 0; k < steps; ++k) {
    for (int q = 0; q < b; ++q) {
      if (pos >= n) {  // Fisher-Yates shuffle of the rows per epoch
        for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[int(rng.next() % uint32_t(i + 1))]);
        pos = 0;
      }
      hidx[q] = perm[pos++];
    }
    if (cudaMemcpyAsync(d->idx, hidx.data(), sizeof(int) * b, cudaMemcpyHostToDevice, st) != cudaSuccess)
      return E2D_ERR_CUDA;
    gather_kernel<<<256, 256, 0, st>>>(X, T, d->idx, b, d->xb, d->tb);
    if (cudaGetLastError() != cudaSuccess) return E2D_ERR_CUDA;
    double l = 0.0;
    if ((rc = gradient_rows(d, b, loss_hist ? &l : nullptr, st))) return rc;
    if (loss_hist) loss_hist[k] = float(l / double(b));
    ++d->adam_t;
    const float c1 = 1.0f - powf(b1, float(d->adam_t)), c2 = 1.0f - powf(b2, float(d->adam_t));
    adam_kernel<<<256, 256, 0, st>>>(d->p, d->g, d->m, d->v, NPARAM, lr, b1, b2, eps, c1, c2);
    if (cudaGetLastError() != cudaSuccess || refresh(d, st)) return E2D_ERR_CUDA;
  }
  return check_err(d, st);
}

}  // extern "C"
