// e2d_capi.cu — the C ABI of include/cffc_e2d.h: handle life cycle, device
// memory, and the launch sequences of the reference's per-block routines.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/cffc_e2d.h"
#include "e2d_handle.h"
#include "e2d_smooth.cuh"

using namespace e2d;

namespace e2d_host {

#define CK(call)                                                               \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      fprintf(stderr, "cffc_e2d: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
      return E2D_ERR_CUDA;                                                     \
    }                                                                          \
  } while (0)


template <class T> int upload(e2d_handle* h, T** p, const T* src, size_t n) {
  int rc = dalloc(h, p, n);
  if (rc) return rc;
  CK(cudaMemcpy(*p, src, sizeof(T) * n, cudaMemcpyHostToDevice));
  return 0;
}

int check_status(e2d_handle* h) {
  int st[2] = {0, 0};
  CK(cudaMemcpyAsync(st, h->B.status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (st[0] == ST_NEGATIVE) return 1 + st[1];
  return st[0] ? E2D_ERR_CUDA : 0;
}

// Runge_Kutta (CFD.cc:901-940) and MultiStage_Optimally_Smoothing
// (CFD.cc:953-1031): the update coefficient of stage s of an n-stage scheme.
// The optimally smoothing values are van Leer, Tai and Powell's published
// coefficients (product of the stage factor and the scheme's CFL factor).
double rk_coefficient(int s, int n) {
  double beta = 1.0;
  if (n == 2 && s == 2) beta = 0.5 * beta;
  if (n == 4) {
    if (s == 1 || s == 2) beta = 0.5 * beta;
    if (s == 4) beta = beta / 6.0;
  }
  if (n == 5) {
    static const double f[4] = {0.059, 0.14, 0.273, 0.5};
    if (s <= 4) beta *= f[s - 1];
  }
  return beta;
}
double os_coefficient(int s, int n, int limiter) {
  static const double zero_lim[7][6] = {{0}, {1.0}, {1.0, 0.3333}, {1.50, 0.1481, 0.4000},
                                        {2.00, 0.0833, 0.2069, 0.4265}, {2.50, 0.0533, 0.1263, 0.2375, 0.4414},
                                        {3.00, 0.0370, 0.0851, 0.1521, 0.2562, 0.4512}};
  static const double lim[7][6] = {{0}, {1.0}, {0.4693, 0.4242}, {0.6936, 0.1918, 0.4929},
                                   {0.9214, 0.1084, 0.2602, 0.5052}, {1.1508, 0.0695, 0.1602, 0.2898, 0.5060},
                                   {1.3805, 0.0482, 0.1085, 0.1885, 0.3050, 0.5063}};
  if (n < 1 || n > 6) return 1.0;
  const double(&t)[6] = limiter == E2D_LIMITER_ZERO ? zero_lim[n] : lim[n];
  double beta = t[0];
  if (s < n) beta = t[s] * beta;  // stage s < n scales the scheme's factor
  return beta;
}

// Is the stage sequence of (time_integration, n_stage) one this library runs?
bool scheme_supported(const e2d_scheme* sc) {
  switch (sc->time_integration) {
    case E2D_TIME_EXPLICIT_EULER: return sc->n_stage == 1 || sc->n_stage == 2;
    case E2D_TIME_PREDICTOR_CORRECTOR: return sc->n_stage == 2;
    case E2D_TIME_RUNGE_KUTTA: return sc->n_stage == 1 || sc->n_stage == 2 || sc->n_stage == 4 || sc->n_stage == 5;
    case E2D_TIME_OPTIMAL_SMOOTHING: return sc->n_stage >= 1 && sc->n_stage <= 6;
    default: return false;
  }
}

// Stage s of the handle's scheme: the state it reads (in) and writes (out)
// -- 0 = (W, U), 1 = (W2, U2), 2 = (W3, U3) -- its update coefficient, the
// residual slot it stores (0 = dUdt, 1 = R1, 2 = R2) and whether its
// residual starts from the stored one (the two-stage Runge-Kutta and
// predictor-corrector schemes, and RK4's last stage; every other stage
// starts from zero, dUdt_Multistage_Explicit, Euler2DQuad.cc:1304-1342).
// A stage never writes the state it reads its halo from; the last one
// writes (W, U) (one-stage schemes copy their result there).
struct StagePlan {
  int mode, in, out, slot;
  bool rk4;
  double omega;
};
StagePlan stage_plan(const e2d_scheme& sc, int s) {
  const int n = sc.n_stage;
  const bool os = sc.time_integration == E2D_TIME_OPTIMAL_SMOOTHING;
  StagePlan p{1, 0, 1, 0, false, os ? os_coefficient(s, n, sc.limiter) : rk_coefficient(s, n)};
  if (s == 1) return p;
  p.in = (s == 2) ? 1 : ((s % 2 == 0) ? 1 : 2);
  p.out = (s == n) ? 0 : (p.in == 1 ? 2 : 1);
  if (!os && n == 2) p.mode = 2;
  if (!os && n == 4) {
    p.slot = s - 1;
    if (s == 4) { p.mode = 2; p.slot = 0; p.rk4 = true; }
  }
  return p;
}

// (W, U) <- (sW, sU) on the ghost cells (ghost) or the interior cells (!ghost).
__global__ void copy_cells_kernel(Blocks B, const double* sW, const double* sU, long long ncell, int ghost) {
  const long long per = (long long)B.NCi * B.NCj;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const long long b = q / per, r = q % per;
    const int i = int(r % B.NCi), j = int(r / B.NCi);
    const bool interior = i >= NG && i < NG + B.nci && j >= NG && j < NG + B.ncj;
    if (interior == bool(ghost)) continue;
    const size_t s = size_t(per);
    const size_t base = size_t(b) * 4 * s + size_t(r);
    for (int v = 0; v < 4; ++v) {
      B.W[base + v * s] = sW[base + v * s];
      B.U[base + v * s] = sU[base + v * s];
    }
  }
}
cudaError_t copy_cells(e2d_handle* h, const double* sW, const double* sU, bool ghost) {
  const int grid = int(std::min<size_t>((h->ncell + 255) / 256, 4096));
  copy_cells_kernel<<<grid, 256, 0, h->stream>>>(h->B, sW, sU, (long long)h->ncell, ghost ? 1 : 0);
  return cudaGetLastError();
}

void stage_buffers(e2d_handle* h, int k, double*& W, double*& U) {
  W = k == 0 ? h->B.W : (k == 1 ? h->B.W2 : h->W3);
  U = k == 0 ? h->B.U : (k == 1 ? h->B.U2 : h->U3);
}

// The stage kernel for a stage: the column-marching kernel where the handle
// allows it (even block width, no degenerate edges) and the autotuner chose
// it, else the tiled stage kernel.
cudaError_t launch_stage_args(e2d_handle* h, StageArgs& a) {
  if (h->march) {
    const bool ex = h->sc.precision == E2D_PREC_FP64_EXACT;
    const CUtensorMap* tw = nullptr;
    if (a.Win == h->B.W) tw = &h->tmW[0];
    else if (a.Win == h->B.W2) tw = &h->tmW[1];
    else if (a.Win == h->W3 && h->W3) tw = &h->tmW[2];
    if (tw) {
      MarchArgs m;
      memset(&m, 0, sizeof(m));
      m.a = a;
      m.tmW = *tw;
      m.tmG = ex ? h->tmGx : h->tmG;
      m.tmN = h->tmN;
      m.geom = ex ? h->geomx : h->geom;
      m.mask = h->gmask;
      m.bcside = h->bcside;
      // update inputs by TMA: explicit stages over U or U2 whose second
      // stage adds to dUdt (RK4's slot combination reads global memory)
      const bool ubase = a.Ubase == h->B.U || a.Ubase == h->B.U2;
      if (h->upd_ok && (a.mode == 1 || a.mode == 2) && !a.no_update && ubase &&
          (a.mode == 1 || (a.res_out == h->B.dUdt && !a.acc1))) {
        m.upd = 1;
        m.tmU = a.Ubase == h->B.U ? h->tmU[0] : h->tmU[1];
        m.tmR = h->tmR;
        m.tmGA = ex ? h->tmGAx : h->tmGA;
        m.tmGF = ex ? h->tmGFx : h->tmGF;
      }
      const int mi = fast::march_strip_cols();
      m.strips = (h->B.nci + mi - 1) / mi;
      m.ch = h->march_rows;
      m.cps = fast::march_chunks(h->B.ncj, m.ch);
      m.nchunk = (long long)m.strips * m.cps * h->B.nblk;
      const int grid = int(std::min<long long>(m.nchunk, h->march_grid));
      if (ex) return exact::launch_march(m, grid, h->stream);
      return h->sc.precision == E2D_PREC_FP32 ? f32::launch_march(m, grid, h->stream)
                                              : fast::launch_march(m, grid, h->stream);
    }
  }
  int ti, tj;
  stage_tile(h->sc.precision, &ti, &tj);
  a.tiles_i = (h->B.nci + ti - 1) / ti;
  a.tiles_j = (h->B.ncj + tj - 1) / tj;
  return launch_stage_prec(h->sc.precision, a, h->stream);
}

// ---- column-marching kernel set-up -------------------------------------------

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

// 3D tensor map of doubles [d2][d1][d0] (rows of d0), box b0 x b1 x b2,
// zero fill outside.
bool encode3(CUtensorMap* map, void* base, uint64_t d0, uint64_t d1, uint64_t d2, uint32_t b0, uint32_t b1,
             uint32_t b2) {
  const EncodeTiled fn = encode_fn();
  if (!fn || !base) return false;
  const cuuint64_t dims[3] = {d0, d1, d2};
  const cuuint64_t strides[2] = {d0 * sizeof(double), d0 * d1 * sizeof(double)};
  const cuuint32_t box[3] = {b0, b1, b2};
  const cuuint32_t es[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Geometry, padded nodes and tensor maps of the marching kernel.  The handle
// keeps the tiled stage kernel when the marching kernel does not apply: an
// odd block width (row strides of the tensor maps must be multiples of 16
// bytes) or a degenerate edge.
int setup_march(e2d_handle* h) {
  h->march = h->march_ok = false;
  const Blocks& B = h->B;
  if (B.NCi % 2 || !encode_fn()) return 0;
  const int mi = fast::march_strip_cols(), wj = fast::march_window_rows();
  const int NNp = B.NNi + 1;  // NNi is odd for an even NCi
  int rc;
  int* degenerate = nullptr;
  if ((rc = dalloc(h, &h->geom, size_t(GEOM_NF) * h->ncell)) || (rc = dalloc(h, &h->geomx, size_t(GEOM_NF) * h->ncell)) ||
      (rc = dalloc(h, &h->gmask, h->ncell)) ||
      (rc = dalloc(h, &h->bcside, B.nblk)) || (rc = dalloc(h, &h->nodes_pad, size_t(B.nblk) * 2 * B.NNj * NNp)) ||
      (rc = dalloc(h, &degenerate, 1)))
    return rc;
  CK(cudaMemsetAsync(degenerate, 0, sizeof(int), h->stream));
  CK(cudaMemsetAsync(h->nodes_pad, 0, sizeof(double) * size_t(B.nblk) * 2 * B.NNj * NNp, h->stream));
  // the exact build's geometry first: the fast one then writes the same mask,
  // side bits and padded nodes again, and both flag degenerate edges
  CK(exact::launch_geometry(B, h->geomx, h->gmask, h->bcside, degenerate, NNp, h->nodes_pad, h->stream));
  CK(fast::launch_geometry(B, h->geom, h->gmask, h->bcside, degenerate, NNp, h->nodes_pad, h->stream));
  int deg = 0;
  CK(cudaMemcpyAsync(&deg, degenerate, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (deg) return 0;
  const uint32_t wi = mi + 4, nwi = mi + 6;
  bool ok = encode3(&h->tmW[0], B.W, B.NCi, B.NCj, 4ull * B.nblk, wi, wj, 4) &&
            encode3(&h->tmW[1], B.W2, B.NCi, B.NCj, 4ull * B.nblk, wi, wj, 4) &&
            encode3(&h->tmG, h->geom, B.NCi, B.NCj, uint64_t(GEOM_NF) * B.nblk, wi, wj, G_K2 + 1) &&
            encode3(&h->tmGx, h->geomx, B.NCi, B.NCj, uint64_t(GEOM_NF) * B.nblk, wi, wj, G_K2 + 1) &&
            encode3(&h->tmN, h->nodes_pad, NNp, B.NNj, 2ull * B.nblk, nwi, wj, 2);
  if (ok && h->W3) ok = encode3(&h->tmW[2], h->W3, B.NCi, B.NCj, 4ull * B.nblk, wi, wj, 4);
  if (!ok) return 0;
  // update inputs of the explicit stages: boxes of the strip's columns x the
  // most rows of a chunk
  const uint32_t mj = fast::march_max_rows();
  h->upd_ok = encode3(&h->tmU[0], B.U, B.NCi, B.NCj, 4ull * B.nblk, mi, mj, 4) &&
              encode3(&h->tmU[1], B.U2, B.NCi, B.NCj, 4ull * B.nblk, mi, mj, 4) &&
              encode3(&h->tmR, B.dUdt, B.NCi, B.NCj, 4ull * B.nblk, mi, mj, 4) &&
              encode3(&h->tmGA, h->geom, B.NCi, B.NCj, uint64_t(GEOM_NF) * B.nblk, mi, mj, 1) &&
              encode3(&h->tmGF, h->geom, B.NCi, B.NCj, uint64_t(GEOM_NF) * B.nblk, mi, mj, GEOM_NF - G_RA) &&
              encode3(&h->tmGAx, h->geomx, B.NCi, B.NCj, uint64_t(GEOM_NF) * B.nblk, mi, mj, 1) &&
              encode3(&h->tmGFx, h->geomx, B.NCi, B.NCj, uint64_t(GEOM_NF) * B.nblk, mi, mj, GEOM_NF - G_RA);
  const int per_sm =
      std::min(std::min(f32::march_ctas_per_sm(), fast::march_ctas_per_sm()), exact::march_ctas_per_sm());
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
  if (per_sm < 1 || sms < 1) return 0;
  h->march_grid = per_sm * sms;
  h->march_ok = true;
  return 0;
}

// ---- stage-kernel autotuner --------------------------------------------------
// The candidates -- the tiled kernel and the marching kernel with 4 to 8
// rows per chunk -- are timed on the handle's own block set (a uniform
// state, an explicit stage 1 per launch, one warm-up and three timed
// launches each) when the handle is created; the fastest is kept.  Choices
// are cached per (block shape, block count, precision, flux function) for
// the process.
struct TuneKey {
  int nci, ncj, nblk, prec, flux;
  bool operator<(const TuneKey& o) const {
    return std::tie(nci, ncj, nblk, prec, flux) < std::tie(o.nci, o.ncj, o.nblk, o.prec, o.flux);
  }
};
struct TuneChoice {
  bool march;
  int rows;
  float us;
};
std::map<TuneKey, TuneChoice> g_tune;
std::mutex g_tune_mutex;

__global__ void uniform_state_kernel(Blocks B, long long ncell) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const long long b = q / ((long long)B.NCi * B.NCj), r = q % ((long long)B.NCi * B.NCj);
    const size_t s = size_t(B.NCi) * B.NCj;
    const size_t base = size_t(b) * 4 * s + size_t(r);
    const PState<double> w{1.0, 0.5, 0.1, 1.0};
    const CState<double> u = U_of_W(w, B.gm1i);
    B.W[base] = w.d; B.W[base + s] = w.u; B.W[base + 2 * s] = w.v; B.W[base + 3 * s] = w.p;
    B.U[base] = u.d; B.U[base + s] = u.mx; B.U[base + 2 * s] = u.my; B.U[base + 3 * s] = u.E;
  }
}

// Tunes one precision into sel_*[prec].
int autotune_precision(e2d_handle* h, int prec) {
  const TuneKey key{h->B.nci, h->B.ncj, h->B.nblk, prec, h->sc.flux};
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      h->sel_march[prec] = it->second.march;
      h->sel_rows[prec] = it->second.rows;
      h->sel_us[prec] = it->second.us;
      return 0;
    }
  }
  const int saved = h->sc.precision;
  h->sc.precision = prec;
  StageArgs a{};
  a.B = h->B;
  a.B.dWdx = a.B.dWdy = a.B.phi = nullptr;
  a.mode = 1;
  a.hist = h->hist;
  a.step = h->step;
  a.Win = h->B.W2;
  a.Ubase = h->B.U2;
  a.Wout = h->B.W;
  a.Uout = h->B.U;
  a.res_out = h->B.dUdt;
  a.omega = 1.0;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  TuneChoice best{true, h->march_rows, 1e30f};
  for (int cand = 0; cand <= 5; ++cand) {  // 0: tiled; 1..5: marching, 4..8 rows
    h->march = cand > 0;
    h->march_rows = cand > 0 ? 3 + cand : h->march_rows;
    if (cand > 0 && h->march_rows > fast::march_max_rows()) continue;
    StageArgs t = a;
    CK(launch_stage_args(h, t));
    CK(cudaEventRecord(e0, h->stream));
    for (int r = 0; r < 3; ++r) {
      t = a;
      CK(launch_stage_args(h, t));
    }
    CK(cudaEventRecord(e1, h->stream));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    const float us = 1000.f * ms / 3.f;
    if (us < best.us) best = TuneChoice{h->march, h->march_rows, us};
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->sc.precision = saved;
  h->sel_march[prec] = best.march;
  h->sel_rows[prec] = best.rows;
  h->sel_us[prec] = best.us;
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune[key] = best;
  return 0;
}

// The kernel of the handle's current precision.
void apply_selection(e2d_handle* h) {
  const int p = h->sc.precision;
  if (!h->march_ok) {
    h->march = false;
    return;
  }
  h->march = h->sel_march[p];
  h->march_rows = h->sel_rows[p];
  h->tune_us = h->sel_us[p];
}

// Every precision is tuned when the handle is created (a handle may switch
// between them, e2d_set_precision) on a uniform state in (W2, U2); the state
// arrays are cleared afterwards.
int autotune_stage(e2d_handle* h) {
  if (!h->march_ok) return 0;
  // "tiled" / "march": one kernel without tuning (tests and comparisons of
  // the two kernels; "march" with its default rows per chunk)
  const char* kind = getenv("CFFC_E2D_STAGE_KERNEL");
  if (kind && (strcmp(kind, "tiled") == 0 || strcmp(kind, "march") == 0)) {
    h->sel_march[0] = h->sel_march[1] = h->sel_march[2] = strcmp(kind, "march") == 0;
    h->sel_rows[0] = h->sel_rows[1] = h->sel_rows[2] = fast::march_chunk_rows();
    apply_selection(h);
    return 0;
  }
  Blocks Bs = h->B;
  Bs.W = h->B.W2;
  Bs.U = h->B.U2;
  const int grid = int(std::min<size_t>((h->ncell + 255) / 256, 4096));
  uniform_state_kernel<<<grid, 256, 0, h->stream>>>(Bs, (long long)h->ncell);
  CK(cudaGetLastError());
  CK(cudaMemsetAsync(h->hist, 0, sizeof(double) * 4 * size_t(h->hist_cap) * h->B.ncase, h->stream));
  int rc;
  if ((rc = autotune_precision(h, E2D_PREC_FP64)) || (rc = autotune_precision(h, E2D_PREC_FP32)) ||
      (rc = autotune_precision(h, E2D_PREC_FP64_EXACT)))
    return rc;
  apply_selection(h);
  // the handle starts from a clean slate
  const size_t nb = sizeof(double) * 4 * h->ncell;
  CK(cudaMemsetAsync(h->B.W, 0, nb, h->stream));
  CK(cudaMemsetAsync(h->B.U, 0, nb, h->stream));
  CK(cudaMemsetAsync(h->B.W2, 0, nb, h->stream));
  CK(cudaMemsetAsync(h->B.U2, 0, nb, h->stream));
  CK(cudaMemsetAsync(h->B.dUdt, 0, nb, h->stream));
  CK(cudaMemsetAsync(h->B.dt, 0, sizeof(double) * h->ncell, h->stream));
  CK(cudaMemsetAsync(h->B.status, 0, sizeof(int) * 2, h->stream));
  if (h->B.phi_keep) CK(cudaMemsetAsync(h->B.phi_keep, 0, nb, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

// Residual (mode 0) or Frechet product (mode 3) of the state (W, U).
cudaError_t launch_stage_any(e2d_handle* h, int mode, int fuse_next) {
  StageArgs a{};
  a.B = h->B;
  a.mode = mode;
  a.fuse_next = fuse_next;
  a.hist = h->hist;
  a.step = h->step;
  a.Win = h->B.W;
  a.Ubase = h->B.U;
  a.Wout = h->B.W;
  a.Uout = h->B.U;
  a.res_out = h->B.dUdt;
  a.omega = 1.0;
  return launch_stage_args(h, a);
}

// Explicit stage s (1-based) of the handle's scheme, per its StagePlan.
cudaError_t launch_explicit_stage(e2d_handle* h, int s, int fuse_next) {
  const StagePlan p = stage_plan(h->sc, s);
  StageArgs a{};
  a.B = h->B;
  a.mode = p.mode;
  a.fuse_next = fuse_next;
  a.hist = h->hist;
  a.step = h->step;
  double *W_in, *U_in;
  stage_buffers(h, p.in, W_in, U_in);
  a.Win = W_in;
  a.Ubase = h->B.U;
  stage_buffers(h, p.out, a.Wout, a.Uout);
  a.omega = p.omega;
  a.res_out = p.slot == 0 ? h->B.dUdt : (p.slot == 1 ? h->R1 : h->R2);
  if (p.rk4) { a.acc1 = h->R1; a.acc2 = h->R2; }
  cudaError_t e = launch_stage_args(h, a);
  // single-stage scheme: the stage's interior result is the new solution
  if (e == cudaSuccess && h->sc.n_stage == 1) e = copy_cells(h, h->B.W2, h->B.U2, false);
  return e;
}

// Ghost fill of the state stage s reads (s = 0: the solution (W, U)).
cudaError_t ghost_fill_for(e2d_handle* h, int s) {
  Blocks B = h->B;
  if (s > 0) stage_buffers(h, stage_plan(h->sc, s).in, B.W, B.U);
  return launch_ghost_fill(B, h->stream);
}

int ensure_recon(e2d_handle* h) {
  if (h->recon_out) return 0;
  int rc;
  if ((rc = dalloc(h, &h->B.dWdx, 4 * h->ncell))) return rc;
  if ((rc = dalloc(h, &h->B.dWdy, 4 * h->ncell))) return rc;
  if ((rc = dalloc(h, &h->B.phi, 4 * h->ncell))) return rc;
  CK(cudaMemsetAsync(h->B.dWdx, 0, sizeof(double) * 4 * h->ncell, h->stream));
  CK(cudaMemsetAsync(h->B.dWdy, 0, sizeof(double) * 4 * h->ncell, h->stream));
  CK(cudaMemsetAsync(h->B.phi, 0, sizeof(double) * 4 * h->ncell, h->stream));
  h->recon_out = true;
  return 0;
}

int ensure_hist(e2d_handle* h, int n) {
  if (n <= h->hist_cap) return 0;
  int cap = n < 64 ? 64 : n;
  double* p = nullptr;
  if (cudaMalloc(&p, sizeof(double) * 4 * size_t(cap) * h->B.ncase) != cudaSuccess) return E2D_ERR_NOMEM;
  if (h->hist) {
    for (auto& q : h->allocs)
      if (q == h->hist) { cudaFree(q); q = p; }
  } else {
    h->allocs.push_back(p);
  }
  h->hist = p;
  h->hist_cap = cap;
  if (h->step_graph) { cudaGraphExecDestroy(h->step_graph); h->step_graph = nullptr; }
  return 0;
}

// CFL + global minimum and the residual norms of the current state into the
// current step's history slot: the head of the reference's explicit step
// (Euler2DQuadSolvers.cc:657-696).  Needed before the first step only; every
// step's last stage computes them for the following step.
cudaError_t enqueue_step_head(e2d_handle* h) {
  cudaError_t e;
  if ((e = launch_slot_init(h->hist, h->step, 0, h->B.ncase, h->stream))) return e;
  if ((e = launch_cfl(h->B, h->hist, h->step, h->stream))) return e;
  return launch_norms(h->B, h->part, h->hist, h->step, h->stream);
}

// The frozen flags ([ncase], cleared), the first-step flag (set) and the
// stored limiters of a scheme with Freeze_Limiter.
int alloc_freeze(e2d_handle* h) {
  if (!h->sc.freeze_limiter) return 0;
  int rc;
  if ((rc = dalloc(h, &h->freeze, size_t(h->B.ncase))) || (rc = dalloc(h, &h->first, 1))) return rc;
  if (!h->B.phi_keep) {
    if ((rc = dalloc(h, &h->B.phi_keep, 4 * h->ncell))) return rc;
    CK(cudaMemset(h->B.phi_keep, 0, sizeof(double) * 4 * h->ncell));
  }
  const int one = 1;
  CK(cudaMemset(h->freeze, 0, sizeof(int) * h->B.ncase));
  CK(cudaMemcpy(h->first, &one, sizeof(int), cudaMemcpyHostToDevice));
  h->B.freeze = h->freeze;
  return 0;
}

// A new initial state starts a new run: limiters unfrozen, first step next.
int reset_run(e2d_handle* h) {
  if (!h->freeze) return 0;
  const int one = 1;
  CK(cudaMemsetAsync(h->freeze, 0, sizeof(int) * h->B.ncase, h->stream));
  CK(cudaMemcpyAsync(h->first, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  return 0;
}

cudaError_t launch_freeze_check(e2d_handle* h) {
  if (!h->freeze) return cudaSuccess;
  freeze_check_kernel<<<1, 32, 0, h->stream>>>(h->hist, h->step, h->B.ncase, h->sc.freeze_level, h->freeze,
                                                h->first);
  return cudaGetLastError();
}

// Stage s with residual smoothing: the stage's residual (no update), the
// Gauss-Seidel smoothing of it, then the update.
cudaError_t launch_smoothed_stage(e2d_handle* h, int s) {
  const StagePlan p = stage_plan(h->sc, s);
  StageArgs a{};
  a.B = h->B;
  a.mode = p.mode;
  a.fuse_next = 0;
  a.hist = h->hist;
  a.step = h->step;
  double *W_in, *U_in, *W_out, *U_out;
  stage_buffers(h, p.in, W_in, U_in);
  stage_buffers(h, p.out, W_out, U_out);
  a.Win = W_in;
  a.Ubase = h->B.U;
  a.Wout = W_out;
  a.Uout = U_out;
  a.omega = p.omega;
  a.res_out = h->B.dUdt;
  a.no_update = 1;
  cudaError_t e = launch_stage_args(h, a);
  if (e != cudaSuccess) return e;
  if (h->smooth_smem)
    residual_smoothing_kernel<true><<<h->B.nblk, SMOOTH_THREADS, h->smooth_smem, h->stream>>>(
        h->B, h->B.dUdt, nullptr, h->sc.rs_epsilon, h->sc.rs_iterations);
  else
    residual_smoothing_kernel<false><<<h->B.nblk, SMOOTH_THREADS, 0, h->stream>>>(
        h->B, h->B.dUdt, h->smooth_scratch, h->sc.rs_epsilon, h->sc.rs_iterations);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  const long long n = (long long)h->B.nblk * h->B.nci * h->B.ncj;
  const int grid = int(std::min<long long>((n + 255) / 256, 4096));
  stage_update_kernel<<<grid, 256, 0, h->stream>>>(h->B, h->B.U, h->B.dUdt, p.omega, W_out, U_out);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (h->sc.n_stage == 1) e = copy_cells(h, h->B.W2, h->B.U2, false);
  return e;
}

// One explicit time step in the reference's order (Euler2DQuadSolvers.cc:657-898):
// limiter-freezing test, then per stage ghost fill + fused residual/update;
// the last stage also reduces the next step's CFL minimum and residual
// norms.  With residual smoothing the stages are split (residual,
// smoothing, update) and every step starts with its own CFL and norms.
cudaError_t enqueue_step(e2d_handle* h) {
  cudaError_t e;
  const bool smooth = h->sc.rs_epsilon > 0.0;
  if (smooth && (e = enqueue_step_head(h))) return e;
  if ((e = launch_slot_init(h->hist, h->step, 1, h->B.ncase, h->stream))) return e;
  if ((e = launch_freeze_check(h))) return e;
  for (int stage = 1; stage <= h->sc.n_stage; ++stage) {
    if ((e = ghost_fill_for(h, stage))) return e;
    if (smooth) {
      if ((e = launch_smoothed_stage(h, stage))) return e;
    } else if ((e = launch_explicit_stage(h, stage, stage == h->sc.n_stage))) {
      return e;
    }
  }
  return launch_step_end(h->hist, h->step, smooth ? 0 : 1, h->B.ncase, h->stream);
}

}  // namespace e2d_host

using namespace e2d_host;

// ---- batches of cases with different block shapes ---------------------------
// One uniform sub-batch per shape (cases grouped in order of first
// appearance); the handle dispatches every call to them and moves each
// case's host arrays between the callers' concatenation (cases in the order
// given, each in its own shape) and the sub-batches' own concatenations.

static e2d_handle* create_mixed_batch(const e2d_blocks_desc* cases, int ncase, const e2d_scheme* sc, int device,
                                      int* err) {
  std::vector<std::vector<int>> groups;
  std::vector<int> group_of(ncase, -1);
  for (int c = 0; c < ncase; ++c) {
    for (size_t g = 0; g < groups.size() && group_of[c] < 0; ++g) {
      const e2d_blocks_desc& r = cases[groups[g][0]];
      if (r.nci == cases[c].nci && r.ncj == cases[c].ncj && r.ng == cases[c].ng) group_of[c] = int(g);
    }
    if (group_of[c] < 0) {
      group_of[c] = int(groups.size());
      groups.emplace_back();
    }
    groups[group_of[c]].push_back(c);
  }
  e2d_handle* h = new e2d_handle;
  h->device = device;
  h->sc = *sc;
  h->B.ncase = ncase;
  h->sub_of.resize(ncase);
  h->local_of.resize(ncase);
  for (size_t g = 0; g < groups.size(); ++g) {
    std::vector<e2d_blocks_desc> d;
    for (size_t k = 0; k < groups[g].size(); ++k) {
      d.push_back(cases[groups[g][k]]);
      h->sub_of[groups[g][k]] = int(g);
      h->local_of[groups[g][k]] = int(k);
    }
    e2d_handle* sub = e2d_create_batch(d.data(), int(d.size()), sc, device, err);
    if (!sub) {
      e2d_destroy(h);
      return nullptr;
    }
    h->subs.push_back(sub);
  }
  size_t o4 = 0, o1 = 0;
  for (int c = 0; c < ncase; ++c) {
    const size_t plane = size_t(cases[c].nci + 2 * cases[c].ng) * (cases[c].ncj + 2 * cases[c].ng);
    h->off4.push_back(o4);
    h->size4.push_back(size_t(cases[c].nblk) * 4 * plane);
    h->off1.push_back(o1);
    h->size1.push_back(size_t(cases[c].nblk) * plane);
    o4 += h->size4.back();
    o1 += h->size1.back();
  }
  return h;
}

namespace e2d_host {

// Cases of sub-batch s in its own order.
static std::vector<int> sub_cases(const e2d_handle* h, int s) {
  std::vector<int> out;
  for (int c = 0; c < int(h->sub_of.size()); ++c)
    if (h->sub_of[c] == s) out.push_back(c);
  return out;
}

// Caller array (per case off/size) -> sub-batch s's concatenation, or back.
static void gather_sub(const e2d_handle* h, int s, const double* all, const std::vector<size_t>& off,
                       const std::vector<size_t>& size, std::vector<double>& out) {
  out.clear();
  for (int c : sub_cases(h, s)) out.insert(out.end(), all + off[c], all + off[c] + size[c]);
}
static void scatter_sub(const e2d_handle* h, int s, const std::vector<double>& in, const std::vector<size_t>& off,
                        const std::vector<size_t>& size, double* all) {
  size_t q = 0;
  for (int c : sub_cases(h, s)) {
    std::copy(in.begin() + q, in.begin() + q + size[c], all + off[c]);
    q += size[c];
  }
}
static size_t sub_total(const e2d_handle* h, int s, const std::vector<size_t>& size) {
  size_t t = 0;
  for (int c : sub_cases(h, s)) t += size[c];
  return t;
}

// Newton-Krylov over the sub-batches, one after another: per-case reference
// levels go to each sub-batch, histories ([case][max_newton]) and step
// counts come back to the caller's case order.
int composite_nks(e2d_handle* h, const e2d_nks_params* p, e2d_nks_step* hist, int* n_steps) {
  const int m = std::max(p->max_newton, 1);
  int rc = 0;
  for (int s = 0; s < int(h->subs.size()); ++s) {
    const std::vector<int> cs = sub_cases(h, s);
    e2d_nks_params q = *p;
    std::vector<double> l2, cfl;
    for (int c : cs) {
      if (p->l2_reference) l2.push_back(p->l2_reference[c]);
      if (p->cfl_reference) cfl.push_back(p->cfl_reference[c]);
    }
    q.l2_reference = p->l2_reference ? l2.data() : nullptr;
    q.cfl_reference = p->cfl_reference ? cfl.data() : nullptr;
    std::vector<e2d_nks_step> hs(size_t(m) * cs.size());
    std::vector<int> ns(cs.size(), 0);
    const int r = e2d_nks(h->subs[s], &q, hist ? hs.data() : nullptr, ns.data());
    if (r < 0) return r;
    if (r > 0 && rc == 0) rc = r;
    for (size_t k = 0; k < cs.size(); ++k) {
      if (n_steps) n_steps[cs[k]] = ns[k];
      if (hist) std::copy(hs.begin() + k * m, hs.begin() + (k + 1) * m, hist + size_t(cs[k]) * m);
    }
  }
  return rc;
}

}  // namespace e2d_host

extern "C" {

e2d_handle* e2d_create(const e2d_blocks_desc* d, const e2d_scheme* sc, int device, int* err) {
  auto fail = [&](int code, e2d_handle* h) -> e2d_handle* {
    if (err) *err = code;
    if (h) e2d_destroy(h);
    return nullptr;
  };
  if (err) *err = 0;
  if (!d || !sc || d->nblk < 1 || d->nci < 2 || d->ncj < 2 || d->ng != NG) return fail(E2D_ERR_ARG, nullptr);
  if (!scheme_supported(sc)) return fail(E2D_ERR_ARG, nullptr);
  // residual smoothing keeps its scratch in the reference's residual slot
  // k_residual+1, which RK4's stages occupy: not a combination to run
  if (sc->rs_epsilon > 0.0 && (sc->rs_iterations < 0 || stage_plan(*sc, sc->n_stage).rk4))
    return fail(E2D_ERR_ARG, nullptr);
  if (!e2d_flux_supported(sc->flux)) return fail(E2D_ERR_ARG, nullptr);
  if (sc->precision != E2D_PREC_FP64 && sc->precision != E2D_PREC_FP64_EXACT && sc->precision != E2D_PREC_FP32)
    return fail(E2D_ERR_ARG, nullptr);
  if (sc->limiter != E2D_LIMITER_VENKATAKRISHNAN && sc->limiter != E2D_LIMITER_BARTH_JESPERSEN &&
      sc->limiter != E2D_LIMITER_ONE && sc->limiter != E2D_LIMITER_ZERO)
    return fail(E2D_ERR_ARG, nullptr);
  const int NCi = d->nci + 2 * NG, NCj = d->ncj + 2 * NG;
  // Supported BC codes only (others would need reference code paths not built here).
  auto bc_ok = [](const int32_t* a, size_t n) {
    for (size_t q = 0; q < n; ++q) {
      const int c = a[q];
      if (c != E2D_BC_NONE && c != E2D_BC_CONSTANT_EXTRAPOLATION && c != E2D_BC_PERIODIC &&
          c != E2D_BC_REFLECTION && c != E2D_BC_CHARACTERISTIC && c != E2D_BC_FIXED)
        return false;
    }
    return true;
  };
  if (!bc_ok(d->bc_w, size_t(d->nblk) * NCj) || !bc_ok(d->bc_e, size_t(d->nblk) * NCj) ||
      !bc_ok(d->bc_s, size_t(d->nblk) * NCi) || !bc_ok(d->bc_n, size_t(d->nblk) * NCi))
    return fail(E2D_ERR_ARG, nullptr);
  for (int q = 0; q < 8 * d->nblk; ++q)
    if (d->neighbour[q] < -1 || d->neighbour[q] >= d->nblk) return fail(E2D_ERR_ARG, nullptr);
  if (cudaSetDevice(device) != cudaSuccess) return fail(E2D_ERR_CUDA, nullptr);

  e2d_handle* h = new e2d_handle;
  h->device = device;
  h->sc = *sc;
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) return fail(E2D_ERR_CUDA, h);
  h->stream = h->own_stream;
  Blocks& B = h->B;
  B.nblk = d->nblk; B.nci = d->nci; B.ncj = d->ncj;
  B.NCi = NCi; B.NCj = NCj; B.NNi = NCi + 1; B.NNj = NCj + 1;
  h->ncell = size_t(B.nblk) * NCi * NCj;
  h->nnode = size_t(B.nblk) * B.NNi * B.NNj;
  B.g = sc->gamma; B.gm1 = B.g - 1.0; B.gm1i = 1.0 / B.gm1;
  B.cfl = sc->cfl; B.limiter = sc->limiter; B.flux = sc->flux; B.n_stage = sc->n_stage; B.local_dt = sc->local_dt;
  B.case_of = nullptr; B.case_start = nullptr; B.ncase = 1; B.case_active = nullptr;
  int rc = 0;
  int *neigh, *bcw, *bce, *bcs, *bcn;
  double *X, *Y, *wow, *woe, *wos, *won;
  if ((rc = upload(h, &neigh, d->neighbour, size_t(8) * B.nblk)) ||
      (rc = upload(h, &bcw, d->bc_w, size_t(B.nblk) * NCj)) || (rc = upload(h, &bce, d->bc_e, size_t(B.nblk) * NCj)) ||
      (rc = upload(h, &bcs, d->bc_s, size_t(B.nblk) * NCi)) || (rc = upload(h, &bcn, d->bc_n, size_t(B.nblk) * NCi)) ||
      (rc = upload(h, &X, d->node_x, h->nnode)) || (rc = upload(h, &Y, d->node_y, h->nnode)) ||
      (rc = upload(h, &wow, d->wo_w, size_t(B.nblk) * 4 * NCj)) ||
      (rc = upload(h, &woe, d->wo_e, size_t(B.nblk) * 4 * NCj)) ||
      (rc = upload(h, &wos, d->wo_s, size_t(B.nblk) * 4 * NCi)) ||
      (rc = upload(h, &won, d->wo_n, size_t(B.nblk) * 4 * NCi)))
    return fail(rc, h);
  B.neigh = neigh; B.bcw = bcw; B.bce = bce; B.bcs = bcs; B.bcn = bcn;
  B.X = X; B.Y = Y; B.wow = wow; B.woe = woe; B.wos = wos; B.won = won;
  if ((rc = dalloc(h, &B.W, 4 * h->ncell)) || (rc = dalloc(h, &B.U, 4 * h->ncell)) ||
      (rc = dalloc(h, &B.W2, 4 * h->ncell)) || (rc = dalloc(h, &B.U2, 4 * h->ncell)) ||
      (rc = dalloc(h, &B.dUdt, 4 * h->ncell)) ||
      (rc = dalloc(h, &B.dt, h->ncell)) || (rc = dalloc(h, &B.status, 2)) ||
      (rc = dalloc(h, &h->step, 1)) || (rc = dalloc(h, &h->part, size_t(3) * B.nblk)))
    return fail(rc, h);
  if (cudaMemset(B.W, 0, sizeof(double) * 4 * h->ncell) || cudaMemset(B.U, 0, sizeof(double) * 4 * h->ncell) ||
      cudaMemset(B.W2, 0, sizeof(double) * 4 * h->ncell) ||
      cudaMemset(B.U2, 0, sizeof(double) * 4 * h->ncell) || cudaMemset(B.dUdt, 0, sizeof(double) * 4 * h->ncell) ||
      cudaMemset(B.dt, 0, sizeof(double) * h->ncell) || cudaMemset(B.status, 0, sizeof(int) * 2) ||
      cudaMemset(h->step, 0, sizeof(int)))
    return fail(E2D_ERR_CUDA, h);
  if (sc->n_stage >= 3) {
    if ((rc = dalloc(h, &h->W3, 4 * h->ncell)) || (rc = dalloc(h, &h->U3, 4 * h->ncell))) return fail(rc, h);
    if (cudaMemset(h->W3, 0, sizeof(double) * 4 * h->ncell) || cudaMemset(h->U3, 0, sizeof(double) * 4 * h->ncell))
      return fail(E2D_ERR_CUDA, h);
  }
  if (stage_plan(*sc, sc->n_stage).rk4) {
    if ((rc = dalloc(h, &h->R1, 4 * h->ncell)) || (rc = dalloc(h, &h->R2, 4 * h->ncell))) return fail(rc, h);
    if (cudaMemset(h->R1, 0, sizeof(double) * 4 * h->ncell) || cudaMemset(h->R2, 0, sizeof(double) * 4 * h->ncell))
      return fail(E2D_ERR_CUDA, h);
  }
  if (sc->rs_epsilon > 0.0) {
    // the smoothing region and its zero ring, [4][ncj][nci] doubles per block,
    // in shared memory when it fits
    const size_t bytes = sizeof(double) * 4 * size_t(d->nci) * d->ncj;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (bytes <= size_t(max_smem) &&
        cudaFuncSetAttribute(residual_smoothing_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(bytes)) == cudaSuccess) {
      h->smooth_smem = bytes;
    } else {
      cudaGetLastError();
      if ((rc = dalloc(h, &h->smooth_scratch, 4 * size_t(d->nci) * d->ncj * B.nblk))) return fail(rc, h);
    }
  }
  if ((rc = alloc_freeze(h))) return fail(rc, h);
  if ((rc = ensure_hist(h, 64))) return fail(rc, h);
  B.dWdx = B.dWdy = B.phi = nullptr;
  if ((rc = setup_march(h)) || (rc = autotune_stage(h))) return fail(rc, h);
  return h;
}

e2d_handle* e2d_create_batch(const e2d_blocks_desc* cases, int ncase, const e2d_scheme* sc, int device, int* err) {
  if (err) *err = 0;
  if (!cases || ncase < 1 || !sc) {
    if (err) *err = E2D_ERR_ARG;
    return nullptr;
  }
  const int nci = cases[0].nci, ncj = cases[0].ncj, ng = cases[0].ng;
  int nblk = 0;
  for (int c = 0; c < ncase; ++c) {
    if (cases[c].nblk < 1) {
      if (err) *err = E2D_ERR_ARG;
      return nullptr;
    }
    if (cases[c].nci != nci || cases[c].ncj != ncj || cases[c].ng != ng)
      return create_mixed_batch(cases, ncase, sc, device, err);
    nblk += cases[c].nblk;
  }
  const size_t NCi = nci + 2 * ng, NCj = ncj + 2 * ng, NN = (NCi + 1) * (NCj + 1);
  std::vector<int32_t> nb, bcw, bce, bcs, bcn, case_of, case_start(1, 0);
  std::vector<double> X, Y, wow, woe, wos, won;
  auto app = [](auto& v, const auto* p, size_t n) { v.insert(v.end(), p, p + n); };
  for (int c = 0; c < ncase; ++c) {
    const e2d_blocks_desc& d = cases[c];
    const int b0 = case_start.back();
    for (int q = 0; q < 8 * d.nblk; ++q) {
      const int v = d.neighbour[q];
      if (v < -1 || v >= d.nblk) {
        if (err) *err = E2D_ERR_ARG;
        return nullptr;
      }
      nb.push_back(v < 0 ? -1 : v + b0);  // neighbours never cross cases
    }
    app(bcw, d.bc_w, d.nblk * NCj); app(bce, d.bc_e, d.nblk * NCj);
    app(bcs, d.bc_s, d.nblk * NCi); app(bcn, d.bc_n, d.nblk * NCi);
    app(X, d.node_x, d.nblk * NN); app(Y, d.node_y, d.nblk * NN);
    app(wow, d.wo_w, d.nblk * 4 * NCj); app(woe, d.wo_e, d.nblk * 4 * NCj);
    app(wos, d.wo_s, d.nblk * 4 * NCi); app(won, d.wo_n, d.nblk * 4 * NCi);
    for (int b = 0; b < d.nblk; ++b) case_of.push_back(c);
    case_start.push_back(b0 + d.nblk);
  }
  e2d_blocks_desc all = cases[0];
  all.nblk = nblk;
  all.neighbour = nb.data();
  all.bc_w = bcw.data(); all.bc_e = bce.data(); all.bc_s = bcs.data(); all.bc_n = bcn.data();
  all.node_x = X.data(); all.node_y = Y.data();
  all.wo_w = wow.data(); all.wo_e = woe.data(); all.wo_s = wos.data(); all.wo_n = won.data();
  e2d_handle* h = e2d_create(&all, sc, device, err);
  if (!h) return nullptr;
  int* dcase = nullptr;
  int* dstart = nullptr;
  int rc;
  if ((rc = upload(h, &dcase, case_of.data(), case_of.size())) ||
      (rc = upload(h, &dstart, case_start.data(), case_start.size()))) {
    if (err) *err = rc;
    e2d_destroy(h);
    return nullptr;
  }
  h->B.case_of = dcase;
  h->B.case_start = dstart;
  h->B.ncase = ncase;
  // the step history holds one slot per case and step
  const int cap = h->hist_cap;
  h->hist_cap = 0;
  if ((rc = ensure_hist(h, cap)) || (rc = alloc_freeze(h))) {
    if (err) *err = rc;
    e2d_destroy(h);
    return nullptr;
  }
  return h;
}

int e2d_batch_cases(e2d_handle* h) { return h ? h->B.ncase : E2D_ERR_ARG; }

void e2d_destroy(e2d_handle* h) {
  if (!h) return;
  if (!h->subs.empty()) {
    for (e2d_handle* s : h->subs) e2d_destroy(s);
    delete h;
    return;
  }
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->step_graph) cudaGraphExecDestroy(h->step_graph);
  nks_free(h);
  for (void* p : h->allocs) cudaFree(p);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

// U = U(W) for every cell (Euler2D_pState::U, Euler2DState.h:1748).
__global__ void u_of_w_kernel(Blocks B, long long ncell) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const long long b = q / ((long long)B.NCi * B.NCj), r = q % ((long long)B.NCi * B.NCj);
    const size_t s = size_t(B.NCi) * B.NCj;
    const size_t base = size_t(b) * 4 * s + size_t(r);
    PState<double> w{B.W[base], B.W[base + s], B.W[base + 2 * s], B.W[base + 3 * s]};
    const CState<double> u = U_of_W(w, B.gm1i);
    B.U[base] = u.d; B.U[base + s] = u.mx; B.U[base + 2 * s] = u.my; B.U[base + 3 * s] = u.E;
  }
}

// The stage buffers (W2, U2) and (W3, U3) take the whole state, ghost cells
// included: a ghost cell that neither an exchange nor a BC fills (an edge
// with BC_NONE and no neighbour) keeps its value in the reference's single
// state array, so it must hold it in every buffer a stage reads.
static int mirror_stage_buffers(e2d_handle* h) {
  const size_t n = sizeof(double) * 4 * h->ncell;
  CK(cudaMemcpyAsync(h->B.W2, h->B.W, n, cudaMemcpyDeviceToDevice, h->stream));
  CK(cudaMemcpyAsync(h->B.U2, h->B.U, n, cudaMemcpyDeviceToDevice, h->stream));
  if (h->W3) {
    CK(cudaMemcpyAsync(h->W3, h->B.W, n, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->U3, h->B.U, n, cudaMemcpyDeviceToDevice, h->stream));
  }
  return 0;
}

int e2d_set_state(e2d_handle* h, const double* W) {
  if (!h || !W) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    std::vector<double> t;
    for (int s = 0; s < int(h->subs.size()); ++s) {
      gather_sub(h, s, W, h->off4, h->size4, t);
      if (int rc = e2d_set_state(h->subs[s], t.data())) return rc;
    }
    return 0;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->B.W, W, sizeof(double) * 4 * h->ncell, cudaMemcpyHostToDevice, h->stream));
  int grid = int((h->ncell + 255) / 256);
  if (grid > 4096) grid = 4096;
  u_of_w_kernel<<<grid, 256, 0, h->stream>>>(h->B, (long long)h->ncell);
  CK(cudaGetLastError());
  if (int rc = mirror_stage_buffers(h)) return rc;
  CK(cudaMemsetAsync(h->B.status, 0, sizeof(int) * 2, h->stream));
  if (int rc = reset_run(h)) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

// W = W(U) for every cell (Euler2D_cState::W, Euler2DState.h:1741; the
// state a restart file's U gives, Euler2DQuad.h:1359-1362).
__global__ void w_of_u_kernel(Blocks B, long long ncell) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ncell; q += (long long)gridDim.x * blockDim.x) {
    const long long b = q / ((long long)B.NCi * B.NCj), r = q % ((long long)B.NCi * B.NCj);
    const size_t s = size_t(B.NCi) * B.NCj;
    const size_t base = size_t(b) * 4 * s + size_t(r);
    CState<double> u{B.U[base], B.U[base + s], B.U[base + 2 * s], B.U[base + 3 * s]};
    const PState<double> w = W_of_U(u, B.gm1);
    B.W[base] = w.d; B.W[base + s] = w.u; B.W[base + 2 * s] = w.v; B.W[base + 3 * s] = w.p;
  }
}

int e2d_set_conserved(e2d_handle* h, const double* U) {
  if (!h || !U) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    std::vector<double> t;
    for (int s = 0; s < int(h->subs.size()); ++s) {
      gather_sub(h, s, U, h->off4, h->size4, t);
      if (int rc = e2d_set_conserved(h->subs[s], t.data())) return rc;
    }
    return 0;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaMemcpyAsync(h->B.U, U, sizeof(double) * 4 * h->ncell, cudaMemcpyHostToDevice, h->stream));
  int grid = int((h->ncell + 255) / 256);
  if (grid > 4096) grid = 4096;
  w_of_u_kernel<<<grid, 256, 0, h->stream>>>(h->B, (long long)h->ncell);
  CK(cudaGetLastError());
  if (int rc = mirror_stage_buffers(h)) return rc;
  CK(cudaMemsetAsync(h->B.status, 0, sizeof(int) * 2, h->stream));
  if (int rc = reset_run(h)) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int e2d_get_state(e2d_handle* h, double* W, double* U) {
  if (!h) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    for (int s = 0; s < int(h->subs.size()); ++s) {
      const size_t n = sub_total(h, s, h->size4);
      std::vector<double> w(W ? n : 0), u(U ? n : 0);
      if (int rc = e2d_get_state(h->subs[s], W ? w.data() : nullptr, U ? u.data() : nullptr)) return rc;
      if (W) scatter_sub(h, s, w, h->off4, h->size4, W);
      if (U) scatter_sub(h, s, u, h->off4, h->size4, U);
    }
    return 0;
  }
  CK(cudaSetDevice(h->device));
  if (W) CK(cudaMemcpyAsync(W, h->B.W, sizeof(double) * 4 * h->ncell, cudaMemcpyDeviceToHost, h->stream));
  if (U) CK(cudaMemcpyAsync(U, h->B.U, sizeof(double) * 4 * h->ncell, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int e2d_fill_ghosts(e2d_handle* h) {
  if (!h) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    for (e2d_handle* s : h->subs)
      if (int rc = e2d_fill_ghosts(s)) return rc;
    return 0;
  }
  CK(cudaSetDevice(h->device));
  CK(launch_ghost_fill(h->B, h->stream));
  return check_status(h);
}

int e2d_residual(e2d_handle* h, double* dUdt) {
  if (!h) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    int rc = 0;
    for (int s = 0; s < int(h->subs.size()); ++s) {
      std::vector<double> r(dUdt ? sub_total(h, s, h->size4) : 0);
      const int q = e2d_residual(h->subs[s], dUdt ? r.data() : nullptr);
      if (q < 0) return q;
      if (q > 0 && rc == 0) rc = q;
      if (dUdt) scatter_sub(h, s, r, h->off4, h->size4, dUdt);
    }
    return rc;
  }
  CK(cudaSetDevice(h->device));
  int rc = ensure_recon(h);
  if (rc) return rc;
  CK(launch_ghost_fill(h->B, h->stream));
  CK(launch_stage_any(h, 0, 0));
  if (dUdt) CK(cudaMemcpyAsync(dUdt, h->B.dUdt, sizeof(double) * 4 * h->ncell, cudaMemcpyDeviceToHost, h->stream));
  return check_status(h);
}

int e2d_get_reconstruction(e2d_handle* h, double* dWdx, double* dWdy, double* phi) {
  if (!h || !h->subs.empty()) return E2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int rc = ensure_recon(h);
  if (rc) return rc;
  const size_t n = sizeof(double) * 4 * h->ncell;
  if (dWdx) CK(cudaMemcpyAsync(dWdx, h->B.dWdx, n, cudaMemcpyDeviceToHost, h->stream));
  if (dWdy) CK(cudaMemcpyAsync(dWdy, h->B.dWdy, n, cudaMemcpyDeviceToHost, h->stream));
  if (phi) CK(cudaMemcpyAsync(phi, h->B.phi, n, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return 0;
}

int e2d_rk_steps(e2d_handle* h, int n_steps, double* hist) {
  if (!h || n_steps < 0) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    const int C = h->B.ncase;
    int rc = 0;
    for (int s = 0; s < int(h->subs.size()); ++s) {
      const std::vector<int> cs = sub_cases(h, s);
      std::vector<double> hs(hist ? size_t(n_steps) * cs.size() * 4 : 0);
      const int q = e2d_rk_steps(h->subs[s], n_steps, hist ? hs.data() : nullptr);
      if (q < 0) return q;
      if (q > 0 && rc == 0) rc = q;
      if (hist)
        for (int t = 0; t < n_steps; ++t)
          for (size_t k = 0; k < cs.size(); ++k)
            for (int f = 0; f < 4; ++f)
              hist[(size_t(t) * C + cs[k]) * 4 + f] = hs[(size_t(t) * cs.size() + k) * 4 + f];
    }
    return rc;
  }
  if (n_steps == 0) return 0;
  CK(cudaSetDevice(h->device));
  int rc = ensure_hist(h, n_steps + 1);  // the last step fills slot n_steps
  if (rc) return rc;
  // the stage kernels do not write the optional reconstruction arrays
  const Blocks saved = h->B;
  h->B.dWdx = h->B.dWdy = h->B.phi = nullptr;
  CK(cudaMemsetAsync(h->step, 0, sizeof(int), h->stream));
  CK(enqueue_step_head(h));
  if (!h->step_graph) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_step(h);
    cudaError_t e2 = cudaStreamEndCapture(h->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      h->B = saved;
      fprintf(stderr, "cffc_e2d: step capture failed: %s\n", cudaGetErrorString(e ? e : e2));
      return E2D_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&h->step_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { h->B = saved; h->step_graph = nullptr; return E2D_ERR_CUDA; }
  }
  h->B = saved;
  for (int s = 0; s < n_steps; ++s) CK(cudaGraphLaunch(h->step_graph, h->stream));
  if (h->sc.n_stage >= 2) {
    // The reference keeps one state array, so after a multistage step its
    // ghost cells hold the last stage's exchange and BCs; here those went
    // to the buffer that stage read.  Copy them so the final state matches
    // the reference's in every cell (what a restart file records).
    double *W, *U;
    stage_buffers(h, stage_plan(h->sc, h->sc.n_stage).in, W, U);
    CK(copy_cells(h, W, U, true));
  }
  if (hist)
    CK(cudaMemcpyAsync(hist, h->hist, sizeof(double) * 4 * size_t(n_steps) * h->B.ncase, cudaMemcpyDeviceToHost,
                       h->stream));
  return check_status(h);
}

int e2d_norms(e2d_handle* h, double* out) {
  if (!h || !out) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    for (int s = 0; s < int(h->subs.size()); ++s) {
      const std::vector<int> cs = sub_cases(h, s);
      std::vector<double> o(3 * cs.size());
      if (int rc = e2d_norms(h->subs[s], o.data())) return rc;
      for (size_t k = 0; k < cs.size(); ++k)
        for (int f = 0; f < 3; ++f) out[3 * size_t(cs[k]) + f] = o[3 * k + f];
    }
    return 0;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaMemsetAsync(h->step, 0, sizeof(int), h->stream));
  CK(launch_norms(h->B, h->part, h->hist, h->step, h->stream));
  std::vector<double> tmp(4 * size_t(h->B.ncase));
  CK(cudaMemcpyAsync(tmp.data(), h->hist, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  for (int c = 0; c < h->B.ncase; ++c)
    for (int k = 0; k < 3; ++k) out[3 * c + k] = tmp[4 * c + 1 + k];
  return 0;
}

int e2d_cfl(e2d_handle* h, double* dt, double* dtmin) {
  if (!h) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    for (int s = 0; s < int(h->subs.size()); ++s) {
      const std::vector<int> cs = sub_cases(h, s);
      std::vector<double> d(dt ? sub_total(h, s, h->size1) : 0), m(cs.size());
      if (int rc = e2d_cfl(h->subs[s], dt ? d.data() : nullptr, m.data())) return rc;
      if (dt) scatter_sub(h, s, d, h->off1, h->size1, dt);
      if (dtmin)
        for (size_t k = 0; k < cs.size(); ++k) dtmin[cs[k]] = m[k];
    }
    return 0;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaMemsetAsync(h->step, 0, sizeof(int), h->stream));
  CK(launch_slot_init(h->hist, h->step, 0, h->B.ncase, h->stream));
  Blocks B = h->B;
  B.local_dt = 1;  // every interior cell's step into B.dt
  CK(launch_cfl(B, h->hist, h->step, h->stream));
  std::vector<double> tmp(4 * size_t(h->B.ncase));
  CK(cudaMemcpyAsync(tmp.data(), h->hist, sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost, h->stream));
  if (dt) CK(cudaMemcpyAsync(dt, h->B.dt, sizeof(double) * h->ncell, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (dtmin)
    for (int c = 0; c < h->B.ncase; ++c) dtmin[c] = tmp[4 * c];
  return 0;
}

int e2d_set_precision(e2d_handle* h, int precision) {
  if (!h || (precision != E2D_PREC_FP64 && precision != E2D_PREC_FP32 && precision != E2D_PREC_FP64_EXACT))
    return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    for (e2d_handle* s : h->subs)
      if (int rc = e2d_set_precision(s, precision)) return rc;
    h->sc.precision = precision;
    return 0;
  }
  if (precision == h->sc.precision) return 0;
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  h->sc.precision = precision;
  apply_selection(h);
  // captured launches hold the previous precision's kernels
  if (h->step_graph) {
    cudaGraphExecDestroy(h->step_graph);
    h->step_graph = nullptr;
  }
  nks_drop_graphs(h);
  return 0;
}

int e2d_stage_config(e2d_handle* h, int* kernel, int* rows, double* us) {
  if (!h) return E2D_ERR_ARG;
  if (!h->subs.empty()) return e2d_stage_config(h->subs[0], kernel, rows, us);  // the first shape's
  if (kernel) *kernel = h->march ? 1 : 0;
  if (rows) *rows = h->march ? h->march_rows : 0;
  if (us) *us = h->tune_us;
  return 0;
}

int e2d_status(e2d_handle* h) {
  if (!h) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    for (e2d_handle* s : h->subs)
      if (int rc = e2d_status(s)) return rc;
    return 0;
  }
  return check_status(h);
}

int e2d_device_state(e2d_handle* h, double** W, double** U, double** dUdt) {
  if (!h || !h->subs.empty()) return E2D_ERR_ARG;
  if (W) *W = h->B.W;
  if (U) *U = h->B.U;
  if (dUdt) *dUdt = h->B.dUdt;
  return 0;
}

int e2d_set_stream(e2d_handle* h, void* stream) {
  if (!h) return E2D_ERR_ARG;
  if (!h->subs.empty()) {
    for (e2d_handle* s : h->subs)
      if (int rc = e2d_set_stream(s, stream)) return rc;
    return 0;
  }
  CK(cudaSetDevice(h->device));
  CK(cudaStreamSynchronize(h->stream));
  if (!h->own_stream) {
    CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
  }
  h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
  return 0;
}

int e2d_kernel_times(e2d_handle* h, int n_steps, double out[6]) {
  if (!h || !out || n_steps < 1 || !h->subs.empty()) return E2D_ERR_ARG;
  CK(cudaSetDevice(h->device));
  int rc = ensure_hist(h, n_steps + 1);
  if (rc) return rc;
  const Blocks saved = h->B;
  h->B.dWdx = h->B.dWdy = h->B.phi = nullptr;
  cudaEvent_t ev[10];
  for (auto& e : ev) CK(cudaEventCreate(&e));
  double acc[6] = {0, 0, 0, 0, 0, 0};
  CK(cudaMemsetAsync(h->step, 0, sizeof(int), h->stream));
  for (int s = 0; s < n_steps; ++s) {
    // the standalone CFL and norm kernels run before the first step only in
    // e2d_rk_steps; they are timed on every step here for the record
    CK(cudaEventRecord(ev[0], h->stream));
    CK(launch_slot_init(h->hist, h->step, 0, h->B.ncase, h->stream));
    CK(launch_cfl(h->B, h->hist, h->step, h->stream));
    CK(cudaEventRecord(ev[1], h->stream));
    CK(launch_norms(h->B, h->part, h->hist, h->step, h->stream));
    CK(cudaEventRecord(ev[2], h->stream));
    CK(launch_slot_init(h->hist, h->step, 1, h->B.ncase, h->stream));
    CK(ghost_fill_for(h, 1));
    CK(cudaEventRecord(ev[3], h->stream));
    CK(launch_explicit_stage(h, 1, h->sc.n_stage == 1));
    CK(cudaEventRecord(ev[4], h->stream));
    if (h->sc.n_stage == 2) {
      CK(ghost_fill_for(h, 2));
      CK(cudaEventRecord(ev[5], h->stream));
      CK(launch_explicit_stage(h, 2, 1));
      CK(cudaEventRecord(ev[6], h->stream));
    }
    CK(launch_step_end(h->hist, h->step, 1, h->B.ncase, h->stream));
    CK(cudaEventRecord(ev[7], h->stream));
    CK(cudaEventSynchronize(ev[7]));
    float t[8] = {0};
    for (int k = 1; k <= 7; ++k)
      if (h->sc.n_stage == 2 || (k != 5 && k != 6)) CK(cudaEventElapsedTime(&t[k], ev[0], ev[k]));
    acc[3] += t[1];
    acc[4] += t[2] - t[1];
    acc[0] += t[3] - t[2];
    acc[1] += t[4] - t[3];
    if (h->sc.n_stage == 2) {
      acc[0] += t[5] - t[4];
      acc[2] += t[6] - t[5];
    }
    acc[5] += t[7];
  }
  for (auto& e : ev) cudaEventDestroy(e);
  h->B = saved;
  const double gf = h->sc.n_stage == 2 ? 2.0 * n_steps : double(n_steps);
  out[0] = acc[0] / gf;
  for (int k = 1; k < 6; ++k) out[k] = acc[k] / n_steps;
  return check_status(h);
}

}  // extern "C"
