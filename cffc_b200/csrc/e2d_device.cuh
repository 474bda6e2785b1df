// e2d_device.cuh — device-side state layout and the Euler2D physics of the
// CFFC reference, restated for sm_100a.
//
// Physics functions keep the reference's floating-point operation order
// (Euler2D_pState / cState / Vector2D operators evaluate component-wise, left
// to right).  Compiled with -fmad=false (the "exact" kernels) they reproduce
// the reference's FP64 results bit for bit: CUDA's double division and
// square root are IEEE round-to-nearest, as the reference's x86-64 SSE2 code
// is.  Compiled with contraction on (the "fast" kernels) they differ from it
// only by FMA rounding.
//
// Reference sources (paths relative to the CFFC tree):
//   state algebra           src_2D/Euler2D/Euler2DState.h:1033-1110, 1741-1860
//   RoeAverage, FluxRoe_x/n  src_2D/Euler2D/Euler2DState.cc:654-685, 2311-2495
//   lambda_x, rc_x, lp_x     src_2D/Euler2D/Euler2DState.h:2153, 2702, 2968
//   HartenFixPos/Neg         src_2D/CFD/CFD.cc:605-646
//   Limiters                 src_2D/CFD/CFD.cc:696-751
//   Reflect                  src_2D/Euler2D/Euler2DState.cc:751-787
//   BC_Characteristic_Pressure src_2D/Euler2D/Euler2DState.cc:1383-1450
//   quadCentroid             src_2D/Math/Math.h:311-351
#pragma once
#include <cstdint>

#include "../../include/cffc_e2d.h"

namespace e2d {

constexpr int NG = 2;  // ghost layers (Euler2D_Quad_Block::allocate asserts Ng > 1)
constexpr double HALF = 0.5;
constexpr double TOLER = 0.0000001;  // src_2D/Math/Math.h:52
constexpr double NANO = 0.000000001; // src_2D/Math/Math.h:53

// Status word codes recorded by kernels (first error wins).
constexpr int ST_OK = 0;
constexpr int ST_NEGATIVE = 1;  // non-positive density/energy: value = 1 + cell index

// Everything a kernel needs about the resident block set.  Cell arrays are
// [nblk][4][NCj][NCi] (SoA per variable, rows of i), node arrays
// [nblk][NNj][NNi], per-cell scalars [nblk][NCj][NCi].
struct Blocks {
  int nblk, nci, ncj, NCi, NCj, NNi, NNj;
  const int* neigh;                // [nblk][8]  W E S N SW SE NW NE
  const int *bcw, *bce, *bcs, *bcn;
  const double *X, *Y;             // nodes
  const double *wow, *woe, *wos, *won;
  double *W, *U, *dUdt;            // cell state (the solution lives in W, U)
  double *W2, *U2;                 // intermediate RK stage state
  double *dWdx, *dWdy, *phi;       // optional reconstruction output (may be null)
  double* dt;                      // local time step per cell (local dt only)
  int* status;                     // device status word (2 ints: code, cell)
  double g, gm1, gm1i, cfl;
  int limiter, n_stage, local_dt;
  // Batches of independent cases: the blocks of case c are
  // case_start[c] .. case_start[c+1]-1 and case_of[b] names the case of block b
  // (null for a single case).  Per-case quantities (time-step minimum, residual
  // norms) live in slot (step, case) of the step history: hist + 4*(step*ncase + case).
  const int* case_of;
  const int* case_start;
  int ncase;
  const int* case_active;  // per case, null = all: residual/JVP stages skip inactive cases
};

__host__ __device__ inline int case_id(const Blocks& B, int b) { return B.case_of ? B.case_of[b] : 0; }

// Arguments of the fused stage kernel.  mode: 0 = dUdt_Residual_Evaluation,
// 1 = RK stage 1, 2 = RK stage 2.  The global time step of the current
// explicit step is hist[4 * *step] (the step history lives on the device so
// that a captured step replays without host involvement).
//
// A stage never updates the array it reads its halo from (tiles read their
// neighbours' cells while those are being updated): stage 1 reads (W, U) and
// writes (W2, U2); stage 2 reads the halo from W2 and the stage-1 base state
// U^0 from U, and writes (W, U).  U^0 is the reference's Uo.
struct StageArgs {
  Blocks B;
  int mode;
  int tiles_i, tiles_j;
  const double* hist;
  const int* step;
  const double* Win;   // primitive state the residual is evaluated on
  const double* Ubase; // U^0 of the update U = U^0 + omega * dUdt
  double* Wout;        // updated state
  double* Uout;
  int fuse_next;       // last stage of a step: also accumulate the next step's
                       // CFL minimum and residual norms into hist[4*(*step+1)..]
  // mode 3 (Frechet Jacobian-vector product of the NKS, GMRES2D.h:445-488):
  // v = (R(U)/normR - b)/eps - (z/dt)*normU/normR on interior cells, with the
  // GMRES vectors b, z, v in the reference's cell-major layout
  // [nblk][NCj][NCi][4].
  const double* nks_b;
  const double* nks_z;
  double* nks_v;
  const double* nks_eps;  // device scalar
  double normU[4], normR[4];
};

__host__ __device__ inline size_t cell_var(const Blocks& B, int b, int v, int j, int i) {
  return ((size_t(b) * 4 + v) * B.NCj + j) * B.NCi + i;
}
__host__ __device__ inline size_t cell_sc(const Blocks& B, int b, int j, int i) {
  return (size_t(b) * B.NCj + j) * B.NCi + i;
}
__host__ __device__ inline size_t node_ix(const Blocks& B, int b, int j, int i) {
  return (size_t(b) * B.NNj + j) * B.NNi + i;
}

template <class T> struct PState { T d, u, v, p; };  // Euler2D_pState
template <class T> struct CState { T d, mx, my, E; }; // Euler2D_cState

template <class T> __device__ __forceinline__ T dmin(T x, T y) { return (x < y) ? x : y; }
template <class T> __device__ __forceinline__ T dmax(T x, T y) { return (x > y) ? x : y; }
template <class T> __device__ __forceinline__ T sqr(T x) { return x * x; }

struct Gas {
  double g, gm1, gm1i;
};

template <class T> __device__ __forceinline__ CState<T> U_of_W(const PState<T>& w, T gm1i) {
  CState<T> u;
  u.d = w.d; u.mx = w.d * w.u; u.my = w.d * w.v;
  u.E = w.p * gm1i + T(HALF) * w.d * (w.u * w.u + w.v * w.v);
  return u;
}
template <class T> __device__ __forceinline__ PState<T> W_of_U(const CState<T>& u, T gm1) {
  PState<T> w;
  w.d = u.d; w.u = u.mx / u.d; w.v = u.my / u.d;
  w.p = gm1 * (u.E - T(HALF) * (u.mx * u.mx + u.my * u.my) / u.d);
  return w;
}
template <class T> __device__ __forceinline__ T a_of(const PState<T>& w, T g) { return sqrt(g * w.p / w.d); }
template <class T> __device__ __forceinline__ T h_of(const PState<T>& w, T g, T gm1) {
  return g * w.p / (gm1 * w.d) + T(HALF) * (w.u * w.u + w.v * w.v);
}
template <class T> __device__ __forceinline__ T e_of_U(const CState<T>& u) {
  return u.E / u.d - T(HALF) * (u.mx * u.mx + u.my * u.my) / sqr(u.d);
}

template <class T> __device__ __forceinline__ PState<T> reflect(const PState<T>& w, T c, T s) {
  T ur = w.u * c + w.v * s;
  T vr = -w.u * s + w.v * c;
  ur = -ur;
  PState<T> r;
  r.d = w.d; r.u = ur * c - vr * s; r.v = ur * s + vr * c; r.p = w.p;
  return r;
}

template <class T>
__device__ inline PState<T> bc_char_pressure(const PState<T>& wi, const PState<T>& wo, T c, T s,
                                             T g, T gm1i) {
  PState<T> ir, orr, r;
  T mi, db, pb, ab, ubr, vbr;
  ir.d = wi.d; ir.u = wi.u * c + wi.v * s; ir.v = -wi.u * s + wi.v * c; ir.p = wi.p;
  orr.d = wo.d; orr.u = wo.u * c + wo.v * s; orr.v = -wo.u * s + wo.v * c; orr.p = wo.p;
  mi = ir.u / a_of(ir, g);
  if (mi >= T(1)) {
    db = ir.d; ubr = ir.u; vbr = ir.v; pb = ir.p;
  } else if (mi >= T(0)) {
    pb = orr.p;
    db = ir.d * pow(pb / ir.p, T(1) / g);
    ab = sqrt(g * pb / db);
    ubr = ir.u + T(2) * (a_of(ir, g) - ab) * gm1i;
    vbr = ir.v;
  } else if (mi >= T(-1)) {
    pb = orr.p; db = orr.d; vbr = orr.v;
    ab = sqrt(g * pb / db);
    ubr = ir.u + T(2) * (a_of(ir, g) - ab) * gm1i;
  } else {
    db = orr.d; ubr = orr.u; vbr = orr.v; pb = orr.p;
  }
  r.d = db; r.u = ubr * c - vbr * s; r.v = ubr * s + vbr * c; r.p = pb;
  return r;
}

template <class T> __device__ __forceinline__ T harten_delta(T la, T ll, T lr) {
  T delta = dmax(T(0), T(2) * (lr - ll));
  if (fabs(la) > delta || delta < T(TOLER)) delta = T(0);
  else delta = T(HALF) * (sqr(la) / delta + delta) - fabs(la);
  return delta;
}

// FluxRoe_n: Roe flux with Harten's entropy fix on the acoustic waves, in
// the frame of the unit normal (c, s).
template <class T>
__device__ inline CState<T> flux_roe_n(const PState<T>& wl0, const PState<T>& wr0, T c, T s,
                                       T g, T gm1, T gm1i) {
  PState<T> wl, wr;
  wl.d = wl0.d; wl.u = wl0.u * c + wl0.v * s; wl.v = -wl0.u * s + wl0.v * c; wl.p = wl0.p;
  wr.d = wr0.d; wr.u = wr0.u * c + wr0.v * s; wr.v = -wr0.u * s + wr0.v * c; wr.p = wr0.p;
  // RoeAverage
  const T hl = h_of(wl, g, gm1), hr = h_of(wr, g, gm1);
  const T sdl = sqrt(wl.d), sdr = sqrt(wr.d);
  PState<T> wa;
  wa.d = sdl * sdr;
  wa.u = (sdl * wl.u + sdr * wr.u) / (sdl + sdr);
  wa.v = (sdl * wl.v + sdr * wr.v) / (sdl + sdr);
  const T ha = (sdl * hl + sdr * hr) / (sdl + sdr);
  const T aa2 = gm1 * (ha - T(HALF) * (sqr(wa.u) + sqr(wa.v)));
  wa.p = wa.d * aa2 / g;
  const T dW0 = wr.d - wl.d, dW1 = wr.u - wl.u, dW2 = wr.v - wl.v, dW3 = wr.p - wl.p;
  const T cl = a_of(wl, g), cr = a_of(wr, g), ca = a_of(wa, g);
  const bool up = wa.u >= T(0);
  const PState<T>& w = up ? wl : wr;
  CState<T> F;
  F.d = w.d * w.u;
  F.mx = w.d * sqr(w.u) + w.p;
  F.my = w.d * w.u * w.v;
  F.E = w.u * (g * gm1i * w.p + T(HALF) * w.d * (w.u * w.u + w.v * w.v));
  T ws[4];
  {
    const T la0 = wa.u - ca, la3 = wa.u + ca;
    const T d0 = harten_delta(la0, wl.u - cl, wr.u - cr);
    const T d3 = harten_delta(la3, wl.u + cl, wr.u + cr);
    if (up) {
      ws[0] = T(HALF) * (la0 - fabs(la0) - d0);
      ws[1] = T(HALF) * (wa.u - fabs(wa.u));
      ws[2] = ws[1];
      ws[3] = T(HALF) * (la3 - fabs(la3) - d3);
    } else {
      ws[0] = T(HALF) * (la0 + fabs(la0) + d0);
      ws[1] = T(HALF) * (wa.u + fabs(wa.u));
      ws[2] = ws[1];
      ws[3] = T(HALF) * (la3 + fabs(la3) + d3);
    }
  }
  const T sgn = up ? T(1) : T(-1);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!(up ? (ws[k] < T(0)) : (ws[k] > T(0)))) continue;
    T coef, r0, r1, r2, r3;
    if (k == 0 || k == 3) {
      // lp_x(1|4) = (0, -+HALF*d/c, 0, HALF/c^2); rc_x(1|4) = (1, u-+c, v, h-+u*c)
      const T lp1 = (k == 0) ? (-T(HALF) * wa.d / ca) : (T(HALF) * wa.d / ca);
      const T lp3 = T(HALF) / sqr(ca);
      coef = ws[k] * (T(0) * dW0 + (lp1 * dW1 + T(0) * dW2) + lp3 * dW3);
      const T hA = h_of(wa, g, gm1);
      r0 = T(1);
      r1 = (k == 0) ? (wa.u - ca) : (wa.u + ca);
      r2 = wa.v;
      r3 = (k == 0) ? (hA - wa.u * ca) : (hA + wa.u * ca);
    } else if (k == 1) {
      // lp_x(2) = (1, 0, 0, -1/a^2); rc_x(2) = (1, u, v, HALF*|v|^2)
      const T lp3 = T(-1) / (g * wa.p / wa.d);
      coef = ws[k] * (T(1) * dW0 + (T(0) * dW1 + T(0) * dW2) + lp3 * dW3);
      r0 = T(1); r1 = wa.u; r2 = wa.v; r3 = T(HALF) * (wa.u * wa.u + wa.v * wa.v);
    } else {
      // lp_x(3) = (0, 0, 1, 0); rc_x(3) = (0, 0, d, d*v)
      coef = ws[k] * (T(0) * dW0 + (T(0) * dW1 + T(1) * dW2) + T(0) * dW3);
      r0 = T(0); r1 = T(0); r2 = wa.d; r3 = wa.d * wa.v;
    }
    // Flux +=/-= coef*rc  (the sign follows the upwind side)
    if (up) {
      F.d += coef * r0; F.mx += coef * r1; F.my += coef * r2; F.E += coef * r3;
    } else {
      F.d -= coef * r0; F.mx -= coef * r1; F.my -= coef * r2; F.E -= coef * r3;
    }
  }
  (void)sgn;
  CState<T> R;
  R.d = F.d;
  R.mx = F.mx * c - F.my * s;
  R.my = F.mx * s + F.my * c;
  R.E = F.E;
  return R;
}

// Limiter_BarthJespersen / Limiter_Venkatakrishnan over the 4 face points.
template <class T>
__device__ __forceinline__ T limiter(int kind, const T* uq, T u0, T umin, T umax) {
  if (kind == E2D_LIMITER_ONE) return T(1);
  if (kind == E2D_LIMITER_ZERO) return T(0);
  T phi = T(1);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const T d = uq[q] - u0;
    if (d > T(TOLER) || d < -T(TOLER)) {
      const T y = ((d > T(TOLER)) ? (umax - u0) : (umin - u0)) / d;
      if (kind == E2D_LIMITER_VENKATAKRISHNAN)
        phi = dmin(phi, (sqr(y) + T(2) * y) / (sqr(y) + y + T(2)));
      else
        phi = dmin(phi, dmin(T(1), y));
    } else {
      phi = dmin(phi, T(1));
    }
  }
  return phi;
}

// quadCentroid on (SW, SE, NE, NW): area and centroid.  The cross products
// of absolute node coordinates cancel heavily away from the origin (the
// reference's own reason for its optional local-coordinate mode), so every
// build evaluates them with explicitly rounded operations: a fused
// multiply-add here would move centroids by ~1e-11 and the residual by
// ~1e-8 relative on the benchmark grid.
__device__ __forceinline__ double rn_cross(double a, double b, double c, double d) {
  return __dsub_rn(__dmul_rn(a, b), __dmul_rn(c, d));  // a*b - c*d
}
__device__ __forceinline__ void quad_moments(double x0, double y0, double x1, double y1,
                                             double x2, double y2, double x3, double y3,
                                             double& atmp, double& xt, double& yt) {
  double ai;
  atmp = 0; xt = 0; yt = 0;
  ai = rn_cross(x3, y0, x0, y3); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x0, x3), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y0, y3), ai));
  ai = rn_cross(x0, y1, x1, y0); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x1, x0), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y1, y0), ai));
  ai = rn_cross(x1, y2, x2, y1); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x2, x1), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y2, y1), ai));
  ai = rn_cross(x2, y3, x3, y2); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x3, x2), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y3, y2), ai));
}
__device__ __forceinline__ void quad_centroid(double x0, double y0, double x1, double y1,
                                              double x2, double y2, double x3, double y3,
                                              double& xc, double& yc, double& area) {
  double ai, atmp = 0, xt = 0, yt = 0;
  ai = rn_cross(x3, y0, x0, y3); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x0, x3), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y0, y3), ai));
  ai = rn_cross(x0, y1, x1, y0); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x1, x0), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y1, y0), ai));
  ai = rn_cross(x1, y2, x2, y1); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x2, x1), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y2, y1), ai));
  ai = rn_cross(x2, y3, x3, y2); atmp = __dadd_rn(atmp, ai);
  xt = __dadd_rn(xt, __dmul_rn(__dadd_rn(x3, x2), ai)); yt = __dadd_rn(yt, __dmul_rn(__dadd_rn(y3, y2), ai));
  area = __dmul_rn(0.5, atmp);
  if (atmp != 0) {
    const double a3 = __dmul_rn(3.0, atmp);
    xc = xt / a3;
    yc = yt / a3;
  } else {
    xc = 0; yc = 0;
  }
}

// Records the first error in the status word.
__device__ __forceinline__ void set_status(int* st, int code, int cell) {
  if (atomicCAS(st, 0, code) == 0) st[1] = cell;
}

}  // namespace e2d
