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
  int limiter, flux, n_stage, local_dt;
  // Batches of independent cases: the blocks of case c are
  // case_start[c] .. case_start[c+1]-1 and case_of[b] names the case of block b
  // (null for a single case).  Per-case quantities (time-step minimum, residual
  // norms) live in slot (step, case) of the step history: hist + 4*(step*ncase + case).
  const int* case_of;
  const int* case_start;
  int ncase;
  const int* case_active;  // per case, null = all: residual/JVP stages skip inactive cases
  // Limiter freezing (Freeze_Limiter): with freeze set, *freeze != 0 means
  // the limiters are frozen and every reconstruction takes phi from
  // phi_keep; while *freeze == 0 each reconstruction stores its phi there
  // (cells of the tiles and their one-cell rings).  freeze null: off.
  const int* freeze;
  double* phi_keep;
};

__host__ __device__ inline int case_id(const Blocks& B, int b) { return B.case_of ? B.case_of[b] : 0; }

// The flux functions of i_Flux_Function built here: all of CFD.h:768-778 but
// Osher (7, which the reference's Euler2D dispatch does not offer either).
__host__ __device__ inline bool e2d_flux_supported(int f) { return f >= E2D_FLUX_GODUNOV && f <= E2D_FLUX_AUSMPLUS && f != 7; }

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
  // explicit stages (modes 1, 2): U = Ubase + omega*dUdt, the stage's dUdt
  // stored to res_out; mode 2 starts dUdt from res_out's previous content
  // (the two-stage schemes) or, with acc1/acc2 set, from
  // res_out + 2*acc1 + 2*acc2 (stage 4 of RK4, Euler2DQuad.cc:1322-1334)
  double omega;
  double* res_out;
  const double* acc1;
  const double* acc2;
  int no_update;  // modes 1, 2: store the stage's residual only (residual smoothing follows)
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

// ---- the other flux functions of i_Flux_Function ----------------------------
// Each *_n routine of the reference rotates both states into the frame of the
// unit normal (c, s), evaluates the x-direction flux and rotates the momentum
// flux back; flux_n does the same around the x-direction functions below.

template <class T> __device__ __forceinline__ PState<T> rotate_in(const PState<T>& w, T c, T s) {
  PState<T> r;
  r.d = w.d; r.u = w.u * c + w.v * s; r.v = -w.u * s + w.v * c; r.p = w.p;
  return r;
}
template <class T> __device__ __forceinline__ CState<T> rotate_out(const CState<T>& f, T c, T s) {
  CState<T> r;
  r.d = f.d; r.mx = f.mx * c - f.my * s; r.my = f.mx * s + f.my * c; r.E = f.E;
  return r;
}
// Euler2D_pState::H (total enthalpy per volume, Euler2DState.h:1077) and Fx (:1845).
template <class T> __device__ __forceinline__ T ht_of(const PState<T>& w, T g, T gm1i) {
  return g * gm1i * w.p + T(HALF) * w.d * (w.u * w.u + w.v * w.v);
}
template <class T> __device__ __forceinline__ CState<T> fx_of(const PState<T>& w, T g, T gm1i) {
  CState<T> F;
  F.d = w.d * w.u; F.mx = w.d * sqr(w.u) + w.p; F.my = w.d * w.u * w.v; F.E = w.u * ht_of(w, g, gm1i);
  return F;
}
// RoeAverage (Euler2DState.cc:654-683).
template <class T> __device__ __forceinline__ PState<T> roe_average(const PState<T>& wl, const PState<T>& wr, T g,
                                                                   T gm1) {
  const T hl = h_of(wl, g, gm1), hr = h_of(wr, g, gm1);
  const T sdl = sqrt(wl.d), sdr = sqrt(wr.d);
  PState<T> wa;
  wa.d = sdl * sdr;
  wa.u = (sdl * wl.u + sdr * wr.u) / (sdl + sdr);
  wa.v = (sdl * wl.v + sdr * wr.v) / (sdl + sdr);
  const T ha = (sdl * hl + sdr * hr) / (sdl + sdr);
  const T aa2 = gm1 * (ha - T(HALF) * (sqr(wa.u) + sqr(wa.v)));
  wa.p = wa.d * aa2 / g;
  return wa;
}
template <class T> __device__ __forceinline__ PState<T> pstate(T d, T u, T v, T p) {
  PState<T> w;
  w.d = d; w.u = u; w.v = v; w.p = p;
  return w;
}

// Riemann_x (Euler2DState.cc:245-449): exact Riemann solver of Gottlieb and
// Groth, Newton-Raphson on the intermediate velocity (at most 11 passes),
// returning the state on the ray x/t = 0.
template <class T>
__device__ inline PState<T> riemann_x(const PState<T>& wl, const PState<T>& wr, T g, T gm1) {
  const T al = a_of(wl, g), ar = a_of(wr, g);
  const T CL = wl.u + T(2) * al / gm1;
  const T CR = wr.u - T(2) * ar / gm1;
  if (CL - CR <= T(0)) return pstate(T(0), T(0), T(0), T(0));
  const T Z = (ar / al) * pow((wl.p / wr.p), T(HALF) * gm1 / g);
  T um = (CL * Z + CR) / (T(1) + Z);
  T pm, aml = T(0), amr = T(0);
  if (um >= wl.u && um <= wr.u) {  // two rarefactions: exact without iteration
    if (um >= T(0)) {
      aml = al - T(HALF) * gm1 * (um - wl.u);
      pm = wl.p * pow((aml / al), T(2) * g / gm1);
      if (wl.u - al >= T(0)) return wl;
      if (um - aml <= T(0)) return pstate(g * pm / sqr(aml), um, wl.v, pm);
      um = (gm1 * wl.u + T(2) * al) / (g + T(1));
      pm = wl.p * pow((um / al), T(2) * g / gm1);
      return pstate(g * pm / sqr(um), um, wl.v, pm);
    }
    amr = ar + T(HALF) * gm1 * (um - wr.u);
    pm = wr.p * pow((amr / ar), T(2) * g / gm1);
    if (wr.u + ar <= T(0)) return wr;
    if (um + amr >= T(0)) return pstate(g * pm / sqr(amr), um, wr.v, pm);
    um = (gm1 * wr.u - T(2) * ar) / (g + T(1));
    pm = wr.p * pow((-um / ar), T(2) * g / gm1);
    return pstate(g * pm / sqr(um), um, wr.v, pm);
  }
  T msl = T(0), msr = T(0), pml, pmr, dpl, dpr;
  for (int it = 1;; ++it) {
    if (um < wl.u) {
      msl = (g + T(1)) * (um - wl.u) / (T(4) * al);
      msl = msl - sqrt(T(1) + sqr(msl));
      pml = wl.p * (T(1) + g * (um - wl.u) * msl / al);
      dpl = T(2) * g * wl.p * (msl * msl * msl) / (al * (T(1) + sqr(msl)));
    } else {
      aml = al - T(HALF) * gm1 * (um - wl.u);
      pml = wl.p * pow((aml / al), T(2) * g / gm1);
      dpl = -g * pml / aml;
    }
    if (um > wr.u) {
      msr = (g + T(1)) * (um - wr.u) / (T(4) * ar);
      msr = msr + sqrt(T(1) + sqr(msr));
      pmr = wr.p * (T(1) + g * (um - wr.u) * msr / ar);
      dpr = T(2) * g * wr.p * (msr * msr * msr) / (ar * (T(1) + sqr(msr)));
    } else {
      amr = ar + T(HALF) * gm1 * (um - wr.u);
      pmr = wr.p * pow((amr / ar), T(2) * g / gm1);
      dpr = g * pmr / amr;
    }
    if (fabs(T(1) - pml / pmr) <= T(TOLER)) break;
    if (it > 10) break;  // the reference reports non-convergence and carries on
    um = um - (pml - pmr) / (dpl - dpr);
  }
  pm = T(HALF) * (pml + pmr);
  if (um >= T(0)) {
    if (um < wl.u) {  // left shock
      aml = al * sqrt(((g + T(1)) + gm1 * pm / wl.p) / ((g + T(1)) + gm1 * wl.p / pm));
      if (wl.u + msl * al >= T(0)) return wl;
      return pstate(g * pm / sqr(aml), um, wl.v, pm);
    }
    if (wl.u - al >= T(0)) return wl;
    if (um - aml <= T(0)) return pstate(g * pm / sqr(aml), um, wl.v, pm);
    um = (gm1 * wl.u + T(2) * al) / (g + T(1));
    pm = wl.p * pow((um / al), T(2) * g / gm1);
    return pstate(g * pm / sqr(um), um, wl.v, pm);
  }
  if (um > wr.u) {  // right shock
    amr = ar * sqrt(((g + T(1)) + gm1 * pm / wr.p) / ((g + T(1)) + gm1 * wr.p / pm));
    if (wr.u + msr * ar <= T(0)) return wr;
    return pstate(g * pm / sqr(amr), um, wr.v, pm);
  }
  if (wr.u + ar <= T(0)) return wr;
  if (um + amr >= T(0)) return pstate(g * pm / sqr(amr), um, wr.v, pm);
  um = (gm1 * wr.u - T(2) * ar) / (g + T(1));
  pm = wr.p * pow((-um / ar), T(2) * g / gm1);
  return pstate(g * pm / sqr(um), um, wr.v, pm);
}

// FluxRusanov_x (Euler2DState.cc:2673-2713): central flux less half the
// largest Harten-fixed |lambda| times the jump in U (HartenFixAbs, CFD.cc:655).
template <class T>
__device__ inline CState<T> flux_rusanov_x(const PState<T>& wl, const PState<T>& wr, T g, T gm1, T gm1i) {
  const PState<T> wa = roe_average(wl, wr, g, gm1);
  const CState<T> ul = U_of_W(wl, gm1i), ur = U_of_W(wr, gm1i);
  const CState<T> fl = fx_of(wl, g, gm1i), fr = fx_of(wr, g, gm1i);
  const T cl = a_of(wl, g), cr = a_of(wr, g), ca = a_of(wa, g);
  const T la0 = wa.u - ca, la3 = wa.u + ca;
  T m = fabs(la0) + harten_delta(la0, wl.u - cl, wr.u - cr);
  m = dmax(m, fabs(wa.u));
  m = dmax(m, fabs(wa.u));
  m = dmax(m, fabs(la3) + harten_delta(la3, wl.u + cl, wr.u + cr));
  const T k = T(HALF) * m;
  CState<T> F;
  F.d = T(HALF) * (fl.d + fr.d);
  F.mx = T(HALF) * (fl.mx + fr.mx);
  F.my = T(HALF) * (fl.my + fr.my);
  F.E = T(HALF) * (fl.E + fr.E);
  F.d -= k * (ur.d - ul.d);
  F.mx -= k * (ur.mx - ul.mx);
  F.my -= k * (ur.my - ul.my);
  F.E -= k * (ur.E - ul.E);
  return F;
}

// FluxHLLE_x (Euler2DState.cc:2921-2963) and FluxLinde_x (:3321-3383): HLL
// flux with the Einfeldt wave-speed bounds; Linde's variant restores part of
// the contact through the coefficient alpha.
template <class T, bool LINDE>
__device__ inline CState<T> flux_hll_x(const PState<T>& wl, const PState<T>& wr, T g, T gm1, T gm1i) {
  const PState<T> wa = roe_average(wl, wr, g, gm1);
  const T ca = a_of(wa, g);
  const T sl = dmin(wl.u - a_of(wl, g), wa.u - ca);
  const T sr = dmax(wr.u + a_of(wr, g), wa.u + ca);
  if (sl >= T(0)) return fx_of(wl, g, gm1i);
  if (sr <= T(0)) return fx_of(wr, g, gm1i);
  const CState<T> ul = U_of_W(wl, gm1i), ur = U_of_W(wr, gm1i);
  const CState<T> fl = fx_of(wl, g, gm1i), fr = fx_of(wr, g, gm1i);
  CState<T> dU;
  dU.d = ur.d - ul.d; dU.mx = ur.mx - ul.mx; dU.my = ur.my - ul.my; dU.E = ur.E - ul.E;
  T k = sl * sr;
  if (LINDE) {
    const T sm = wa.u, da = wa.d;
    T du = fabs(dU.d) / da + fabs(dU.mx) / (da * ca) + fabs(dU.my) / (da * ca) + fabs(dU.E) / (da * ca * ca);
    T alpha;
    if (du <= T(TOLER)) {
      alpha = T(0);
    } else {
      du = T(1) / du;
      const T w0 = (fr.d - fl.d) - sm * dU.d, w1 = (fr.mx - fl.mx) - sm * dU.mx;
      const T w2 = (fr.my - fl.my) - sm * dU.my, w3 = (fr.E - fl.E) - sm * dU.E;
      alpha = T(1) - (fabs(w0) / (da * ca) + fabs(w1) / (da * ca * ca) + fabs(w2) / (da * ca * ca) +
                      fabs(w3) / (da * ca * ca * ca)) * du;
      alpha = dmax(T(0), alpha);
    }
    k = k * (T(1) - (T(1) - dmax(sm / sr, sm / sl)) * alpha);
  }
  const T den = sr - sl;
  CState<T> F;
  F.d = ((sr * fl.d - sl * fr.d) + k * dU.d) / den;
  F.mx = ((sr * fl.mx - sl * fr.mx) + k * dU.mx) / den;
  F.my = ((sr * fl.my - sl * fr.my) + k * dU.my) / den;
  F.E = ((sr * fl.E - sl * fr.E) + k * dU.E) / den;
  return F;
}

// FluxHLLC_x (Euler2DState.cc:3630-3694): Toro's HLLC with wave speeds from
// the two-rarefaction pressure estimate.
template <class T>
__device__ inline CState<T> flux_hllc_x(const PState<T>& wl, const PState<T>& wr, T g, T gm1, T gm1i) {
  const T al = a_of(wl, g), ar = a_of(wr, g);
  const T CL = wl.u + T(2) * al / gm1;
  const T CR = wr.u - T(2) * ar / gm1;
  const T Z = (ar / al) * pow((wl.p / wr.p), T(HALF) * gm1 / g);
  const T um = (CL * Z + CR) / (T(1) + Z);
  const T aml = al - T(HALF) * gm1 * (um - wl.u);
  T pm = wl.p * pow((aml / al), T(2) * g / gm1);
  const T amr = ar + T(HALF) * gm1 * (um - wr.u);
  pm = T(HALF) * (pm + wr.p * pow((amr / ar), T(2) * g / gm1));
  const T ql = (pm / wl.p <= T(1)) ? T(1) : sqrt(T(1) + T(HALF) * ((g + T(1)) / g) * (pm / wl.p));
  const T sl = wl.u - ql * al;
  const T qr = (pm / wr.p <= T(1)) ? T(1) : sqrt(T(1) + T(HALF) * ((g + T(1)) / g) * (pm / wr.p));
  const T sr = wr.u + qr * ar;
  if (sl >= T(0)) return fx_of(wl, g, gm1i);
  if (sr <= T(0)) return fx_of(wr, g, gm1i);
  const bool left = um >= T(0);
  const PState<T>& w = left ? wl : wr;
  const T sk = left ? sl : sr;
  const CState<T> uk = U_of_W(w, gm1i), fk = fx_of(w, g, gm1i);
  const T f = (sk - w.u) / (sk - um);
  CState<T> us;  // intermediate state on the upwind side of the contact
  us.d = w.d * f;
  us.mx = (w.d * um) * f;
  us.my = (w.d * w.v) * f;
  us.E = (uk.E + w.d * (um - w.u) * (um + w.p / (w.d * (sk - w.u)))) * f;
  CState<T> F;
  F.d = fk.d + sk * (us.d - uk.d);
  F.mx = fk.mx + sk * (us.mx - uk.mx);
  F.my = fk.my + sk * (us.my - uk.my);
  F.E = fk.E + sk * (us.E - uk.E);
  return F;
}

// FluxVanLeer (Euler2DState.cc:3862-3903): flux-vector splitting.
template <class T>
__device__ inline CState<T> flux_vanleer_x(const PState<T>& wl, const PState<T>& wr, T g, T gm1, T gm1i) {
  CState<T> fl, fr;
  // Euler2D_cState's default value, reached only by a NaN Mach number
  fl.d = fr.d = T(1.225); fl.mx = fr.mx = fl.my = fr.my = T(0); fl.E = fr.E = T(101325.0 / (1.4 - 1.0));
  T M = wl.u / a_of(wl, g);
  if (M < T(-1)) {
    fl.d = fl.mx = fl.my = fl.E = T(0);
  } else if (fabs(M) <= T(1)) {
    const T a = a_of(wl, g);
    const T Mp = T(0.25) * wl.d * a * sqr(T(1) + M);
    fl.d = Mp;
    fl.mx = Mp * ((T(2) * a / g) * (T(HALF) * gm1 * M + T(1)));
    fl.my = Mp * wl.v;
    fl.E = Mp * ((T(2) * (g * wl.p / wl.d) / (g * g - T(1))) * sqr(T(HALF) * gm1 * M + T(1)) + T(HALF) * sqr(wl.v));
  } else if (M > T(1)) {
    fl = fx_of(wl, g, gm1i);
  }
  M = wr.u / a_of(wr, g);
  if (-M < T(-1)) {
    fr.d = fr.mx = fr.my = fr.E = T(0);
  } else if (fabs(M) <= T(1)) {
    const T a = a_of(wr, g);
    const T Mn = T(-0.25) * wr.d * a * sqr(T(1) - M);
    fr.d = Mn;
    fr.mx = Mn * ((T(2) * a / g) * (T(HALF) * gm1 * M - T(1)));
    fr.my = Mn * wr.v;
    fr.E = Mn * ((T(2) * (g * wr.p / wr.d) / (g * g - T(1))) * sqr(T(HALF) * gm1 * M - T(1)) + T(HALF) * sqr(wr.v));
  } else if (-M > T(1)) {
    fr = fx_of(wr, g, gm1i);
  }
  CState<T> F;
  F.d = fl.d + fr.d; F.mx = fl.mx + fr.mx; F.my = fl.my + fr.my; F.E = fl.E + fr.E;
  return F;
}

// FluxAUSM (Euler2DState.cc:4056-4106, Liou and Steffen) and FluxAUSMplus
// (:4170-4231, Liou 1994): split Mach numbers and pressures.
template <class T>
__device__ inline CState<T> flux_ausm_x(const PState<T>& wl, const PState<T>& wr, T g, T gm1i) {
  const T al = a_of(wl, g), Ml = wl.u / al;
  const T ar = a_of(wr, g), Mr = wr.u / ar;
  T Mplus, pplus, Mminus, pminus;
  if (fabs(Ml) <= T(1)) {
    Mplus = T(0.25) * sqr(Ml + T(1));
    pplus = T(0.25) * wl.p * sqr(Ml + T(1)) * (T(2) - Ml);
  } else {
    Mplus = T(0.5) * (Ml + fabs(Ml));
    pplus = T(0.5) * wl.p * (Ml + fabs(Ml)) / Ml;
  }
  if (fabs(Mr) <= T(1)) {
    Mminus = T(-0.25) * sqr(Mr - T(1));
    pminus = T(0.25) * wr.p * sqr(Mr - T(1)) * (T(2) + Mr);
  } else {
    Mminus = T(0.5) * (Mr - fabs(Mr));
    pminus = T(0.5) * wr.p * (Mr - fabs(Mr)) / Mr;
  }
  const T Mh = Mplus + Mminus, ph = pplus + pminus;
  const T Hl = ht_of(wl, g, gm1i), Hr = ht_of(wr, g, gm1i);
  const T k = T(0.5) * Mh, q = T(0.5) * fabs(Mh);
  CState<T> F;
  F.d = k * (wl.d * al + wr.d * ar);
  F.mx = k * (wl.d * al * wl.u + wr.d * ar * wr.u);
  F.my = k * (wl.d * al * wl.v + wr.d * ar * wr.v);
  F.E = k * (al * Hl + ar * Hr);
  F.d -= q * (wr.d * ar - wl.d * al);
  F.mx -= q * (wr.d * ar * wr.u - wl.d * al * wl.u);
  F.my -= q * (wr.d * ar * wr.v - wl.d * al * wl.v);
  F.E -= q * (ar * Hr - al * Hl);
  F.mx += ph;
  return F;
}
template <class T>
__device__ inline CState<T> flux_ausmplus_x(const PState<T>& wl, const PState<T>& wr, T g, T gm1i) {
  const T beta = T(0.125), alpha = T(0.1875);
  const T ah = T(HALF) * (a_of(wl, g) + a_of(wr, g));
  const T Ml = wl.u / ah, Mr = wr.u / ah;
  T Mplus, pplus, Mminus, pminus;
  if (fabs(Ml) < T(1)) {
    Mplus = T(0.25) * sqr(Ml + T(1)) + beta * sqr(Ml * Ml - T(1));
    pplus = (T(0.25) * sqr(Ml + T(1)) * (T(2) - Ml) + alpha * Ml * sqr(Ml * Ml - T(1))) * wl.p;
  } else {
    Mplus = T(0.5) * (Ml + fabs(Ml));
    pplus = T(0.5) * wl.p * (T(1) + ((Ml < T(0)) ? T(-1) : T(1)));
  }
  if (fabs(Mr) < T(1)) {
    Mminus = T(-0.25) * sqr(Mr - T(1)) - beta * sqr(Mr * Mr - T(1));
    pminus = (T(0.25) * sqr(Mr - T(1)) * (T(2) + Mr) - alpha * Mr * sqr(Mr * Mr - T(1))) * wr.p;
  } else {
    Mminus = T(0.5) * (Mr - fabs(Mr));
    pminus = T(0.5) * wr.p * (T(1) - ((Mr < T(0)) ? T(-1) : T(1)));
  }
  const T Mh = Mplus + Mminus, ph = pplus + pminus;
  const T Hl = ht_of(wl, g, gm1i), Hr = ht_of(wr, g, gm1i);
  const T k = T(0.5) * Mh, q = T(0.5) * fabs(Mh);
  CState<T> F;
  F.d = k * (wl.d + wr.d);
  F.mx = k * (wl.d * wl.u + wr.d * wr.u);
  F.my = k * (wl.d * wl.v + wr.d * wr.v);
  F.E = k * (Hl + Hr);
  F.d -= q * (wr.d - wl.d);
  F.mx -= q * (wr.d * wr.u - wl.d * wl.u);
  F.my -= q * (wr.d * wr.v - wl.d * wl.v);
  F.E -= q * (Hr - Hl);
  F.d *= ah; F.mx *= ah; F.my *= ah; F.E *= ah;
  F.mx += ph;
  return F;
}

// Face flux of i_Flux_Function `kind` other than Roe (dispatch of
// dUdt_Residual_Evaluation, Euler2DQuad.cc:968-1003).  Kept out of line so
// that the Roe path's register allocation does not carry these.
template <class T>
__device__ inline CState<T> flux_n(int kind, PState<T> wl, PState<T> wr, T c, T s, T g, T gm1, T gm1i) {
  wl = rotate_in(wl, c, s);
  wr = rotate_in(wr, c, s);
  CState<T> F;
  switch (kind) {
    case E2D_FLUX_GODUNOV: F = fx_of(riemann_x(wl, wr, g, gm1), g, gm1i); break;
    case E2D_FLUX_RUSANOV: F = flux_rusanov_x(wl, wr, g, gm1, gm1i); break;
    case E2D_FLUX_HLLE: F = flux_hll_x<T, false>(wl, wr, g, gm1, gm1i); break;
    case E2D_FLUX_LINDE: F = flux_hll_x<T, true>(wl, wr, g, gm1, gm1i); break;
    case E2D_FLUX_HLLC: F = flux_hllc_x(wl, wr, g, gm1, gm1i); break;
    case E2D_FLUX_VANLEER: F = flux_vanleer_x(wl, wr, g, gm1, gm1i); break;
    case E2D_FLUX_AUSM: F = flux_ausm_x(wl, wr, g, gm1i); break;
    default: F = flux_ausmplus_x(wl, wr, g, gm1i); break;
  }
  return rotate_out(F, c, s);
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
