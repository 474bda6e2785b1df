// e2d_fastmath.cuh — the fast FP64 path's arithmetic: reciprocal and
// reciprocal square root by Newton–Raphson refinement of the PTX approximate
// instructions, and division-lean restatements of the Roe flux, the
// least-squares gradient and the limiters.
//
// Refinement (Newton–Raphson on f(r) = 1/r - x and f(r) = 1/r^2 - x; each step
// squares the relative error): starting from rcp.approx / rsqrt.approx
// (relative error below 2^-22), two steps reach the double-precision
// rounding level.  tests/test_gpu_fastmath.py bounds the error against IEEE
// division and square root.
//
// The algebra keeps the reference's quantities but removes divisions:
//   c^2 = g p / d,  h = c^2/(g-1) + |v|^2/2,  u H = d u h,
//   Roe average: a_a^2 = (g-1)(h_a - |v_a|^2/2), and g p_a / d_a = a_a^2, so
//   lp_x(1|4) = (0, -+d_a/(2 a_a), 0, 1/(2 a_a^2)),  lp_x(2) = (1, 0, 0, -1/a_a^2),
//   rc_x(1|4) = (1, u_a -+ a_a, v_a, h_a -+ u_a a_a)  (h of the Roe state is h_a);
//   least-squares: the 1/n averaging cancels in the gradient;
//   limiters: phi increases with y, so the smallest y = |a|/|b| over the
//   face points is found by cross-multiplication and phi is evaluated once,
//   (a^2 + 2ab)/(a^2 + ab + 2b^2) (Venkatakrishnan) or a/b (Barth–Jespersen),
//   capped at 1, with one reciprocal.
#pragma once
#include "e2d_device.cuh"

namespace e2d {
namespace fm {

__device__ __forceinline__ double rcp_approx(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
}
__device__ __forceinline__ double rsqrt_approx(double x) {
  double r;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
}
// 1/x for normal, non-zero x.
__device__ __forceinline__ double rcp(double x) {
  double r = rcp_approx(x);
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
// 1/sqrt(x) for normal x > 0.
__device__ __forceinline__ double rsqrt(double x) {
  double r = rsqrt_approx(x);
  const double h = 0.5 * x;
  double e = fma(-h * r, r, 0.5);
  r = fma(r, e, r);
  e = fma(-h * r, r, 0.5);
  return fma(r, e, r);
}
// sqrt(x) = x / sqrt(x) with one Newton correction; x > 0.
__device__ __forceinline__ double sqrt_from_rsqrt(double x, double r) {
  const double s = x * r;
  const double d = fma(-s, s, x);
  return fma(0.5 * r, d, s);
}

// Single precision counterparts for the FP32 build (compiled with the
// approximate single-precision division and square root).
__device__ __forceinline__ float rcp(float x) { return 1.0f / x; }
__device__ __forceinline__ float rsqrt(float x) { return rsqrtf(x); }
__device__ __forceinline__ float sqrt_from_rsqrt(float x, float r) {
  const float s = x * r;
  const float d = fmaf(-s, s, x);
  return fmaf(0.5f * r, d, s);
}

template <class T>
__device__ __forceinline__ T harten_delta(T la, T ll, T lr) {
  T delta = dmax(T(0), T(2) * (lr - ll));
  if (fabs(la) > delta || delta < T(TOLER)) return T(0);
  return T(0.5) * (la * la * rcp(delta) + delta) - fabs(la);
}

// FluxRoe_n in the frame of the unit normal (c, s), division-lean form (T =
// double for the fast FP64 build, float for the FP32 one).
template <class T>
__device__ __forceinline__ CState<T> flux_roe_n(const PState<T>& wl0, const PState<T>& wr0, T c, T s, T g, T gm1,
                                                T gm1i) {
  const T dl = wl0.d, pl = wl0.p, dr = wr0.d, pr = wr0.p;
  const T ul = wl0.u * c + wl0.v * s, vl = -wl0.u * s + wl0.v * c;
  const T ur = wr0.u * c + wr0.v * s, vr = -wr0.u * s + wr0.v * c;
  const T rsdl = rsqrt(dl), rsdr = rsqrt(dr);
  const T sdl = sqrt_from_rsqrt(dl, rsdl), sdr = sqrt_from_rsqrt(dr, rsdr);
  const T cl2 = g * pl * (rsdl * rsdl), cr2 = g * pr * (rsdr * rsdr);
  const T hl = cl2 * gm1i + T(0.5) * (ul * ul + vl * vl);
  const T hr = cr2 * gm1i + T(0.5) * (ur * ur + vr * vr);
  const T inv = rcp(sdl + sdr);
  const T ua = (sdl * ul + sdr * ur) * inv;
  const T va = (sdl * vl + sdr * vr) * inv;
  const T ha = (sdl * hl + sdr * hr) * inv;
  const T qa2 = ua * ua + va * va;
  const T aa2 = gm1 * (ha - T(0.5) * qa2);
  const T rca = rsqrt(aa2);
  const T ca = sqrt_from_rsqrt(aa2, rca);
  const T da = sdl * sdr;
  const T dW1 = ur - ul, dW3 = pr - pl;
  const bool up = ua >= T(0);
  const T d = up ? dl : dr, u = up ? ul : ur, v = up ? vl : vr, p = up ? pl : pr;
  const T h = up ? hl : hr;
  const T du = d * u;
  T F0 = du, F1 = du * u + p, F2 = du * v, F3 = du * h;
  const T la0 = ua - ca, la3 = ua + ca;
  // Harten's fix acts on a wave only where |la| <= delta = max(0, 2 (lr - ll)),
  // lr - ll = (ur - ul) -+ (cr - cl).  Since |cr - cl| <= sqrt|cr^2 - cl^2|,
  // delta <= 2 (|ur - ul| + sqrt|cr^2 - cl^2|): faces whose wave speeds
  // exceed that bound (computed in single precision with a wide margin)
  // skip the exact sound speeds.
  const float dbound = 2.0f * (float(fabs(ur - ul)) + sqrtf(float(fabs(cr2 - cl2)))) * 1.001f + 1e-30f;
  T d0 = T(0), d3 = T(0);
  if (!(float(fabs(la0)) > dbound) || !(float(fabs(la3)) > dbound)) {
    const T cl = sqrt_from_rsqrt(cl2, rsqrt(cl2)), cr = sqrt_from_rsqrt(cr2, rsqrt(cr2));
    d0 = harten_delta(la0, ul - cl, ur - cr);
    d3 = harten_delta(la3, ul + cl, ur + cr);
  }
  // The entropy and shear waves travel at ua itself: with the upwind side
  // taken from the sign of ua their strengths (ua -+ |ua|) / 2 are exactly
  // zero, so only the two acoustic waves can contribute.
  T ws0, ws3;
  if (up) {
    ws0 = T(0.5) * (la0 - fabs(la0) - d0);
    ws3 = T(0.5) * (la3 - fabs(la3) - d3);
  } else {
    ws0 = T(0.5) * (la0 + fabs(la0) + d0);
    ws3 = T(0.5) * (la3 + fabs(la3) + d3);
  }
  const T sg = up ? T(1) : T(-1);
  const T rca2 = rca * rca;
  const T hdr = T(0.5) * da * rca * dW1, pdr = T(0.5) * rca2 * dW3;
  // Each wave contributes only where the reference's upwind test selects it;
  // a wave speed of exactly zero contributes nothing either way.
  const bool on0 = up ? (ws0 < T(0)) : (ws0 > T(0));
  const bool on3 = up ? (ws3 < T(0)) : (ws3 > T(0));
  if (on0) {
    const T k = sg * ws0 * (pdr - hdr);
    F0 += k; F1 += k * (ua - ca); F2 += k * va; F3 += k * (ha - ua * ca);
  }
  if (on3) {
    const T k = sg * ws3 * (pdr + hdr);
    F0 += k; F1 += k * (ua + ca); F2 += k * va; F3 += k * (ha + ua * ca);
  }
  CState<T> R;
  R.d = F0;
  R.mx = F1 * c - F2 * s;
  R.my = F1 * s + F2 * c;
  R.E = F3;
  return R;
}

// Limiter over the 4 face points with one reciprocal.  The reference takes
// the smallest of phi(y_q) over the face points q, y_q = (u_max or u_min -
// u0) / (u_q - u0) >= 0, skipping points within TOLER of u0
// (CFD.cc:696-751).  Both phi here -- Venkatakrishnan's (y^2 + 2y) /
// (y^2 + y + 2) and Barth-Jespersen's min(1, y) -- increase with y, so that
// minimum is phi at the smallest y_q, capped at 1: the smallest ratio is found
// by cross-multiplying |a| / |b| pairs and phi is evaluated once.
__device__ __forceinline__ double rcp_t(double x) { return rcp(x); }
__device__ __forceinline__ float rcp_t(float x) { return rcp(x); }
template <class T>
__device__ __forceinline__ T limiter(int kind, const T* uq, T u0, T umin, T umax) {
  if (kind == E2D_LIMITER_ONE) return T(1);
  if (kind == E2D_LIMITER_ZERO) return T(0);
  T A = T(1), Bm = T(0);  // smallest ratio A / Bm so far; 1/0 stands for "none"
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const T b = uq[q] - u0;
    const T ab = fabs(b);
    if (ab > T(TOLER)) {
      const T a = fabs((b > T(0) ? umax : umin) - u0);
      if (a * Bm < A * ab) { A = a; Bm = ab; }
    }
  }
  if (kind == E2D_LIMITER_VENKATAKRISHNAN) {
    const T n = A * A + T(2) * A * Bm;         // y^2 + 2y, times Bm^2
    const T d = A * A + A * Bm + T(2) * Bm * Bm;  // y^2 + y + 2, times Bm^2
    return n < d ? n * rcp_t(d) : T(1);
  }
  return A < Bm ? A * rcp_t(Bm) : T(1);  // Barth-Jespersen
}

// The same limiter from the face-point differences dq[q] = u_q - u0 and the
// neighbour extremes as differences dmax = u_max - u0 >= 0, dmin = u_min - u0
// <= 0 (the marching kernel forms dq directly from the gradient, without
// the round trip through u_q).  Among the points that rise (dq > TOLER) the
// smallest ratio dmax / dq is at the largest rise, among those that fall
// (dq < -TOLER) the smallest dmin / dq at the largest fall, so the smallest
// ratio over all points is the smaller of those two: two extremes of the
// four differences and one comparison instead of a test per point.
template <int KIND, class T>
__device__ __forceinline__ T limiter_diff_k(const T* dq, T dmin, T dmax) {
  if (KIND == E2D_LIMITER_ONE) return T(1);
  if (KIND == E2D_LIMITER_ZERO) return T(0);
  const T rise = e2d::dmax(e2d::dmax(dq[0], dq[1]), e2d::dmax(dq[2], dq[3]));
  const T fall = e2d::dmin(e2d::dmin(dq[0], dq[1]), e2d::dmin(dq[2], dq[3]));
  T A = T(1), Bm = T(0);  // smallest ratio A / Bm; 1/0 stands for "none"
  if (rise > T(TOLER)) { A = dmax; Bm = rise; }
  if (fall < -T(TOLER) && -dmin * Bm < A * -fall) { A = -dmin; Bm = -fall; }
  if (KIND == E2D_LIMITER_VENKATAKRISHNAN) {
    const T n = A * A + T(2) * A * Bm;
    const T d = A * A + A * Bm + T(2) * Bm * Bm;
    return n < d ? n * rcp_t(d) : T(1);
  }
  return A < Bm ? A * rcp_t(Bm) : T(1);
}
template <class T>
__device__ __forceinline__ T limiter_diff(int kind, const T* dq, T dmin, T dmax) {
  switch (kind) {
    case E2D_LIMITER_ONE: return T(1);
    case E2D_LIMITER_ZERO: return T(0);
    case E2D_LIMITER_VENKATAKRISHNAN: return limiter_diff_k<E2D_LIMITER_VENKATAKRISHNAN>(dq, dmin, dmax);
    default: return limiter_diff_k<E2D_LIMITER_BARTH_JESPERSEN>(dq, dmin, dmax);
  }
}

// quadCentroid with the reference-rounded moments and one reciprocal.
__device__ __forceinline__ void quad_centroid(double x0, double y0, double x1, double y1,
                                              double x2, double y2, double x3, double y3,
                                              double& xc, double& yc, double& area) {
  double atmp, xt, yt;
  quad_moments(x0, y0, x1, y1, x2, y2, x3, y3, atmp, xt, yt);
  area = 0.5 * atmp;
  if (atmp != 0) {
    const double r = rcp(3.0 * atmp);
    xc = xt * r;
    yc = yt * r;
  } else {
    xc = 0; yc = 0;
  }
}

__device__ __forceinline__ PState<double> W_of_U(const CState<double>& u, double gm1) {
  const double rd = rcp(u.d);
  PState<double> w;
  w.d = u.d; w.u = u.mx * rd; w.v = u.my * rd;
  w.p = gm1 * (u.E - 0.5 * (u.mx * u.mx + u.my * u.my) * rd);
  return w;
}

}  // namespace fm
}  // namespace e2d
