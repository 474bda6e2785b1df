/*
 * e2d_oracle.c — CPU restatement of the CFFC reference's Euler2D path.
 * TEST INFRASTRUCTURE ONLY (see e2d_oracle.h): the checker, never the product.
 *
 * Each function names the reference routine it restates (paths relative to
 * the CFFC source tree).  Floating-point expressions keep the reference's
 * operation order (C++ operator overloads on Euler2D_pState / cState /
 * Vector2D evaluate component-wise, left to right), so with contraction off
 * (-ffp-contract=off) results match the compiled reference bit for bit.
 */
#include "e2d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define HALF 0.5
#define TOLER 0.0000001   /* src_2D/Math/Math.h:52 */
#define NANO 0.000000001  /* src_2D/Math/Math.h:53 */
#define MILLION 1000000.0

typedef struct { double x, y; } vec2;
typedef struct { double d, u, v, p; } pst; /* Euler2D_pState */
typedef struct { double d, mx, my, E; } cst; /* Euler2D_cState */

struct e2d_oracle {
  int nblk, nci, ncj, ng, NCi, NCj, NNi, NNj, ICl, ICu, JCl, JCu;
  e2d_scheme sc;
  double g, gm1, gm1i;
  int *neigh, *bcw, *bce, *bcs, *bcn;
  double *X, *Y, *wow, *woe, *wos, *won;
  double *xc, *yc, *A;                                  /* [nblk][NCj][NCi] */
  double *W, *U, *Uo, *dUdt, *dWdx, *dWdy, *phi, *dt;  /* cell arrays */
  double *dUdt1, *dUdt2;  /* residual slots 1, 2 (dUdt[i][j][1..2], RK4) */
  int frozen, first;      /* limiters frozen; next explicit step is a run's first */
};

static inline double dmin(double x, double y) { return (x < y) ? x : y; } /* Math.h */
static inline double dmax(double x, double y) { return (x > y) ? x : y; }
static inline double sqr(double x) { return x * x; }

#define SC(o, b, j, i) ((((size_t)(b) * (o)->NCj) + (j)) * (o)->NCi + (i))
#define CV(o, b, v, j, i) ((((size_t)(b) * 4 + (v)) * (o)->NCj + (j)) * (o)->NCi + (i))
#define ND(o, b, j, i) ((((size_t)(b) * (o)->NNj) + (j)) * (o)->NNi + (i))

static vec2 node(const e2d_oracle *o, int b, int i, int j) {
  vec2 r = {o->X[ND(o, b, j, i)], o->Y[ND(o, b, j, i)]};
  return r;
}
static vec2 vsub(vec2 a, vec2 b) { vec2 r = {a.x - b.x, a.y - b.y}; return r; }
static vec2 vmid(vec2 a, vec2 b) { vec2 r = {HALF * (a.x + b.x), HALF * (a.y + b.y)}; return r; }
static double vabs(vec2 a) { return sqrt(a.x * a.x + a.y * a.y); }

/* Face geometry, Grid2D_Quad_Block_HO accessors (src_2D/Grid/HO_Grid2DQuad.h:1755-2003). */
static vec2 xfaceE(const e2d_oracle *o, int b, int i, int j) { return vmid(node(o, b, i + 1, j), node(o, b, i + 1, j + 1)); }
static vec2 xfaceW(const e2d_oracle *o, int b, int i, int j) { return vmid(node(o, b, i, j), node(o, b, i, j + 1)); }
static vec2 xfaceN(const e2d_oracle *o, int b, int i, int j) { return vmid(node(o, b, i, j + 1), node(o, b, i + 1, j + 1)); }
static vec2 xfaceS(const e2d_oracle *o, int b, int i, int j) { return vmid(node(o, b, i, j), node(o, b, i + 1, j)); }
static double lfaceN(const e2d_oracle *o, int b, int i, int j) { return vabs(vsub(node(o, b, i, j + 1), node(o, b, i + 1, j + 1))); }
static double lfaceS(const e2d_oracle *o, int b, int i, int j) { return vabs(vsub(node(o, b, i, j), node(o, b, i + 1, j))); }
static double lfaceE(const e2d_oracle *o, int b, int i, int j) { return vabs(vsub(node(o, b, i + 1, j), node(o, b, i + 1, j + 1))); }
static double lfaceW(const e2d_oracle *o, int b, int i, int j) { return vabs(vsub(node(o, b, i, j), node(o, b, i, j + 1))); }
static double perim(const e2d_oracle *o, int b, int i, int j) {
  return lfaceE(o, b, i, j) + lfaceN(o, b, i, j) + lfaceW(o, b, i, j) + lfaceS(o, b, i, j);
}
/* Outward unit normal of the edge from node a to node c (a->c counter-clockwise
 * around the cell): (a.y - c.y, -(a.x - c.x)) / |a - c|, or ihat when the
 * edge is degenerate. */
static vec2 nface(vec2 a, vec2 c, double l, double per) {
  vec2 r = {1.0, 0.0};
  if (l > NANO * per) {
    double n = vabs(vsub(a, c));
    r.x = (a.y - c.y) / n;
    r.y = -(a.x - c.x) / n;
  }
  return r;
}
static vec2 nfaceN(const e2d_oracle *o, int b, int i, int j) {
  return nface(node(o, b, i, j + 1), node(o, b, i + 1, j + 1), lfaceN(o, b, i, j), perim(o, b, i, j));
}
static vec2 nfaceS(const e2d_oracle *o, int b, int i, int j) {
  return nface(node(o, b, i + 1, j), node(o, b, i, j), lfaceS(o, b, i, j), perim(o, b, i, j));
}
static vec2 nfaceE(const e2d_oracle *o, int b, int i, int j) {
  return nface(node(o, b, i + 1, j + 1), node(o, b, i + 1, j), lfaceE(o, b, i, j), perim(o, b, i, j));
}
static vec2 nfaceW(const e2d_oracle *o, int b, int i, int j) {
  return nface(node(o, b, i, j), node(o, b, i, j + 1), lfaceW(o, b, i, j), perim(o, b, i, j));
}

/* quadCentroid (src_2D/Math/Math.h:311-351) on SW, SE, NE, NW in global
 * coordinates (Minimize_Error_Calculation_Of_Geometric_Properties is OFF by
 * default, HO_Grid2DQuad.cc:80). */
static void quad_centroid(vec2 X0, vec2 X1, vec2 X2, vec2 X3, vec2 *c, double *area) {
  double ai, atmp = 0, xtmp = 0, ytmp = 0;
  ai = X3.x * X0.y - X0.x * X3.y; atmp += ai; xtmp += (X0.x + X3.x) * ai; ytmp += (X0.y + X3.y) * ai;
  ai = X0.x * X1.y - X1.x * X0.y; atmp += ai; xtmp += (X1.x + X0.x) * ai; ytmp += (X1.y + X0.y) * ai;
  ai = X1.x * X2.y - X2.x * X1.y; atmp += ai; xtmp += (X2.x + X1.x) * ai; ytmp += (X2.y + X1.y) * ai;
  ai = X2.x * X3.y - X3.x * X2.y; atmp += ai; xtmp += (X3.x + X2.x) * ai; ytmp += (X3.y + X2.y) * ai;
  *area = 0.5 * atmp;
  if (atmp != 0) { c->x = xtmp / (3 * atmp); c->y = ytmp / (3 * atmp); }
}

/* State algebra (src_2D/Euler2D/Euler2DState.h:1033-1110, :1741-1760). */
static pst getW(const e2d_oracle *o, const double *A, int b, int i, int j) {
  pst w = {A[CV(o, b, 0, j, i)], A[CV(o, b, 1, j, i)], A[CV(o, b, 2, j, i)], A[CV(o, b, 3, j, i)]};
  return w;
}
static void putW(const e2d_oracle *o, double *A, int b, int i, int j, pst w) {
  A[CV(o, b, 0, j, i)] = w.d; A[CV(o, b, 1, j, i)] = w.u; A[CV(o, b, 2, j, i)] = w.v; A[CV(o, b, 3, j, i)] = w.p;
}
static cst getU(const e2d_oracle *o, const double *A, int b, int i, int j) {
  cst u = {A[CV(o, b, 0, j, i)], A[CV(o, b, 1, j, i)], A[CV(o, b, 2, j, i)], A[CV(o, b, 3, j, i)]};
  return u;
}
static void putU(const e2d_oracle *o, double *A, int b, int i, int j, cst u) {
  A[CV(o, b, 0, j, i)] = u.d; A[CV(o, b, 1, j, i)] = u.mx; A[CV(o, b, 2, j, i)] = u.my; A[CV(o, b, 3, j, i)] = u.E;
}
static cst U_of_W(const e2d_oracle *o, pst w) {
  cst u;
  u.d = w.d; u.mx = w.d * w.u; u.my = w.d * w.v;
  u.E = w.p * o->gm1i + HALF * w.d * (w.u * w.u + w.v * w.v);
  return u;
}
static pst W_of_U(const e2d_oracle *o, cst u) {
  pst w;
  w.d = u.d; w.u = u.mx / u.d; w.v = u.my / u.d;
  w.p = o->gm1 * (u.E - HALF * (u.mx * u.mx + u.my * u.my) / u.d);
  return w;
}
static double a_of(const e2d_oracle *o, pst w) { return sqrt(o->g * w.p / w.d); }
static double h_of(const e2d_oracle *o, pst w) { return o->g * w.p / (o->gm1 * w.d) + HALF * (w.u * w.u + w.v * w.v); }
static double Ht_of(const e2d_oracle *o, pst w) { return o->g * o->gm1i * w.p + HALF * w.d * (w.u * w.u + w.v * w.v); }
static double e_of_U(cst u) { return u.E / u.d - HALF * (u.mx * u.mx + u.my * u.my) / sqr(u.d); }

/* Reflect (src_2D/Euler2D/Euler2DState.cc:751-787). */
static pst reflect(pst w, vec2 n) {
  double c = n.x, s = n.y, ur, vr;
  pst r;
  ur = w.u * c + w.v * s;
  vr = -w.u * s + w.v * c;
  ur = -ur;
  r.d = w.d; r.u = ur * c - vr * s; r.v = ur * s + vr * c; r.p = w.p;
  return r;
}

/* BC_Characteristic_Pressure (src_2D/Euler2D/Euler2DState.cc:1383-1450). */
static pst bc_char_pressure(const e2d_oracle *o, pst wi, pst wo, vec2 n) {
  double c = n.x, s = n.y, mi, db, ub, vb, pb, ab, ubr, vbr;
  pst ir, orr, r;
  ir.d = wi.d; ir.u = wi.u * c + wi.v * s; ir.v = -wi.u * s + wi.v * c; ir.p = wi.p;
  orr.d = wo.d; orr.u = wo.u * c + wo.v * s; orr.v = -wo.u * s + wo.v * c; orr.p = wo.p;
  mi = ir.u / a_of(o, ir);
  if (mi >= 1.0) {
    db = ir.d; ubr = ir.u; vbr = ir.v; pb = ir.p;
  } else if (mi >= 0.0) {
    pb = orr.p;
    db = ir.d * pow(pb / ir.p, 1.0 / o->g);
    ab = sqrt(o->g * pb / db);
    ubr = ir.u + 2.0 * (a_of(o, ir) - ab) * o->gm1i;
    vbr = ir.v;
  } else if (mi >= -1.0) {
    pb = orr.p; db = orr.d; vbr = orr.v;
    ab = sqrt(o->g * pb / db);
    ubr = ir.u + 2.0 * (a_of(o, ir) - ab) * o->gm1i;
  } else {
    db = orr.d; ubr = orr.u; vbr = orr.v; pb = orr.p;
  }
  ub = ubr * c - vbr * s;
  vb = ubr * s + vbr * c;
  r.d = db; r.u = ub; r.v = vb; r.p = pb;
  return r;
}

/* HartenFixPos / HartenFixNeg (src_2D/CFD/CFD.cc:605-646). */
static double harten_delta(double la, double ll, double lr) {
  double delta = dmax(0.0, 2.0 * (lr - ll));
  if (fabs(la) > delta || delta < TOLER) delta = 0.0;
  else delta = HALF * (sqr(la) / delta + delta) - fabs(la);
  return delta;
}
static double harten_pos(double la, double ll, double lr) {
  double delta = harten_delta(la, ll, lr);
  return HALF * (la + fabs(la) + delta);
}
static double harten_neg(double la, double ll, double lr) {
  double delta = harten_delta(la, ll, lr);
  return HALF * (la - fabs(la) - delta);
}

/* FluxRoe_x (src_2D/Euler2D/Euler2DState.cc:2311-2354) with RoeAverage
 * (:654-685), lambda_x, lp_x, rc_x, Fx (Euler2DState.h:2153, 2968, 2702, 1845). */
static cst flux_roe_x(const e2d_oracle *o, pst wl, pst wr) {
  const double g = o->g, gm1 = o->gm1;
  double hl, hr, sdl, sdr, da, ua, va, ha, aa2, pa;
  double dW[4], ll[4], lr[4], la[4], ws[4], cl, cr, ca;
  cst F;
  pst wa, wup;
  int k;
  hl = h_of(o, wl); hr = h_of(o, wr);
  sdl = sqrt(wl.d); sdr = sqrt(wr.d);
  da = sdl * sdr;
  ua = (sdl * wl.u + sdr * wr.u) / (sdl + sdr);
  va = (sdl * wl.v + sdr * wr.v) / (sdl + sdr);
  ha = (sdl * hl + sdr * hr) / (sdl + sdr);
  aa2 = gm1 * (ha - HALF * (sqr(ua) + sqr(va)));
  pa = da * aa2 / g;
  wa.d = da; wa.u = ua; wa.v = va; wa.p = pa;
  dW[0] = wr.d - wl.d; dW[1] = wr.u - wl.u; dW[2] = wr.v - wl.v; dW[3] = wr.p - wl.p;
  cl = a_of(o, wl); cr = a_of(o, wr); ca = a_of(o, wa);
  ll[0] = wl.u - cl; ll[1] = wl.u; ll[2] = wl.u; ll[3] = wl.u + cl;
  lr[0] = wr.u - cr; lr[1] = wr.u; lr[2] = wr.u; lr[3] = wr.u + cr;
  la[0] = wa.u - ca; la[1] = wa.u; la[2] = wa.u; la[3] = wa.u + ca;
  if (wa.u >= 0.0) {
    wup = wl;
    ws[0] = harten_neg(la[0], ll[0], lr[0]);
    ws[1] = HALF * (la[1] - fabs(la[1]));
    ws[2] = HALF * (la[2] - fabs(la[2]));
    ws[3] = harten_neg(la[3], ll[3], lr[3]);
  } else {
    wup = wr;
    ws[0] = harten_pos(la[0], ll[0], lr[0]);
    ws[1] = HALF * (la[1] + fabs(la[1]));
    ws[2] = HALF * (la[2] + fabs(la[2]));
    ws[3] = harten_pos(la[3], ll[3], lr[3]);
  }
  F.d = wup.d * wup.u;
  F.mx = wup.d * sqr(wup.u) + wup.p;
  F.my = wup.d * wup.u * wup.v;
  F.E = wup.u * Ht_of(o, wup);
  for (k = 0; k < 4; ++k) {
    double lp[4], rc[4], coef, c = ca;
    if (!((wa.u >= 0.0) ? (ws[k] < 0.0) : (ws[k] > 0.0))) continue;
    switch (k) {
      case 0:
        lp[0] = 0.0; lp[1] = -HALF * wa.d / c; lp[2] = 0.0; lp[3] = HALF / sqr(c);
        rc[0] = 1.0; rc[1] = wa.u - c; rc[2] = wa.v; rc[3] = h_of(o, wa) - wa.u * c;
        break;
      case 1:
        lp[0] = 1.0; lp[1] = 0.0; lp[2] = 0.0; lp[3] = -1.0 / (g * wa.p / wa.d);
        rc[0] = 1.0; rc[1] = wa.u; rc[2] = wa.v; rc[3] = HALF * (wa.u * wa.u + wa.v * wa.v);
        break;
      case 2:
        lp[0] = 0.0; lp[1] = 0.0; lp[2] = 1.0; lp[3] = 0.0;
        rc[0] = 0.0; rc[1] = 0.0; rc[2] = wa.d; rc[3] = wa.d * wa.v;
        break;
      default:
        lp[0] = 0.0; lp[1] = HALF * wa.d / c; lp[2] = 0.0; lp[3] = HALF / sqr(c);
        rc[0] = 1.0; rc[1] = wa.u + c; rc[2] = wa.v; rc[3] = h_of(o, wa) + wa.u * c;
        break;
    }
    /* pState inner product: d*d + (v.v) + p*p */
    coef = ws[k] * (lp[0] * dW[0] + (lp[1] * dW[1] + lp[2] * dW[2]) + lp[3] * dW[3]);
    if (wa.u >= 0.0) {
      F.d += coef * rc[0]; F.mx += coef * rc[1]; F.my += coef * rc[2]; F.E += coef * rc[3];
    } else {
      F.d -= coef * rc[0]; F.mx -= coef * rc[1]; F.my -= coef * rc[2]; F.E -= coef * rc[3];
    }
  }
  return F;
}

/* FluxRoe_n (src_2D/Euler2D/Euler2DState.cc:2446-2495). */
static cst flux_roe_n(const e2d_oracle *o, pst wl, pst wr, vec2 n) {
  double c = n.x, s = n.y;
  pst lr, rr;
  cst Fr, F;
  lr.d = wl.d; lr.u = wl.u * c + wl.v * s; lr.v = -wl.u * s + wl.v * c; lr.p = wl.p;
  rr.d = wr.d; rr.u = wr.u * c + wr.v * s; rr.v = -wr.u * s + wr.v * c; rr.p = wr.p;
  Fr = flux_roe_x(o, lr, rr);
  F.d = Fr.d;
  F.mx = Fr.mx * c - Fr.my * s;
  F.my = Fr.mx * s + Fr.my * c;
  F.E = Fr.E;
  return F;
}

/* ---- the other flux functions of i_Flux_Function (Euler2DQuad.cc:968-1003) ----
 * All evaluate an x-direction flux between states rotated into the frame of
 * the face normal and rotate the momentum flux back (FluxXxx_n). */

static cst Fx_of(const e2d_oracle *o, pst w) { /* Euler2D_pState::Fx, Euler2DState.h:1845 */
  cst F;
  F.d = w.d * w.u; F.mx = w.d * sqr(w.u) + w.p; F.my = w.d * w.u * w.v; F.E = w.u * Ht_of(o, w);
  return F;
}
static pst mkp(double d, double u, double v, double p) { pst w; w.d = d; w.u = u; w.v = v; w.p = p; return w; }
static cst cdiff(cst a, cst b) { cst r; r.d = a.d - b.d; r.mx = a.mx - b.mx; r.my = a.my - b.my; r.E = a.E - b.E; return r; }

/* RoeAverage (src_2D/Euler2D/Euler2DState.cc:654-683). */
static pst roe_average(const e2d_oracle *o, pst wl, pst wr) {
  double hl = h_of(o, wl), hr = h_of(o, wr), sdl = sqrt(wl.d), sdr = sqrt(wr.d), ha, aa2;
  pst wa;
  wa.d = sdl * sdr;
  wa.u = (sdl * wl.u + sdr * wr.u) / (sdl + sdr);
  wa.v = (sdl * wl.v + sdr * wr.v) / (sdl + sdr);
  ha = (sdl * hl + sdr * hr) / (sdl + sdr);
  aa2 = o->gm1 * (ha - HALF * (sqr(wa.u) + sqr(wa.v)));
  wa.p = wa.d * aa2 / o->g;
  return wa;
}

/* Riemann_x (Euler2DState.cc:245-449): exact solver, Newton-Raphson on the
 * intermediate velocity, state on x/t = 0. */
static pst riemann_x(const e2d_oracle *o, pst wl, pst wr) {
  const double g = o->g, gm1 = o->gm1;
  double al = a_of(o, wl), ar = a_of(o, wr), CL, CR, Z, um, pm, aml = 0.0, amr = 0.0;
  double msl = 0.0, msr = 0.0, pml = 0.0, pmr = 0.0, dpl, dpr;
  int it;
  CL = wl.u + 2.0 * al / gm1;
  CR = wr.u - 2.0 * ar / gm1;
  if (CL - CR <= 0.0) return mkp(0.0, 0.0, 0.0, 0.0);
  Z = (ar / al) * pow((wl.p / wr.p), HALF * gm1 / g);
  um = (CL * Z + CR) / (1.0 + Z);
  if (um >= wl.u && um <= wr.u) {
    if (um >= 0.0) {
      aml = al - HALF * gm1 * (um - wl.u);
      pm = wl.p * pow((aml / al), 2.0 * g / gm1);
      if (wl.u - al >= 0.0) return wl;
      if (um - aml <= 0.0) return mkp(g * pm / sqr(aml), um, wl.v, pm);
      um = (gm1 * wl.u + 2.0 * al) / (g + 1.0);
      pm = wl.p * pow((um / al), 2.0 * g / gm1);
      return mkp(g * pm / sqr(um), um, wl.v, pm);
    }
    amr = ar + HALF * gm1 * (um - wr.u);
    pm = wr.p * pow((amr / ar), 2.0 * g / gm1);
    if (wr.u + ar <= 0.0) return wr;
    if (um + amr >= 0.0) return mkp(g * pm / sqr(amr), um, wr.v, pm);
    um = (gm1 * wr.u - 2.0 * ar) / (g + 1.0);
    pm = wr.p * pow((-um / ar), 2.0 * g / gm1);
    return mkp(g * pm / sqr(um), um, wr.v, pm);
  }
  for (it = 1;; ++it) {
    if (um < wl.u) {
      msl = (g + 1.0) * (um - wl.u) / (4.0 * al);
      msl = msl - sqrt(1.0 + sqr(msl));
      pml = wl.p * (1.0 + g * (um - wl.u) * msl / al);
      dpl = 2.0 * g * wl.p * (msl * msl * msl) / (al * (1.0 + sqr(msl)));
    } else {
      aml = al - HALF * gm1 * (um - wl.u);
      pml = wl.p * pow((aml / al), 2.0 * g / gm1);
      dpl = -g * pml / aml;
    }
    if (um > wr.u) {
      msr = (g + 1.0) * (um - wr.u) / (4.0 * ar);
      msr = msr + sqrt(1.0 + sqr(msr));
      pmr = wr.p * (1.0 + g * (um - wr.u) * msr / ar);
      dpr = 2.0 * g * wr.p * (msr * msr * msr) / (ar * (1.0 + sqr(msr)));
    } else {
      amr = ar + HALF * gm1 * (um - wr.u);
      pmr = wr.p * pow((amr / ar), 2.0 * g / gm1);
      dpr = g * pmr / amr;
    }
    if (fabs(1.0 - pml / pmr) <= TOLER) break;
    if (it > 10) break;
    um = um - (pml - pmr) / (dpl - dpr);
  }
  pm = HALF * (pml + pmr);
  if (um >= 0.0) {
    if (um < wl.u) {
      aml = al * sqrt(((g + 1.0) + gm1 * pm / wl.p) / ((g + 1.0) + gm1 * wl.p / pm));
      if (wl.u + msl * al >= 0.0) return wl;
      return mkp(g * pm / sqr(aml), um, wl.v, pm);
    }
    if (wl.u - al >= 0.0) return wl;
    if (um - aml <= 0.0) return mkp(g * pm / sqr(aml), um, wl.v, pm);
    um = (gm1 * wl.u + 2.0 * al) / (g + 1.0);
    pm = wl.p * pow((um / al), 2.0 * g / gm1);
    return mkp(g * pm / sqr(um), um, wl.v, pm);
  }
  if (um > wr.u) {
    amr = ar * sqrt(((g + 1.0) + gm1 * pm / wr.p) / ((g + 1.0) + gm1 * wr.p / pm));
    if (wr.u + msr * ar <= 0.0) return wr;
    return mkp(g * pm / sqr(amr), um, wr.v, pm);
  }
  if (wr.u + ar <= 0.0) return wr;
  if (um + amr >= 0.0) return mkp(g * pm / sqr(amr), um, wr.v, pm);
  um = (gm1 * wr.u - 2.0 * ar) / (g + 1.0);
  pm = wr.p * pow((-um / ar), 2.0 * g / gm1);
  return mkp(g * pm / sqr(um), um, wr.v, pm);
}

/* FluxRusanov_x (Euler2DState.cc:2673-2713) with HartenFixAbs (CFD.cc:655-669). */
static cst flux_rusanov_x(const e2d_oracle *o, pst wl, pst wr) {
  pst wa = roe_average(o, wl, wr);
  cst fl = Fx_of(o, wl), fr = Fx_of(o, wr), dU = cdiff(U_of_W(o, wr), U_of_W(o, wl)), F;
  double cl = a_of(o, wl), cr = a_of(o, wr), ca = a_of(o, wa), ws[4], m;
  int k;
  ws[0] = fabs(wa.u - ca) + harten_delta(wa.u - ca, wl.u - cl, wr.u - cr);
  ws[1] = fabs(wa.u);
  ws[2] = fabs(wa.u);
  ws[3] = fabs(wa.u + ca) + harten_delta(wa.u + ca, wl.u + cl, wr.u + cr);
  m = ws[0];
  for (k = 1; k < 4; ++k) m = dmax(m, ws[k]);
  F.d = HALF * (fl.d + fr.d); F.mx = HALF * (fl.mx + fr.mx);
  F.my = HALF * (fl.my + fr.my); F.E = HALF * (fl.E + fr.E);
  F.d -= HALF * m * dU.d; F.mx -= HALF * m * dU.mx; F.my -= HALF * m * dU.my; F.E -= HALF * m * dU.E;
  return F;
}

/* FluxHLLE_x (Euler2DState.cc:2921-2963); linde != 0: FluxLinde_x (:3321-3383). */
static cst flux_hll_x(const e2d_oracle *o, pst wl, pst wr, int linde) {
  pst wa = roe_average(o, wl, wr);
  double ca = a_of(o, wa), sl, sr, k, alpha, du, sm, da;
  cst fl, fr, dU, dF, F;
  sl = dmin(wl.u - a_of(o, wl), wa.u - ca);
  sr = dmax(wr.u + a_of(o, wr), wa.u + ca);
  if (sl >= 0.0) return Fx_of(o, wl);
  if (sr <= 0.0) return Fx_of(o, wr);
  fl = Fx_of(o, wl); fr = Fx_of(o, wr);
  dU = cdiff(U_of_W(o, wr), U_of_W(o, wl));
  k = sl * sr;
  if (linde) {
    sm = wa.u; da = wa.d;
    du = fabs(dU.d) / da + fabs(dU.mx) / (da * ca) + fabs(dU.my) / (da * ca) + fabs(dU.E) / (da * ca * ca);
    if (du <= TOLER) {
      alpha = 0.0;
    } else {
      du = 1.0 / du;
      dF = cdiff(fr, fl);
      dF.d = dF.d - sm * dU.d; dF.mx = dF.mx - sm * dU.mx; dF.my = dF.my - sm * dU.my; dF.E = dF.E - sm * dU.E;
      alpha = 1.0 - (fabs(dF.d) / (da * ca) + fabs(dF.mx) / (da * ca * ca) + fabs(dF.my) / (da * ca * ca) +
                     fabs(dF.E) / (da * ca * ca * ca)) * du;
      alpha = dmax(0.0, alpha);
    }
    k = k * (1.0 - (1.0 - dmax(sm / sr, sm / sl)) * alpha);
  }
  F.d = ((sr * fl.d - sl * fr.d) + k * dU.d) / (sr - sl);
  F.mx = ((sr * fl.mx - sl * fr.mx) + k * dU.mx) / (sr - sl);
  F.my = ((sr * fl.my - sl * fr.my) + k * dU.my) / (sr - sl);
  F.E = ((sr * fl.E - sl * fr.E) + k * dU.E) / (sr - sl);
  return F;
}

/* FluxHLLC_x (Euler2DState.cc:3630-3694). */
static cst flux_hllc_x(const e2d_oracle *o, pst wl, pst wr) {
  const double g = o->g, gm1 = o->gm1;
  double al = a_of(o, wl), ar = a_of(o, wr), CL, CR, Z, um, aml, amr, pm, ql, qr, sl, sr, sk, f;
  pst w;
  cst uk, fk, us, F;
  CL = wl.u + 2.0 * al / gm1;
  CR = wr.u - 2.0 * ar / gm1;
  Z = (ar / al) * pow((wl.p / wr.p), HALF * gm1 / g);
  um = (CL * Z + CR) / (1.0 + Z);
  aml = al - HALF * gm1 * (um - wl.u);
  pm = wl.p * pow((aml / al), 2.0 * g / gm1);
  amr = ar + HALF * gm1 * (um - wr.u);
  pm = HALF * (pm + wr.p * pow((amr / ar), 2.0 * g / gm1));
  ql = (pm / wl.p <= 1.0) ? 1.0 : sqrt(1.0 + HALF * ((g + 1.0) / g) * (pm / wl.p));
  sl = wl.u - ql * al;
  qr = (pm / wr.p <= 1.0) ? 1.0 : sqrt(1.0 + HALF * ((g + 1.0) / g) * (pm / wr.p));
  sr = wr.u + qr * ar;
  if (sl >= 0.0) return Fx_of(o, wl);
  if (sr <= 0.0) return Fx_of(o, wr);
  if (um >= 0.0) { w = wl; sk = sl; } else { w = wr; sk = sr; }
  uk = U_of_W(o, w); fk = Fx_of(o, w);
  f = (sk - w.u) / (sk - um);
  us.d = w.d * f;
  us.mx = (w.d * um) * f;
  us.my = (w.d * w.v) * f;
  us.E = (uk.E + w.d * (um - w.u) * (um + w.p / (w.d * (sk - w.u)))) * f;
  F.d = fk.d + sk * (us.d - uk.d);
  F.mx = fk.mx + sk * (us.mx - uk.mx);
  F.my = fk.my + sk * (us.my - uk.my);
  F.E = fk.E + sk * (us.E - uk.E);
  return F;
}

/* FluxVanLeer (Euler2DState.cc:3862-3903). */
static cst flux_vanleer_x(const e2d_oracle *o, pst wl, pst wr) {
  const double g = o->g, gm1 = o->gm1;
  cst fl, fr, F;
  double M, a, m;
  /* Euler2D_cState() defaults: only a NaN Mach number leaves them */
  fl.d = fr.d = 1.225; fl.mx = fr.mx = fl.my = fr.my = 0.0; fl.E = fr.E = 101325.0 / (1.4 - 1.0);
  M = wl.u / a_of(o, wl);
  if (M < -1.0) {
    fl.d = fl.mx = fl.my = fl.E = 0.0;
  } else if (fabs(M) <= 1.0) {
    a = a_of(o, wl);
    m = 0.25 * wl.d * a * sqr(1.0 + M);
    fl.d = m;
    fl.mx = m * ((2.0 * a / g) * (HALF * gm1 * M + 1.0));
    fl.my = m * wl.v;
    fl.E = m * ((2.0 * (g * wl.p / wl.d) / (g * g - 1.0)) * sqr(HALF * gm1 * M + 1.0) + HALF * sqr(wl.v));
  } else if (M > 1.0) {
    fl = Fx_of(o, wl);
  }
  M = wr.u / a_of(o, wr);
  if (-M < -1.0) {
    fr.d = fr.mx = fr.my = fr.E = 0.0;
  } else if (fabs(M) <= 1.0) {
    a = a_of(o, wr);
    m = -0.25 * wr.d * a * sqr(1.0 - M);
    fr.d = m;
    fr.mx = m * ((2.0 * a / g) * (HALF * gm1 * M - 1.0));
    fr.my = m * wr.v;
    fr.E = m * ((2.0 * (g * wr.p / wr.d) / (g * g - 1.0)) * sqr(HALF * gm1 * M - 1.0) + HALF * sqr(wr.v));
  } else if (-M > 1.0) {
    fr = Fx_of(o, wr);
  }
  F.d = fl.d + fr.d; F.mx = fl.mx + fr.mx; F.my = fl.my + fr.my; F.E = fl.E + fr.E;
  return F;
}

/* FluxAUSM (Euler2DState.cc:4056-4106). */
static cst flux_ausm_x(const e2d_oracle *o, pst wl, pst wr) {
  double al = a_of(o, wl), Ml = wl.u / al, ar = a_of(o, wr), Mr = wr.u / ar;
  double Mp, pp, Mn, pn, Mh, ph, Hl, Hr;
  cst F;
  if (fabs(Ml) <= 1.0) { Mp = 0.25 * sqr(Ml + 1.0); pp = 0.25 * wl.p * sqr(Ml + 1.0) * (2.0 - Ml); }
  else { Mp = 0.5 * (Ml + fabs(Ml)); pp = 0.5 * wl.p * (Ml + fabs(Ml)) / Ml; }
  if (fabs(Mr) <= 1.0) { Mn = -0.25 * sqr(Mr - 1.0); pn = 0.25 * wr.p * sqr(Mr - 1.0) * (2.0 + Mr); }
  else { Mn = 0.5 * (Mr - fabs(Mr)); pn = 0.5 * wr.p * (Mr - fabs(Mr)) / Mr; }
  Mh = Mp + Mn; ph = pp + pn;
  Hl = Ht_of(o, wl); Hr = Ht_of(o, wr);
  F.d = 0.5 * Mh * (wl.d * al + wr.d * ar);
  F.mx = 0.5 * Mh * (wl.d * al * wl.u + wr.d * ar * wr.u);
  F.my = 0.5 * Mh * (wl.d * al * wl.v + wr.d * ar * wr.v);
  F.E = 0.5 * Mh * (al * Hl + ar * Hr);
  F.d -= 0.5 * fabs(Mh) * (wr.d * ar - wl.d * al);
  F.mx -= 0.5 * fabs(Mh) * (wr.d * ar * wr.u - wl.d * al * wl.u);
  F.my -= 0.5 * fabs(Mh) * (wr.d * ar * wr.v - wl.d * al * wl.v);
  F.E -= 0.5 * fabs(Mh) * (ar * Hr - al * Hl);
  F.mx += ph;
  return F;
}

/* FluxAUSMplus (Euler2DState.cc:4170-4231). */
static cst flux_ausmplus_x(const e2d_oracle *o, pst wl, pst wr) {
  const double beta = 0.125, alpha = 0.1875;
  double ah = HALF * (a_of(o, wl) + a_of(o, wr)), Ml = wl.u / ah, Mr = wr.u / ah;
  double Mp, pp, Mn, pn, Mh, ph, Hl, Hr;
  cst F;
  if (fabs(Ml) < 1.0) {
    Mp = 0.25 * sqr(Ml + 1.0) + beta * sqr(Ml * Ml - 1.0);
    pp = (0.25 * sqr(Ml + 1.0) * (2.0 - Ml) + alpha * Ml * sqr(Ml * Ml - 1.0)) * wl.p;
  } else {
    Mp = 0.5 * (Ml + fabs(Ml));
    pp = 0.5 * wl.p * (1.0 + ((Ml < 0.0) ? -1.0 : 1.0));
  }
  if (fabs(Mr) < 1.0) {
    Mn = -0.25 * sqr(Mr - 1.0) - beta * sqr(Mr * Mr - 1.0);
    pn = (0.25 * sqr(Mr - 1.0) * (2.0 + Mr) - alpha * Mr * sqr(Mr * Mr - 1.0)) * wr.p;
  } else {
    Mn = 0.5 * (Mr - fabs(Mr));
    pn = 0.5 * wr.p * (1.0 - ((Mr < 0.0) ? -1.0 : 1.0));
  }
  Mh = Mp + Mn; ph = pp + pn;
  Hl = Ht_of(o, wl); Hr = Ht_of(o, wr);
  F.d = 0.5 * Mh * (wl.d + wr.d);
  F.mx = 0.5 * Mh * (wl.d * wl.u + wr.d * wr.u);
  F.my = 0.5 * Mh * (wl.d * wl.v + wr.d * wr.v);
  F.E = 0.5 * Mh * (Hl + Hr);
  F.d -= 0.5 * fabs(Mh) * (wr.d - wl.d);
  F.mx -= 0.5 * fabs(Mh) * (wr.d * wr.u - wl.d * wl.u);
  F.my -= 0.5 * fabs(Mh) * (wr.d * wr.v - wl.d * wl.v);
  F.E -= 0.5 * fabs(Mh) * (Hr - Hl);
  F.d *= ah; F.mx *= ah; F.my *= ah; F.E *= ah;
  F.mx += ph;
  return F;
}

/* Face flux of the scheme's i_Flux_Function (dispatch of Euler2DQuad.cc:968-1003). */
static cst face_flux_n(const e2d_oracle *o, pst wl, pst wr, vec2 n) {
  double c = n.x, s = n.y;
  pst lr, rr;
  cst Fr, F;
  if (o->sc.flux == E2D_FLUX_ROE) return flux_roe_n(o, wl, wr, n);
  lr.d = wl.d; lr.u = wl.u * c + wl.v * s; lr.v = -wl.u * s + wl.v * c; lr.p = wl.p;
  rr.d = wr.d; rr.u = wr.u * c + wr.v * s; rr.v = -wr.u * s + wr.v * c; rr.p = wr.p;
  switch (o->sc.flux) {
    case E2D_FLUX_GODUNOV: Fr = Fx_of(o, riemann_x(o, lr, rr)); break;
    case E2D_FLUX_RUSANOV: Fr = flux_rusanov_x(o, lr, rr); break;
    case E2D_FLUX_HLLE: Fr = flux_hll_x(o, lr, rr, 0); break;
    case E2D_FLUX_LINDE: Fr = flux_hll_x(o, lr, rr, 1); break;
    case E2D_FLUX_HLLC: Fr = flux_hllc_x(o, lr, rr); break;
    case E2D_FLUX_VANLEER: Fr = flux_vanleer_x(o, lr, rr); break;
    case E2D_FLUX_AUSM: Fr = flux_ausm_x(o, lr, rr); break;
    default: Fr = flux_ausmplus_x(o, lr, rr); break;
  }
  F.d = Fr.d;
  F.mx = Fr.mx * c - Fr.my * s;
  F.my = Fr.mx * s + Fr.my * c;
  F.E = Fr.E;
  return F;
}

/* Limiter_BarthJespersen / Limiter_Venkatakrishnan (src_2D/CFD/CFD.cc:696-751). */
static double limiter(int kind, const double *uq, double u0, double umin, double umax) {
  double phi = 1.0, y;
  int q;
  if (kind == E2D_LIMITER_ONE) return 1.0;
  if (kind == E2D_LIMITER_ZERO) return 0.0;
  for (q = 0; q < 4; ++q) {
    if (uq[q] - u0 > TOLER) {
      y = (umax - u0) / (uq[q] - u0);
      phi = (kind == E2D_LIMITER_VENKATAKRISHNAN) ? dmin(phi, (sqr(y) + 2.0 * y) / (sqr(y) + y + 2.0))
                                                  : dmin(phi, dmin(1.0, y));
    } else if (uq[q] - u0 < -TOLER) {
      y = (umin - u0) / (uq[q] - u0);
      phi = (kind == E2D_LIMITER_VENKATAKRISHNAN) ? dmin(phi, (sqr(y) + 2.0 * y) / (sqr(y) + y + 2.0))
                                                  : dmin(phi, dmin(1.0, y));
    } else {
      phi = dmin(phi, 1.0);
    }
  }
  return phi;
}

/* Least-squares stencil selection (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:3692-3990).
 * Returns n_pts and fills the neighbour offsets. */
static int lsq_stencil(const e2d_oracle *o, int b, int i, int j, int *ii, int *jj) {
  const int Ng = o->ng, ICl = o->ICl, ICu = o->ICu, JCl = o->JCl, JCu = o->JCu;
  int n = 0;
#define P(a, c) (ii[n] = (a), jj[n] = (c), ++n)
  const int bcw = o->bcw[(size_t)b * o->NCj + j], bce = o->bce[(size_t)b * o->NCj + j];
  const int bcs = o->bcs[(size_t)b * o->NCi + i], bcn = o->bcn[(size_t)b * o->NCi + i];
#define EXTRAP(t) ((t) == E2D_BC_PERIODIC || (t) == E2D_BC_CONSTANT_EXTRAPOLATION || (t) == 4002 || (t) == E2D_BC_CHARACTERISTIC)
  if (i == ICl - Ng || i == ICu + Ng || j == JCl - Ng || j == JCu + Ng) return 0;
  if (i == ICl - Ng + 1 && bcw != E2D_BC_NONE) {
    if (j == JCl - Ng + 1 || j == JCu + Ng - 1) return 0;
    if (EXTRAP(bcw)) {
      if (j == JCl) { P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1); }
      else if (j == JCu) { P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); }
      else { P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1); }
    } else {
      if (j == JCl) { P(i+1,j); P(i,j+1); P(i+1,j+1); }
      else if (j == JCu) { P(i,j-1); P(i+1,j-1); P(i+1,j); }
      else { P(i,j-1); P(i+1,j-1); P(i+1,j); P(i,j+1); P(i+1,j+1); }
    }
  } else if (i == ICu + Ng - 1 && bce != E2D_BC_NONE) {
    if (j == JCl - Ng + 1 || j == JCu + Ng - 1) return 0;
    if (EXTRAP(bce)) {
      if (j == JCl) { P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1); }
      else if (j == JCu) { P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); }
      else { P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1); }
    } else {
      if (j == JCl) { P(i-1,j); P(i-1,j+1); P(i,j+1); }
      else if (j == JCu) { P(i-1,j-1); P(i,j-1); P(i-1,j); }
      else { P(i-1,j-1); P(i,j-1); P(i-1,j); P(i-1,j+1); P(i,j+1); }
    }
  } else if (j == JCl - Ng + 1 && bcs != E2D_BC_NONE) {
    if (i == ICl - Ng + 1 || i == ICu + Ng - 1) return 0;
    if (EXTRAP(bcs)) {
      if (i == ICl) { P(i,j-1); P(i+1,j-1); P(i+1,j); P(i,j+1); P(i+1,j+1); }
      else if (i == ICu) { P(i-1,j-1); P(i,j-1); P(i-1,j); P(i-1,j+1); P(i,j+1); }
      else { P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1); }
    } else {
      if (i == ICl) { P(i+1,j); P(i,j+1); P(i+1,j+1); }
      else if (i == ICu) { P(i-1,j); P(i-1,j+1); P(i,j+1); }
      else { P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1); }
    }
  } else if (j == JCu + Ng - 1 && bcn != E2D_BC_NONE) {
    if (i == ICl - Ng + 1 || i == ICu + Ng - 1) return 0;
    if (EXTRAP(bcn)) {
      if (i == ICl) { P(i,j-1); P(i+1,j-1); P(i+1,j); P(i,j+1); P(i+1,j+1); }
      else if (i == ICu) { P(i-1,j-1); P(i,j-1); P(i-1,j); P(i-1,j+1); P(i,j+1); }
      else { P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1); }
    } else {
      if (i == ICl) { P(i,j-1); P(i+1,j-1); P(i+1,j); }
      else if (i == ICu) { P(i-1,j-1); P(i,j-1); P(i-1,j); }
      else { P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); }
    }
  } else {
    P(i-1,j-1); P(i,j-1); P(i+1,j-1); P(i-1,j); P(i+1,j); P(i-1,j+1); P(i,j+1); P(i+1,j+1);
  }
#undef P
#undef EXTRAP
  return n;
}

/* Linear_Reconstruction_LeastSquares for one cell
 * (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:3678-4087). */
static void lsq_cell(e2d_oracle *o, int b, int i, int j) {
  int ii[8], jj[8], n, n2, v, q;
  const size_t c = SC(o, b, j, i);
  n = lsq_stencil(o, b, i, j, ii, jj);
  if (n > 0) {
    double DUDx[4] = {0, 0, 0, 0}, DUDy[4] = {0, 0, 0, 0}, DxDx = 0, DxDy = 0, DyDy = 0, det;
    double dWx[4], dWy[4];
    for (n2 = 0; n2 < n; ++n2) {
      const size_t s = SC(o, b, jj[n2], ii[n2]);
      const double dx = o->xc[s] - o->xc[c], dy = o->yc[s] - o->yc[c];
      for (v = 0; v < 4; ++v) {
        const double DU = o->W[CV(o, b, v, jj[n2], ii[n2])] - o->W[CV(o, b, v, j, i)];
        DUDx[v] += DU * dx;
        DUDy[v] += DU * dy;
      }
      DxDx += dx * dx; DxDy += dx * dy; DyDy += dy * dy;
    }
    for (v = 0; v < 4; ++v) { DUDx[v] = DUDx[v] / (double)n; DUDy[v] = DUDy[v] / (double)n; }
    DxDx = DxDx / (double)n; DxDy = DxDy / (double)n; DyDy = DyDy / (double)n;
    det = DxDx * DyDy - DxDy * DxDy;
    for (v = 0; v < 4; ++v) {
      dWx[v] = (DUDx[v] * DyDy - DUDy[v] * DxDy) / det;
      dWy[v] = (DUDy[v] * DxDx - DUDx[v] * DxDy) / det;
      o->dWdx[CV(o, b, v, j, i)] = dWx[v];
      o->dWdy[CV(o, b, v, j, i)] = dWy[v];
    }
    {
      vec2 xf[4];
      xf[0] = xfaceE(o, b, i, j); xf[1] = xfaceW(o, b, i, j);
      xf[2] = xfaceN(o, b, i, j); xf[3] = xfaceS(o, b, i, j);
      for (v = 0; v < 4; ++v) {
        const double u0 = o->W[CV(o, b, v, j, i)];
        double umin = u0, umax = u0, uq[4];
        for (n2 = 0; n2 < n; ++n2) {
          const double w = o->W[CV(o, b, v, jj[n2], ii[n2])];
          umin = dmin(umin, w);
          umax = dmax(umax, w);
        }
        for (q = 0; q < 4; ++q) {
          const double dx = xf[q].x - o->xc[c], dy = xf[q].y - o->yc[c];
          uq[q] = u0 + dWx[v] * dx + dWy[v] * dy;
        }
        /* Freeze_Limiter: a frozen block keeps its stored phi
           (Linear_Reconstruction_LeastSquares, Euler2DQuadSingleBlock.cc:3572) */
        if (!o->frozen) o->phi[CV(o, b, v, j, i)] = limiter(o->sc.limiter, uq, u0, umin, umax);
      }
    }
  } else {
    for (v = 0; v < 4; ++v) {
      o->dWdx[CV(o, b, v, j, i)] = 0.0;
      o->dWdy[CV(o, b, v, j, i)] = 0.0;
      o->phi[CV(o, b, v, j, i)] = 0.0;
    }
  }
}

/* Limited linear face state W + (phi^dWdx)*dX.x + (phi^dWdy)*dX.y. */
static pst face_state(const e2d_oracle *o, int b, int i, int j, vec2 xf) {
  const size_t c = SC(o, b, j, i);
  const double dx = xf.x - o->xc[c], dy = xf.y - o->yc[c];
  double r[4];
  int v;
  pst w;
  for (v = 0; v < 4; ++v) {
    const size_t q = CV(o, b, v, j, i);
    r[v] = o->W[q] + (o->phi[q] * o->dWdx[q]) * dx + (o->phi[q] * o->dWdy[q]) * dy;
  }
  w.d = r[0]; w.u = r[1]; w.v = r[2]; w.p = r[3];
  return w;
}

/* Face states at a block-boundary face with a reflection or characteristic
 * BC (src_2D/Euler2D/Euler2DQuad.cc:855-957). */
static pst bc_face_state(const e2d_oracle *o, int bc, pst inner, pst wo, vec2 n) {
  return (bc == E2D_BC_REFLECTION) ? reflect(inner, n) : bc_char_pressure(o, inner, wo, n);
}
static int face_bc(int bc) { return bc == E2D_BC_REFLECTION || bc == E2D_BC_CHARACTERISTIC; }
static pst wo_at(const e2d_oracle *o, const double *wo, int b, int len, int k) {
  pst w;
  const double *p = wo + (size_t)b * 4 * len;
  w.d = p[k]; w.u = p[len + k]; w.v = p[2 * len + k]; w.p = p[3 * len + k];
  return w;
}

/* i-direction face flux between cells (i, j) and (i+1, j). */
static cst iface_flux(const e2d_oracle *o, int b, int i, int j) {
  pst wl, wr;
  const int bcw = o->bcw[(size_t)b * o->NCj + j], bce = o->bce[(size_t)b * o->NCj + j];
  if (i == o->ICl - 1 && face_bc(bcw)) {
    wr = face_state(o, b, i + 1, j, xfaceW(o, b, i + 1, j));
    wl = bc_face_state(o, bcw, wr, wo_at(o, o->wow, b, o->NCj, j), nfaceW(o, b, i + 1, j));
  } else if (i == o->ICu && face_bc(bce)) {
    wl = face_state(o, b, i, j, xfaceE(o, b, i, j));
    wr = bc_face_state(o, bce, wl, wo_at(o, o->woe, b, o->NCj, j), nfaceE(o, b, i, j));
  } else {
    wl = face_state(o, b, i, j, xfaceE(o, b, i, j));
    wr = face_state(o, b, i + 1, j, xfaceW(o, b, i + 1, j));
  }
  return face_flux_n(o, wl, wr, nfaceE(o, b, i, j));
}

/* j-direction face flux between cells (i, j) and (i, j+1). */
static cst jface_flux(const e2d_oracle *o, int b, int i, int j) {
  pst wl, wr;
  const int bcs = o->bcs[(size_t)b * o->NCi + i], bcn = o->bcn[(size_t)b * o->NCi + i];
  if (j == o->JCl - 1 && face_bc(bcs)) {
    wr = face_state(o, b, i, j + 1, xfaceS(o, b, i, j + 1));
    wl = bc_face_state(o, bcs, wr, wo_at(o, o->wos, b, o->NCi, i), nfaceS(o, b, i, j + 1));
  } else if (j == o->JCu && face_bc(bcn)) {
    wl = face_state(o, b, i, j, xfaceN(o, b, i, j));
    wr = bc_face_state(o, bcn, wl, wo_at(o, o->won, b, o->NCi, i), nfaceN(o, b, i, j));
  } else {
    wl = face_state(o, b, i, j, xfaceN(o, b, i, j));
    wr = face_state(o, b, i, j + 1, xfaceS(o, b, i, j + 1));
  }
  return face_flux_n(o, wl, wr, nfaceN(o, b, i, j));
}

/* The explicit schemes' stage structure (dUdt_Multistage_Explicit and
 * Update_Solution_Multistage_Explicit, Euler2DQuad.cc:1235-1342,
 * Euler2DQuadSingleBlock.cc:5300-5350): the update coefficient of stage s
 * (Runge_Kutta, CFD.cc:901-940; MultiStage_Optimally_Smoothing, CFD.cc:953-1031),
 * the residual slot k_residual it fills, and how its residual starts: 0
 * from zero, 1 from the stored slot-0 residual (the two-stage Runge-Kutta
 * and predictor-corrector schemes), 2 from slot0 + 2 slot1 + 2 slot2 (RK4's
 * last stage). */
static double stage_omega(const e2d_scheme *sc, int s) {
  const int n = sc->n_stage;
  double beta = 1.0;
  if (sc->time_integration == E2D_TIME_OPTIMAL_SMOOTHING) {
    static const double z[7][6] = {{0}, {1.0}, {1.0, 0.3333}, {1.50, 0.1481, 0.4000},
                                   {2.00, 0.0833, 0.2069, 0.4265}, {2.50, 0.0533, 0.1263, 0.2375, 0.4414},
                                   {3.00, 0.0370, 0.0851, 0.1521, 0.2562, 0.4512}};
    static const double l[7][6] = {{0}, {1.0}, {0.4693, 0.4242}, {0.6936, 0.1918, 0.4929},
                                   {0.9214, 0.1084, 0.2602, 0.5052}, {1.1508, 0.0695, 0.1602, 0.2898, 0.5060},
                                   {1.3805, 0.0482, 0.1085, 0.1885, 0.3050, 0.5063}};
    const double *t = sc->limiter == E2D_LIMITER_ZERO ? z[n] : l[n];
    beta = t[0];
    if (s < n) beta = t[s] * beta;
    return beta;
  }
  if (n == 2 && s == 2) beta = HALF * beta;
  if (n == 4) {
    if (s == 1 || s == 2) beta = HALF * beta;
    if (s == 4) beta = beta / 6.0;
  }
  if (n == 5) {
    static const double f[4] = {0.059, 0.14, 0.273, 0.5};
    if (s <= 4) beta *= f[s - 1];
  }
  return beta;
}
static int stage_slot(const e2d_scheme *sc, int s) {
  return (sc->time_integration != E2D_TIME_OPTIMAL_SMOOTHING && sc->n_stage == 4 && s < 4) ? s - 1 : 0;
}
static int stage_start(const e2d_scheme *sc, int s) {
  if (s == 1 || sc->time_integration == E2D_TIME_OPTIMAL_SMOOTHING) return 0;
  if (sc->n_stage == 2) return 1;
  if (sc->n_stage == 4 && s == 4) return 2;
  return 0;
}
static double *slot_array(e2d_oracle *o, int slot) {
  return slot == 0 ? o->dUdt : (slot == 1 ? o->dUdt1 : o->dUdt2);
}

/* Residual of one block: dUdt_Residual_Evaluation (stage == 0,
 * src_2D/Euler2D/Euler2DQuad.cc:814-1227) or stage `stage` of
 * dUdt_Multistage_Explicit (:1235-1727).  Each interior cell accumulates, in
 * the reference's loop order, D + west - east + south - north into the
 * stage's residual slot, D per stage_start. */
static void residual_block(e2d_oracle *o, int b, int stage) {
  const int ICl = o->ICl, ICu = o->ICu, JCl = o->JCl, JCu = o->JCu;
  int i, j, v;
  cst *Fi = (cst *)malloc(sizeof(cst) * (size_t)(ICu - ICl + 2) * (JCu - JCl + 1));
  cst *Fj = (cst *)malloc(sizeof(cst) * (size_t)(ICu - ICl + 1) * (JCu - JCl + 2));
  const int ni = ICu - ICl + 2, nj = JCu - JCl + 2;
  const int start = stage ? stage_start(&o->sc, stage) : 0;
  double *R = slot_array(o, stage ? stage_slot(&o->sc, stage) : 0);
  for (j = JCl - 1; j <= JCu + 1; ++j)
    for (i = ICl - 1; i <= ICu + 1; ++i) lsq_cell(o, b, i, j);
  if (stage == 1) {
    for (j = JCl - 1; j <= JCu + 1; ++j)
      for (i = ICl - 1; i <= ICu + 1; ++i)
        for (v = 0; v < 4; ++v) o->Uo[CV(o, b, v, j, i)] = o->U[CV(o, b, v, j, i)];
  }
  for (j = JCl; j <= JCu; ++j)
    for (i = ICl - 1; i <= ICu; ++i) Fi[(size_t)(j - JCl) * ni + (i - ICl + 1)] = iface_flux(o, b, i, j);
  for (j = JCl - 1; j <= JCu; ++j)
    for (i = ICl; i <= ICu; ++i) Fj[(size_t)(j - JCl + 1) * (ICu - ICl + 1) + (i - ICl)] = jface_flux(o, b, i, j);
  (void)nj;
  for (j = 0; j < o->NCj; ++j)
    for (i = 0; i < o->NCi; ++i) {
      const int interior = (i >= ICl && i <= ICu && j >= JCl && j <= JCu);
      if (!interior) {
        for (v = 0; v < 4; ++v) R[CV(o, b, v, j, i)] = 0.0;
        continue;
      }
      {
        const size_t c = SC(o, b, j, i);
        const double A = o->A[c];
        const double lW = lfaceW(o, b, i, j), lE = lfaceE(o, b, i, j);
        const double lS = lfaceS(o, b, i, j), lN = lfaceN(o, b, i, j);
        const cst fw = Fi[(size_t)(j - JCl) * ni + (i - ICl)];
        const cst fe = Fi[(size_t)(j - JCl) * ni + (i - ICl + 1)];
        const cst fs = Fj[(size_t)(j - JCl) * (ICu - ICl + 1) + (i - ICl)];
        const cst fn = Fj[(size_t)(j - JCl + 1) * (ICu - ICl + 1) + (i - ICl)];
        const double k = stage ? o->sc.cfl * o->dt[c] : 1.0;
        const double fwv[4] = {fw.d, fw.mx, fw.my, fw.E}, fev[4] = {fe.d, fe.mx, fe.my, fe.E};
        const double fsv[4] = {fs.d, fs.mx, fs.my, fs.E}, fnv[4] = {fn.d, fn.mx, fn.my, fn.E};
        for (v = 0; v < 4; ++v) {
          const size_t q = CV(o, b, v, j, i);
          double d = 0.0;
          if (start == 1) d = o->dUdt[q];
          if (start == 2) d = o->dUdt[q] + 2.0 * o->dUdt1[q] + 2.0 * o->dUdt2[q];
          if (stage) {
            d += k * fwv[v] * lW / A;
            d -= k * fev[v] * lE / A;
            d += k * fsv[v] * lS / A;
            d -= k * fnv[v] * lN / A;
          } else {
            d += fwv[v] * lW / A;
            d -= fev[v] * lE / A;
            d += fsv[v] * lS / A;
            d -= fnv[v] * lN / A;
          }
          R[q] = d;
        }
      }
    }
  free(Fi);
  free(Fj);
}

/* Same-resolution ghost exchange: copy of the neighbours' two edge layers of
 * U, then W = U.W() (Euler2D_Quad_Block::LoadSendBuffer/UnloadReceiveBuffer,
 * src_2D/Euler2D/Euler2DQuad.h:1570-1650). */
static void exchange(e2d_oracle *o) {
  const int g = o->ng, ICl = o->ICl, ICu = o->ICu, JCl = o->JCl, JCu = o->JCu;
  int b, k, i, j;
  for (b = 0; b < o->nblk; ++b)
    for (k = 0; k < 8; ++k) {
      const int s = o->neigh[b * 8 + k];
      int i0, i1, j0, j1, di, dj;
      const int wi = (k == 0 || k == 4 || k == 6), ei = (k == 1 || k == 5 || k == 7);
      const int sj = (k == 2 || k == 4 || k == 5), nj = (k == 3 || k == 6 || k == 7);
      if (s < 0) continue;
      if (wi) { i0 = ICl - g; i1 = ICl - 1; di = (ICu + 1) - ICl; }
      else if (ei) { i0 = ICu + 1; i1 = ICu + g; di = ICl - (ICu + 1); }
      else { i0 = ICl; i1 = ICu; di = 0; }
      if (sj) { j0 = JCl - g; j1 = JCl - 1; dj = (JCu + 1) - JCl; }
      else if (nj) { j0 = JCu + 1; j1 = JCu + g; dj = JCl - (JCu + 1); }
      else { j0 = JCl; j1 = JCu; dj = 0; }
      for (j = j0; j <= j1; ++j)
        for (i = i0; i <= i1; ++i) {
          const cst u = getU(o, o->U, s, i + di, j + dj);
          putU(o, o->U, b, i, j, u);
          putW(o, o->W, b, i, j, W_of_U(o, u));
        }
    }
}

/* One ghost cell assignment W[dst] = w with U = U(W). */
static void set_ghost_W(e2d_oracle *o, int b, int i, int j, pst w) {
  putW(o, o->W, b, i, j, w);
  putU(o, o->U, b, i, j, U_of_W(o, w));
}
static void copy_cell(e2d_oracle *o, int b, int id, int jd, int is, int js) {
  putW(o, o->W, b, id, jd, getW(o, o->W, b, is, js));
  putU(o, o->U, b, id, jd, getU(o, o->U, b, is, js));
}

/* BCs (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:2354-2995) for the
 * supported types. */
static void bcs_block(e2d_oracle *o, int b) {
  const int Ng = o->ng, ICl = o->ICl, ICu = o->ICu, JCl = o->JCl, JCu = o->JCu;
  const int NCi = o->NCi, NCj = o->NCj;
  int i, j, g;
  for (j = 0; j < NCj; ++j) {
    const int bw = o->bcw[(size_t)b * NCj + j], be = o->bce[(size_t)b * NCj + j];
    if ((j >= JCl && j <= JCu) || (j < JCl && o->bcs[(size_t)b * NCi + ICl - 1] == E2D_BC_NONE) ||
        (j > JCu && o->bcn[(size_t)b * NCi + ICl - 1] == E2D_BC_NONE)) {
      switch (bw) {
        case E2D_BC_NONE: break;
        case E2D_BC_FIXED:
          for (g = 1; g <= Ng; ++g) set_ghost_W(o, b, ICl - g, j, wo_at(o, o->wow, b, NCj, j));
          break;
        case E2D_BC_REFLECTION:
          for (g = 1; g <= Ng; ++g)
            set_ghost_W(o, b, ICl - g, j, reflect(getW(o, o->W, b, ICl + g - 1, j), nfaceW(o, b, ICl, j)));
          break;
        case E2D_BC_PERIODIC:
          for (g = 1; g <= Ng; ++g) copy_cell(o, b, ICl - g, j, ICu - g + 1, j);
          break;
        case E2D_BC_CHARACTERISTIC:
          set_ghost_W(o, b, ICl - 1, j,
                      bc_char_pressure(o, getW(o, o->W, b, ICl, j), wo_at(o, o->wow, b, NCj, j), nfaceW(o, b, ICl, j)));
          for (g = 2; g <= Ng; ++g) copy_cell(o, b, ICl - g, j, ICl - 1, j);
          break;
        default: /* BC_CONSTANT_EXTRAPOLATION and the reference's default */
          for (g = 1; g <= Ng; ++g) copy_cell(o, b, ICl - g, j, ICl, j);
          break;
      }
    }
    if ((j >= JCl && j <= JCu) || (j < JCl && o->bcs[(size_t)b * NCi + ICu + 1] == E2D_BC_NONE) ||
        (j > JCu && o->bcn[(size_t)b * NCi + ICu + 1] == E2D_BC_NONE)) {
      switch (be) {
        case E2D_BC_NONE: break;
        case E2D_BC_FIXED:
          for (g = 1; g <= Ng; ++g) set_ghost_W(o, b, ICu + g, j, wo_at(o, o->woe, b, NCj, j));
          break;
        case E2D_BC_REFLECTION:
          for (g = 1; g <= Ng; ++g)
            set_ghost_W(o, b, ICu + g, j, reflect(getW(o, o->W, b, ICu - g + 1, j), nfaceE(o, b, ICu, j)));
          break;
        case E2D_BC_PERIODIC:
          for (g = 1; g <= Ng; ++g) copy_cell(o, b, ICu + g, j, ICl + g - 1, j);
          break;
        case E2D_BC_CHARACTERISTIC:
          set_ghost_W(o, b, ICu + 1, j,
                      bc_char_pressure(o, getW(o, o->W, b, ICu, j), wo_at(o, o->woe, b, NCj, j), nfaceE(o, b, ICu, j)));
          for (g = 2; g <= Ng; ++g) copy_cell(o, b, ICu + g, j, ICu + 1, j);
          break;
        default:
          for (g = 1; g <= Ng; ++g) copy_cell(o, b, ICu + g, j, ICu, j);
          break;
      }
    }
  }
  for (i = 0; i < NCi; ++i) {
    const int bs = o->bcs[(size_t)b * NCi + i], bn = o->bcn[(size_t)b * NCi + i];
    switch (bs) {
      case E2D_BC_NONE: break;
      case E2D_BC_FIXED:
        for (g = 1; g <= Ng; ++g) set_ghost_W(o, b, i, JCl - g, wo_at(o, o->wos, b, NCi, i));
        break;
      case E2D_BC_REFLECTION:
        for (g = 1; g <= Ng; ++g)
          set_ghost_W(o, b, i, JCl - g, reflect(getW(o, o->W, b, i, JCl + g - 1), nfaceS(o, b, i, JCl)));
        break;
      case E2D_BC_PERIODIC:
        for (g = 1; g <= Ng; ++g) copy_cell(o, b, i, JCl - g, i, JCu - g + 1);
        break;
      case E2D_BC_CHARACTERISTIC:
        set_ghost_W(o, b, i, JCl - 1,
                    bc_char_pressure(o, getW(o, o->W, b, i, JCl), wo_at(o, o->wos, b, NCi, i), nfaceS(o, b, i, JCl)));
        for (g = 2; g <= Ng; ++g) copy_cell(o, b, i, JCl - g, i, JCl - 1);
        break;
      default:
        for (g = 1; g <= Ng; ++g) copy_cell(o, b, i, JCl - g, i, JCl);
        break;
    }
    switch (bn) {
      case E2D_BC_NONE: break;
      case E2D_BC_FIXED:
        for (g = 1; g <= Ng; ++g) set_ghost_W(o, b, i, JCu + g, wo_at(o, o->won, b, NCi, i));
        break;
      case E2D_BC_REFLECTION:
        for (g = 1; g <= Ng; ++g)
          set_ghost_W(o, b, i, JCu + g, reflect(getW(o, o->W, b, i, JCu - g + 1), nfaceN(o, b, i, JCu)));
        break;
      case E2D_BC_PERIODIC:
        for (g = 1; g <= Ng; ++g) copy_cell(o, b, i, JCu + g, i, JCl + g - 1);
        break;
      case E2D_BC_CHARACTERISTIC:
        set_ghost_W(o, b, i, JCu + 1,
                    bc_char_pressure(o, getW(o, o->W, b, i, JCu), wo_at(o, o->won, b, NCi, i), nfaceN(o, b, i, JCu)));
        for (g = 2; g <= Ng; ++g) copy_cell(o, b, i, JCu + g, i, JCu + 1);
        break;
      default:
        for (g = 1; g <= Ng; ++g) copy_cell(o, b, i, JCu + g, i, JCu);
        break;
    }
  }
}

/* CFL (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:3019-3080): local dt in each
 * interior cell, ghosts get the block minimum; returns the block minimum. */
static double cfl_block(e2d_oracle *o, int b) {
  double dtMin = MILLION;
  int i, j;
  for (j = 0; j < o->NCj; ++j)
    for (i = 0; i < o->NCi; ++i) {
      const size_t c = SC(o, b, j, i);
      if (i < o->ICl || i > o->ICu || j < o->JCl || j > o->JCu) {
        o->dt[c] = 0.0;
      } else {
        const pst w = getW(o, o->W, b, i, j);
        const vec2 nE = nfaceE(o, b, i, j), nW = nfaceW(o, b, i, j);
        const vec2 nN = nfaceN(o, b, i, j), nS = nfaceS(o, b, i, j);
        const double d_i = 2.0 * (o->A[c] / (lfaceE(o, b, i, j) + lfaceW(o, b, i, j)));
        const double d_j = 2.0 * (o->A[c] / (lfaceN(o, b, i, j) + lfaceS(o, b, i, j)));
        const double v_i = HALF * (w.u * (nE.x - nW.x) + w.v * (nE.y - nW.y));
        const double v_j = HALF * (w.u * (nN.x - nS.x) + w.v * (nN.y - nS.y));
        const double a = a_of(o, w);
        o->dt[c] = dmin(d_i / (a + fabs(v_i)), d_j / (a + fabs(v_j)));
        dtMin = dmin(dtMin, o->dt[c]);
      }
    }
  for (j = 0; j < o->NCj; ++j)
    for (i = 0; i < o->NCi; ++i)
      if (i < o->ICl || i > o->ICu || j < o->JCl || j > o->JCu) o->dt[SC(o, b, j, i)] = dtMin;
  return dtMin;
}

/* Residual_Smoothing (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:4521-4563):
 * Gauss-Seidel sweeps in lexicographic order over the cells one away from
 * the block edges, on a copy whose other entries are zero (the reference's
 * second residual slot, never written on this path); the result replaces
 * the residual there. */
static void residual_smoothing_block(e2d_oracle *o, int b, double *R) {
  const int il = o->ICl + 1, iu = o->ICu - 1, jl = o->JCl + 1, ju = o->JCu - 1;
  const double eps = o->sc.rs_epsilon;
  const size_t n = 4 * (size_t)o->NCi * o->NCj;
  double *S = (double *)calloc(n, sizeof(double));
  int i, j, v, it;
  /* S indexed as R of block 0 */
  for (v = 0; v < 4; ++v)
    for (j = jl; j <= ju; ++j)
      for (i = il; i <= iu; ++i) S[CV(o, 0, v, j, i)] = R[CV(o, b, v, j, i)];
  for (it = 1; it <= o->sc.rs_iterations; ++it)
    for (j = jl; j <= ju; ++j)
      for (i = il; i <= iu; ++i)
        for (v = 0; v < 4; ++v)
          S[CV(o, 0, v, j, i)] = (R[CV(o, b, v, j, i)] +
                                  eps * (S[CV(o, 0, v, j - 1, i)] + S[CV(o, 0, v, j, i - 1)] +
                                         S[CV(o, 0, v, j, i + 1)] + S[CV(o, 0, v, j + 1, i)])) /
                                 (1.0 + 4.0 * eps);
  for (v = 0; v < 4; ++v)
    for (j = jl; j <= ju; ++j)
      for (i = il; i <= iu; ++i) R[CV(o, b, v, j, i)] = S[CV(o, 0, v, j, i)];
  free(S);
}

/* Update_Solution_Multistage_Explicit for RK (src_2D/Euler2D/Euler2DQuadSingleBlock.cc:5300-5507)
 * and Runge_Kutta (src_2D/CFD/CFD.cc:901-937).  Returns 0 or 1 + the linear
 * cell index of the failing cell. */
static int update_block(e2d_oracle *o, int b, int stage) {
  const double omega = stage_omega(&o->sc, stage);
  double *R = slot_array(o, stage_slot(&o->sc, stage));
  int i, j, v, nr;
  for (j = o->JCl; j <= o->JCu; ++j)
    for (i = o->ICl; i <= o->ICu; ++i) {
      const size_t c = SC(o, b, j, i);
      cst uo = getU(o, o->Uo, b, i, j), du = getU(o, R, b, i, j), u;
      u.d = uo.d + omega * du.d; u.mx = uo.mx + omega * du.mx;
      u.my = uo.my + omega * du.my; u.E = uo.E + omega * du.E;
      if (u.d <= 0.0 || u.E <= 0.0 || e_of_U(u) <= 0.0) {
        if (!o->sc.local_dt) return 1 + (int)c;
        {
          double rrf = 1.0;
          for (nr = 1; nr <= 10; ++nr) {
            rrf = HALF * rrf;
            o->dt[c] = rrf * o->dt[c];
            du.d = rrf * du.d; du.mx = rrf * du.mx; du.my = rrf * du.my; du.E = rrf * du.E;
            u.d = uo.d + omega * du.d; u.mx = uo.mx + omega * du.mx;
            u.my = uo.my + omega * du.my; u.E = uo.E + omega * du.E;
            if (u.d > 0.0 && u.E > 0.0 && e_of_U(u) > 0.0) break;
          }
          putU(o, R, b, i, j, du);
          if (u.d <= 0.0 || u.E <= 0.0 || e_of_U(u) <= 0.0) return 1 + (int)c;
        }
      }
      putU(o, o->U, b, i, j, u);
      putW(o, o->W, b, i, j, W_of_U(o, u));
      (void)v;
    }
  return 0;
}

e2d_oracle *e2d_oracle_create(const e2d_blocks_desc *d, const e2d_scheme *sc, int *err) {
  e2d_oracle *o;
  int b, i, j;
  size_t ncell, nnode;
  if (err) *err = 0;
  if (!d || !sc || d->nblk < 1 || d->nci < 2 || d->ncj < 2 || d->ng != 2 ||
      sc->n_stage < 1 || sc->n_stage > 6 || sc->flux < E2D_FLUX_GODUNOV || sc->flux > E2D_FLUX_AUSMPLUS ||
      sc->flux == 7) {
    if (err) *err = E2D_ERR_ARG;
    return NULL;
  }
  o = (e2d_oracle *)calloc(1, sizeof(*o));
  o->nblk = d->nblk; o->nci = d->nci; o->ncj = d->ncj; o->ng = d->ng;
  o->NCi = d->nci + 2 * d->ng; o->NCj = d->ncj + 2 * d->ng;
  o->NNi = o->NCi + 1; o->NNj = o->NCj + 1;
  o->ICl = d->ng; o->ICu = d->nci + d->ng - 1; o->JCl = d->ng; o->JCu = d->ncj + d->ng - 1;
  o->sc = *sc;
  o->g = sc->gamma; o->gm1 = o->g - 1.0; o->gm1i = 1.0 / o->gm1;
  ncell = (size_t)o->nblk * o->NCi * o->NCj;
  nnode = (size_t)o->nblk * o->NNi * o->NNj;
#define DUP(dst, src, n, T) do { dst = (T *)malloc(sizeof(T) * (n)); memcpy(dst, src, sizeof(T) * (n)); } while (0)
  DUP(o->neigh, d->neighbour, (size_t)o->nblk * 8, int);
  DUP(o->bcw, d->bc_w, (size_t)o->nblk * o->NCj, int);
  DUP(o->bce, d->bc_e, (size_t)o->nblk * o->NCj, int);
  DUP(o->bcs, d->bc_s, (size_t)o->nblk * o->NCi, int);
  DUP(o->bcn, d->bc_n, (size_t)o->nblk * o->NCi, int);
  DUP(o->X, d->node_x, nnode, double);
  DUP(o->Y, d->node_y, nnode, double);
  DUP(o->wow, d->wo_w, (size_t)o->nblk * 4 * o->NCj, double);
  DUP(o->woe, d->wo_e, (size_t)o->nblk * 4 * o->NCj, double);
  DUP(o->wos, d->wo_s, (size_t)o->nblk * 4 * o->NCi, double);
  DUP(o->won, d->wo_n, (size_t)o->nblk * 4 * o->NCi, double);
#undef DUP
  o->xc = (double *)calloc(ncell, sizeof(double));
  o->yc = (double *)calloc(ncell, sizeof(double));
  o->A = (double *)calloc(ncell, sizeof(double));
  o->dt = (double *)calloc(ncell, sizeof(double));
  o->W = (double *)calloc(4 * ncell, sizeof(double));
  o->U = (double *)calloc(4 * ncell, sizeof(double));
  o->Uo = (double *)calloc(4 * ncell, sizeof(double));
  o->dUdt = (double *)calloc(4 * ncell, sizeof(double));
  o->dUdt1 = (double *)calloc(4 * ncell, sizeof(double));
  o->dUdt2 = (double *)calloc(4 * ncell, sizeof(double));
  o->dWdx = (double *)calloc(4 * ncell, sizeof(double));
  o->dWdy = (double *)calloc(4 * ncell, sizeof(double));
  o->phi = (double *)calloc(4 * ncell, sizeof(double));
  for (b = 0; b < o->nblk; ++b)
    for (j = 0; j < o->NCj; ++j)
      for (i = 0; i < o->NCi; ++i) {
        vec2 c = {0, 0};
        double area = 0;
        quad_centroid(node(o, b, i, j), node(o, b, i + 1, j), node(o, b, i + 1, j + 1), node(o, b, i, j + 1), &c, &area);
        o->xc[SC(o, b, j, i)] = c.x; o->yc[SC(o, b, j, i)] = c.y; o->A[SC(o, b, j, i)] = area;
      }
  return o;
}

void e2d_oracle_destroy(e2d_oracle *o) {
  if (!o) return;
  free(o->neigh); free(o->bcw); free(o->bce); free(o->bcs); free(o->bcn);
  free(o->X); free(o->Y); free(o->wow); free(o->woe); free(o->wos); free(o->won);
  free(o->xc); free(o->yc); free(o->A); free(o->dt);
  free(o->W); free(o->U); free(o->Uo); free(o->dUdt); free(o->dWdx); free(o->dWdy); free(o->phi);
  free(o->dUdt1); free(o->dUdt2);
  free(o);
}

int e2d_oracle_set_state(e2d_oracle *o, const double *W) {
  int b, i, j;
  memcpy(o->W, W, sizeof(double) * 4 * (size_t)o->nblk * o->NCi * o->NCj);
  for (b = 0; b < o->nblk; ++b)
    for (j = 0; j < o->NCj; ++j)
      for (i = 0; i < o->NCi; ++i) putU(o, o->U, b, i, j, U_of_W(o, getW(o, o->W, b, i, j)));
  o->frozen = 0;
  o->first = 1;
  return 0;
}

int e2d_oracle_get_state(e2d_oracle *o, double *W, double *U) {
  const size_t n = sizeof(double) * 4 * (size_t)o->nblk * o->NCi * o->NCj;
  if (W) memcpy(W, o->W, n);
  if (U) memcpy(U, o->U, n);
  return 0;
}

int e2d_oracle_fill_ghosts(e2d_oracle *o) {
  int b;
  exchange(o);
  for (b = 0; b < o->nblk; ++b) bcs_block(o, b);
  return 0;
}

int e2d_oracle_residual(e2d_oracle *o, double *dUdt) {
  int b;
  e2d_oracle_fill_ghosts(o);
  for (b = 0; b < o->nblk; ++b) residual_block(o, b, 0);
  if (dUdt) memcpy(dUdt, o->dUdt, sizeof(double) * 4 * (size_t)o->nblk * o->NCi * o->NCj);
  return 0;
}

int e2d_oracle_get_reconstruction(e2d_oracle *o, double *dWdx, double *dWdy, double *phi) {
  const size_t n = sizeof(double) * 4 * (size_t)o->nblk * o->NCi * o->NCj;
  if (dWdx) memcpy(dWdx, o->dWdx, n);
  if (dWdy) memcpy(dWdy, o->dWdy, n);
  if (phi) memcpy(phi, o->phi, n);
  return 0;
}

int e2d_oracle_geometry(e2d_oracle *o, double *xc, double *yc, double *area) {
  const size_t n = sizeof(double) * (size_t)o->nblk * o->NCi * o->NCj;
  if (xc) memcpy(xc, o->xc, n);
  if (yc) memcpy(yc, o->yc, n);
  if (area) memcpy(area, o->A, n);
  return 0;
}

/* The explicit time-marching loop of src_2D/Euler2D/Euler2DQuadSolvers.cc:657-898. */
int e2d_oracle_rk_steps(e2d_oracle *o, int n_steps, double *hist) {
  int n, b, stage, i, j, err;
  for (n = 0; n < n_steps; ++n) {
    double dtmin = MILLION, l1 = 0, l2 = 0, lmax = 0;
    for (b = 0; b < o->nblk; ++b) dtmin = dmin(dtmin, cfl_block(o, b));
    if (!o->sc.local_dt)
      for (b = 0; b < o->nblk; ++b)
        for (j = o->JCl; j <= o->JCu; ++j)
          for (i = o->ICl; i <= o->ICu; ++i) o->dt[SC(o, b, j, i)] = dtmin;
    for (b = 0; b < o->nblk; ++b) {
      double s1 = 0, s2 = 0, mx = 0;
      for (j = o->JCl; j <= o->JCu; ++j)
        for (i = o->ICl; i <= o->ICu; ++i) {
          const double r = o->dUdt[CV(o, b, 0, j, i)];
          s1 += fabs(r);
          s2 += sqr(r);
          mx = dmax(mx, fabs(r));
        }
      l1 += s1;
      l2 += sqr(sqrt(s2));
      lmax = dmax(lmax, mx);
    }
    if (hist) {
      /* multi-block L2 (Euler2DQuadMultiBlock.cc:1049), squared, summed and
       rooted again by the solver loop (Euler2DQuadSolvers.cc:690-693) */
      hist[4 * n] = dtmin; hist[4 * n + 1] = l1; hist[4 * n + 2] = sqrt(sqr(sqrt(l2))); hist[4 * n + 3] = lmax;
    }
    /* limiter freezing at the head of every step but a run's first
       (Euler2DQuadSolvers.cc:794-803) */
    if (!o->first && o->sc.freeze_limiter && sqrt(sqr(sqrt(l2))) <= o->sc.freeze_level) o->frozen = 1;
    o->first = 0;
    for (stage = 1; stage <= o->sc.n_stage; ++stage) {
      e2d_oracle_fill_ghosts(o);
      for (b = 0; b < o->nblk; ++b) residual_block(o, b, stage);
      if (o->sc.rs_epsilon > 0.0)
        for (b = 0; b < o->nblk; ++b) residual_smoothing_block(o, b, slot_array(o, stage_slot(&o->sc, stage)));
      for (b = 0; b < o->nblk; ++b) {
        err = update_block(o, b, stage);
        if (err) return err;
      }
    }
  }
  return 0;
}
