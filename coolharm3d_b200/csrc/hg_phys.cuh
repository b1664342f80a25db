// hg_phys.cuh -- per-zone GRMHD physics of the step, as device functions.
//
// Every function restates the reference routine named beside it (paths
// relative to scnastro/coolharm3d src/) with the same operation order, and the
// library is compiled with -fmad=false, so FP64 results are bit-identical to
// the reference's gcc build (which has no fused multiply-add either).
#pragma once
#include "hg_internal.h"

namespace hg {

#define HG_SMALL 1.e-15
#define HG_SAFE 1.3
#define HG_GAMMAMAX 50.
#define HG_GAMMAMAX2 1.e4
#define HG_BETA_MIN 1.e-2
#define HG_PPM_FACTOR 0.16666666666666666667
#define HG_MAX_NEWT_ITER 30
#define HG_NEWT_TOL 1.0e-10
#define HG_MIN_NEWT_TOL 1.0e-10
#define HG_EXTRA_NEWT_ITER 2
#define HG_NEWT_TOL2 1.0e-15
#define HG_W_TOO_BIG 1.e20
#define HG_UTSQ_TOO_BIG 1.e20
#define HG_FAIL_VAL 1.e30

template <class T>
struct StateT {
  T ucon[4], ucov[4], bcon[4], bcov[4];
  T bsq, p, eta, ptot;
};
typedef StateT<double> State;

__device__ __forceinline__ int off3(const GridDev &G, int i, int j, int k)  // 32-bit: planes < 2^31 entries
{
  return i * G.st[0] + j * G.st[1] + k * G.st[2];
}

// get_geometry (macros.h:605): metric_dim 0 uses one struct, metric_dim 2
// the (pos,i,j) tables, metric_dim 3 the (pos,i,j,k) table of time level
// `slot` (0 n_beg, 1 n_mid, 2 n_end; the buffer of each level is in
// DevScalars::lev, rotated on the device every step).
__device__ __forceinline__ void load_geom(const GridDev &G, int pos, int i, int j, Geom &g, int k = 0, int slot = 0)
{
  if (G.mdim == 0) {
    g = G.g0;
    return;
  }
  const double *t;
  long s;
  if (G.mdim == 3) {
    const int L = G.sc->lev[slot];
    t = (L == 0 ? G.geomL[0] : L == 1 ? G.geomL[1] : G.geomL[2]) + (long)pos * G.S + off3(G, i, j, k);
    s = G.gS3;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = a; b < 4; b++) {
        const double cn = __ldg(t + (HG_DP_GCON + dyn_sym(a, b)) * s), cv = __ldg(t + (HG_DP_GCOV + dyn_sym(a, b)) * s);
        g.gcon[a][b] = cn;
        g.gcon[b][a] = cn;
        g.gcov[a][b] = cv;
        g.gcov[b][a] = cv;
      }
    g.g = __ldg(t + HG_DP_G * s);
    g.g_inv = __ldg(t + HG_DP_GINV * s);
    g.alpha = __ldg(t + HG_DP_ALPHA * s);
    g.beta[0] = __ldg(t + (HG_DP_BETA + 0) * s);
    g.beta[1] = __ldg(t + (HG_DP_BETA + 1) * s);
    g.beta[2] = __ldg(t + (HG_DP_BETA + 2) * s);
    g.ncon[0] = __ldg(t + HG_DP_NCON0 * s);
    g.ncon[1] = -g.alpha * g.gcon[0][1];
    g.ncon[2] = -g.alpha * g.gcon[0][2];
    g.ncon[3] = -g.alpha * g.gcon[0][3];
    return;
  } else {
    const int ii = G.deg[0] ? 0 : i, jj = G.deg[1] ? 0 : j;
    const long o = ((long)pos * G.T[1] + jj) * G.T[0] + ii;
    t = G.geomT + o;
    s = G.gS;
  }
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      g.gcon[a][b] = __ldg(t + (a * 4 + b) * s);
      g.gcov[a][b] = __ldg(t + (16 + a * 4 + b) * s);
    }
  g.g = __ldg(t + 32 * s);
  g.g_inv = __ldg(t + 33 * s);
  g.alpha = __ldg(t + 34 * s);
  g.beta[0] = __ldg(t + 35 * s);
  g.beta[1] = __ldg(t + 36 * s);
  g.beta[2] = __ldg(t + 37 * s);
  g.ncon[0] = __ldg(t + 38 * s);
  g.ncon[1] = __ldg(t + 39 * s);
  g.ncon[2] = __ldg(t + 40 * s);
  g.ncon[3] = __ldg(t + 41 * s);
}

template <class T, class GT>
__device__ __forceinline__ void lower4(const T *v, const GT &g, T *w)  // metric.c:338
{
#pragma unroll
  for (int a = 0; a < 4; a++)
    w[a] = g.cov(a, 0) * v[0] + g.cov(a, 1) * v[1] + g.cov(a, 2) * v[2] + g.cov(a, 3) * v[3];
}

__device__ __forceinline__ void raise4(const double *v, const Geom &g, double *w)  // metric.c:362
{
#pragma unroll
  for (int a = 0; a < 4; a++)
    w[a] = g.gcon[a][0] * v[0] + g.gcon[a][1] * v[1] + g.gcon[a][2] * v[2] + g.gcon[a][3] * v[3];
}

// The gcov-weighted spatial quadratic form of gamma_calc (phys.c:249-255),
// Utoprim_new_body's Bsq and utsq (utoprim_2d_fast.c:255-304).
template <class T, class GT>
__device__ __forceinline__ T quad3(const GT &g, T a, T b, T c)
{
  return g.cov(1, 1) * a * a + g.cov(2, 2) * b * b + g.cov(3, 3) * c * c +
         2 * (g.cov(1, 2) * a * b + g.cov(1, 3) * a * c + g.cov(2, 3) * b * c);
}

template <class T, class GT>
__device__ __forceinline__ int gamma_calc(const T *pr, const GT &g, T *gamma)  // phys.c:244-270
{
  T qsq = quad3(g, pr[U1], pr[U2], pr[U3]);
  if (qsq < T(0)) {
    if (fabs(qsq) > T(1.E-10)) {
      *gamma = T(1);
      return 1;
    }
    qsq = T(1.E-10);
  }
  *gamma = sqrt(T(1) + qsq);
  return 0;
}

// get_state (phys.c:199), with ucon_calc (phys.c:216) and bcon_calc (phys.c:75).
// Returns 1 if gamma_calc failed (the caller books FAIL_GAMMA_CALC).
template <class T, class GT>
__device__ __forceinline__ int get_state(const T *pr, const GT &g, T gam, StateT<T> &q)
{
  T gamma;
  const int bad = gamma_calc(pr, g, &gamma);
  q.ucon[0] = gamma * g.nc(0);
  q.ucon[1] = pr[U1] - q.ucon[0] * g.bet(0);
  q.ucon[2] = pr[U2] - q.ucon[0] * g.bet(1);
  q.ucon[3] = pr[U3] - q.ucon[0] * g.bet(2);
  lower4(q.ucon, g, q.ucov);
  const T inv_ut = T(1) / q.ucon[0];
  q.bcon[0] = pr[B1] * q.ucov[1] + pr[B2] * q.ucov[2] + pr[B3] * q.ucov[3];
  q.bcon[1] = (pr[B1] + q.bcon[0] * q.ucon[1]) * inv_ut;
  q.bcon[2] = (pr[B2] + q.bcon[0] * q.ucon[2]) * inv_ut;
  q.bcon[3] = (pr[B3] + q.bcon[0] * q.ucon[3]) * inv_ut;
  lower4(q.bcon, g, q.bcov);
  q.bsq = q.bcon[0] * q.bcov[0] + q.bcon[1] * q.bcov[1] + q.bcon[2] * q.bcov[2] + q.bcon[3] * q.bcov[3];
  q.p = (gam - T(1)) * pr[UU];
  q.eta = q.p + pr[RHO] + pr[UU] + q.bsq;
  q.ptot = q.p + T(0.5) * q.bsq;
  return bad;
}

__device__ __forceinline__ void mhd_row(const State &q, int dir, double *mhd)  // phys.c:93
{
  const double eta_ucon = q.eta * q.ucon[dir];
  const double bcon_dir = q.bcon[dir];
  mhd[0] = eta_ucon * q.ucov[0] - bcon_dir * q.bcov[0];
  mhd[1] = eta_ucon * q.ucov[1] - bcon_dir * q.bcov[1];
  mhd[2] = eta_ucon * q.ucov[2] - bcon_dir * q.bcov[2];
  mhd[3] = eta_ucon * q.ucov[3] - bcon_dir * q.bcov[3];
  mhd[dir] += q.ptot;
}

__device__ __forceinline__ void primtoflux(const double *pr, const State &q, int dir, const Geom &g,
                                           double *f)  // phys.c:28-63
{
  double mhd[4];
  mhd_row(q, dir, mhd);
  f[RHO] = pr[RHO] * q.ucon[dir];
  f[UU] = mhd[0] + f[RHO];
  f[U1] = mhd[1];
  f[U2] = mhd[2];
  f[U3] = mhd[3];
  f[B1] = q.bcon[1] * q.ucon[dir] - q.bcon[dir] * q.ucon[1];
  f[B2] = q.bcon[2] * q.ucon[dir] - q.bcon[dir] * q.ucon[2];
  f[B3] = q.bcon[3] * q.ucon[dir] - q.bcon[dir] * q.ucon[3];
#pragma unroll
  for (int l = 0; l < HG_NPR; l++) f[l] *= g.g;
}

template <class T, class GT>
__device__ __forceinline__ void vchar_fast(const StateT<T> &q, const GT &g, int js, T gam, T *vmax,
                                           T *vmin)  // phys.c:432-501
{
  T cms2 = (gam * q.p + q.bsq) / q.eta;
  if (cms2 < T(0)) cms2 = T(HG_SMALL);
  else if (cms2 > T(1)) cms2 = T(1);
  const T Au2 = q.ucon[js] * q.ucon[js];
  const T Bu2 = q.ucon[0] * q.ucon[0];
  const T AuBu = q.ucon[js] * q.ucon[0];
  const T A = Bu2 - (g.con(0, 0) + Bu2) * cms2;
  const T B = AuBu - (g.con(0, js) + AuBu) * cms2;
  const T C = Au2 - (g.con(js, js) + Au2) * cms2;
  T discr = B * B - A * C;
  if (discr < T(0)) discr = T(0);
  discr = sqrt(discr);
  const T denom = T(1) / A;
  const T vp = -(-B + discr) * denom;
  const T vm = -(-B - discr) * denom;
  if (vp > vm) {
    *vmax = vp;
    *vmin = vm;
  } else {
    *vmax = vm;
    *vmin = vp;
  }
}

// One component of primtoflux(pr, q, dir) (phys.c:28-63), same operations.
template <class T>
__device__ __forceinline__ T flux_comp(const T *pr, const StateT<T> &q, int dir, T gg, int l)
{
  const T eta_ucon = q.eta * q.ucon[dir];
  const T bcon_dir = q.bcon[dir];
  T f;
  if (l == RHO) {
    f = pr[RHO] * q.ucon[dir];
  } else if (l <= U3) {
    const int a = l - 1;  // UU -> 0, U1 -> 1, ...
    T m = eta_ucon * q.ucov[a] - bcon_dir * q.bcov[a];
    if (a == dir) m += q.ptot;
    f = (l == UU) ? m + pr[RHO] * q.ucon[dir] : m;
  } else {
    const int a = l - 4;
    f = q.bcon[a] * q.ucon[dir] - q.bcon[dir] * q.ucon[a];
  }
  return f * gg;
}

// ---------------------------------------------------------------------------
// Reconstruction of one variable at one face from the six zones around it.
// y[0..5] are zones f-3 .. f+2 along the direction; *yl is the left state
// (right edge of zone f-1, p_L[f]) and *yr the right state (left edge of zone
// f, p_R[f]).  PPM: linear_recon_vect (recon.c:237-264) + para_vect
// (recon.c:611-641); limiters: linear_recon (recon.c:86-125).

// Both limiters are written as selections among candidates computed up
// front instead of early returns, so a warp takes no data-dependent branch;
// every value selected is the one the reference's branch returns.
template <class T>
__device__ __forceinline__ T slope_vect(int rt, T a, T b)  // recon.c:246-260
{
  const T s = a * b;
  T r;
  if (rt == 2 || rt == 5) {
    const T a_abs = fabs(a), b_abs = fabs(b);
    const T a3 = a_abs + a_abs + a_abs, b3 = b_abs + b_abs + b_abs;
    r = T(0.5) * (a + b);
    r = (b3 <= a_abs) ? b + b : r;
    r = (a3 <= b_abs) ? a + a : r;
  } else if (rt == 0 || rt == 3) {
    r = (fabs(a) <= fabs(b)) ? a : b;
  } else {
    r = T(2) * s / (a + b);
  }
  return (s <= T(0)) ? T(0) : r;
}

template <class T>
__device__ __forceinline__ void para_cell(T yi, T l, T r, T *lnew, T *rnew)  // recon.c:624-638
{
  const T qa = (r - yi) * (yi - l);
  const T r2 = r + r, l2 = l + l, y3 = yi + yi + yi;
  const T cl = l + r2, cr = l2 + r;
  const bool up = r > l;
  const bool movel = up ? (y3 > cl) : (y3 < cl);
  const bool mover = up ? (y3 < cr) : (y3 > cr);
  const bool flat = qa <= T(0);
  *lnew = flat ? yi : (movel ? y3 - r2 : l);
  *rnew = flat ? yi : (mover ? y3 - l2 : r);
}

template <class T>
__device__ __forceinline__ T linear_recon(int rt, T y1, T y2, T y3)  // recon.c:86-125
{
  T Dqm, Dqp, s;
  if (rt == 2) {
    Dqm = T(2) * (y2 - y1);
    Dqp = T(2) * (y3 - y2);
    const T Dqc = T(0.5) * (y3 - y1);
    s = Dqm * Dqp;
    if (s <= T(0)) return T(0);
    const T aDqm = fabs(Dqm), aDqp = fabs(Dqp), aDqc = fabs(Dqc);
    if ((aDqm <= aDqp) && (aDqm <= aDqc)) return Dqm;
    if (aDqp <= aDqc) return Dqp;
    return Dqc;
  }
  Dqm = (y2 - y1);
  Dqp = (y3 - y2);
  s = Dqm * Dqp;
  if (s <= T(0)) return T(0);
  if (rt == 0) return (fabs(Dqm) < fabs(Dqp)) ? Dqm : Dqp;
  return T(2) * s / (Dqm + Dqp);
}

// PPM states at face f from y[0..5] = zones f-3 .. f+2: *yl = right edge of
// zone f-1, *yr = left edge of zone f.  The slope limiter is the one of
// linear_recon_vect for RECON_TYPE_CHOICE rt (also used by the EMF
// reconstruction of flux_ct_para_fast2 whatever rt is).
template <class T>
__device__ __forceinline__ void ppm_face(int rt, const T *y, T *yl, T *yr)
{
  // slopes of zones f-2 .. f+1
  const T d0 = y[1] - y[0], d1 = y[2] - y[1], d2 = y[3] - y[2], d3 = y[4] - y[3], d4 = y[5] - y[4];
  const T q1 = slope_vect(rt, d0, d1);  // zone f-2
  const T q2 = slope_vect(rt, d1, d2);  // zone f-1
  const T q3 = slope_vect(rt, d2, d3);  // zone f
  const T q4 = slope_vect(rt, d3, d4);  // zone f+1
  // face values between zones (f-2,f-1), (f-1,f), (f,f+1)
  const T rA = T(0.5) * (y[2] + y[1]) - T(HG_PPM_FACTOR) * (q2 - q1);
  const T rB = T(0.5) * (y[3] + y[2]) - T(HG_PPM_FACTOR) * (q3 - q2);
  const T rC = T(0.5) * (y[4] + y[3]) - T(HG_PPM_FACTOR) * (q4 - q3);
  T ln, rn;
  para_cell(y[2], rA, rB, &ln, &rn);  // zone f-1
  *yl = rn;
  para_cell(y[3], rB, rC, &ln, &rn);  // zone f
  *yr = ln;
}

// Face states from 6 zone values (y[0] = zone f-3).
template <class T>
__device__ __forceinline__ void recon_face(int rt, const T *y, T *yl, T *yr)
{
  if (rt >= 3) {
    ppm_face(rt, y, yl, yr);
  } else {
    const T dl = T(0.5) * linear_recon(rt, y[1], y[2], y[3]);  // zone f-1
    const T dr = T(0.5) * linear_recon(rt, y[2], y[3], y[4]);  // zone f
    *yl = y[2] + dl;
    *yr = y[3] - dr;
  }
}

// PPM edge values of zone c on a line: *ln = left edge, *rn = right edge,
// from y[0..4] = zones c-2 .. c+2 (the EMF reconstruction of flux_ct.c:759-939).
template <class T>
__device__ __forceinline__ void ppm_zone(int rt, const T *y, T *ln, T *rn)
{
  const T d0 = y[1] - y[0], d1 = y[2] - y[1], d2 = y[3] - y[2], d3 = y[4] - y[3];
  const T q1 = slope_vect(rt, d0, d1);
  const T q2 = slope_vect(rt, d1, d2);
  const T q3 = slope_vect(rt, d2, d3);
  const T l = T(0.5) * (y[2] + y[1]) - T(HG_PPM_FACTOR) * (q2 - q1);
  const T r = T(0.5) * (y[3] + y[2]) - T(HG_PPM_FACTOR) * (q3 - q2);
  para_cell(y[2], l, r, ln, rn);
}

// ---------------------------------------------------------------------------
// Con2prim (utoprim_2d_fast.c:135-740).  Returns the reference's codes.
__device__ __forceinline__ int utoprim_2d(const double *U, const Geom &g, double gam, double *prim, double *gamma_out,
                                          double *bsq_out)
{
  if (U[0] <= 0.) return -100;
  const double inv_gdet = g.g_inv, alpha = g.alpha, gf = alpha * inv_gdet;
  prim[B1] = U[B1] * inv_gdet;
  prim[B2] = U[B2] * inv_gdet;
  prim[B3] = U[B3] * inv_gdet;
  const double UtRHO = gf * U[RHO];
  const double Qcov[4] = {gf * (U[UU] - U[RHO]), gf * U[U1], gf * U[U2], gf * U[U3]};
  const double Bcon[4] = {0., gf * U[B1], gf * U[B2], gf * U[B3]};
  const double gmog = (gam - 1.) / gam;
  const double Bsq = quad3(g, Bcon[1], Bcon[2], Bcon[3]);
  double Qcon[4];
  raise4(Qcov, g, Qcon);
  const double QdotB = Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  const double QdotBsq = QdotB * QdotB;
  const double Qdotn = -alpha * Qcon[0];
  const double Qsq = Qcov[0] * Qcon[0] + Qcov[1] * Qcon[1] + Qcov[2] * Qcon[2] + Qcov[3] * Qcon[3];
  const double Qtsq = Qsq + Qdotn * Qdotn;
  const double D = UtRHO;
  const double half_Bsq = 0.5 * Bsq;
  double utsq = quad3(g, prim[U1], prim[U2], prim[U3]);
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > HG_UTSQ_TOO_BIG) return 2;
  const double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = D / gamma;
  double u = prim[UU];
  double p = (gam - 1.) * u;
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * Bsq) - QdotBsq * (2. * W_last + Bsq)) <=
          W_last * W_last * (Qtsq - Bsq * Bsq)) &&
         (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  double x0 = fabs(W_last), x1;
  {
    const double Wsq = W_last * W_last, Bsq_W = Bsq + W_last, Xsq = Bsq_W * Bsq_W;
    const double vsq = fabs((Wsq * Qtsq + QdotBsq * (Bsq_W + W_last)) / (Wsq * Xsq));
    x1 = (vsq > 1.) ? (1.0 - 1.e-15) : vsq;
  }
  // general_newton_raphson (utoprim_2d_fast.c:489-592) with func_vsq (:613-665)
  double f = 1., df = 1., errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    const double W = x0, vsq = x1;
    const double ftmp = 1. - vsq, gtmp = sqrt(ftmp);
    const double dPdW = gmog * ftmp;
    const double dPdvsq = gmog * (0.5 * D / gtmp - W);
    const double p_tmp = gmog * (W * ftmp - D * gtmp);
    const double t2 = -half_Bsq + dPdvsq;
    const double t3 = Bsq + W;
    const double t4 = t3 * t3;
    const double t23 = 1 / W;
    const double t16 = QdotBsq * t23 * t23;
    const double t11 = Qtsq - vsq * t4 + t16 * (Bsq + W + W);
    const double t18 = -Qdotn - half_Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
    const double t24 = t16 * t23;
    const double t25 = -1.0 + dPdW - t24;
    const double t35 = t25 * t3 + (Bsq - 2.0 * dPdvsq) * (t16 + vsq * W) * t23;
    const double t21 = 1 / (t3 * t35);
    const double dx0 = -(t2 * t11 + t4 * t18) * t21;
    const double t40 = -2 * (vsq + t24) * t3;
    const double dx1 = -(-t25 * t11 + t40 * t18) * t21;
    df = -t11 * t11 - t18 * t18;
    f = -0.5 * df;
    const double xo0 = x0;
    x0 += dx0;
    x1 += dx1;
    errx = (x0 == 0.) ? fabs(dx0) : fabs(dx0 / x0);
    if (x0 < 0.) x0 = fabs(x0);
    else if (x0 > HG_W_TOO_BIG) x0 = xo0;
    if (x1 < 0.) x1 = 0.;
    else if (x1 > 1.) x1 = (1. - 1.e-15);
    if ((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0) && (HG_EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0)) || (i_extra > HG_EXTRA_NEWT_ITER) ||
        (n_iter >= (HG_MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  int retval;
  if (!isfinite(f) || !isfinite(df)) retval = 2;
  else if (fabs(errx) <= HG_NEWT_TOL) retval = 0;
  else if ((fabs(errx) <= HG_MIN_NEWT_TOL) && (fabs(errx) > HG_NEWT_TOL)) retval = 0;
  else retval = 1;
  const double W = x0, vsq = x1;
  if ((retval != 0) || (W == HG_FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > HG_W_TOO_BIG) return 3;
  if (vsq >= 1.) return 4;
  const double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = D * gtmp;
  *gamma_out = gamma;
  w = W * (1. - vsq);
  p = (gam - 1.) * (w - rho0) / gam;
  u = w - (rho0 + p);
  const double g_o_WBsq = gamma / (W + Bsq);
  const double QdB_o_W = QdotB / W;
  *bsq_out = Bsq * (1. - vsq) + QdB_o_W * QdB_o_W;
  prim[RHO] = rho0;
  prim[UU] = u;
  prim[U1] = g_o_WBsq * (Qcon[1] + g.ncon[1] * Qdotn + QdB_o_W * Bcon[1]);
  prim[U2] = g_o_WBsq * (Qcon[2] + g.ncon[2] * Qdotn + QdB_o_W * Bcon[2]);
  prim[U3] = g_o_WBsq * (Qcon[3] + g.ncon[3] * Qdotn + QdB_o_W * Bcon[3]);
  return 0;
}

__device__ __forceinline__ int check_gamma(double gamma)  // fixup.c:133-141
{
  if (gamma <= HG_GAMMAMAX) return 0;
  if (gamma > HG_GAMMAMAX2) return 2;
  return 1;
}

}  // namespace hg
