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

struct State {
  double ucon[4], ucov[4], bcon[4], bcov[4];
  double bsq, p, eta, ptot;
};

__device__ __forceinline__ long off3(const GridDev &G, int i, int j, int k)
{
  return i * G.st[0] + j * G.st[1] + k * G.st[2];
}

// get_geometry (macros.h:605) for the static metrics: metric_dim 0 uses one
// struct, metric_dim 2 the (pos,i,j) tables.
__device__ __forceinline__ void load_geom(const GridDev &G, int pos, int i, int j, Geom &g)
{
  if (G.mdim == 0) {
    g = G.g0;
    return;
  }
  const int ii = G.deg[0] ? 0 : i, jj = G.deg[1] ? 0 : j;
  const long o = ((long)pos * G.T[1] + jj) * G.T[0] + ii;
  const double *t = G.geomT + o;
  const long s = G.gS;
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

__device__ __forceinline__ void lower4(const double *v, const Geom &g, double *w)  // metric.c:338
{
#pragma unroll
  for (int a = 0; a < 4; a++)
    w[a] = g.gcov[a][0] * v[0] + g.gcov[a][1] * v[1] + g.gcov[a][2] * v[2] + g.gcov[a][3] * v[3];
}

__device__ __forceinline__ void raise4(const double *v, const Geom &g, double *w)  // metric.c:362
{
#pragma unroll
  for (int a = 0; a < 4; a++)
    w[a] = g.gcon[a][0] * v[0] + g.gcon[a][1] * v[1] + g.gcon[a][2] * v[2] + g.gcon[a][3] * v[3];
}

// The gcov-weighted spatial quadratic form of gamma_calc (phys.c:249-255),
// Utoprim_new_body's Bsq and utsq (utoprim_2d_fast.c:255-304).
__device__ __forceinline__ double quad3(const Geom &g, double a, double b, double c)
{
  return g.gcov[1][1] * a * a + g.gcov[2][2] * b * b + g.gcov[3][3] * c * c +
         2 * (g.gcov[1][2] * a * b + g.gcov[1][3] * a * c + g.gcov[2][3] * b * c);
}

__device__ __forceinline__ int gamma_calc(const double *pr, const Geom &g, double *gamma)  // phys.c:244-270
{
  double qsq = quad3(g, pr[U1], pr[U2], pr[U3]);
  if (qsq < 0.) {
    if (fabs(qsq) > 1.E-10) {
      *gamma = 1.;
      return 1;
    }
    qsq = 1.E-10;
  }
  *gamma = sqrt(1. + qsq);
  return 0;
}

// get_state (phys.c:199), with ucon_calc (phys.c:216) and bcon_calc (phys.c:75).
// Returns 1 if gamma_calc failed (the caller books FAIL_GAMMA_CALC).
__device__ __forceinline__ int get_state(const double *pr, const Geom &g, double gam, State &q)
{
  double gamma;
  const int bad = gamma_calc(pr, g, &gamma);
  q.ucon[0] = gamma * g.ncon[0];
  q.ucon[1] = pr[U1] - q.ucon[0] * g.beta[0];
  q.ucon[2] = pr[U2] - q.ucon[0] * g.beta[1];
  q.ucon[3] = pr[U3] - q.ucon[0] * g.beta[2];
  lower4(q.ucon, g, q.ucov);
  const double inv_ut = 1. / q.ucon[0];
  q.bcon[0] = pr[B1] * q.ucov[1] + pr[B2] * q.ucov[2] + pr[B3] * q.ucov[3];
  q.bcon[1] = (pr[B1] + q.bcon[0] * q.ucon[1]) * inv_ut;
  q.bcon[2] = (pr[B2] + q.bcon[0] * q.ucon[2]) * inv_ut;
  q.bcon[3] = (pr[B3] + q.bcon[0] * q.ucon[3]) * inv_ut;
  lower4(q.bcon, g, q.bcov);
  q.bsq = q.bcon[0] * q.bcov[0] + q.bcon[1] * q.bcov[1] + q.bcon[2] * q.bcov[2] + q.bcon[3] * q.bcov[3];
  q.p = (gam - 1.) * pr[UU];
  q.eta = q.p + pr[RHO] + pr[UU] + q.bsq;
  q.ptot = q.p + 0.5 * q.bsq;
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

__device__ __forceinline__ void vchar_fast(const State &q, const Geom &g, int js, double gam, double *vmax,
                                           double *vmin)  // phys.c:432-501
{
  double cms2 = (gam * q.p + q.bsq) / q.eta;
  if (cms2 < 0.) cms2 = HG_SMALL;
  else if (cms2 > 1.) cms2 = 1.;
  const double Au2 = q.ucon[js] * q.ucon[js];
  const double Bu2 = q.ucon[0] * q.ucon[0];
  const double AuBu = q.ucon[js] * q.ucon[0];
  const double A = Bu2 - (g.gcon[0][0] + Bu2) * cms2;
  const double B = AuBu - (g.gcon[0][js] + AuBu) * cms2;
  const double C = Au2 - (g.gcon[js][js] + Au2) * cms2;
  double discr = B * B - A * C;
  if (discr < 0.) discr = 0.;
  discr = sqrt(discr);
  const double denom = 1. / A;
  const double vp = -(-B + discr) * denom;
  const double vm = -(-B - discr) * denom;
  if (vp > vm) {
    *vmax = vp;
    *vmin = vm;
  } else {
    *vmax = vm;
    *vmin = vp;
  }
}

// ---------------------------------------------------------------------------
// Reconstruction of one variable at one face from the six zones around it.
// y[0..5] are zones f-3 .. f+2 along the direction; *yl is the left state
// (right edge of zone f-1, p_L[f]) and *yr the right state (left edge of zone
// f, p_R[f]).  PPM: linear_recon_vect (recon.c:237-264) + para_vect
// (recon.c:611-641); limiters: linear_recon (recon.c:86-125).

__device__ __forceinline__ double slope_vect(int rt, double a, double b)  // recon.c:246-260
{
  const double s = a * b;
  if (s <= 0.) return 0.;
  if (rt == 2 || rt == 5) {
    const double a_abs = fabs(a), b_abs = fabs(b);
    const double a3 = a_abs + a_abs + a_abs, b3 = b_abs + b_abs + b_abs;
    if (a3 <= b_abs) return a + a;
    if (b3 <= a_abs) return b + b;
    return 0.5 * (a + b);
  }
  if (rt == 0 || rt == 3) return (fabs(a) <= fabs(b)) ? a : b;
  return 2 * s / (a + b);
}

__device__ __forceinline__ void para_cell(double yi, double l, double r, double *lnew, double *rnew)  // recon.c:624-638
{
  const double qa = (r - yi) * (yi - l);
  if (qa <= 0.) {
    *lnew = *rnew = yi;
    return;
  }
  const double r2 = r + r, l2 = l + l, y3 = yi + yi + yi;
  double ln = l, rn = r;
  if (r > l) {
    if (y3 > (l + r2)) ln = y3 - r2;
    if (y3 < (l2 + r)) rn = y3 - l2;
  } else {
    if (y3 < (l + r2)) ln = y3 - r2;
    if (y3 > (l2 + r)) rn = y3 - l2;
  }
  *lnew = ln;
  *rnew = rn;
}

__device__ __forceinline__ double linear_recon(int rt, double y1, double y2, double y3)  // recon.c:86-125
{
  double Dqm, Dqp, s;
  if (rt == 2) {
    Dqm = 2. * (y2 - y1);
    Dqp = 2. * (y3 - y2);
    const double Dqc = 0.5 * (y3 - y1);
    s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    const double aDqm = fabs(Dqm), aDqp = fabs(Dqp), aDqc = fabs(Dqc);
    if ((aDqm <= aDqp) && (aDqm <= aDqc)) return Dqm;
    if (aDqp <= aDqc) return Dqp;
    return Dqc;
  }
  Dqm = (y2 - y1);
  Dqp = (y3 - y2);
  s = Dqm * Dqp;
  if (s <= 0.) return 0.;
  if (rt == 0) return (fabs(Dqm) < fabs(Dqp)) ? Dqm : Dqp;
  return 2. * s / (Dqm + Dqp);
}

// PPM states at face f from y[0..5] = zones f-3 .. f+2: *yl = right edge of
// zone f-1, *yr = left edge of zone f.  The slope limiter is the one of
// linear_recon_vect for RECON_TYPE_CHOICE rt (also used by the EMF
// reconstruction of flux_ct_para_fast2 whatever rt is).
__device__ __forceinline__ void ppm_face(int rt, const double *y, double *yl, double *yr)
{
  // slopes of zones f-2 .. f+1
  const double d0 = y[1] - y[0], d1 = y[2] - y[1], d2 = y[3] - y[2], d3 = y[4] - y[3], d4 = y[5] - y[4];
  const double q1 = slope_vect(rt, d0, d1);  // zone f-2
  const double q2 = slope_vect(rt, d1, d2);  // zone f-1
  const double q3 = slope_vect(rt, d2, d3);  // zone f
  const double q4 = slope_vect(rt, d3, d4);  // zone f+1
  // face values between zones (f-2,f-1), (f-1,f), (f,f+1)
  const double rA = 0.5 * (y[2] + y[1]) - HG_PPM_FACTOR * (q2 - q1);
  const double rB = 0.5 * (y[3] + y[2]) - HG_PPM_FACTOR * (q3 - q2);
  const double rC = 0.5 * (y[4] + y[3]) - HG_PPM_FACTOR * (q4 - q3);
  double ln, rn;
  para_cell(y[2], rA, rB, &ln, &rn);  // zone f-1
  *yl = rn;
  para_cell(y[3], rB, rC, &ln, &rn);  // zone f
  *yr = ln;
}

// Face states from 6 zone values (y[0] = zone f-3).
__device__ __forceinline__ void recon_face(int rt, const double *y, double *yl, double *yr)
{
  if (rt >= 3) {
    ppm_face(rt, y, yl, yr);
  } else {
    const double dl = 0.5 * linear_recon(rt, y[1], y[2], y[3]);  // zone f-1
    const double dr = 0.5 * linear_recon(rt, y[2], y[3], y[4]);  // zone f
    *yl = y[2] + dl;
    *yr = y[3] - dr;
  }
}

// PPM edge values of zone c on a line: *ln = left edge, *rn = right edge,
// from y[0..4] = zones c-2 .. c+2 (the EMF reconstruction of flux_ct.c:759-939).
__device__ __forceinline__ void ppm_zone(int rt, const double *y, double *ln, double *rn)
{
  const double d0 = y[1] - y[0], d1 = y[2] - y[1], d2 = y[3] - y[2], d3 = y[4] - y[3];
  const double q1 = slope_vect(rt, d0, d1);
  const double q2 = slope_vect(rt, d1, d2);
  const double q3 = slope_vect(rt, d2, d3);
  const double l = 0.5 * (y[2] + y[1]) - HG_PPM_FACTOR * (q2 - q1);
  const double r = 0.5 * (y[3] + y[2]) - HG_PPM_FACTOR * (q3 - q2);
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
