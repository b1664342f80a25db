// hg_fallback.cuh -- the rarely taken branches of recover_primitives():
// Utoprim_1d, the entropy-equation fix with Utoprim_1d_ee / Utoprim_1d_ee2,
// run by the fallback kernel over a compacted queue of zones whose 2D Newton
// inversion failed or that need the entropy fix.  Same operation order as the
// reference routines named beside each function.  Every power of the density
// goes through hg_cr_pow (correctly rounded, hg_crpow.h) instead of pow().
#pragma once
#include "hg_crpow.h"
#include "hg_phys.cuh"

namespace hg {

// Utoprim_1d (utoprim_1d.c:118-629)
static __device__ __noinline__ int utoprim_1d(const double *U, const Geom &g, double gam, double *prim, double *gamma_out,
                                       double *bsq_out)
{
  double Ut[HG_NPR], pt[HG_NPR];
  const double gdet = g.g;
  for (int i = B1; i <= B3; i++) prim[i] = U[i] / gdet;
  const double alpha = 1.0 / sqrt(-g.gcon[0][0]);
  Ut[RHO] = alpha * U[RHO] / gdet;
  Ut[UU] = alpha * (U[UU] - U[RHO]) / gdet;
  for (int i = U1; i <= U3; i++) Ut[i] = alpha * U[i] / gdet;
  for (int i = B1; i <= B3; i++) Ut[i] = alpha * U[i] / gdet;
  for (int i = 0; i < B1; i++) pt[i] = prim[i];
  double Bcon[4], Bcov[4], Qcov[4], Qcon[4], ncov[4], ncon[4];
  Bcon[0] = 0.;
  for (int i = 1; i < 4; i++) Bcon[i] = Ut[B1 + i - 1];
  lower4(Bcon, g, Bcov);
  for (int i = 0; i < 4; i++) Qcov[i] = Ut[UU + i];
  raise4(Qcov, g, Qcon);
  double Bsq = 0.;
  for (int i = 1; i < 4; i++) Bsq += Bcon[i] * Bcov[i];
  double QdotB = 0.;
  for (int i = 0; i < 4; i++) QdotB += Qcov[i] * Bcon[i];
  const double QdotBsq = QdotB * QdotB;
  ncov[0] = -sqrt(-1. / g.gcon[0][0]);
  ncov[1] = ncov[2] = ncov[3] = 0.;
  raise4(ncov, g, ncon);
  const double Qdotn = Qcon[0] * ncov[0];
  double Qsq = 0.;
  for (int i = 0; i < 4; i++) Qsq += Qcov[i] * Qcon[i];
  const double Qtsq = Qsq + Qdotn * Qdotn;
  const double D = Ut[RHO];
  double utsq = 0.;
  for (int i = 1; i < 4; i++)
    for (int j = 1; j < 4; j++) utsq += g.gcov[i][j] * pt[U1 + i - 1] * pt[U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > HG_UTSQ_TOO_BIG) return 2;
  const double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = D / gamma, u = pt[UU], p = (gam - 1.) * u, w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * Bsq) - QdotBsq * (2. * W_last + Bsq)) <=
          W_last * W_last * (Qtsq - Bsq * Bsq)) &&
         (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  double x = W_last, f = 1., df = 1., errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    // func_1d_orig (utoprim_1d.c:560-600)
    const double dv = 1.0e-15;
    const double W = x, Wsq = W * W;
    double vsq = (Wsq * Qtsq + QdotBsq * (Bsq + 2. * W)) / (Wsq * ((Bsq + W) * (Bsq + W)));
    vsq = (vsq < -dv) ? 0. : fabs(vsq);
    vsq = (vsq > 1.) ? (1. - dv) : vsq;
    const double gtmp = 1. - vsq;
    const double p_tmp = (gam - 1.) * (W * gtmp - D * sqrt(gtmp)) / gam;
    const double X = Bsq + W, W3 = W * W * W, X3 = X * X * X;
    const double dvsq = -2. * (Qtsq / X3 + QdotBsq * (3 * W * X + Bsq * Bsq) / (W3 * X3));
    const double dp1 = (gam - 1.) * (1. - vsq) / gam;
    const double dp2 = (gam - 1.) * (0.5 * D / sqrt(1. - vsq) - W) / gam;
    const double dpdW = dp1 + dp2 * dvsq;
    const double resid = +W + 0.5 * Bsq * (1. + vsq) - 0.5 * QdotBsq / Wsq + Qdotn - p_tmp;
    const double drdW = 1. - dpdW + QdotBsq / (Wsq * W) + 0.5 * Bsq * dvsq;
    const double dx = -resid / drdW;
    f = 0.5 * resid * resid;
    df = -2. * f;
    x += dx;
    i_increase = 0;
    while (((x * x * x * (x + 2. * Bsq) - QdotBsq * (2. * x + Bsq)) <= x * x * (Qtsq - Bsq * Bsq)) &&
           (i_increase < 10)) {
      x -= (1. * i_increase) * dx / 10.;
      i_increase++;
    }
    errx = (x == 0.) ? fabs(dx) : fabs(dx / x);
    x = fabs(x);
    if ((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0) && (HG_EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0)) || (i_extra > HG_EXTRA_NEWT_ITER) ||
        (n_iter >= (HG_MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  int retval;
  if (!isfinite(f) || !isfinite(df)) retval = 2;
  else if (fabs(errx) > HG_MIN_NEWT_TOL) retval = 1;
  else retval = 0;
  const double W = x;
  if ((retval != 0) || (W == HG_FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > HG_W_TOO_BIG) return 3;
  const double Wsq = W * W;
  const double vsq = (Wsq * Qtsq + QdotBsq * (Bsq + 2. * W)) / (Wsq * ((Bsq + W) * (Bsq + W)));
  if (vsq >= 1.) return 4;
  const double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = D * gtmp;
  *gamma_out = gamma;
  w = W * (1. - vsq);
  p = (gam - 1.) * (w - rho0) / gam;
  u = w - (rho0 + p);
  pt[RHO] = rho0;
  pt[UU] = u;
  *bsq_out = Bsq * (1. - vsq) + QdotBsq / (W * W);
  for (int i = 1; i < 4; i++) {
    const double Qtcon = Qcon[i] + ncon[i] * Qdotn;
    pt[U1 + i - 1] = gamma / (W + Bsq) * (Qtcon + QdotB * Bcon[i] / W);
  }
  for (int i = 0; i < B1; i++) prim[i] = pt[i];
  return 0;
}

// Utoprim_1d_ee (utoprim_1d_ee.c:156-847): W Newton with an inner rho Newton.
// The two Newton loops are inlined into utoprim_1d_ee, so EEState lives in
// registers instead of the stack for the whole nested iteration (the
// fallback kernel's time is the longest of these chains).
struct EEState {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, Sc, rho_gm1, two_Bsq;
  double W_for_gnr2, rho_for_gnr2, W_for_gnr2_old, rho_for_gnr2_old, drho_dW;
  double g_o_gm1, gm1, gm1_inv, gam;
  double t2, t4, t7, t24, t300, t400, s100, s200;
};

static __device__ __forceinline__ int ee_gnr2(EEState &s, double *x)  // gnr2 + func_rho (utoprim_1d_ee.c:640-847)
{
  double f = 1., df = 1., errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    const double rho = x[0], W = s.W_for_gnr2;
    const double t40 = hg_cr_pow(rho, s.gm1);
    s.rho_gm1 = t40;
    const double resid = (rho * W + (-t40 * s.s100 - s.D) * s.D);
    const double t14 = t40 / rho;
    const double jac = -t14 * s.s200 + W;
    const double dx = -resid / jac;
    df = -resid * resid;
    f = -0.5 * df;
    x[0] += dx;
    errx = (x[0] == 0.) ? fabs(dx) : fabs(dx / x[0]);
    x[0] = fabs(x[0]);
    // the reference sets doing_extra = 0 here, so no extra iterations are made
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= HG_NEWT_TOL2) && (doing_extra == 0)) || (i_extra > HG_EXTRA_NEWT_ITER) ||
        (n_iter >= (HG_MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x[0])) return 2;
  if (fabs(errx) <= HG_NEWT_TOL) return 0;
  if ((fabs(errx) <= HG_MIN_NEWT_TOL) && (fabs(errx) > HG_NEWT_TOL)) return 0;
  return 1;
}

static __device__ __forceinline__ int ee_gnr(EEState &s, double *x)  // general_newton_raphson + func_W
{
  double f = 1., df = 1., errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    const double W = x[0];
    double x_rho[1], rho_g;
    s.W_for_gnr2_old = s.W_for_gnr2;
    s.W_for_gnr2 = W;
    rho_g = x_rho[0] = s.rho_for_gnr2;
    int ntries = 0;
    while (ee_gnr2(s, x_rho) && (ntries++ < 10)) {
      rho_g *= 10.;
      x_rho[0] = rho_g;
    }
    s.rho_for_gnr2_old = s.rho_for_gnr2;
    const double rho = s.rho_for_gnr2 = x_rho[0];
    s.rho_gm1 = hg_cr_pow(rho, s.gm1);
    s.drho_dW = -rho * rho / (-s.rho_gm1 * s.s200 + W * rho);
    const double t15 = -(s.D - rho) * (s.D + rho);
    const double t200 = W + s.two_Bsq;
    const double t1000 = rho * s.drho_dW;
    const double resid = (s.t300 + (s.t4 + s.t4 + (s.t400 + t15 * (s.t7 + (t200)*W)) * W) * W) * s.t24;
    const double jac =
        2 * (s.t4 + (s.t400 + t15 * s.t7 + (3.0 * t15 * s.Bsq + s.t7 * t1000 + (t15 + t15 + t1000 * (t200)) * W) * W) * W) *
        s.t24;
    const double dx = -resid / jac;
    df = -resid * resid;
    f = -0.5 * df;
    x[0] += dx;
    errx = (x[0] == 0.) ? fabs(dx) : fabs(dx / x[0]);
    x[0] = fabs(x[0]);
    if ((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0) && (HG_EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0)) || (i_extra > HG_EXTRA_NEWT_ITER) ||
        (n_iter >= (HG_MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x[0])) return 2;
  if (fabs(errx) <= HG_NEWT_TOL) return 0;
  if ((fabs(errx) <= HG_MIN_NEWT_TOL) && (fabs(errx) > HG_NEWT_TOL)) return 0;
  return 1;
}

static __device__ __noinline__ int utoprim_1d_ee(const double *U, double S, const Geom &g, double gam, double *prim,
                                          double *gamma_out)
{
  if (U[0] <= 0.) return -100;
  EEState s;
  s.gam = gam;
  s.gm1 = (gam - 1.);
  s.gm1_inv = 1. / s.gm1;
  s.g_o_gm1 = gam * s.gm1_inv;
  const double inv_gdet = g.g_inv, alpha = g.alpha, gf = alpha * inv_gdet;
  prim[B1] = U[B1] * inv_gdet;
  prim[B2] = U[B2] * inv_gdet;
  prim[B3] = U[B3] * inv_gdet;
  s.Sc = gf * S;
  const double Qcov[4] = {gf * (U[UU] - U[RHO]), gf * U[U1], gf * U[U2], gf * U[U3]};
  const double Bcon[4] = {0., gf * U[B1], gf * U[B2], gf * U[B3]};
  s.Bsq = quad3(g, Bcon[1], Bcon[2], Bcon[3]);
  double Qcon[4];
  raise4(Qcov, g, Qcon);
  const double QdotB = Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  s.QdotBsq = QdotB * QdotB;
  s.Qdotn = -alpha * Qcon[0];
  const double Qsq = Qcov[0] * Qcon[0] + Qcov[1] * Qcon[1] + Qcov[2] * Qcon[2] + Qcov[3] * Qcon[3];
  s.Qtsq = Qsq + s.Qdotn * s.Qdotn;
  s.D = gf * U[RHO];
  s.t2 = s.D * s.D;
  s.t4 = s.QdotBsq * s.t2;
  s.t7 = s.Bsq * s.Bsq;
  s.t24 = 1 / s.t2;
  s.two_Bsq = s.Bsq + s.Bsq;
  s.t300 = s.QdotBsq * s.Bsq * s.t2;
  s.t400 = s.Qtsq * s.t2;
  s.s200 = s.D * gam * s.Sc;
  s.s100 = s.g_o_gm1 * s.Sc;
  double utsq = quad3(g, prim[U1], prim[U2], prim[U3]);
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > HG_UTSQ_TOO_BIG) return 2;
  const double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = s.D / gamma;
  s.rho_gm1 = hg_cr_pow(rho0, s.gm1);
  double p = s.Sc * s.rho_gm1 / gamma;
  double u = p * s.gm1_inv;
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) - s.QdotBsq * (2. * W_last + s.Bsq)) <=
          W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) &&
         (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  s.W_for_gnr2 = s.W_for_gnr2_old = W_last;
  s.rho_for_gnr2 = s.rho_for_gnr2_old = rho0;
  double x1[1] = {W_last};
  int retval = ee_gnr(s, x1);
  const double W = x1[0];
  if ((retval != 0) || (W == HG_FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > HG_W_TOO_BIG) return 3;
  double x_rho[1], rho_g;
  rho_g = x_rho[0] = s.rho_for_gnr2;
  int ntries = 0;
  while ((retval = ee_gnr2(s, x_rho)) && (ntries++ < 10)) {
    rho_g *= 10.;
    x_rho[0] = rho_g;
  }
  s.rho_for_gnr2 = x_rho[0];
  if (retval != 0) return 10;
  rho0 = s.rho_for_gnr2;
  s.rho_gm1 = hg_cr_pow(rho0, s.gm1);
  utsq = (s.D - rho0) * (s.D + rho0) / (rho0 * rho0);
  const double gamma_sq = 1. + utsq;
  gamma = sqrt(gamma_sq);
  *gamma_out = gamma;
  if (utsq < 0.) return 4;
  p = s.Sc * s.rho_gm1 / gamma;
  u = p * s.gm1_inv;
  const double g_o_WBsq = gamma / (W + s.Bsq);
  const double QdB_o_W = QdotB / W;
  prim[RHO] = rho0;
  prim[UU] = u;
  prim[U1] = g_o_WBsq * (Qcon[1] + g.ncon[1] * s.Qdotn + QdB_o_W * Bcon[1]);
  prim[U2] = g_o_WBsq * (Qcon[2] + g.ncon[2] * s.Qdotn + QdB_o_W * Bcon[2]);
  prim[U3] = g_o_WBsq * (Qcon[3] + g.ncon[3] * s.Qdotn + QdB_o_W * Bcon[3]);
  return 0;
}

// Utoprim_1d_ee2 (utoprim_1d_ee2.c:152-590): one Newton iteration in rho.
static __device__ __noinline__ int utoprim_1d_ee2(const double *U, double S, const Geom &g, double gam, double *prim,
                                           double *gamma_out)
{
  if (U[0] <= 0.) return -100;
  const double g_o_gm1 = gam / (gam - 1.);
  const double inv_gdet = 1. / g.g;
  prim[B1] = U[B1] * inv_gdet;
  prim[B2] = U[B2] * inv_gdet;
  prim[B3] = U[B3] * inv_gdet;
  const double alpha = g.alpha, gf = alpha * inv_gdet;
  const double Sc = gf * S;
  const double Qcov[4] = {gf * (U[UU] - U[RHO]), gf * U[U1], gf * U[U2], gf * U[U3]};
  const double Bcon[4] = {0., gf * U[B1], gf * U[B2], gf * U[B3]};
  double Bcov[4], Qcon[4];
  lower4(Bcon, g, Bcov);
  raise4(Qcov, g, Qcon);
  const double Bsq = Bcon[1] * Bcov[1] + Bcon[2] * Bcov[2] + Bcon[3] * Bcov[3];
  const double QdotB = Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  const double QdotBsq = QdotB * QdotB;
  const double ncov0 = -g.alpha;
  const double ncon[4] = {-g.alpha * g.gcon[0][0], -g.alpha * g.gcon[0][1], -g.alpha * g.gcon[0][2],
                          -g.alpha * g.gcon[0][3]};
  const double Qdotn = Qcon[0] * ncov0;
  const double Qsq = Qcov[0] * Qcon[0] + Qcov[1] * Qcon[1] + Qcov[2] * Qcon[2] + Qcov[3] * Qcon[3];
  const double Qtsq = Qsq + Qdotn * Qdotn;
  const double D = gf * U[RHO];
  double utsq = quad3(g, prim[U1], prim[U2], prim[U3]);
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > HG_UTSQ_TOO_BIG) return 2;
  double gamma = sqrt(1. + utsq);
  double x = D / gamma, f = 1., df = 1., errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0;
  bool keep = true;
  while (keep) {
    // func_rho (utoprim_1d_ee2.c:540-585)
    const double rho = x, rhosq = rho * rho;
    const double t200 = 1. / (D * D);
    const double t100 = g_o_gm1 * Sc * hg_cr_pow(rho, (gam - 1.));
    const double W = D * (D + t100) / rho;
    const double dWdrho = D * (-D + t100 * (gam - 2.)) / rhosq;
    const double t1 = W * W, t2 = Bsq + W, t3 = t2 * t2;
    const double vsq = (D - rho) * (D + rho) * t200;
    const double dvsqdrho = -2 * rho * t200;
    const double resid = t1 * (Qtsq - vsq * t3) + QdotBsq * (t2 + W);
    const double t12 = Bsq * Bsq, t17 = dWdrho * vsq;
    const double jac = 2 * QdotBsq * dWdrho +
                       ((Qtsq - vsq * t12) * 2 * dWdrho +
                        (-6 * t17 * Bsq - dvsqdrho * t12 + (-2 * dvsqdrho * Bsq - 4 * t17 - dvsqdrho * W) * W) * W) *
                           W;
    const double dx = -resid / jac;
    f = 0.5 * resid * resid;
    df = -2. * f;
    x += dx;
    errx = (x == 0.) ? fabs(dx) : fabs(dx / x);
    x = fabs(x);
    if ((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0) && (HG_EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= HG_NEWT_TOL) && (doing_extra == 0)) || (i_extra > HG_EXTRA_NEWT_ITER) ||
        (n_iter >= (HG_MAX_NEWT_ITER - 1)))
      keep = false;
    n_iter++;
  }
  int retval;
  if (!isfinite(f) || !isfinite(df) || !isfinite(x)) retval = 2;
  else if (fabs(errx) > HG_MIN_NEWT_TOL) retval = 1;
  else retval = 0;
  const double rho0 = x;
  if ((retval != 0) || (rho0 == HG_FAIL_VAL)) return retval * 100 + 1;
  if (rho0 > HG_W_TOO_BIG) return 3;
  utsq = (D - rho0) * (D + rho0) / (rho0 * rho0);
  const double gamma_sq = 1. + utsq;
  gamma = sqrt(gamma_sq);
  *gamma_out = gamma;
  if (utsq < 0.) return 4;
  const double rho_gm1 = hg_cr_pow(rho0, (gam - 1.));
  const double p = Sc * rho_gm1 / gamma;
  const double u = p / (gam - 1.);
  const double w = rho0 + u + p;
  const double W = w * gamma_sq;
  const double g_o_WBsq = gamma / (W + Bsq);
  const double QdB_o_W = QdotB / W;
  prim[RHO] = rho0;
  prim[UU] = u;
  prim[U1] = g_o_WBsq * (Qcon[1] + ncon[1] * Qdotn + QdB_o_W * Bcon[1]);
  prim[U2] = g_o_WBsq * (Qcon[2] + ncon[2] * Qdotn + QdB_o_W * Bcon[2]);
  prim[U3] = g_o_WBsq * (Qcon[3] + ncon[3] * Qdotn + QdB_o_W * Bcon[3]);
  return 0;
}

}  // namespace hg
