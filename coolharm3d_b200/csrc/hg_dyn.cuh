// hg_dyn.cuh -- geometry of the time-dependent metric path (metric_dim 3,
// the reference's METRIC_GENERAL_DYNAMIC): the metric at any position and
// time, evaluated on the device, and the connection rebuilt from it every
// substep by 4th-order differences.
//
// The reference stores the geometry of three time levels -- the step's start
// n_beg, its half step n_mid and its end n_end -- at the five positions of
// every cell (set_general_geometry, metric.c:3390-3499), rotates them each
// step (advance_geometry, metric.c:398-430), and rebuilds the connection
// before each substep from those tables (set_general_conn,
// metric.c:3507-3648; conn_func_fd4 and the backward-differenced _lo2/_hi2
// variants at physical x2 boundaries, metric.c:212-340; stencils conn.h).
// Here the three levels are tables in HBM filled by k_geom_level from the
// metric function at the level's time; the connection is a 3D table filled
// by k_conn_dyn before each substep.  Spacetimes: the reference's
// Minkowski-spherical test spacetime (METRIC_DYNAMIC_MINK_SPHERICAL), in
// COORD_DIAGONAL3 modified spherical coordinates (coord.c:270-276,
// 468-472).  A post-Newtonian metric plugs in as one more gcov function.
//
// Every function restates the reference routine named beside it in the same
// operation order; the elementary functions (exp, sincos, pow) are the
// platform's, so the device's tables agree with the reference's to their
// last-bit rounding, not bit for bit.
#pragma once
#include <math.h>

#include "hg_internal.h"

namespace hg {

#define HG_DYN_HD __host__ __device__ __forceinline__
#define HG_GCON_EPS (-1.e-3)  // set_general_geometry's bound on gcon[0][0] (metric.c:3392)
#define HG_SINGSMALL 1.e-16   // options.h:271 (COORDSINGFIX 1)

// seesaw(x, 0, 1) (coord.c:4316-4324) with PERIODIC (macros.h:489-490)
HG_DYN_HD double dyn_seesaw(double x)
{
  const double x0 = 0., xn = 1.;
  const double xn2 = 2 * xn - x0;
  const int shift = (x < x0) ? (1 + (int)(fabs(x - x0) / (xn2 - x0))) : (-(int)(fabs(x - x0) / (xn2 - x0)));
  const double x1 = x + (xn2 - x0) * shift;
  return (x1 < xn) ? (x1 - x0) : (xn2 - x1);
}

// numerical coordinates of a cell position (coord(), coord.c:182-233)
HG_DYN_HD void dyn_xp(const GridDev &G, int pos, int i, int j, int k, double t, double *xp)
{
  xp[0] = t;
  xp[1] = G.startx[1] + (pos == 0 || pos == 4 ? (double)i : (i + 0.5)) * G.dx[1];
  xp[2] = G.startx[2] + (pos == 1 || pos == 4 ? (double)j : (j + 0.5)) * G.dx[2];
  xp[3] = G.startx[3] + (pos == 2 || pos == 4 ? (double)k : (k + 0.5)) * G.dx[3];
}

// x_of_xp, dx_dxp_calc, dxp_dx_calc2_default, det_dx_dxp_calc2_default for
// COORD_DIAGONAL3 (coord.c:270-276, 468-472, 1629-1652, 837-841)
HG_DYN_HD void dyn_coords(const DynMetric &m, const double *xp, double *x, double dx_dxp[4][4], double dxp_dx[4][4],
                          double *det)
{
  const double ftmp = 2 * dyn_seesaw(xp[2]) - 1.;
  x[0] = xp[0];
  x[1] = m.R0 + exp(xp[1]);
  x[2] = 0.5 * M_PI * (1. + m.h_slope * ftmp + m.diag3_factor * pow(ftmp, (double)m.diag3_exponent));
  x[3] = xp[3];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) dx_dxp[a][b] = (a == b) ? 1. : 0.;
  dx_dxp[1][1] = x[1] - m.R0;
  dx_dxp[2][2] = M_PI * (m.h_slope + m.diag3_exponent * m.diag3_factor * pow(ftmp, (double)(m.diag3_exponent - 1)));
  const double a11 = dx_dxp[1][1], a12 = dx_dxp[1][2], a21 = dx_dxp[2][1], a22 = dx_dxp[2][2];
  const double inv_det = 1. / (a11 * a22 - a12 * a21);
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) dxp_dx[a][b] = (a == b) ? 1. : 0.;
  dxp_dx[1][1] = a22 * inv_det;
  dxp_dx[1][2] = -a12 * inv_det;
  dxp_dx[2][1] = -a21 * inv_det;
  dxp_dx[2][2] = a11 * inv_det;
  *det = dx_dxp[0][0] * dx_dxp[3][3] * (dx_dxp[1][1] * dx_dxp[2][2] - dx_dxp[1][2] * dx_dxp[2][1]);
}

// trigvalues (metric.c:29-41): sincos with COORDSINGFIX
HG_DYN_HD void dyn_trig(double th, double *cth, double *sth)
{
  sincos(th, sth, cth);
  if (fabs(*sth) < HG_SINGSMALL) {
    if ((*sth) >= 0) *sth = HG_SINGSMALL;
    if ((*sth) < 0) *sth = -HG_SINGSMALL;
  }
}

// the spacetime's metric in its own coordinates (t, r, th, phi): the
// general_gcov_func of the dynamic path (metric.h:165-167) and, for the
// tables, gcon and sqrt(-g) (mink_spherical_gcov/gcon/gdet_func,
// metric.c:2015-2095)
HG_DYN_HD void dyn_gcov_sth(const double *x, double t1, double gcov[4][4])
{
  const double r = x[1];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) gcov[a][b] = 0.;
  gcov[0][0] = -1.;
  gcov[1][1] = 1.;
  gcov[2][2] = r * r;
  gcov[3][3] = gcov[2][2] * t1 * t1;
}

HG_DYN_HD void dyn_gcov_x(const DynMetric &m, const double *x, double gcov[4][4])
{
  double cth, t1;
  dyn_trig(x[2], &cth, &t1);
  dyn_gcov_sth(x, t1, gcov);
}

// gcon and sqrt(-g) from the same sin(th) (trigvalues is a pure function of
// th: the reference's three calls return the same value)
HG_DYN_HD void dyn_gcon_sth(const double *x, double t2, double gcon[4][4])
{
  const double r = x[1];
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) gcon[a][b] = 0.;
  const double t1 = r * r, t3 = t2 * t2;
  gcon[0][0] = -1.;
  gcon[1][1] = 1.;
  gcon[2][2] = 1. / t1;
  gcon[3][3] = gcon[2][2] / t3;
}

HG_DYN_HD double dyn_gdet_sth(const double *x, double t1) { return x[1] * x[1] * fabs(t1); }

// The struct of_geom of one position at time t: set_general_geometry's loop
// body (metric.c:3453-3483) with transform_all (coord.c:2340-2355:
// transform_rank2cov2 / transform_rank2con2, coord.c:1852-1879, 1975-2002).
HG_DYN_HD void dyn_geom(const GridDev &G, int pos, int i, int j, int k, double t, Geom &g)
{
  const DynMetric &m = G.dyn;
  double xp[4], x[4], dx_dxp[4][4], dxp_dx[4][4], det;
  dyn_xp(G, pos, i, j, k, t, xp);
  dyn_coords(m, xp, x, dx_dxp, dxp_dx, &det);
  double gc[4][4], gn[4][4], cth, sth;
  dyn_trig(x[2], &cth, &sth);
  dyn_gcov_sth(x, sth, gc);
  dyn_gcon_sth(x, sth, gn);
  g.g = dyn_gdet_sth(x, sth);
  // The sums of transform_rank2cov2/con2 in their order, leaving out the
  // terms whose Jacobian factor is exactly zero (most of them: COORD_DIAGONAL3
  // couples only r-x1 and th-x2); adding those zero products changes no sum.
#pragma unroll
  for (int ip = 0; ip < 4; ip++)
#pragma unroll
    for (int jp = 0; jp < 4; jp++) {
      double c = 0., n = 0.;
#pragma unroll
      for (int a = 0; a < 4; a++) {
        const double ja = dx_dxp[a][ip], ka = dxp_dx[ip][a];
#pragma unroll
        for (int b = 0; b < 4; b++) {
          if (ja != 0. && dx_dxp[b][jp] != 0.) c += gc[a][b] * ja * dx_dxp[b][jp];
          if (ka != 0. && dxp_dx[jp][b] != 0.) n += gn[a][b] * ka * dxp_dx[jp][b];
        }
      }
      g.gcov[ip][jp] = c;
      g.gcon[ip][jp] = n;
    }
  g.g *= det;
  g.g_inv = 1. / g.g;
  if (g.gcon[0][0] >= HG_GCON_EPS) g.gcon[0][0] = HG_GCON_EPS;
  g.ncon[0] = sqrt(-g.gcon[0][0]);
  g.alpha = 1. / g.ncon[0];
  g.ncon[1] = -g.alpha * g.gcon[0][1];
  g.ncon[2] = -g.alpha * g.gcon[0][2];
  g.ncon[3] = -g.alpha * g.gcon[0][3];
  g.beta[0] = -g.gcon[0][1] / g.gcon[0][0];
  g.beta[1] = -g.gcon[0][2] / g.gcon[0][0];
  g.beta[2] = -g.gcon[0][3] / g.gcon[0][0];
}

// gcov_func() of the dynamic path (metric.c:3943-3981): the spacetime's
// metric at a position, in its own coordinates (the reference does not
// transform it here; it enters only the time derivative of the connection).
HG_DYN_HD void dyn_gcov_func(const GridDev &G, int pos, int i, int j, int k, double t, double gcov[4][4])
{
  double xp[4], x[4], dx_dxp[4][4], dxp_dx[4][4], det;
  dyn_xp(G, pos, i, j, k, t, xp);
  dyn_coords(G.dyn, xp, x, dx_dxp, dxp_dx, &det);
  dyn_gcov_x(G.dyn, x, gcov);
}

}  // namespace hg
