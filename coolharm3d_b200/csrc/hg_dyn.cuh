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
// operation order.  The elementary functions of the coordinates (exp of x1,
// the power of x2 and sincos of th; sincos of phi for spacetimes that need
// Cartesian positions) depend on one index each: the host evaluates them with
// the platform's libm into per-axis tables at faces and centres
// (dyn_coord_tables), and the device and host evaluations read those, so the
// device's geometry is the host's -- and the reference's -- bit for bit.
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

// Layout of GridDev::ctab (T = stored extents, every direction resolved):
// per axis a value at 2*index + h, h = 0 at the face (index), 1 at the centre
// (index + 1/2).
struct DynTab {
  int r, dr, th, dth, sth, cth, sph, cph, total;
};
HG_DYN_HD DynTab dyn_tab_layout(const int *T)
{
  DynTab L;
  L.r = 0;
  L.dr = L.r + 2 * T[0];
  L.th = L.dr + 2 * T[0];
  L.dth = L.th + 2 * T[1];
  L.sth = L.dth + 2 * T[1];
  L.cth = L.sth + 2 * T[1];
  L.sph = L.cth + 2 * T[1];
  L.cph = L.sph + 2 * T[2];
  L.total = L.cph + 2 * T[2];
  return L;
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

// Kerr-Schild, M = 1, spin a, from cos/sin th: ks_gcov_func, ks_gcon_func
// (metric.c:1168-1250) and ks_gdet_func = bl_gdet_func (metric.c:523-540,
// 1905-1910), in their operation order
HG_DYN_HD void dyn_ks(double r, double cth, double sth, double a, double gcov[4][4], double gcon[4][4],
                      double *gdet)
{
  const double M = 1., asq = a * a;
#pragma unroll
  for (int p = 0; p < 4; p++)
#pragma unroll
    for (int q = 0; q < 4; q++) gcov[p][q] = gcon[p][q] = 0.;
  {
    const double t2 = r * r, t3 = asq, t5 = cth * cth, t7 = t2 + t3 * t5, t9 = M * r / t7, t10 = 2.0 * t9;
    const double t13 = sth * sth;
    gcov[0][0] = t10 - 1.0;
    gcov[0][1] = t10;
    gcov[0][3] = -2.0 * t9 * a * t13;
    gcov[1][0] = t10;
    gcov[1][1] = 1.0 + t10;
    gcov[1][3] = -a * gcov[1][1] * t13;
    gcov[2][2] = t7;
    gcov[3][0] = gcov[0][3];
    gcov[3][1] = gcov[1][3];
    gcov[3][3] = t13 * (t2 + t3 * (1.0 + 2.0 * t9 * t13));
  }
  {
    const double t1 = M * r, t2 = r * r, t3 = asq, t5 = cth * cth, t8 = 1 / (t2 + t3 * t5), t10 = 2.0 * t1 * t8;
    gcon[0][0] = -1.0 - t10;
    gcon[0][1] = t10;
    gcon[1][0] = t10;
    gcon[1][1] = (t2 - 2.0 * t1 + t3) * t8;
    gcon[1][3] = a * t8;
    gcon[2][2] = t8;
    gcon[3][1] = gcon[1][3];
    const double t14 = sth * sth;
    gcon[3][3] = t8 / t14;
  }
  const double cos_2th = (cth - sth) * (cth + sth), r2 = r * r;
  *gdet = r2 * fabs(sth) * (1. + 0.5 * (asq / r2) * (1. + cos_2th));
}

// The coordinates of a position from the tables: x (t, r, th, phi), the
// diagonal Jacobian entries, sin/cos th, and dyn_coords' inverse and
// determinant formed from them as dyn_coords forms them.
struct DynPoint {
  double x[4], a11, a22, i11, i22, det, sth, cth, sph, cph;
};
HG_DYN_HD void dyn_point(const GridDev &G, int pos, int i, int j, int k, double t, DynPoint &q)
{
  const DynTab L = dyn_tab_layout(G.T);
  const double *c = G.ctab;
  const int hi = (pos == 0 || pos == 4) ? 0 : 1, hj = (pos == 1 || pos == 4) ? 0 : 1;
  const int hk = (pos == 2 || pos == 4) ? 0 : 1;
  const int ti = 2 * i + hi, tj = 2 * j + hj, tk = 2 * k + hk;
  q.x[0] = t;
  q.x[1] = c[L.r + ti];
  q.x[2] = c[L.th + tj];
  q.x[3] = G.startx[3] + (pos == 2 || pos == 4 ? (double)k : (k + 0.5)) * G.dx[3];
  q.a11 = c[L.dr + ti];
  q.a22 = c[L.dth + tj];
  q.sth = c[L.sth + tj];
  q.cth = c[L.cth + tj];
  q.sph = c[L.sph + tk];
  q.cph = c[L.cph + tk];
  const double a12 = 0., a21 = 0.;
  const double inv_det = 1. / (q.a11 * q.a22 - a12 * a21);
  q.i11 = q.a22 * inv_det;
  q.i22 = q.a11 * inv_det;
  q.det = 1. * 1. * (q.a11 * q.a22 - a12 * a21);
}

// The tables on the host: r = R0 + exp(x1), th and the Jacobian by
// dyn_coords, sin/cos th by trigvalues, sin/cos phi by sincos, at the face
// and the centre of every index of each axis.
inline void dyn_coord_tables(const GridDev &G, double *c)
{
  const DynTab L = dyn_tab_layout(G.T);
  const int T0 = G.T[0], T1 = G.T[1], T2 = G.T[2];
  for (int n = 0; n < 2 * (T0 > T1 ? (T0 > T2 ? T0 : T2) : (T1 > T2 ? T1 : T2)); n++) {
    const double h = (n & 1) ? 0.5 : 0.;
    const int idx = n >> 1;
    double xp[4] = {0., G.startx[1] + (idx + h) * G.dx[1], G.startx[2] + (idx + h) * G.dx[2],
                    G.startx[3] + (idx + h) * G.dx[3]};
    double x[4], J[4][4], Ji[4][4], det;
    dyn_coords(G.dyn, xp, x, J, Ji, &det);
    if (idx < T0) {
      c[L.r + n] = x[1];
      c[L.dr + n] = J[1][1];
    }
    if (idx < T1) {
      double cth, sth;
      dyn_trig(x[2], &cth, &sth);
      c[L.th + n] = x[2];
      c[L.dth + n] = J[2][2];
      c[L.sth + n] = sth;
      c[L.cth + n] = cth;
    }
    if (idx < T2) {
      double sp, cp;
      sincos(x[3], &sp, &cp);
      c[L.sph + n] = sp;
      c[L.cph + n] = cp;
    }
  }
}

// ---------------------------------------------------------------------------
// HG_DYN_PN_BINARY: the binary's positions and velocities at time t, and the
// first post-Newtonian harmonic-gauge metric of two point masses
//   g00 = -1 + 2V - 2V^2,  g0i = -4 V_i,  gij = (1 + 2V) delta_ij,
//   V = sum m_a / r_a,  V_i = sum m_a v_a^i / r_a
// (the 1PN metric written with the potentials V, V_i, e.g. Blanchet, Faye &
// Ponsot 1998, Phys. Rev. D 58 124002, eq. 7.2 at this order, with V and V_i
// at their instantaneous point-mass values).  No counterpart in the
// reference's sources, whose PN metric bodies are absent.
struct PNBinary {
  double y[2][3], v[2][3], m[2];
};

// Quasi-circular orbit: the separation shrinks by the quadrupole formula
// (Peters 1964): r^4 = r0^4 - (256/5) eta M^3 t, dr/dt = -(64/5) eta M^3 / r^3,
// phase phi0 + (r0^(5/2) - r^(5/2)) / (32 eta M^(5/2)) (the integral of
// Omega = sqrt(M / r^3)); without inspiral r = r0, phi = phi0 + Omega t.
// m1 sits at +m2/M r n, m2 at -m1/M r n, n = (cos phi, sin phi, 0).
HG_DYN_HD void pn_binary(const DynMetric &dm, double t, PNBinary &b)
{
  const double M = dm.m1 + dm.m2, eta = dm.m1 * dm.m2 / (M * M);
  const double r0 = dm.sep, M3 = M * M * M;
  double r = r0, rdot = 0., phi;
  if (dm.inspiral) {
    double q = r0 * r0 * r0 * r0 - (256. / 5.) * eta * M3 * t;
    const double qmin = 1.e-12 * r0 * r0 * r0 * r0;  // past coalescence: hold the smallest orbit
    if (q < qmin) q = qmin;
    r = sqrt(sqrt(q));
    rdot = -(64. / 5.) * eta * M3 / (r * r * r);
    phi = dm.phase0 + (r0 * r0 * sqrt(r0) - r * r * sqrt(r)) / (32. * eta * M * M * sqrt(M));
  } else {
    phi = dm.phase0 + sqrt(M / (r * r * r)) * t;
  }
  const double om = sqrt(M / (r * r * r));
  double sp, cp;
  sincos(phi, &sp, &cp);
  const double f[2] = {dm.m2 / M, -dm.m1 / M};
  b.m[0] = dm.m1;
  b.m[1] = dm.m2;
  for (int a = 0; a < 2; a++) {
    b.y[a][0] = f[a] * r * cp;
    b.y[a][1] = f[a] * r * sp;
    b.y[a][2] = 0.;
    b.v[a][0] = f[a] * (rdot * cp - r * om * sp);
    b.v[a][1] = f[a] * (rdot * sp + r * om * cp);
    b.v[a][2] = 0.;
  }
}

// gcov, gcon and sqrt(-g) of the PN metric at a position, in the grid's
// numerical coordinates: gcov = J^T g_cart J with J = d(t,x,y,z)/d(t,x1,x2,x3)
// (Cartesian of the spherical r, th, phi of the COORD_DIAGONAL3 point), gcon
// = K g_cart^-1 K^T with K = J^-1, and g_cart^-1 from the block form of
// g_cart: with A = 1 + 2V, w = g0i and s = g00 - w.w / A,
// g^00 = 1/s, g^0i = -w_i / (A s), g^ij = delta_ij / A + w_i w_j / (A^2 s),
// det g_cart = A^3 s.
template <bool WITH_GCON = true>
HG_DYN_HD void pn_metric(const PNBinary &b, const DynPoint &q, double gcov[4][4], double gcon[4][4], double *gdet,
                         double *s_out)
{
  const double r = q.x[1];
  const double X[3] = {r * q.sth * q.cph, r * q.sth * q.sph, r * q.cth};
  double V = 0., Vi[3] = {0., 0., 0.};
  for (int a = 0; a < 2; a++) {
    const double d0 = X[0] - b.y[a][0], d1 = X[1] - b.y[a][1], d2 = X[2] - b.y[a][2];
    const double ma = b.m[a] / sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    V += ma;
    for (int c = 0; c < 3; c++) Vi[c] += ma * b.v[a][c];
  }
  const double A = 1. + 2. * V;
  const double g00 = -1. + 2. * V - 2. * V * V;
  const double w[3] = {-4. * Vi[0], -4. * Vi[1], -4. * Vi[2]};
  // columns of J (x1, x2, x3) and rows of K = J^-1
  const double J[3][3] = {{q.a11 * q.sth * q.cph, q.a11 * q.sth * q.sph, q.a11 * q.cth},
                          {q.a22 * r * q.cth * q.cph, q.a22 * r * q.cth * q.sph, -q.a22 * r * q.sth},
                          {-r * q.sth * q.sph, r * q.sth * q.cph, 0.}};
  const double ir = 1. / r, irs = 1. / (r * q.sth);
  const double K[3][3] = {{q.i11 * q.sth * q.cph, q.i11 * q.sth * q.sph, q.i11 * q.cth},
                          {q.i22 * ir * q.cth * q.cph, q.i22 * ir * q.cth * q.sph, -q.i22 * ir * q.sth},
                          {-irs * q.sph, irs * q.cph, 0.}};
  gcov[0][0] = g00;
  for (int a = 0; a < 3; a++) {
    const double c = w[0] * J[a][0] + w[1] * J[a][1] + w[2] * J[a][2];
    gcov[0][a + 1] = c;
    gcov[a + 1][0] = c;
    for (int e = 0; e < 3; e++) gcov[a + 1][e + 1] = A * (J[a][0] * J[e][0] + J[a][1] * J[e][1] + J[a][2] * J[e][2]);
  }
  if (!WITH_GCON) return;  // gcov alone: the connection's time derivative
  const double iA = 1. / A;
  const double s = g00 - (w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) * iA;
  const double is = 1. / s, iAs = iA * is;
  double Kw[3];
  for (int a = 0; a < 3; a++) Kw[a] = K[a][0] * w[0] + K[a][1] * w[1] + K[a][2] * w[2];
  gcon[0][0] = is;
  for (int a = 0; a < 3; a++) {
    gcon[0][a + 1] = -Kw[a] * iAs;
    gcon[a + 1][0] = gcon[0][a + 1];
    for (int e = 0; e < 3; e++)
      gcon[a + 1][e + 1] = (K[a][0] * K[e][0] + K[a][1] * K[e][1] + K[a][2] * K[e][2]) * iA + Kw[a] * Kw[e] * iAs * iA;
  }
  *gdet = sqrt(-(A * A * A * s)) * fabs(q.det * r * r * q.sth);
  *s_out = s;
}

// The struct of_geom of one position at time t: set_general_geometry's loop
// body (metric.c:3453-3483) with transform_all (coord.c:2340-2355:
// transform_rank2cov2 / transform_rank2con2, coord.c:1852-1879, 1975-2002).
// bin: the PN binary at time t when the caller has it (kernels evaluate it
// once per level), else it is evaluated here.
HG_DYN_HD void dyn_geom(const GridDev &G, int pos, int i, int j, int k, double t, Geom &g,
                        const PNBinary *bin = nullptr)
{
  DynPoint q;
  dyn_point(G, pos, i, j, k, t, q);
  if (G.dyn.spacetime == HG_DYN_PN_BINARY) {
    PNBinary b0;
    if (!bin) {
      pn_binary(G.dyn, t, b0);
      bin = &b0;
    }
    double s;
    pn_metric(*bin, q, g.gcov, g.gcon, &g.g, &s);
    // the derived quantities of set_general_geometry, with 1/gcon[0][0] = s
    g.g_inv = 1. / g.g;
    double inv00 = s;
    if (g.gcon[0][0] >= HG_GCON_EPS) {
      g.gcon[0][0] = HG_GCON_EPS;
      inv00 = 1. / HG_GCON_EPS;
    }
    g.ncon[0] = sqrt(-g.gcon[0][0]);
    g.alpha = 1. / g.ncon[0];
    g.ncon[1] = -g.alpha * g.gcon[0][1];
    g.ncon[2] = -g.alpha * g.gcon[0][2];
    g.ncon[3] = -g.alpha * g.gcon[0][3];
    g.beta[0] = -g.gcon[0][1] * inv00;
    g.beta[1] = -g.gcon[0][2] * inv00;
    g.beta[2] = -g.gcon[0][3] * inv00;
    return;
  } else {
  double gc[4][4], gn[4][4];
  if (G.dyn.spacetime == HG_DYN_KS_SPHERICAL) {
    dyn_ks(q.x[1], q.cth, q.sth, G.dyn.spin, gc, gn, &g.g);
  } else {
    dyn_gcov_sth(q.x, q.sth, gc);
    dyn_gcon_sth(q.x, q.sth, gn);
    g.g = dyn_gdet_sth(q.x, q.sth);
  }
  // The sums of transform_rank2cov2/con2 in their order, leaving out the
  // terms whose Jacobian factor is exactly zero (most of them: COORD_DIAGONAL3
  // couples only r-x1 and th-x2); adding those zero products changes no sum.
  const double J[4] = {1., q.a11, q.a22, 1.}, Ji[4] = {1., q.i11, q.i22, 1.};
#pragma unroll
  for (int ip = 0; ip < 4; ip++)
#pragma unroll
    for (int jp = 0; jp < 4; jp++) {
      g.gcov[ip][jp] = gc[ip][jp] * J[ip] * J[jp] + 0.;
      g.gcon[ip][jp] = gn[ip][jp] * Ji[ip] * Ji[jp] + 0.;
    }
  g.g *= q.det;
  }
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
// metric at a position, for the time derivative of the connection.  A
// spacetime in the grid's own (spherical) topology is not transformed there;
// a Cartesian one -- the PN binary -- is taken to the numerical coordinates
// (transform_rank2cov2 with dxc_dxp, metric.c:3968-3976).
HG_DYN_HD void dyn_gcov_func(const GridDev &G, int pos, int i, int j, int k, double t, double gcov[4][4],
                             const PNBinary *bin = nullptr)
{
  DynPoint q;
  dyn_point(G, pos, i, j, k, t, q);
  if (G.dyn.spacetime == HG_DYN_PN_BINARY) {
    PNBinary b0;
    if (!bin) {
      pn_binary(G.dyn, t, b0);
      bin = &b0;
    }
    pn_metric<false>(*bin, q, gcov, nullptr, nullptr, nullptr);
  } else {
    dyn_gcov_sth(q.x, q.sth, gcov);
  }
}

}  // namespace hg
