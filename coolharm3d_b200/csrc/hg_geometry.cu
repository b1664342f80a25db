// hg_geometry.cu -- host-side builder of the static geometry tables for
// Kerr-Schild space-time in modified Kerr-Schild coordinates (COORD_DIAGONAL3),
// the init-time work calc_all_geom() does for METRIC_KS_SPHERICAL
// (metric.c:4111-4265; coord.c:270-276, 3754-3800), and of the H/R cooling
// tables cooling_func_hr_disk() fills on its first call (phys.c:683-704).
//
// The metric is the Kerr-Schild form (M = 1); the MKS map is
//   r = R0 + exp(x1),  th = pi/2 (1 + h f + c f^n),  f = 2 seesaw(x2) - 1
// with its diagonal Jacobian.  The connection Gamma^a_bc is built here from
// the metric's own first derivatives, taken by complex-step differentiation
// (d/dx f(x) = Im f(x + i eps) / eps, free of cancellation, exact to
// rounding), rather than from closed-form expressions, so the tables agree
// with the reference's to rounding, not bit for bit.
#include <cmath>
#include <complex>

#include "harmgpu.h"

namespace {

typedef std::complex<double> cd;

struct KSParams {
  double a, R0, h_slope, diag3_factor;
  int diag3_exponent;
};

// seesaw(x, 0, 1) of coord.c:4316-4324: x reflected into [0, 1]
double seesaw01(double x)
{
  const double xn2 = 2.;
  const double shift = (x < 0.) ? (1 + (int)(fabs(x) / xn2)) : (-(int)(fabs(x) / xn2));
  const double x1 = x + xn2 * shift;
  return (x1 < 1.) ? x1 : (xn2 - x1);
}

template <class T>
T ipow(T x, int n)
{
  T r = 1.;
  for (int k = 0; k < n; k++) r *= x;
  return r;
}

// (r, th) at numerical (x1, x2), with x2 already reflected, and the diagonal
// Jacobian entries dr/dx1, dth/dx2 (coord.c:270-276, 466-485)
template <class T>
void mks_map(const KSParams &P, T x1, T x2, T &r, T &th, T &J1, T &J2)
{
  const T f = 2. * x2 - 1.;
  r = P.R0 + exp(x1);
  th = 0.5 * M_PI * (1. + P.h_slope * f + P.diag3_factor * ipow(f, P.diag3_exponent));
  J1 = r - P.R0;
  J2 = M_PI * (P.h_slope + (double)P.diag3_exponent * P.diag3_factor * ipow(f, P.diag3_exponent - 1));
}

// cos, sin of th; |sin th| is held at 1e-16 or above (SINGSMALL of trigvalues)
template <class T>
void trig(T th, T &c, T &s)
{
  c = cos(th);
  s = sin(th);
}

template <>
void trig<double>(double th, double &c, double &s)
{
  c = cos(th);
  s = sin(th);
  if (fabs(s) < 1e-16) s = (s >= 0) ? 1e-16 : -1e-16;
}

// Kerr-Schild covariant metric in (t, r, th, phi), M = 1
template <class T>
void ks_gcov(double a, T r, T th, T g[4][4])
{
  T c, s;
  trig(th, c, s);
  const T rho2 = r * r + a * a * c * c;
  const T z = 2. * r / rho2;
  const T s2 = s * s;
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) g[p][q] = 0.;
  g[0][0] = z - 1.;
  g[0][1] = g[1][0] = z;
  g[0][3] = g[3][0] = -z * a * s2;
  g[1][1] = 1. + z;
  g[1][3] = g[3][1] = -a * (1. + z) * s2;
  g[2][2] = rho2;
  g[3][3] = s2 * (r * r + a * a * (1. + z * s2));
}

// its inverse
void ks_gcon(double a, double r, double th, double g[4][4])
{
  double c, s;
  trig(th, c, s);
  const double rho2 = r * r + a * a * c * c;
  const double im = 1. / rho2;
  const double z = 2. * r * im;
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) g[p][q] = 0.;
  g[0][0] = -1. - z;
  g[0][1] = g[1][0] = z;
  g[1][1] = (r * r - 2. * r + a * a) * im;
  g[1][3] = g[3][1] = a * im;
  g[2][2] = im;
  g[3][3] = im / (s * s);
}

// MKS covariant metric at (x1, x2)
template <class T>
void mks_gcov(const KSParams &P, T x1, T x2, T g[4][4])
{
  T r, th, J1, J2;
  mks_map(P, x1, x2, r, th, J1, J2);
  ks_gcov(P.a, r, th, g);
  const T J[4] = {1., J1, J2, 1.};
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) g[p][q] *= J[p] * J[q];
}

// the 42 doubles of struct of_geom at MKS (x1, x2): gcon, gcov, g, g_inv,
// alpha, beta[3], ncon[4] (globals.h:90-98, metric.c:4170-4247)
void geom_at(const KSParams &P, double x1, double x2, double *out)
{
  double r, th, J1, J2;
  mks_map(P, x1, x2, r, th, J1, J2);
  double gco[4][4], gcn[4][4];
  ks_gcov(P.a, r, th, gco);
  ks_gcon(P.a, r, th, gcn);
  const double J[4] = {1., J1, J2, 1.};
  double c, s;
  trig(th, c, s);
  const double gdet_ks = (r * r + P.a * P.a * c * c) * fabs(s);
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) {
      out[p * 4 + q] = gcn[p][q] / (J[p] * J[q]);
      out[16 + p * 4 + q] = gco[p][q] * J[p] * J[q];
    }
  const double g = gdet_ks * J1 * J2;
  out[32] = g;
  out[33] = 1. / g;
  out[34] = 1. / sqrt(-out[0]);                                  // alpha
  for (int k = 0; k < 3; k++) out[35 + k] = -out[k + 1] / out[0];  // beta^i = -g^{0i}/g^{00}
  out[38] = sqrt(-out[0]);                                        // n^mu = -alpha g^{0mu}
  for (int k = 1; k < 4; k++) out[38 + k] = -out[34] * out[k];
}

// Gamma^a_bc at MKS (x1, x2), conn[(a*4+b)*4+c]
void conn_at(const KSParams &P, double x1, double x2, double *conn)
{
  const double eps = 1e-30;
  cd g1[4][4], g2[4][4];
  mks_gcov(P, cd(x1, eps), cd(x2, 0.), g1);
  mks_gcov(P, cd(x1, 0.), cd(x2, eps), g2);
  double dg[4][4][4];  // dg[c][p][q] = d g_pq / d x^c
  for (int p = 0; p < 4; p++)
    for (int q = 0; q < 4; q++) {
      dg[0][p][q] = 0.;
      dg[1][p][q] = g1[p][q].imag() / eps;
      dg[2][p][q] = g2[p][q].imag() / eps;
      dg[3][p][q] = 0.;
    }
  double geom[HG_NGEOM];
  geom_at(P, x1, x2, geom);
  for (int a = 0; a < 4; a++)
    for (int b = 0; b < 4; b++)
      for (int c = 0; c < 4; c++) {
        double v = 0.;
        for (int d = 0; d < 4; d++) v += geom[a * 4 + d] * (dg[b][d][c] + dg[c][d][b] - dg[d][b][c]);
        conn[(a * 4 + b) * 4 + c] = 0.5 * v;
      }
}

// Prograde ISCO radius of the Bardeen-Press-Teukolsky formula (M = 1) as the
// torus setup evaluates it: set_special_coord() calls risco_calc() before
// asq = a*a is assigned (init.torus.c:241-242, metric.c:458-472), so the
// 3 a^2 term under Z2's root is 0 there and Z2 = Z1.
double risco_setup(double a)
{
  const double z1 = 1. + cbrt(1. - a * a) * (cbrt(1. + a) + cbrt(1. - a));
  const double z2 = sqrt(z1 * z1);
  return 3. + z2 - sqrt((3. - z1) * (3. + z1 + 2. * z2));
}

// u_t^2 and u_phi^2 of the equatorial circular orbit at r (Novikov-Thorne
// functions C, F, G), as target_temperature() forms them (phys.c:810-850)
void nt_u2(double a, double r, double &ut2, double &up2)
{
  const double rm1 = 1. / r, x = sqrt(r), xm3 = 1. / (x * x * x), t1 = a * a * rm1;
  const double C = 1. - 3 * rm1 + 2 * a * xm3, F = 1. - 2 * a * xm3 + t1 * rm1, Gf = 1. - 2 * rm1 + a * xm3;
  ut2 = Gf * Gf / C;
  up2 = F * F * r / C;
}

}  // namespace

namespace hg {
// The Kerr-Schild connection of the physical zones (i, j) of a
// COORD_DIAGONAL3 grid, rows (j + n2 i) of 64: the static connection of the
// dynamic path's Kerr-Schild test spacetime (ks_conn_func at CENT,
// metric.c:3555-3558), by the complex-step derivatives above.
void ks_conn_rows(double a, double R0, double h_slope, double diag3_factor, int diag3_exponent, const double *startx,
                  const double *dx, int n1, int n2, double *out)
{
  const KSParams P = {a, R0, h_slope, diag3_factor, diag3_exponent};
  for (int i = 0; i < n1; i++)
    for (int j = 0; j < n2; j++) {
      const double x1 = startx[1] + (i + HG_NG + 0.5) * dx[1];
      const double x2 = seesaw01(startx[2] + (j + HG_NG + 0.5) * dx[2]);
      conn_at(P, x1, x2, out + 64L * (j + (long)n2 * i));
    }
}
}  // namespace hg

extern "C" int hg_build_geometry_ks_mks(const hg_grid_desc *d, double a, double R0, double h_slope,
                                        double diag3_factor, int32_t diag3_exponent, double h_o_r, double *geom,
                                        double *conn, double *cell6, double *rface, double *cool_omega,
                                        double *cool_temp)
{
  if (!d || !geom || !conn || !cell6 || !rface || diag3_exponent < 3 || !(fabs(a) < 1.)) return HG_ERR_BADARG;
  if (d->n1 < 1 || d->n2 < 1 || d->n3 < 1) return HG_ERR_BADARG;
  const KSParams P = {a, R0, h_slope, diag3_factor, diag3_exponent};
  const int N1T = d->n1 + 2 * HG_NG, N2T = d->n2 + 2 * HG_NG, N3T = d->n3 + 2 * HG_NG;
  const double RHOMIN = 2.e-10, UUMIN = 2.e-12, RHOPOWER = -1.5, UUPOWER = -2.5;  // options.h:233-240
  // positions FACE1, FACE2, FACE3, CENT, CORN (macros.h:184-188), GEOM_ID order
  for (int pos = 0; pos < 5; pos++)
    for (int i = 0; i < N1T; i++)
      for (int j = 0; j < N2T; j++) {
        const double o1 = (pos == 0 || pos == 4) ? 0. : 0.5, o2 = (pos == 1 || pos == 4) ? 0. : 0.5;
        const double x1 = d->startx[1] + (i + o1) * d->dx[1];
        const double x2 = seesaw01(d->startx[2] + (j + o2) * d->dx[2]);
        geom_at(P, x1, x2, geom + (long)HG_NGEOM * (j + (long)N2T * (i + (long)N1T * pos)));
      }
  for (int i = 0; i < d->n1; i++)
    for (int j = 0; j < d->n2; j++) {
      const double x1 = d->startx[1] + (i + HG_NG + 0.5) * d->dx[1];
      const double x2 = seesaw01(d->startx[2] + (j + HG_NG + 0.5) * d->dx[2]);
      conn_at(P, x1, x2, conn + 64L * (j + (long)d->n2 * i));
    }
  const double ri = risco_setup(a);
  for (int i = 0; i < N1T; i++) {
    const double r = R0 + exp(d->startx[1] + (i + 0.5) * d->dx[1]);
    rface[i] = R0 + exp(d->startx[1] + i * d->dx[1]);
    const double rhoflr = RHOMIN * pow(r, RHOPOWER), uuflr = UUMIN * pow(r, UUPOWER);
    for (int j = 0; j < N2T; j++) {
      const double f = 2. * seesaw01(d->startx[2] + (j + 0.5) * d->dx[2]) - 1.;
      const double th = 0.5 * M_PI * (1. + h_slope * f + diag3_factor * ipow(f, diag3_exponent));
      for (int k = 0; k < N3T; k++) {
        double *c = cell6 + (((long)i * N2T + j) * N3T + k) * 6;
        c[0] = rhoflr;
        c[1] = uuflr;
        c[2] = r;
        c[3] = r;
        c[4] = th;
        c[5] = d->startx[3] + (k + 0.5) * d->dx[3];
      }
    }
    if (cool_omega && cool_temp) {
      // omega_circular_equatorial (phys.c:865-905): Keplerian outside the
      // ISCO; inside it, the ISCO orbit's u_mu raised with the metric at r
      double omega;
      if (r >= ri) {
        omega = 1. / (pow(r, 1.5) + a);
      } else {
        double gi[4][4], gr[4][4];
        const double r32 = pow(ri, 1.5);
        const double uphi = 1. / sqrt(2 * a * r32 + ri * ri * (ri - 3.));
        const double v[4] = {uphi * (r32 + a), 0., 0., uphi};
        ks_gcov(a, ri, 0.5 * M_PI, gi);
        double vc[4];
        for (int p = 0; p < 4; p++) vc[p] = gi[p][0] * v[0] + gi[p][3] * v[3];
        ks_gcon(a, r, 0.5 * M_PI, gr);
        double u0 = 0., u3 = 0.;
        for (int p = 0; p < 4; p++) {
          u0 += gr[0][p] * vc[p];
          u3 += gr[3][p] * vc[p];
        }
        omega = u3 / u0;
      }
      cool_omega[i] = omega;
      // target_temperature (phys.c:805-850): T = pi/2 R_z (H/R)^2 / r, with
      // the ISCO's u_t, u_phi inside the ISCO
      double ut2, up2;
      nt_u2(a, r > ri ? r : ri, ut2, up2);
      const double rm1 = 1. / r, term1 = a * a * rm1;
      const double Rz = up2 * rm1 - term1 * (ut2 - 1.);
      cool_temp[i] = 0.5 * M_PI * Rz * h_o_r * h_o_r * rm1;
    }
  }
  return HG_OK;
}
