/* harm_oracle.c -- CPU restatement of the HARM3D step (TEST INFRASTRUCTURE).
 *
 * The oracle: only tests/ and __graft_entry__.smoke() load it, to verify
 * the engine's results.  The product never does (bench.py's CPU baseline
 * runs the reference's own build in oracle/_ref instead).
 *
 * It restates, loop by loop and in the same floating-point evaluation order,
 * the reference's time step of scnastro/coolharm3d (paths below are relative
 * to the reference's src/ directory); each function names the lines it
 * follows.  Compile with -ffp-contract=off so that no multiply-add is fused,
 * exactly like the reference build in oracle/_ref.
 *
 * Supported switch values: recon 0..5, flux LF/HLLE, para or Toth flux-CT,
 * BC cartesian outflow / periodic / spherical outflow3, METRIC_DIM 0 or 2,
 * FIXUP_TREE 3, USE_ENTROPY_EQ 0/1, cooling 0, RESCALE_R 0/1.
 */
#include "harm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* Test hook: tests/test_pow_sensitivity.py rebuilds the oracle with
 * -DOR_POW_HOOK=<function> to perturb every pow() result. */
#ifdef OR_POW_HOOK
double OR_POW_HOOK(double, double);
#define pow OR_POW_HOOK
#endif

#define NP 8
#define NG 3
#define NDIM 4
#define RHO 0
#define UU 1
#define U1 2
#define U2 3
#define U3 4
#define B1 5
#define B2 6
#define B3 7
#define SMALL 1.e-15
#define SAFE 1.3
#define GAMMAMAX 50.
#define GAMMAMAX2 1.e4
#define BETA_MIN 1.e-2
#define PPM_FACTOR 0.16666666666666666667
#define MAX_NEWT_ITER 30
#define NEWT_TOL 1.0e-10
#define MIN_NEWT_TOL 1.0e-10
#define EXTRA_NEWT_ITER 2
#define NEWT_TOL2 1.0e-15
#define W_TOO_BIG 1.e20
#define UTSQ_TOO_BIG 1.e20
#define FAIL_VAL 1.e30

/* nfail[] indices, src/macros.h:243-258 */
enum { NF_FLOOR = 0, NF_TMAX, NF_GAMMA_MAX, NF_GAMMA_CALC, NF_USE_FULL_INV, NF_USE_EE,
       NF_UTOPRIM, NF_UTOPRIM_EE, NF_USE_INTERP_PRIM, NF_USE_INTERP_V, NF_INTERP_PRIM,
       NF_INTERP_V };
/* fail() types used on this path, src/macros.h:207-219 */
enum { F_FLOOR = 1, F_TMAX, F_GAMMA_MAX, F_GAMMA_CALC, F_USE_FULL_INV, F_USE_EE, F_UTOPRIM,
       F_UTOPRIM_EE, F_USE_INTERP_PRIM, F_USE_INTERP_V, F_INTERP_PRIM, F_INTERP_V };
enum { PF_NONE = 0, PF_INTERP_V = 1, PF_INTERP_PRIM = 2 };

typedef struct {
  double gcon[4][4];
  double gcov[4][4];
  double g, g_inv, alpha;
  double beta[3];
  double ncon[4];
} geom_t;

typedef struct {
  double ucon[4], ucov[4], bcon[4], bcov[4];
  double bsq, p, eta, ptot;
} state_t;

struct or_ctx {
  or_desc d;
  int N1, N2, N3, N1T, N2T, N3T;
  long ntot;
  int do_recon[3];
  int nsd; /* n_spatial_dims */
  int r_s[3], r_e[3]; /* N*_R_S, N*_R_E of src/decomp.c:87-121 */
  double invdx[4];
  geom_t *geom;  /* metric_dim 0: 1 entry; 2: NPOS*N1T*N2T */
  double *conn;  /* metric_dim 2: N1*N2*64 */
  double *cell6;
  double *rscale[6];
  double *cool_omega, *cool_temp; /* Omega_gf, T_r_gf of cooling_func_hr_disk (phys.c:683-704) */
  int cool_tables_built;          /* cooling_func_hr_disk's local_first_time has been cleared */
  double *p, *ph, *p_old, *pL, *pR, *F, *emf[3], *cgf, *uconL, *uconR, *U0, *Un, *p_gamma;
  int32_t *pflag;
  int32_t *nfail;
  uint64_t nfailtot[OR_NFAIL];
  double max_char_speed[4];
  double M_tot;
  int failure_exists, failure_type[3], bnd_phys_pflag;
  int n_substep;
  int icur, jcur, kcur, pcur; /* icurr, jcurr, kcurr, pcurr of the reference */
  double *vec, *dq, *vL, *vR;
};

#define IX(c, i, j, k) ((((long)(i)) * (c)->N2T + (j)) * (c)->N3T + (k))

/* ------------------------------------------------------------------------- */
/* geometry lookup: get_geometry macro, src/macros.h:605, GEOM_ID :592-601   */
static geom_t *G(or_ctx *c, int i, int j, int k, int pos)
{
  c->icur = i; c->jcur = j; c->kcur = k; c->pcur = pos;
  if (c->d.metric_dim == 0) return c->geom;
  return &c->geom[j + (long)c->N2T * (i + (long)c->N1T * pos)];
}

/* fail(), src/diag.c:159-330 (the non-fatal branches reached on this path) */
static void check_boundary_pflag(or_ctx *c, int i, int j, int k) /* src/harm_mpi.c:1388-1426 */
{
  if (i < NG + NG || i > c->N1 + NG - 1 - NG) c->bnd_phys_pflag = 1;
  if (j < NG + NG || j > c->N2 + NG - 1 - NG) c->bnd_phys_pflag = 1;
  if (k < NG + NG || k > c->N3 + NG - 1 - NG) c->bnd_phys_pflag = 1;
}

static void fail(or_ctx *c, int type, int state)
{
  static const int resp[3] = {0, PF_INTERP_PRIM, PF_INTERP_V};
  long id = IX(c, c->icur, c->jcur, c->kcur);
  int nf = -1;
  switch (type) {
    case F_FLOOR: nf = NF_FLOOR; break;
    case F_TMAX: nf = NF_TMAX; break;
    case F_GAMMA_MAX: nf = NF_GAMMA_MAX; break;
    case F_GAMMA_CALC: nf = NF_GAMMA_CALC; break;
    case F_USE_FULL_INV: nf = NF_USE_FULL_INV; break;
    case F_USE_EE: nf = NF_USE_EE; break;
    case F_UTOPRIM: nf = NF_UTOPRIM; break;
    case F_UTOPRIM_EE: nf = NF_UTOPRIM_EE; break;
    case F_USE_INTERP_PRIM: nf = NF_USE_INTERP_PRIM; break;
    case F_USE_INTERP_V: nf = NF_USE_INTERP_V; break;
    case F_INTERP_PRIM: nf = NF_INTERP_PRIM; break;
    case F_INTERP_V: nf = NF_INTERP_V; break;
  }
  if (state && type != F_GAMMA_CALC && type != F_USE_FULL_INV && type != F_USE_EE) {
    c->failure_exists = 1;
    check_boundary_pflag(c, c->icur, c->jcur, c->kcur);
    c->pflag[id] = resp[state];
    c->failure_type[resp[state]] = 1;
  }
  c->nfail[(long)nf * c->ntot + id]++;
  c->nfailtot[nf]++;
}

/* ------------------------------------------------------------------------- */
/* physics, src/phys.c and src/metric.c                                       */
static void lower(const double *v, const geom_t *g, double *w) /* metric.c:338 */
{
  w[0] = g->gcov[0][0] * v[0] + g->gcov[0][1] * v[1] + g->gcov[0][2] * v[2] + g->gcov[0][3] * v[3];
  w[1] = g->gcov[1][0] * v[0] + g->gcov[1][1] * v[1] + g->gcov[1][2] * v[2] + g->gcov[1][3] * v[3];
  w[2] = g->gcov[2][0] * v[0] + g->gcov[2][1] * v[1] + g->gcov[2][2] * v[2] + g->gcov[2][3] * v[3];
  w[3] = g->gcov[3][0] * v[0] + g->gcov[3][1] * v[1] + g->gcov[3][2] * v[2] + g->gcov[3][3] * v[3];
}

static void raise(const double *v, const geom_t *g, double *w) /* metric.c:362 */
{
  w[0] = g->gcon[0][0] * v[0] + g->gcon[0][1] * v[1] + g->gcon[0][2] * v[2] + g->gcon[0][3] * v[3];
  w[1] = g->gcon[1][0] * v[0] + g->gcon[1][1] * v[1] + g->gcon[1][2] * v[2] + g->gcon[1][3] * v[3];
  w[2] = g->gcon[2][0] * v[0] + g->gcon[2][1] * v[1] + g->gcon[2][2] * v[2] + g->gcon[2][3] * v[3];
  w[3] = g->gcon[3][0] * v[0] + g->gcon[3][1] * v[1] + g->gcon[3][2] * v[2] + g->gcon[3][3] * v[3];
}

static double quad3(const geom_t *g, double a, double b, double cc) /* the qsq/utsq/Bsq form */
{
  return g->gcov[1][1] * a * a + g->gcov[2][2] * b * b + g->gcov[3][3] * cc * cc +
         2 * (g->gcov[1][2] * a * b + g->gcov[1][3] * a * cc + g->gcov[2][3] * b * cc);
}

static int gamma_calc(const double *pr, const geom_t *g, double *gamma) /* phys.c:244-270 */
{
  double qsq = quad3(g, pr[U1], pr[U2], pr[U3]);
  if (qsq < 0.) {
    if (fabs(qsq) > 1.E-10) { *gamma = 1.; return 1; }
    qsq = 1.E-10;
  }
  *gamma = sqrt(1. + qsq);
  return 0;
}

static void ucon_calc(or_ctx *c, const double *pr, const geom_t *g, double *ucon) /* phys.c:216 */
{
  double gamma;
  if (gamma_calc(pr, g, &gamma)) fail(c, F_GAMMA_CALC, 0);
  ucon[0] = gamma * g->ncon[0];
  ucon[1] = pr[U1] - ucon[0] * g->beta[0];
  ucon[2] = pr[U2] - ucon[0] * g->beta[1];
  ucon[3] = pr[U3] - ucon[0] * g->beta[2];
}

static void bcon_calc(const double *pr, const double *ucon, const double *ucov, double *bcon) /* phys.c:75 */
{
  double inv_ut = 1. / ucon[0];
  bcon[0] = pr[B1] * ucov[1] + pr[B2] * ucov[2] + pr[B3] * ucov[3];
  bcon[1] = (pr[B1] + bcon[0] * ucon[1]) * inv_ut;
  bcon[2] = (pr[B2] + bcon[0] * ucon[2]) * inv_ut;
  bcon[3] = (pr[B3] + bcon[0] * ucon[3]) * inv_ut;
}

static void get_state(or_ctx *c, const double *pr, const geom_t *g, state_t *q) /* phys.c:199 */
{
  ucon_calc(c, pr, g, q->ucon);
  lower(q->ucon, g, q->ucov);
  bcon_calc(pr, q->ucon, q->ucov, q->bcon);
  lower(q->bcon, g, q->bcov);
  q->bsq = q->bcon[0] * q->bcov[0] + q->bcon[1] * q->bcov[1] + q->bcon[2] * q->bcov[2] + q->bcon[3] * q->bcov[3];
  q->p = (c->d.gam - 1.) * pr[UU];
  q->eta = q->p + pr[RHO] + pr[UU] + q->bsq;
  q->ptot = q->p + 0.5 * q->bsq;
}

static void primtoflux(const double *pr, const state_t *q, int dir, const geom_t *g, double *f) /* phys.c:28-63 */
{
  double eta_ucon = q->eta * q->ucon[dir];
  double bcon_dir = q->bcon[dir];
  double mhd[4];
  int l;
  mhd[0] = eta_ucon * q->ucov[0] - bcon_dir * q->bcov[0];
  mhd[1] = eta_ucon * q->ucov[1] - bcon_dir * q->bcov[1];
  mhd[2] = eta_ucon * q->ucov[2] - bcon_dir * q->bcov[2];
  mhd[3] = eta_ucon * q->ucov[3] - bcon_dir * q->bcov[3];
  mhd[dir] += q->ptot;
  f[RHO] = pr[RHO] * q->ucon[dir];
  f[UU] = mhd[0] + f[RHO];
  f[U1] = mhd[1];
  f[U2] = mhd[2];
  f[U3] = mhd[3];
  f[B1] = q->bcon[1] * q->ucon[dir] - q->bcon[dir] * q->ucon[1];
  f[B2] = q->bcon[2] * q->ucon[dir] - q->bcon[dir] * q->ucon[2];
  f[B3] = q->bcon[3] * q->ucon[dir] - q->bcon[dir] * q->ucon[3];
  for (l = 0; l < NP; l++) f[l] *= g->g;
}

static void mhd_calc(const state_t *q, int dir, double *mhd) /* phys.c:93 */
{
  double eta_ucon = q->eta * q->ucon[dir];
  double bcon_dir = q->bcon[dir];
  mhd[0] = eta_ucon * q->ucov[0] - bcon_dir * q->bcov[0];
  mhd[1] = eta_ucon * q->ucov[1] - bcon_dir * q->bcov[1];
  mhd[2] = eta_ucon * q->ucov[2] - bcon_dir * q->bcov[2];
  mhd[3] = eta_ucon * q->ucov[3] - bcon_dir * q->bcov[3];
  mhd[dir] += q->ptot;
}

static void vchar_fast(const or_ctx *c, const state_t *q, const geom_t *g, int js, double *vmax,
                       double *vmin) /* phys.c:432-501 */
{
  double cms2 = (c->d.gam * q->p + q->bsq) / q->eta;
  if (cms2 < 0.) cms2 = SMALL;
  else if (cms2 > 1.) cms2 = 1.;
  double Au2 = q->ucon[js] * q->ucon[js];
  double Bu2 = q->ucon[0] * q->ucon[0];
  double AuBu = q->ucon[js] * q->ucon[0];
  double A = Bu2 - (g->gcon[0][0] + Bu2) * cms2;
  double B = AuBu - (g->gcon[0][js] + AuBu) * cms2;
  double C = Au2 - (g->gcon[js][js] + Au2) * cms2;
  double discr = B * B - A * C;
  if (discr < 0.) discr = 0.; /* both reference branches set 0 */
  discr = sqrt(discr);
  double denom = 1. / A;
  double vp = -(-B + discr) * denom;
  double vm = -(-B - discr) * denom;
  if (vp > vm) { *vmax = vp; *vmin = vm; }
  else { *vmax = vm; *vmin = vp; }
}

/* source(), phys.c:121-187: T^mu_kappa Gamma^kappa_nu mu for METRIC_DIM 2
 * (U1, U2 only) and the H/R cooling (USE_COOLING_FUNCTION 1), times sqrt(-g).
 * get_state() runs once, as in the reference. */
static void source(or_ctx *c, const double *ph, const geom_t *g, int ii, int jj, double *dU)
{
  int l;
  state_t q;
  for (l = 0; l < NP; l++) dU[l] = 0.;
  if (c->d.metric_dim > 0) {
    double mhd[4][4];
    const double *cn = &c->conn[64L * ((jj - NG) + (long)c->N2 * (ii - NG))];
    get_state(c, ph, g, &q);
    mhd_calc(&q, 0, mhd[0]); mhd_calc(&q, 1, mhd[1]);
    mhd_calc(&q, 2, mhd[2]); mhd_calc(&q, 3, mhd[3]);
    int i, j;
    for (i = 0; i < NDIM; i++)
      for (j = 0; j < NDIM; j++) {
        dU[U1] += mhd[i][j] * cn[(j * 4 + 1) * 4 + i];
        dU[U2] += mhd[i][j] * cn[(j * 4 + 2) * 4 + i];
      }
  }
  if (c->d.cooling == 1) {
    if (c->d.metric_dim == 0) get_state(c, ph, g, &q);
    int bound = ((q.ucov[0] * (q.p + ph[UU] + ph[RHO] + q.bsq)) > (-ph[RHO])) ? 1 : 0;
    double f_cool = 0.;
    if (bound) { /* cooling_func_hr_disk, phys.c:649-784 (s_norm 1, q_exp 0.5) */
      double T_r = c->cool_temp[ii], Omega_r = c->cool_omega[ii];
      double E_ratio = (c->d.gam - 1.) * ph[UU] / (ph[RHO] * T_r);
      double dE = E_ratio - 1.;
      f_cool = 1. * ph[UU] * Omega_r * pow((dE + fabs(dE)), 0.5);
      if (!c->cool_tables_built) {
        /* The reference fills its tables on this first call with
         * get_coord(j, N2S, N3S, ...) for every j (phys.c:683-690), which
         * leaves icurr/jcurr/kcurr at (N1TOT-1, N2S, N3S): the remaining
         * fail() bookings of this zone land on that cell. */
        c->cool_tables_built = 1;
        c->icur = c->N1T - 1;
        c->jcur = NG;
        c->kcur = NG;
      }
    }
    /* source_cooling_func, phys.c:571-575 */
    dU[UU] -= f_cool * q.ucov[0];
    dU[U1] -= f_cool * q.ucov[1];
    dU[U2] -= f_cool * q.ucov[2];
    dU[U3] -= f_cool * q.ucov[3];
  }
  dU[UU] *= g->g;
  dU[U1] *= g->g;
  dU[U2] *= g->g;
  dU[U3] *= g->g;
}

/* ------------------------------------------------------------------------- */
/* reconstruction, src/recon.c                                               */
static double linear_recon(int rt, double y1, double y2, double y3) /* recon.c:86-125 */
{
  double Dqm, Dqp, Dqc, s;
  if (rt == 2 || rt == 5) {
    Dqm = 2. * (y2 - y1);
    Dqp = 2. * (y3 - y2);
    Dqc = 0.5 * (y3 - y1);
    s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    double aDqm = fabs(Dqm), aDqp = fabs(Dqp), aDqc = fabs(Dqc);
    if ((aDqm <= aDqp) && (aDqm <= aDqc)) return Dqm;
    else if (aDqp <= aDqc) return Dqp;
    return Dqc;
  } else if (rt == 0 || rt == 3) {
    Dqm = (y2 - y1);
    Dqp = (y3 - y2);
    s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    else if (fabs(Dqm) < fabs(Dqp)) return Dqm;
    return Dqp;
  } else {
    Dqm = (y2 - y1);
    Dqp = (y3 - y2);
    s = Dqm * Dqp;
    if (s <= 0.) return 0.;
    return 2. * s / (Dqm + Dqp);
  }
}

static void linear_recon_vect(int rt, const double *y, double *Dq, int ibeg, int iend) /* recon.c:237-264 */
{
  int i;
  double a, b, s, Dqi;
  b = y[1] - y[0];
  for (i = ibeg; i <= iend; i++) {
    a = b;
    b = y[i + 1] - y[i];
    s = a * b;
    if (s <= 0.) Dqi = 0.;
    else if (rt == 2 || rt == 5) {
      double a_abs = fabs(a), b_abs = fabs(b);
      double a3 = a_abs + a_abs + a_abs, b3 = b_abs + b_abs + b_abs;
      if (a3 <= b_abs) Dqi = a + a;
      else if (b3 <= a_abs) Dqi = b + b;
      else Dqi = 0.5 * (a + b);
    } else if (rt == 0 || rt == 3) {
      if (fabs(a) <= fabs(b)) Dqi = a;
      else Dqi = b;
    } else {
      Dqi = 2 * s / (a + b);
    }
    Dq[i] = Dqi;
  }
}

static void para_vect(const double *y, const double *dq, double *yL, double *yR, int ibeg, int iend) /* recon.c:611-641 */
{
  int i;
  double l, r, qa, lnew, rnew, yi, r2, l2, y3, yip;
  r = 0.5 * (y[2] + y[1]) - PPM_FACTOR * (dq[2] - dq[1]);
  yip = y[2];
  for (i = ibeg; i <= iend; i++) {
    yi = yip;
    yip = y[i + 1];
    l = r;
    r = 0.5 * (yip + yi) - PPM_FACTOR * (dq[i + 1] - dq[i]);
    qa = (r - yi) * (yi - l);
    if (qa <= 0.) { lnew = rnew = yi; }
    else {
      r2 = r + r; l2 = l + l; y3 = yi + yi + yi;
      lnew = l; rnew = r;
      if (r > l) {
        if (y3 > (l + r2)) lnew = y3 - r2;
        if (y3 < (l2 + r)) rnew = y3 - l2;
      } else {
        if (y3 < (l + r2)) lnew = y3 - r2;
        if (y3 > (l2 + r)) rnew = y3 - l2;
      }
    }
    yL[i] = lnew;
    yR[i] = rnew;
  }
}

#define PL(c, id, d, l) ((c)->pL[((id) * 3 + (d)) * NP + (l)])
#define PR(c, id, d, l) ((c)->pR[((id) * 3 + (d)) * NP + (l)])
#define FX(c, id, d, l) ((c)->F[((id) * 3 + (d)) * NP + (l)])

/* rescale_prims_r(), recon.c:1120-1237 */
static void rescale_prims_r(or_ctx *c, double *ph, int type)
{
  int i, j, k;
  for (i = 0; i < c->N1T; i++) {
    double rf0, rf1, rf2;
    if (type == 0) { rf0 = c->rscale[0][i]; rf1 = c->rscale[1][i]; rf2 = c->rscale[2][i]; }
    else { rf0 = 1 / c->rscale[0][i]; rf1 = 1 / c->rscale[1][i]; rf2 = 1 / c->rscale[2][i]; }
    for (j = 0; j < c->N2T; j++)
      for (k = 0; k < c->N3T; k++) {
        double *q = &ph[IX(c, i, j, k) * NP];
        q[RHO] *= rf0; q[UU] *= rf2; q[U1] *= rf1; q[U2] *= rf1; q[U3] *= rf1;
        q[B1] *= rf1; q[B2] *= rf1; q[B3] *= rf1;
      }
    if (type) {
      double rf3 = 1 / c->rscale[3][i], rf4 = 1 / c->rscale[4][i], rf5 = 1 / c->rscale[5][i];
      for (j = 0; j < c->N2T; j++)
        for (k = 0; k < c->N3T; k++) {
          long id = IX(c, i, j, k);
          double *a = &PL(c, id, 0, 0), *b = &PR(c, id, 0, 0);
          a[RHO] *= rf3; a[UU] *= rf5; a[U1] *= rf4; a[U2] *= rf4; a[U3] *= rf4;
          a[B1] *= rf4; a[B2] *= rf4; a[B3] *= rf4;
          b[RHO] *= rf3; b[UU] *= rf5; b[U1] *= rf4; b[U2] *= rf4; b[U3] *= rf4;
          b[B1] *= rf4; b[B2] *= rf4; b[B3] *= rf4;
        }
    }
  }
}

/* reconstruct_fast(), recon.c:894-1103 */
static void reconstruct_fast(or_ctx *c, double *ph)
{
  int i, j, k, l, d;
  const int rt = c->d.recon_type;
  const int BUF = c->d.use_flux_ct_para ? NG : 1;
  const int Ns[3] = {c->N1T, c->N2T, c->N3T};
  if (rt < 3) {
    for (d = 0; d < 3; d++) {
      if (!c->do_recon[d]) continue;
      int im = d == 0, jm = d == 1, km = d == 2;
      if (c->d.rescale_r && d == 0) rescale_prims_r(c, ph, 0);
      int is = c->r_s[0] + (BUF - 1) * im, js = c->r_s[1] + (BUF - 1) * jm, ks = c->r_s[2] + (BUF - 1) * km;
      int ie = c->r_e[0] - (BUF - 1) * im, je = c->r_e[1] - (BUF - 1) * jm, ke = c->r_e[2] - (BUF - 1) * km;
      for (i = is; i <= ie; i++)
        for (j = js; j <= je; j++)
          for (k = ks; k <= ke; k++) {
            long id = IX(c, i, j, k), idm = IX(c, i - im, j - jm, k - km), idp = IX(c, i + im, j + jm, k + km);
            for (l = 0; l < NP; l++) {
              double dqtmp = 0.5 * linear_recon(rt, ph[idm * NP + l], ph[id * NP + l], ph[idp * NP + l]);
              PL(c, idp, d, l) = ph[id * NP + l] + dqtmp;
              PR(c, id, d, l) = ph[id * NP + l] - dqtmp;
            }
          }
      if (c->d.rescale_r && d == 0) rescale_prims_r(c, ph, 1);
    }
  } else {
    for (d = 0; d < 3; d++) {
      if (!c->do_recon[d]) continue;
      if (c->d.rescale_r && d == 0) rescale_prims_r(c, ph, 0);
      int a1 = d == 0 ? 1 : 0, a2 = d == 2 ? 1 : 2; /* transverse directions */
      int t1, t2, n = Ns[d], e = (d == 0 ? c->N1 : d == 1 ? c->N2 : c->N3) + NG - 1;
      for (t1 = c->r_s[a1]; t1 <= c->r_e[a1]; t1++)
        for (t2 = c->r_s[a2]; t2 <= c->r_e[a2]; t2++)
          for (l = 0; l < NP; l++) {
            int s;
            int ijk[3];
            ijk[a1] = t1; ijk[a2] = t2;
            for (s = 0; s < n; s++) { ijk[d] = s; c->vec[s] = ph[IX(c, ijk[0], ijk[1], ijk[2]) * NP + l]; }
            linear_recon_vect(rt, c->vec, c->dq, NG - 2, e + 2);
            para_vect(c->vec, c->dq, c->vL, c->vR, NG - 1, e + 1);
            for (s = c->r_s[d] + BUF - 1; s <= c->r_e[d] - BUF + 1; s++) {
              ijk[d] = s + 1;
              PL(c, IX(c, ijk[0], ijk[1], ijk[2]), d, l) = c->vR[s];
              ijk[d] = s;
              PR(c, IX(c, ijk[0], ijk[1], ijk[2]), d, l) = c->vL[s];
            }
          }
      if (c->d.rescale_r && d == 0) rescale_prims_r(c, ph, 1);
    }
  }
  /* degenerate-direction copies, recon.c:1050-1075 */
  if (!c->do_recon[0]) {
    for (j = 0; j < c->N2T; j++)
      for (k = 0; k < c->N3T; k++) {
        long i0 = IX(c, NG, j, k);
        for (l = 0; l < NP; l++) PL(c, i0, 0, l) = PR(c, i0, 0, l) = ph[i0 * NP + l];
        for (i = 1; i <= BUF; i++)
          for (d = 0; d < 3; d++)
            for (l = 0; l < NP; l++) {
              PL(c, IX(c, NG - i, j, k), d, l) = PL(c, IX(c, NG + i, j, k), d, l) = PL(c, i0, d, l);
              PR(c, IX(c, NG - i, j, k), d, l) = PR(c, IX(c, NG + i, j, k), d, l) = PR(c, i0, d, l);
            }
      }
  }
  if (!c->do_recon[1]) {
    for (i = 0; i < c->N1T; i++)
      for (k = 0; k < c->N3T; k++) {
        long j0 = IX(c, i, NG, k);
        for (l = 0; l < NP; l++) PL(c, j0, 1, l) = PR(c, j0, 1, l) = ph[j0 * NP + l];
        for (j = 1; j <= BUF; j++)
          for (d = 0; d < 3; d++)
            for (l = 0; l < NP; l++) {
              PL(c, IX(c, i, NG - j, k), d, l) = PL(c, IX(c, i, NG + j, k), d, l) = PL(c, j0, d, l);
              PR(c, IX(c, i, NG - j, k), d, l) = PR(c, IX(c, i, NG + j, k), d, l) = PR(c, j0, d, l);
            }
      }
  }
  if (!c->do_recon[2]) {
    for (i = 0; i < c->N1T; i++)
      for (j = 0; j < c->N2T; j++) {
        long k0 = IX(c, i, j, NG);
        for (l = 0; l < NP; l++) PL(c, k0, 2, l) = PR(c, k0, 2, l) = ph[k0 * NP + l];
        for (k = 1; k <= BUF; k++)
          for (d = 0; d < 3; d++)
            for (l = 0; l < NP; l++) {
              PL(c, IX(c, i, j, NG - k), d, l) = PL(c, IX(c, i, j, NG + k), d, l) = PL(c, k0, d, l);
              PR(c, IX(c, i, j, NG - k), d, l) = PR(c, IX(c, i, j, NG + k), d, l) = PR(c, k0, d, l);
            }
      }
  }
}

/* numerical_flux(), src/step_ch.c:636-790 */
static void numerical_flux(or_ctx *c)
{
  int d, i, j, k, l;
  const int nE[3] = {c->N1 + NG - 1, c->N2 + NG - 1, c->N3 + NG - 1};
  for (i = 0; i < 4; i++) c->max_char_speed[i] = 0.;
  for (d = 0; d < 3; d++) {
    int dir[3] = {d == 0, d == 1, d == 2};
    int s[3], e[3], a;
    for (a = 0; a < 3; a++) {
      if (c->d.use_flux_ct_para) {
        s[a] = NG + NG * (dir[a] - 1);
        e[a] = nE[a] + 1 + (NG - 1) * (1 - dir[a]);
      } else {
        s[a] = NG + dir[a] - 1;
        e[a] = nE[a] + 1;
      }
    }
    int dim = d + 1;
    for (i = s[0]; i <= e[0]; i++)
      for (j = s[1]; j <= e[1]; j++)
        for (k = s[2]; k <= e[2]; k++) {
          geom_t *g = G(c, i, j, k, d);
          long id = IX(c, i, j, k);
          const double *pl = &PL(c, id, d, 0), *pr = &PR(c, id, d, 0);
          state_t ql, qr;
          double Ul[NP], Ur[NP], Fl[NP], Fr[NP], cmaxl, cminl, cmaxr, cminr;
          get_state(c, pl, g, &ql);
          get_state(c, pr, g, &qr);
          primtoflux(pl, &ql, 0, g, Ul);
          primtoflux(pr, &qr, 0, g, Ur);
          primtoflux(pl, &ql, dim, g, Fl);
          primtoflux(pr, &qr, dim, g, Fr);
          vchar_fast(c, &ql, g, dim, &cmaxl, &cminl);
          vchar_fast(c, &qr, g, dim, &cmaxr, &cminr);
          double t0 = 0. > cmaxl ? 0. : cmaxl;
          double cmax = fabs(t0 > cmaxr ? t0 : cmaxr);
          double t1 = 0. > -cminl ? 0. : -cminl;
          double cmin = fabs(t1 > -cminr ? t1 : -cminr);
          double ctop = cmin > cmax ? cmin : cmax;
          if (ctop > c->max_char_speed[dim])
            if (i >= NG && i <= nE[0] && j >= NG && j <= nE[1] && k >= NG && k <= nE[2])
              c->max_char_speed[dim] = ctop;
          if (c->d.use_entropy_eq) {
            c->cgf[(id * 3 + d) * 2 + 0] = cmin;
            c->cgf[(id * 3 + d) * 2 + 1] = cmax;
            c->uconL[(id * 3 + d) * 2 + 0] = g->g * ql.ucon[0];
            c->uconL[(id * 3 + d) * 2 + 1] = g->g * ql.ucon[dim];
            c->uconR[(id * 3 + d) * 2 + 0] = g->g * qr.ucon[0];
            c->uconR[(id * 3 + d) * 2 + 1] = g->g * qr.ucon[dim];
          }
          if (c->d.flux_type == 1) {
            for (l = 0; l < NP; l++)
              FX(c, id, d, l) = (cmax * Fl[l] + cmin * Fr[l] - cmax * cmin * (Ur[l] - Ul[l])) / (cmax + cmin + SMALL);
          } else {
            for (l = 0; l < NP; l++) FX(c, id, d, l) = 0.5 * (Fl[l] + Fr[l] - ctop * (Ur[l] - Ul[l]));
          }
        }
  }
}

/* flux_ct_para_fast2(), src/flux_ct.c:759-939, and flux_ct(), flux_ct.c:26-128 */
static void flux_ct(or_ctx *c)
{
  int i, j, k, d;
  const int e1 = c->N1 + NG - 1, e2 = c->N2 + NG - 1, e3 = c->N3 + NG - 1;
  double *E0 = c->emf[0], *E1 = c->emf[1], *E2 = c->emf[2];
  double fac;
  if (c->d.use_flux_ct_para) {
    const int rt = c->d.recon_type;
    int s;
    for (d = 0; d < 3; d++) memset(c->emf[d], 0, sizeof(double) * c->ntot);
    /* EMF 0 first term: F[1][B3] along k */
    for (i = NG; i <= e1 + 1; i++)
      for (j = NG; j <= e2 + 1; j++) {
        for (s = 0; s < c->N3T; s++) c->vec[s] = FX(c, IX(c, i, j, s), 1, B3);
        linear_recon_vect(rt, c->vec, c->dq, NG - 2, e3 + 2);
        para_vect(c->vec, c->dq, c->vL, c->vR, NG - 1, e3 + 1);
        for (k = NG - 1; k <= e3 + 1; k++) { E0[IX(c, i, j, k)] += c->vL[k]; E0[IX(c, i, j, k + 1)] += c->vR[k]; }
      }
    for (i = NG; i <= e1 + 1; i++)
      for (k = NG; k <= e3 + 1; k++) {
        for (s = 0; s < c->N2T; s++) c->vec[s] = FX(c, IX(c, i, s, k), 2, B2);
        linear_recon_vect(rt, c->vec, c->dq, NG - 2, e2 + 2);
        para_vect(c->vec, c->dq, c->vL, c->vR, NG - 1, e2 + 1);
        for (j = NG - 1; j <= e2 + 1; j++) { E0[IX(c, i, j, k)] -= c->vL[j]; E0[IX(c, i, j + 1, k)] -= c->vR[j]; }
      }
    /* EMF 1 */
    for (j = NG; j <= e2 + 1; j++)
      for (k = NG; k <= e3 + 1; k++) {
        for (s = 0; s < c->N1T; s++) c->vec[s] = FX(c, IX(c, s, j, k), 2, B1);
        linear_recon_vect(rt, c->vec, c->dq, NG - 2, e1 + 2);
        para_vect(c->vec, c->dq, c->vL, c->vR, NG - 1, e1 + 1);
        for (i = NG - 1; i <= e1 + 1; i++) { E1[IX(c, i, j, k)] += c->vL[i]; E1[IX(c, i + 1, j, k)] += c->vR[i]; }
      }
    for (i = NG; i <= e1 + 1; i++)
      for (j = NG; j <= e2 + 1; j++) {
        for (s = 0; s < c->N3T; s++) c->vec[s] = FX(c, IX(c, i, j, s), 0, B3);
        linear_recon_vect(rt, c->vec, c->dq, NG - 2, e3 + 2);
        para_vect(c->vec, c->dq, c->vL, c->vR, NG - 1, e3 + 1);
        for (k = NG - 1; k <= e3 + 1; k++) { E1[IX(c, i, j, k)] -= c->vL[k]; E1[IX(c, i, j, k + 1)] -= c->vR[k]; }
      }
    /* EMF 2 */
    for (i = NG; i <= e1 + 1; i++)
      for (k = NG; k <= e3 + 1; k++) {
        for (s = 0; s < c->N2T; s++) c->vec[s] = FX(c, IX(c, i, s, k), 0, B2);
        linear_recon_vect(rt, c->vec, c->dq, NG - 2, e2 + 2);
        para_vect(c->vec, c->dq, c->vL, c->vR, NG - 1, e2 + 1);
        for (j = NG - 1; j <= e2 + 1; j++) { E2[IX(c, i, j, k)] += c->vL[j]; E2[IX(c, i, j + 1, k)] += c->vR[j]; }
      }
    for (j = NG; j <= e2 + 1; j++)
      for (k = NG; k <= e3 + 1; k++) {
        for (s = 0; s < c->N1T; s++) c->vec[s] = FX(c, IX(c, s, j, k), 1, B1);
        linear_recon_vect(rt, c->vec, c->dq, NG - 2, e1 + 2);
        para_vect(c->vec, c->dq, c->vL, c->vR, NG - 1, e1 + 1);
        for (i = NG - 1; i <= e1 + 1; i++) { E2[IX(c, i, j, k)] -= c->vL[i]; E2[IX(c, i + 1, j, k)] -= c->vR[i]; }
      }
    fac = 0.125;
  } else {
    for (i = NG; i <= e1 + 1; i++)
      for (j = NG; j <= e2 + 1; j++)
        for (k = NG; k <= e3 + 1; k++) {
          long id = IX(c, i, j, k);
          E0[id] = 0.25 * (FX(c, id, 1, B3) + FX(c, IX(c, i, j, k - 1), 1, B3) - FX(c, id, 2, B2) - FX(c, IX(c, i, j - 1, k), 2, B2));
          E1[id] = 0.25 * (FX(c, id, 2, B1) + FX(c, IX(c, i - 1, j, k), 2, B1) - FX(c, id, 0, B3) - FX(c, IX(c, i, j, k - 1), 0, B3));
          E2[id] = 0.25 * (FX(c, id, 0, B2) + FX(c, IX(c, i, j - 1, k), 0, B2) - FX(c, id, 1, B1) - FX(c, IX(c, i - 1, j, k), 1, B1));
        }
    fac = 0.5;
  }
  for (i = NG; i <= e1 + 1; i++)
    for (j = NG; j <= e2 + 1; j++)
      for (k = NG; k <= e3 + 1; k++) {
        long id = IX(c, i, j, k);
        for (d = 0; d < 3; d++) { FX(c, id, d, B1) = 0.; FX(c, id, d, B2) = 0.; FX(c, id, d, B3) = 0.; }
      }
  for (i = NG; i <= e1 + 1; i++)
    for (j = NG; j <= e2; j++)
      for (k = NG; k <= e3; k++) {
        long id = IX(c, i, j, k);
        FX(c, id, 0, B2) += fac * (E2[id] + E2[IX(c, i, j + 1, k)]);
        FX(c, id, 0, B3) += -fac * (E1[id] + E1[IX(c, i, j, k + 1)]);
      }
  for (i = NG; i <= e1; i++)
    for (j = NG; j <= e2 + 1; j++)
      for (k = NG; k <= e3; k++) {
        long id = IX(c, i, j, k);
        FX(c, id, 1, B1) += -fac * (E2[id] + E2[IX(c, i + 1, j, k)]);
        FX(c, id, 1, B3) += fac * (E0[id] + E0[IX(c, i, j, k + 1)]);
      }
  for (i = NG; i <= e1; i++)
    for (j = NG; j <= e2; j++)
      for (k = NG; k <= e3 + 1; k++) {
        long id = IX(c, i, j, k);
        FX(c, id, 2, B1) += fac * (E1[id] + E1[IX(c, i + 1, j, k)]);
        FX(c, id, 2, B2) += -fac * (E0[id] + E0[IX(c, i, j + 1, k)]);
      }
}

/* ------------------------------------------------------------------------- */
/* con2prim                                                                  */
typedef struct {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, half_Bsq, gmog; /* gmog = (gam-1)/gam */
} u2p2d_t;

static void func_vsq(const u2p2d_t *s, const double *x, double *dx, double *f, double *df) /* utoprim_2d_fast.c:613-665 */
{
  double W = x[0], vsq = x[1];
  double ftmp = 1. - vsq, gtmp = sqrt(ftmp);
  double dPdW = s->gmog * ftmp;
  double dPdvsq = s->gmog * (0.5 * s->D / gtmp - W);
  double p_tmp = s->gmog * (W * ftmp - s->D * gtmp);
  double t2 = -s->half_Bsq + dPdvsq;
  double t3 = s->Bsq + W;
  double t4 = t3 * t3;
  double t23 = 1 / W;
  double t16 = s->QdotBsq * t23 * t23;
  double t11 = s->Qtsq - vsq * t4 + t16 * (s->Bsq + W + W);
  double t18 = -s->Qdotn - s->half_Bsq * (1.0 + vsq) + 0.5 * t16 - W + p_tmp;
  double t24 = t16 * t23;
  double t25 = -1.0 + dPdW - t24;
  double t35 = t25 * t3 + (s->Bsq - 2.0 * dPdvsq) * (t16 + vsq * W) * t23;
  double t21 = 1 / (t3 * t35);
  dx[0] = -(t2 * t11 + t4 * t18) * t21;
  double t40 = -2 * (vsq + t24) * t3;
  dx[1] = -(-t25 * t11 + t40 * t18) * t21;
  *df = -t11 * t11 - t18 * t18;
  *f = -0.5 * (*df);
}

static int gnr_2d(const u2p2d_t *s, double *x) /* utoprim_2d_fast.c:489-592 */
{
  double f = 1., df = 1., dx[2], x_old[2], errx = 1.;
  const double dv = (1. - 1.e-15);
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
  while (keep) {
    func_vsq(s, x, dx, &f, &df);
    x_old[0] = x[0]; x_old[1] = x[1];
    x[0] += dx[0];
    x[1] += dx[1];
    errx = (x[0] == 0.) ? fabs(dx[0]) : fabs(dx[0] / x[0]);
    if (x[0] < 0.) x[0] = fabs(x[0]);
    else if (x[0] > W_TOO_BIG) x[0] = x_old[0];
    if (x[1] < 0.) x[1] = 0.;
    else if (x[1] > 1.) x[1] = dv;
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df)) return 2;
  if (fabs(errx) <= NEWT_TOL) return 0;
  if ((fabs(errx) <= MIN_NEWT_TOL) && (fabs(errx) > NEWT_TOL)) return 0;
  return 1;
}

/* Utoprim_2d_fast(), utoprim_2d_fast.c:135-408 */
static int utoprim_2d(or_ctx *c, const double *U, const geom_t *g, double *prim, double *gamma_out, double *bsq)
{
  double Ut[NP], pt[NP];
  if (U[0] <= 0.) return -100;
  double inv_gdet = g->g_inv, alpha = g->alpha, gf = alpha * inv_gdet;
  prim[B1] = U[B1] * inv_gdet;
  prim[B2] = U[B2] * inv_gdet;
  prim[B3] = U[B3] * inv_gdet;
  Ut[RHO] = gf * U[RHO];
  Ut[UU] = gf * (U[UU] - U[RHO]);
  Ut[U1] = gf * U[U1];
  Ut[U2] = gf * U[U2];
  Ut[U3] = gf * U[U3];
  Ut[B1] = gf * U[B1];
  Ut[B2] = gf * U[B2];
  Ut[B3] = gf * U[B3];
  pt[RHO] = prim[RHO]; pt[UU] = prim[UU]; pt[U1] = prim[U1]; pt[U2] = prim[U2]; pt[U3] = prim[U3];
  /* Utoprim_new_body */
  u2p2d_t s;
  double gam = c->d.gam;
  s.gmog = (gam - 1.) / gam;
  double Bcon[4] = {0., Ut[B1], Ut[B2], Ut[B3]};
  s.Bsq = quad3(g, Bcon[1], Bcon[2], Bcon[3]);
  double Qcov[4] = {Ut[UU], Ut[U1], Ut[U2], Ut[U3]}, Qcon[4];
  raise(Qcov, g, Qcon);
  double QdotB = Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  s.QdotBsq = QdotB * QdotB;
  s.Qdotn = -alpha * Qcon[0];
  double Qsq = Qcov[0] * Qcon[0] + Qcov[1] * Qcon[1] + Qcov[2] * Qcon[2] + Qcov[3] * Qcon[3];
  s.Qtsq = Qsq + s.Qdotn * s.Qdotn;
  s.D = Ut[RHO];
  s.half_Bsq = 0.5 * s.Bsq;
  double utsq = quad3(g, pt[U1], pt[U2], pt[U3]);
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > UTSQ_TOO_BIG) return 2;
  double gammasq = 1. + utsq;
  double gamma = sqrt(gammasq);
  double rho0 = s.D / gamma;
  double u = pt[UU];
  double p = (gam - 1.) * u;
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) - s.QdotBsq * (2. * W_last + s.Bsq)) <=
          W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) && (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  double x[2];
  x[0] = fabs(W_last);
  {
    double Wsq = W_last * W_last, Bsq_W = s.Bsq + W_last, Xsq = Bsq_W * Bsq_W;
    double vsq = fabs((Wsq * s.Qtsq + s.QdotBsq * (Bsq_W + W_last)) / (Wsq * Xsq));
    x[1] = (vsq > 1.) ? (1.0 - 1.e-15) : vsq;
  }
  int retval = gnr_2d(&s, x);
  double W = x[0], vsq = x[1];
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  if (vsq >= 1.) return 4;
  double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = s.D * gtmp;
  *gamma_out = gamma;
  w = W * (1. - vsq);
  p = (gam - 1.) * (w - rho0) / gam;
  u = w - (rho0 + p);
  pt[RHO] = rho0;
  pt[UU] = u;
  double g_o_WBsq = gamma / (W + s.Bsq);
  double QdB_o_W = QdotB / W;
  *bsq = s.Bsq * (1. - vsq) + QdB_o_W * QdB_o_W;
  pt[U1] = g_o_WBsq * (Qcon[1] + g->ncon[1] * s.Qdotn + QdB_o_W * Bcon[1]);
  pt[U2] = g_o_WBsq * (Qcon[2] + g->ncon[2] * s.Qdotn + QdB_o_W * Bcon[2]);
  pt[U3] = g_o_WBsq * (Qcon[3] + g->ncon[3] * s.Qdotn + QdB_o_W * Bcon[3]);
  prim[RHO] = pt[RHO]; prim[UU] = pt[UU]; prim[U1] = pt[U1]; prim[U2] = pt[U2]; prim[U3] = pt[U3];
  return 0;
}

/* Utoprim_1d(), utoprim_1d.c:118-629 */
typedef struct { double Bsq, QdotBsq, Qtsq, Qdotn, D, gam; } u2p1d_t;

static double vsq_1d(const u2p1d_t *s, double W)
{
  double Wsq = W * W, Xsq = (s->Bsq + W) * (s->Bsq + W);
  return (Wsq * s->Qtsq + s->QdotBsq * (s->Bsq + 2. * W)) / (Wsq * Xsq);
}

static void func_1d_orig(const u2p1d_t *s, const double *x, double *dx, double *f, double *df)
{
  const double dv = 1.0e-15, G = s->gam;
  double W = x[0], Wsq = W * W;
  double vsq = vsq_1d(s, W);
  vsq = (vsq < -dv) ? 0. : fabs(vsq);
  vsq = (vsq > 1.) ? (1. - dv) : vsq;
  double gtmp = 1. - vsq;
  double p_tmp = (G - 1.) * (W * gtmp - s->D * sqrt(gtmp)) / G;
  double X = s->Bsq + W, W3 = W * W * W, X3 = X * X * X;
  double dvsq = -2. * (s->Qtsq / X3 + s->QdotBsq * (3 * W * X + s->Bsq * s->Bsq) / (W3 * X3));
  double dp1 = (G - 1.) * (1. - vsq) / G;
  double dp2 = (G - 1.) * (0.5 * s->D / sqrt(1. - vsq) - W) / G;
  double dpdW = dp1 + dp2 * dvsq;
  double resid = +W + 0.5 * s->Bsq * (1. + vsq) - 0.5 * s->QdotBsq / Wsq + s->Qdotn - p_tmp;
  double drdW = 1. - dpdW + s->QdotBsq / (Wsq * W) + 0.5 * s->Bsq * dvsq;
  dx[0] = -resid / drdW;
  *f = 0.5 * resid * resid;
  *df = -2. * (*f);
}

static int utoprim_1d(or_ctx *c, const double *U, const geom_t *g, double *prim, double *gamma_out, double *bsq)
{
  int i, j;
  double Ut[NP], pt[NP];
  double gdet = g->g;
  for (i = B1; i <= B3; i++) prim[i] = U[i] / gdet;
  double alpha = 1.0 / sqrt(-g->gcon[0][0]);
  Ut[RHO] = alpha * U[RHO] / gdet;
  Ut[UU] = alpha * (U[UU] - U[RHO]) / gdet;
  for (i = U1; i <= U3; i++) Ut[i] = alpha * U[i] / gdet;
  for (i = B1; i <= B3; i++) Ut[i] = alpha * U[i] / gdet;
  for (i = 0; i < B1; i++) pt[i] = prim[i];
  for (i = B1; i <= B3; i++) pt[i] = alpha * prim[i];
  /* Utoprim_new_body (utoprim_1d.c:227-368) */
  u2p1d_t s;
  s.gam = c->d.gam;
  double Bcon[4], Bcov[4], Qcov[4], Qcon[4], ncov[4], ncon[4], Qtcon[4];
  Bcon[0] = 0.;
  for (i = 1; i < 4; i++) Bcon[i] = Ut[B1 + i - 1];
  lower(Bcon, g, Bcov);
  for (i = 0; i < 4; i++) Qcov[i] = Ut[UU + i];
  raise(Qcov, g, Qcon);
  s.Bsq = 0.;
  for (i = 1; i < 4; i++) s.Bsq += Bcon[i] * Bcov[i];
  double QdotB = 0.;
  for (i = 0; i < 4; i++) QdotB += Qcov[i] * Bcon[i];
  s.QdotBsq = QdotB * QdotB;
  { /* ncov_calc (u2p_util.c) */
    double lapse = sqrt(-1. / g->gcon[0][0]);
    ncov[0] = -lapse; ncov[1] = ncov[2] = ncov[3] = 0.;
  }
  raise(ncov, g, ncon);
  s.Qdotn = Qcon[0] * ncov[0];
  double Qsq = 0.;
  for (i = 0; i < 4; i++) Qsq += Qcov[i] * Qcon[i];
  s.Qtsq = Qsq + s.Qdotn * s.Qdotn;
  s.D = Ut[RHO];
  double utsq = 0.;
  for (i = 1; i < 4; i++)
    for (j = 1; j < 4; j++) utsq += g->gcov[i][j] * pt[U1 + i - 1] * pt[U1 + j - 1];
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > UTSQ_TOO_BIG) return 2;
  double gammasq = 1. + utsq, gamma = sqrt(gammasq);
  double rho0 = s.D / gamma, u = pt[UU], p = (s.gam - 1.) * u, w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) - s.QdotBsq * (2. * W_last + s.Bsq)) <=
          W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) && (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  /* general_newton_raphson (utoprim_1d.c:405-520) */
  double x = W_last, dx, f = 1., df = 1., errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1, retval;
  while (keep) {
    func_1d_orig(&s, &x, &dx, &f, &df);
    x += dx;
    i_increase = 0;
    while (((x * x * x * (x + 2. * s.Bsq) - s.QdotBsq * (2. * x + s.Bsq)) <= x * x * (s.Qtsq - s.Bsq * s.Bsq)) &&
           (i_increase < 10)) {
      x -= (1. * i_increase) * dx / 10.;
      i_increase++;
    }
    errx = (x == 0.) ? fabs(dx) : fabs(dx / x);
    x = fabs(x);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df)) retval = 2;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  else retval = 0;
  double W = x;
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  double vsq = vsq_1d(&s, W);
  if (vsq >= 1.) return 4;
  double gtmp = sqrt(1. - vsq);
  gamma = 1. / gtmp;
  rho0 = s.D * gtmp;
  *gamma_out = gamma;
  w = W * (1. - vsq);
  p = (s.gam - 1.) * (w - rho0) / s.gam;
  u = w - (rho0 + p);
  pt[RHO] = rho0;
  pt[UU] = u;
  *bsq = s.Bsq * (1. - vsq) + s.QdotBsq / (W * W);
  for (i = 1; i < 4; i++) Qtcon[i] = Qcon[i] + ncon[i] * s.Qdotn;
  for (i = 1; i < 4; i++) pt[U1 + i - 1] = gamma / (W + s.Bsq) * (Qtcon[i] + QdotB * Bcon[i] / W);
  for (i = 0; i < B1; i++) prim[i] = pt[i];
  return 0;
}

/* Utoprim_1d_ee(), utoprim_1d_ee.c:156-470 and its Newton routines */
typedef struct {
  double Bsq, QdotBsq, Qtsq, Qdotn, D, Sc, rho_gm1, two_Bsq;
  double W_for_gnr2, rho_for_gnr2, W_for_gnr2_old, rho_for_gnr2_old, drho_dW;
  double g_o_gm1, gm1, gm1_inv, gam;
  double t2, t4, t7, t24, t300, t400, s100, s200;
} ee_t;

static void ee_func_rho(ee_t *s, const double *x, double *dx, double *f, double *df)
{
  double rho = x[0], W = s->W_for_gnr2;
  double t40 = pow(rho, s->gm1);
  s->rho_gm1 = t40;
  double resid = (rho * W + (-t40 * s->s100 - s->D) * s->D);
  double t14 = t40 / rho;
  double jac = -t14 * s->s200 + W;
  dx[0] = -resid / jac;
  *df = -resid * resid;
  *f = -0.5 * (*df);
}

static int ee_gnr2(ee_t *s, double *x)
{
  double f = 1., df = 1., dx, errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
  while (keep) {
    ee_func_rho(s, x, &dx, &f, &df);
    x[0] += dx;
    errx = (x[0] == 0.) ? fabs(dx) : fabs(dx / x[0]);
    x[0] = fabs(x[0]);
    if ((fabs(errx) <= NEWT_TOL2) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 0;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL2) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x[0])) return 2;
  if (fabs(errx) <= NEWT_TOL) return 0;
  if ((fabs(errx) <= MIN_NEWT_TOL) && (fabs(errx) > NEWT_TOL)) return 0;
  return 1;
}

static void ee_func_W(ee_t *s, const double *x, double *dx, double *f, double *df)
{
  double W = x[0], x_rho[1], rho_g;
  int retval, ntries;
  s->W_for_gnr2_old = s->W_for_gnr2;
  s->W_for_gnr2 = W;
  rho_g = x_rho[0] = s->rho_for_gnr2;
  ntries = 0;
  while ((retval = ee_gnr2(s, x_rho)) && (ntries++ < 10)) {
    rho_g *= 10.;
    x_rho[0] = rho_g;
  }
  s->rho_for_gnr2_old = s->rho_for_gnr2;
  double rho = s->rho_for_gnr2 = x_rho[0];
  s->rho_gm1 = pow(rho, s->gm1);
  s->drho_dW = -rho * rho / (-s->rho_gm1 * s->s200 + W * rho);
  double t15 = -(s->D - rho) * (s->D + rho);
  double t200 = W + s->two_Bsq;
  double t1000 = rho * s->drho_dW;
  double resid = (s->t300 + (s->t4 + s->t4 + (s->t400 + t15 * (s->t7 + (t200) * W)) * W) * W) * s->t24;
  double jac = 2 * (s->t4 + (s->t400 + t15 * s->t7 + (3.0 * t15 * s->Bsq + s->t7 * t1000 + (t15 + t15 + t1000 * (t200)) * W) * W) * W) * s->t24;
  dx[0] = -resid / jac;
  *df = -resid * resid;
  *f = -0.5 * (*df);
}

static int ee_gnr(ee_t *s, double *x)
{
  double f = 1., df = 1., dx, errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1;
  while (keep) {
    ee_func_W(s, x, &dx, &f, &df);
    x[0] += dx;
    errx = (x[0] == 0.) ? fabs(dx) : fabs(dx / x[0]);
    x[0] = fabs(x[0]);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x[0])) return 2;
  if (fabs(errx) <= NEWT_TOL) return 0;
  if ((fabs(errx) <= MIN_NEWT_TOL) && (fabs(errx) > NEWT_TOL)) return 0;
  return 1;
}

static int utoprim_1d_ee(or_ctx *c, const double *U, double S, const geom_t *g, double *prim, double *gamma_out)
{
  double Ut[NP], pt[NP];
  if (U[0] <= 0.) return -100;
  ee_t s;
  s.gam = c->d.gam;
  s.gm1 = (s.gam - 1.);
  s.gm1_inv = 1. / s.gm1;
  s.g_o_gm1 = s.gam * s.gm1_inv;
  double inv_gdet = g->g_inv, alpha = g->alpha, gf = alpha * inv_gdet;
  prim[B1] = U[B1] * inv_gdet;
  prim[B2] = U[B2] * inv_gdet;
  prim[B3] = U[B3] * inv_gdet;
  s.Sc = gf * S;
  Ut[RHO] = gf * U[RHO];
  Ut[UU] = gf * (U[UU] - U[RHO]);
  Ut[U1] = gf * U[U1];
  Ut[U2] = gf * U[U2];
  Ut[U3] = gf * U[U3];
  Ut[B1] = gf * U[B1];
  Ut[B2] = gf * U[B2];
  Ut[B3] = gf * U[B3];
  pt[RHO] = prim[RHO]; pt[UU] = prim[UU]; pt[U1] = prim[U1]; pt[U2] = prim[U2]; pt[U3] = prim[U3];
  double Bcon[4] = {0., Ut[B1], Ut[B2], Ut[B3]};
  s.Bsq = quad3(g, Bcon[1], Bcon[2], Bcon[3]);
  double Qcov[4] = {Ut[UU], Ut[U1], Ut[U2], Ut[U3]}, Qcon[4];
  raise(Qcov, g, Qcon);
  double QdotB = Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  s.QdotBsq = QdotB * QdotB;
  s.Qdotn = -alpha * Qcon[0];
  double Qsq = Qcov[0] * Qcon[0] + Qcov[1] * Qcon[1] + Qcov[2] * Qcon[2] + Qcov[3] * Qcon[3];
  s.Qtsq = Qsq + s.Qdotn * s.Qdotn;
  s.D = Ut[RHO];
  s.t2 = s.D * s.D;
  s.t4 = s.QdotBsq * s.t2;
  s.t7 = s.Bsq * s.Bsq;
  s.t24 = 1 / s.t2;
  s.two_Bsq = s.Bsq + s.Bsq;
  s.t300 = s.QdotBsq * s.Bsq * s.t2;
  s.t400 = s.Qtsq * s.t2;
  s.s200 = s.D * s.gam * s.Sc;
  s.s100 = s.g_o_gm1 * s.Sc;
  double utsq = quad3(g, pt[U1], pt[U2], pt[U3]);
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > UTSQ_TOO_BIG) return 2;
  double gammasq = 1. + utsq, gamma = sqrt(gammasq);
  double rho0 = s.D / gamma;
  s.rho_gm1 = pow(rho0, s.gm1);
  double p = s.Sc * s.rho_gm1 / gamma;
  double u = p * s.gm1_inv;
  double w = rho0 + u + p;
  double W_last = w * gammasq;
  int i_increase = 0;
  while (((W_last * W_last * W_last * (W_last + 2. * s.Bsq) - s.QdotBsq * (2. * W_last + s.Bsq)) <=
          W_last * W_last * (s.Qtsq - s.Bsq * s.Bsq)) && (i_increase < 10)) {
    W_last *= 10.;
    i_increase++;
  }
  s.W_for_gnr2 = s.W_for_gnr2_old = W_last;
  s.rho_for_gnr2 = s.rho_for_gnr2_old = rho0;
  double x1[1] = {W_last};
  int retval = ee_gnr(&s, x1);
  double W = x1[0];
  if ((retval != 0) || (W == FAIL_VAL)) return retval * 100 + 1;
  if (W <= 0. || W > W_TOO_BIG) return 3;
  double x_rho[1], rho_g;
  rho_g = x_rho[0] = s.rho_for_gnr2;
  int ntries = 0;
  while ((retval = ee_gnr2(&s, x_rho)) && (ntries++ < 10)) {
    rho_g *= 10.;
    x_rho[0] = rho_g;
  }
  s.rho_for_gnr2 = x_rho[0];
  if (retval != 0) return 10;
  rho0 = s.rho_for_gnr2;
  s.rho_gm1 = pow(rho0, s.gm1);
  utsq = (s.D - rho0) * (s.D + rho0) / (rho0 * rho0);
  double gamma_sq = 1. + utsq;
  gamma = sqrt(gamma_sq);
  *gamma_out = gamma;
  if (utsq < 0.) return 4;
  w = W / gamma_sq;
  p = s.Sc * s.rho_gm1 / gamma;
  u = p * s.gm1_inv;
  double g_o_WBsq = gamma / (W + s.Bsq);
  double QdB_o_W = QdotB / W;
  prim[RHO] = rho0;
  prim[UU] = u;
  prim[U1] = g_o_WBsq * (Qcon[1] + g->ncon[1] * s.Qdotn + QdB_o_W * Bcon[1]);
  prim[U2] = g_o_WBsq * (Qcon[2] + g->ncon[2] * s.Qdotn + QdB_o_W * Bcon[2]);
  prim[U3] = g_o_WBsq * (Qcon[3] + g->ncon[3] * s.Qdotn + QdB_o_W * Bcon[3]);
  return 0;
}

/* Utoprim_1d_ee2(), utoprim_1d_ee2.c:152-590 */
typedef struct { double Bsq, QdotBsq, Qtsq, D, Sc, g_o_gm1, gam; } ee2_t;

static void ee2_func_rho(const ee2_t *s, const double *x, double *dx, double *f, double *df)
{
  double G = s->gam;
  double rho = x[0];
  double rhosq = rho * rho;
  double t200 = 1. / (s->D * s->D);
  double t100 = s->g_o_gm1 * s->Sc * pow(rho, (G - 1.));
  double W = s->D * (s->D + t100) / rho;
  double dWdrho = s->D * (-s->D + t100 * (G - 2.)) / rhosq;
  double t1 = W * W;
  double t2 = s->Bsq + W;
  double t3 = t2 * t2;
  double vsq = (s->D - rho) * (s->D + rho) * t200;
  double dvsqdrho = -2 * rho * t200;
  double resid = t1 * (s->Qtsq - vsq * t3) + s->QdotBsq * (t2 + W);
  double t12 = s->Bsq * s->Bsq;
  double t17 = dWdrho * vsq;
  double jac = 2 * s->QdotBsq * dWdrho +
               ((s->Qtsq - vsq * t12) * 2 * dWdrho +
                (-6 * t17 * s->Bsq - dvsqdrho * t12 + (-2 * dvsqdrho * s->Bsq - 4 * t17 - dvsqdrho * W) * W) * W) * W;
  dx[0] = -resid / jac;
  *f = 0.5 * resid * resid;
  *df = -2. * (*f);
}

static int utoprim_1d_ee2(or_ctx *c, const double *U, double S, const geom_t *g, double *prim, double *gamma_out)
{
  double Ut[NP], pt[NP];
  if (U[0] <= 0.) return -100;
  ee2_t s;
  double G = c->d.gam;
  s.gam = G;
  s.g_o_gm1 = G / (G - 1.);
  double inv_gdet = 1. / g->g;
  prim[B1] = U[B1] * inv_gdet;
  prim[B2] = U[B2] * inv_gdet;
  prim[B3] = U[B3] * inv_gdet;
  double alpha = g->alpha, gf = alpha * inv_gdet;
  s.Sc = gf * S;
  Ut[RHO] = gf * U[RHO];
  Ut[UU] = gf * (U[UU] - U[RHO]);
  Ut[U1] = gf * U[U1];
  Ut[U2] = gf * U[U2];
  Ut[U3] = gf * U[U3];
  Ut[B1] = gf * U[B1];
  Ut[B2] = gf * U[B2];
  Ut[B3] = gf * U[B3];
  pt[RHO] = prim[RHO]; pt[UU] = prim[UU]; pt[U1] = prim[U1]; pt[U2] = prim[U2]; pt[U3] = prim[U3];
  double Bcon[4] = {0., Ut[B1], Ut[B2], Ut[B3]}, Bcov[4], Qcov[4] = {Ut[UU], Ut[U1], Ut[U2], Ut[U3]}, Qcon[4];
  lower(Bcon, g, Bcov);
  raise(Qcov, g, Qcon);
  s.Bsq = Bcon[1] * Bcov[1] + Bcon[2] * Bcov[2] + Bcon[3] * Bcov[3];
  double QdotB = Qcov[1] * Bcon[1] + Qcov[2] * Bcon[2] + Qcov[3] * Bcon[3];
  s.QdotBsq = QdotB * QdotB;
  double ncov0 = -g->alpha;
  double ncon[4];
  ncon[0] = -g->alpha * g->gcon[0][0];
  ncon[1] = -g->alpha * g->gcon[0][1];
  ncon[2] = -g->alpha * g->gcon[0][2];
  ncon[3] = -g->alpha * g->gcon[0][3];
  double Qdotn = Qcon[0] * ncov0;
  double Qsq = Qcov[0] * Qcon[0] + Qcov[1] * Qcon[1] + Qcov[2] * Qcon[2] + Qcov[3] * Qcon[3];
  s.Qtsq = Qsq + Qdotn * Qdotn;
  s.D = Ut[RHO];
  double utsq = quad3(g, pt[U1], pt[U2], pt[U3]);
  if ((utsq < 0.) && (fabs(utsq) < 1.0e-13)) utsq = fabs(utsq);
  if (utsq < 0. || utsq > UTSQ_TOO_BIG) return 2;
  double gammasq = 1. + utsq, gamma = sqrt(gammasq);
  double rho0 = s.D / gamma;
  /* general_newton_raphson (utoprim_1d_ee2.c:421-520) */
  double x = rho0, dx, f = 1., df = 1., errx = 1.;
  int n_iter = 0, i_extra = 0, doing_extra = 0, keep = 1, retval;
  while (keep) {
    ee2_func_rho(&s, &x, &dx, &f, &df);
    x += dx;
    errx = (x == 0.) ? fabs(dx) : fabs(dx / x);
    x = fabs(x);
    if ((fabs(errx) <= NEWT_TOL) && (doing_extra == 0) && (EXTRA_NEWT_ITER > 0)) doing_extra = 1;
    if (doing_extra == 1) i_extra++;
    if (((fabs(errx) <= NEWT_TOL) && (doing_extra == 0)) || (i_extra > EXTRA_NEWT_ITER) ||
        (n_iter >= (MAX_NEWT_ITER - 1)))
      keep = 0;
    n_iter++;
  }
  if (!isfinite(f) || !isfinite(df) || !isfinite(x)) retval = 2;
  else if (fabs(errx) > MIN_NEWT_TOL) retval = 1;
  else retval = 0;
  rho0 = x;
  if ((retval != 0) || (rho0 == FAIL_VAL)) return retval * 100 + 1;
  if (rho0 > W_TOO_BIG) return 3;
  utsq = (s.D - rho0) * (s.D + rho0) / (rho0 * rho0);
  double gamma_sq = 1. + utsq;
  gamma = sqrt(gamma_sq);
  *gamma_out = gamma;
  if (utsq < 0.) return 4;
  double rho_gm1 = pow(rho0, (G - 1.));
  double p = s.Sc * rho_gm1 / gamma;
  double u = p / (G - 1.);
  double w = rho0 + u + p;
  double W = w * gamma_sq;
  double g_o_WBsq = gamma / (W + s.Bsq);
  double QdB_o_W = QdotB / W;
  prim[RHO] = rho0;
  prim[UU] = u;
  prim[U1] = g_o_WBsq * (Qcon[1] + ncon[1] * Qdotn + QdB_o_W * Bcon[1]);
  prim[U2] = g_o_WBsq * (Qcon[2] + ncon[2] * Qdotn + QdB_o_W * Bcon[2]);
  prim[U3] = g_o_WBsq * (Qcon[3] + ncon[3] * Qdotn + QdB_o_W * Bcon[3]);
  return 0;
}

/* ------------------------------------------------------------------------- */
/* fixups, src/fixup.c                                                       */
static int check_gamma(double gamma) /* fixup.c:133-141 */
{
  if (gamma <= GAMMAMAX) return 0;
  if (gamma > GAMMAMAX2) return 2;
  return 1;
}

static void fixup_gamma(or_ctx *c, double *pv, double *gamma) /* fixup.c:148-158 */
{
  double f = sqrt((GAMMAMAX - 1.) * (GAMMAMAX + 1.) / ((*gamma - 1.) * (*gamma + 1.)));
  pv[U1] *= f;
  pv[U2] *= f;
  pv[U3] *= f;
  *gamma = GAMMAMAX;
  fail(c, F_GAMMA_MAX, 0);
}

static void fixup_floor(or_ctx *c, double *pv, long id) /* fixup.c:105-121 */
{
  int ret = 0;
  double rf = c->cell6[id * 6 + 0], uf = c->cell6[id * 6 + 1];
  if (pv[RHO] < rf) { pv[RHO] = rf; ret = 1; }
  if (pv[UU] < uf) { pv[UU] = uf; ret = 1; }
  if (ret) fail(c, F_FLOOR, 0);
}

static int check_entropy_eq(or_ctx *c, double uu, double bsq, double rho) /* fixup.c:313-320 */
{
  if (!c->d.use_entropy_eq) return 0;
  return (uu < BETA_MIN * bsq) || (rho < BETA_MIN * bsq);
}

/* fixup_entropy_eq(), fixup.c:335-454 */
static int fixup_entropy_eq(or_ctx *c, int i, int j, int k, const double *prim_old, double *prim,
                            const geom_t *geom, const geom_t *geom_old, double *gamma_out, double Dt)
{
  int d, l, ret;
  double prim_backup[NP], gamma, Ftot_m[3], Ftot_p[3];
  const double gam = c->d.gam;
  for (l = 0; l < NP; l++) prim_backup[l] = prim[l];
  gamma_calc(prim_old, geom_old, &gamma);
  double S_old = geom_old->g * (gam - 1.) * prim_old[UU] * gamma / (geom_old->alpha * pow(prim_old[RHO], (gam - 1.)));
  for (int side = 0; side < 2; side++) {
    for (d = 0; d < 3; d++) {
      long id = side ? IX(c, i + (d == 0), j + (d == 1), k + (d == 2)) : IX(c, i, j, k);
      double cmin = c->cgf[(id * 3 + d) * 2 + 0], cmax = c->cgf[(id * 3 + d) * 2 + 1];
      double ctop = cmin > cmax ? cmin : cmax;
      double s = (gam - 1.) * PL(c, id, d, UU) * pow(PL(c, id, d, RHO), 1. - gam);
      double Ul = s * c->uconL[(id * 3 + d) * 2 + 0];
      double Fl = s * c->uconL[(id * 3 + d) * 2 + 1];
      s = (gam - 1.) * PR(c, id, d, UU) * pow(PR(c, id, d, RHO), 1. - gam);
      double Ur = s * c->uconR[(id * 3 + d) * 2 + 0];
      double Fr = s * c->uconR[(id * 3 + d) * 2 + 1];
      double Ft;
      if (c->d.flux_type == 1) Ft = (cmax * Fl + cmin * Fr - cmax * cmin * (Ur - Ul)) / (cmax + cmin + SMALL);
      else Ft = 0.5 * (Fl + Fr - ctop * (Ur - Ul));
      if (side) Ftot_p[d] = Ft; else Ftot_m[d] = Ft;
    }
  }
  double S = S_old + Dt * (-(Ftot_p[0] - Ftot_m[0]) * c->invdx[1] - (Ftot_p[1] - Ftot_m[1]) * c->invdx[2] -
                           (Ftot_p[2] - Ftot_m[2]) * c->invdx[3]);
  const double *Un = &c->Un[IX(c, i, j, k) * NP];
  ret = utoprim_1d_ee(c, Un, S, geom, prim, &gamma);
  if ((!ret) && (check_gamma(gamma) == 2)) {
    for (l = 0; l < NP; l++) prim[l] = prim_backup[l];
    ret = 1;
    gamma = 1.;
  }
  if (ret) {
    ret = utoprim_1d_ee2(c, Un, S, geom, prim, &gamma);
    if ((!ret) && (check_gamma(gamma) == 2)) {
      for (l = 0; l < NP; l++) prim[l] = prim_backup[l];
      ret = 1;
    }
    if (ret) gamma = 1.;
  }
  *gamma_out = gamma;
  if (!ret) fail(c, F_USE_EE, 0);
  return ret;
}

/* recover_primitives(), src/step_ch.c:801-1024 (FIXUP_TREE 3) */
static void recover_primitives(or_ctx *c, int i, int j, int k, double *pf, const double *U, const geom_t *geom,
                               const geom_t *geom_old, double Dt)
{
  int l, ret, ret_ee, use_ee = 0;
  double pg[NP], gamma = 0., bsq = 0., pf2[NP];
  long id = IX(c, i, j, k);
  for (l = 0; l < NP; l++) pg[l] = pf[l];
  ret = utoprim_2d(c, U, geom, pf, &gamma, &bsq);
  if ((!ret) && (check_gamma(gamma) == 2)) {
    for (l = 0; l < B1; l++) pf[l] = pg[l];
    ret = 1;
    gamma = 1.;
  }
  if (ret) {
    ret = utoprim_1d(c, U, geom, pf, &gamma, &bsq);
    if ((!ret) && (check_gamma(gamma) == 2)) {
      for (l = 0; l < B1; l++) pf[l] = pg[l];
      ret = 1;
    }
    if (ret) gamma = 1.;
  }
  c->p_gamma[id] = gamma;
  if (c->d.use_entropy_eq)
    if (ret || check_entropy_eq(c, pf[UU], bsq, pf[RHO])) use_ee = 1;
  if (!use_ee) {
    if (!ret) fail(c, F_USE_FULL_INV, 0);
    else fail(c, F_UTOPRIM, 1);
  } else {
    if (!ret) { for (l = 0; l < NP; l++) pf2[l] = pf[l]; }
    else fail(c, F_UTOPRIM, 0);
    for (l = 0; l < B1; l++) pf[l] = pg[l];
    ret_ee = fixup_entropy_eq(c, i, j, k, &c->p_old[id * NP], pf, geom, geom_old, &gamma, Dt);
    if (ret_ee) {
      if (ret) {
        fail(c, F_UTOPRIM_EE, 1);
        return;
      } else {
        fail(c, F_UTOPRIM_EE, 0);
        for (l = 0; l < NP; l++) pf[l] = pf2[l];
        gamma = c->p_gamma[id];
        fail(c, F_USE_FULL_INV, 0);
      }
    }
  }
  c->p_gamma[id] = gamma;
  fixup_floor(c, pf, id);
  if (check_gamma(gamma)) {
    fail(c, F_GAMMA_MAX, 2);
    return;
  }
  c->p_gamma[id] = gamma;
}

/* advance(), src/step_ch.c:248-451 */
static void advance(or_ctx *c, double *p_i, double *p_h, double Dt, double *p_f)
{
  int i, j, k, l;
  const int e1 = c->N1 + NG - 1, e2 = c->N2 + NG - 1, e3 = c->N3 + NG - 1;
  reconstruct_fast(c, p_h);
  numerical_flux(c);
  if (c->d.bc_type == 10) { /* fix_flux(), bounds.c:2263-2275 */
    int j2, k2;
    for (j2 = 0; j2 < c->N2T; j2++)
      for (k2 = 0; k2 < c->N3T; k2++) {
        long lo = IX(c, NG, j2, k2), hi = IX(c, c->N1 + NG, j2, k2);
        if (FX(c, lo, 0, RHO) > 0) FX(c, lo, 0, RHO) = 0.;
        if (FX(c, hi, 0, RHO) < 0) FX(c, hi, 0, RHO) = 0.;
      }
  }
  flux_ct(c);
  c->M_tot = 0.;
  for (i = NG; i <= e1; i++)
    for (j = NG; j <= e2; j++)
      for (k = NG; k <= e3; k++) {
        long id = IX(c, i, j, k);
        double U[NP], dU[NP];
        geom_t *gi = G(c, i, j, k, 3), *gh, *gf;
        if (c->n_substep == 0) {
          gh = gi;
          gf = G(c, i, j, k, 3);
          state_t q;
          get_state(c, &p_i[id * NP], gi, &q);
          primtoflux(&p_i[id * NP], &q, 0, gi, U);
          for (l = 0; l < NP; l++) c->U0[id * NP + l] = U[l];
        } else {
          gh = G(c, i, j, k, 3);
          gf = G(c, i, j, k, 3);
          for (l = 0; l < NP; l++) U[l] = c->U0[id * NP + l];
        }
        source(c, &p_h[id * NP], gh, i, j, dU);
        for (l = 0; l < NP; l++) {
          U[l] += Dt * (-(FX(c, IX(c, i + 1, j, k), 0, l) - FX(c, id, 0, l)) * c->invdx[1] -
                        (FX(c, IX(c, i, j + 1, k), 1, l) - FX(c, id, 1, l)) * c->invdx[2] -
                        (FX(c, IX(c, i, j, k + 1), 2, l) - FX(c, id, 2, l)) * c->invdx[3] + dU[l]);
        }
        for (l = 0; l < NP; l++) c->Un[id * NP + l] = U[l];
        recover_primitives(c, i, j, k, &p_f[id * NP], U, gf, gi, Dt);
        c->M_tot += U[0];
      }
}

/* ------------------------------------------------------------------------- */
/* boundary conditions, src/bounds.c:31-575                                  */
static void copy_cell(or_ctx *c, double *pa, long dst, long src, int flags)
{
  int l;
  for (l = 0; l < NP; l++) pa[dst * NP + l] = pa[src * NP + l];
  if (flags) c->pflag[dst] = c->pflag[src];
}

/* inflow_check(), bounds.c:2304-2370, dir = RR (USE_GAMMA_CEILING_X1DN_BC 0) */
static void inflow_check(or_ctx *c, double *pr, int ii, int jj, int kk, int type)
{
  const int dir = 1;
  double ucon[4];
  geom_t *g = G(c, ii, jj, kk, 3);
  ucon_calc(c, pr, g, ucon);
  if (((ucon[dir] > 0.) && (type == 0)) || ((ucon[dir] < 0.) && (type == 1))) {
    double gamma = g->alpha * ucon[0];
    pr[U1] /= gamma;
    pr[U2] /= gamma;
    pr[U3] /= gamma;
    pr[U1 + dir - 1] = g->beta[dir - 1] * g->ncon[0];
    double vsq = 0.;
    int j, k;
    for (j = 1; j < NDIM; j++)
      for (k = 1; k < NDIM; k++) vsq += g->gcov[j][k] * pr[U1 + j - 1] * pr[U1 + k - 1];
    if (fabs(vsq) < 1.e-13) vsq = fabs(vsq);
    if (vsq < 0.) vsq = 0.;
    if (vsq >= 1.) vsq = 1. - 1. / (GAMMAMAX * GAMMAMAX);
    gamma = 1. / sqrt(1. - vsq);
    pr[U1] *= gamma;
    pr[U2] *= gamma;
    pr[U3] *= gamma;
  }
}

static void bounds(or_ctx *c, double *pa)
{
  int i, j, k, g;
  const int e1 = c->N1 + NG - 1, e2 = c->N2 + NG - 1, e3 = c->N3 + NG - 1;
  const int fl = c->failure_exists;
  const int per = (c->d.bc_type == 1);
  if (c->d.bc_type == 0 || c->d.bc_type == 1) { /* bounds.c:58-211 */
    for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      copy_cell(c, pa, IX(c, NG - 1 - g, j, k), IX(c, per ? e1 - g : NG, j, k), 0);
    if (fl) for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, NG - 1 - g, j, k)] = c->pflag[IX(c, per ? e1 - g : NG, j, k)];
    for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      copy_cell(c, pa, IX(c, e1 + 1 + g, j, k), IX(c, per ? NG + g : e1, j, k), 0);
    if (fl) for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, e1 + 1 + g, j, k)] = c->pflag[IX(c, per ? NG + g : e1, j, k)];
    for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++)
      copy_cell(c, pa, IX(c, i, NG - 1 - g, k), IX(c, i, per ? e2 - g : NG, k), 0);
    if (fl) for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, i, NG - 1 - g, k)] = c->pflag[IX(c, i, per ? e2 - g : NG, k)];
    for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++)
      copy_cell(c, pa, IX(c, i, e2 + 1 + g, k), IX(c, i, per ? NG + g : e2, k), 0);
    if (fl) for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, i, e2 + 1 + g, k)] = c->pflag[IX(c, i, per ? NG + g : e2, k)];
    for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      copy_cell(c, pa, IX(c, i, j, NG - 1 - g), IX(c, i, j, per ? e3 - g : NG), 0);
    if (fl) for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      c->pflag[IX(c, i, j, NG - 1 - g)] = c->pflag[IX(c, i, j, per ? e3 - g : NG)];
    for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      copy_cell(c, pa, IX(c, i, j, e3 + 1 + g), IX(c, i, j, per ? NG + g : e3), 0);
    if (fl) for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      c->pflag[IX(c, i, j, e3 + 1 + g)] = c->pflag[IX(c, i, j, per ? NG + g : e3)];
  } else if (c->d.bc_type == 10) { /* BC_SPHERICAL_OUTFLOW3, bounds.c:492-575 */
    for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      copy_cell(c, pa, IX(c, NG - 1 - g, j, k), IX(c, NG, j, k), 0);
    for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      inflow_check(c, &pa[IX(c, NG - 1 - g, j, k) * NP], NG - 1 - g, j, k, 0);
    if (fl) for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, NG - 1 - g, j, k)] = c->pflag[IX(c, NG, j, k)];
    for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      copy_cell(c, pa, IX(c, e1 + 1 + g, j, k), IX(c, e1, j, k), 0);
    for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      inflow_check(c, &pa[IX(c, e1 + 1 + g, j, k) * NP], e1 + 1 + g, j, k, 1);
    if (fl) for (g = 0; g < NG; g++) for (j = NG; j <= e2; j++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, e1 + 1 + g, j, k)] = c->pflag[IX(c, e1, j, k)];
    for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++) {
      long d = IX(c, i, NG - 1 - g, k);
      copy_cell(c, pa, d, IX(c, i, NG + g, k), 0);
      pa[d * NP + U2] *= -1;
      pa[d * NP + B2] *= -1;
    }
    if (fl) for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, i, NG - 1 - g, k)] = c->pflag[IX(c, i, NG + g, k)];
    for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++) {
      long d = IX(c, i, e2 + 1 + g, k);
      copy_cell(c, pa, d, IX(c, i, e2 - g, k), 0);
      pa[d * NP + U2] *= -1;
      pa[d * NP + B2] *= -1;
    }
    if (fl) for (i = 0; i < c->N1T; i++) for (g = 0; g < NG; g++) for (k = NG; k <= e3; k++)
      c->pflag[IX(c, i, e2 + 1 + g, k)] = c->pflag[IX(c, i, e2 - g, k)];
    for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      copy_cell(c, pa, IX(c, i, j, NG - 1 - g), IX(c, i, j, e3 - g), 0);
    if (fl) for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      c->pflag[IX(c, i, j, NG - 1 - g)] = c->pflag[IX(c, i, j, e3 - g)];
    for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      copy_cell(c, pa, IX(c, i, j, e3 + 1 + g), IX(c, i, j, NG + g), 0);
    if (fl) for (i = 0; i < c->N1T; i++) for (j = 0; j < c->N2T; j++) for (g = 0; g < NG; g++)
      c->pflag[IX(c, i, j, e3 + 1 + g)] = c->pflag[IX(c, i, j, NG + g)];
  } else {
    fprintf(stderr, "harm_oracle: bc_type %d not supported\n", c->d.bc_type);
    abort();
  }
}

/* fixup_interp_prim() / fixup_interp_v(), src/fixup.c:499-761 */
static void fixup_interp(or_ctx *c, double *pv, int which)
{
  static const int ngood_min[] = {13, 9, 6, 4};
  const int o = 13;
  int i, j, k, l, ii, jj, kk;
  const int e1 = c->N1 + NG - 1, e2 = c->N2 + NG - 1, e3 = c->N3 + NG - 1;
  const int lo = which == PF_INTERP_PRIM ? 0 : U1, hi = which == PF_INTERP_PRIM ? B1 - 1 : U3;
  if (!c->failure_exists) return;
  for (i = NG; i <= e1; i++)
    for (j = NG; j <= e2; j++)
      for (k = NG; k <= e3; k++) {
        long id = IX(c, i, j, k);
        if (c->pflag[id] != which) continue;
        int pf[27], ngood = 0, ngood2, i_ret;
        double pold[NP], gamma, f, gamma_old;
        c->icur = i; c->jcur = j; c->kcur = k;
        for (l = lo; l <= hi; l++) pold[l] = pv[id * NP + l];
        for (ii = -1; ii <= 1; ii++) for (jj = -1; jj <= 1; jj++) for (kk = -1; kk <= 1; kk++)
          pf[o + ii + 3 * (jj + 3 * kk)] = !c->pflag[IX(c, i + ii, j + jj, k + kk)];
        for (ii = 1; ii <= 13; ii++) {
          if (pf[o + ii] && pf[o - ii]) ngood++;
          else pf[o + ii] = pf[o - ii] = 0;
        }
        double *pc = &pv[id * NP];
        if (which == PF_INTERP_PRIM) {
          geom_t *g = G(c, i, j, k, 3);
          if (ngood < ngood_min[c->nsd]) {
            gamma_calc(pc, g, &c->p_gamma[id]);
            fail(c, F_INTERP_PRIM, 0);
            continue;
          }
          for (l = lo; l <= hi; l++) pc[l] = 0.;
          for (ii = -1; ii <= 1; ii++) for (jj = -1; jj <= 1; jj++) for (kk = -1; kk <= 1; kk++)
            if (pf[o + ii + 3 * (jj + 3 * kk)])
              for (l = lo; l <= hi; l++) pc[l] += pv[IX(c, i + ii, j + jj, k + kk) * NP + l];
          ngood *= 2;
          for (l = lo; l <= hi; l++) pc[l] /= ngood;
          i_ret = gamma_calc(pc, g, &gamma);
          if (check_gamma(gamma)) {
            gamma_old = gamma; gamma = 0.; ngood2 = 0;
            for (ii = -1; ii <= 1; ii++) for (jj = -1; jj <= 1; jj++) for (kk = -1; kk <= 1; kk++)
              if (pf[o + ii + 3 * (jj + 3 * kk)]) {
                geom_t *g2 = G(c, i + ii, j + jj, k + kk, 3);
                i_ret = gamma_calc(&pv[IX(c, i + ii, j + jj, k + kk) * NP], g2, &f);
                if (!i_ret) { gamma += f; ngood2++; }
              }
            gamma /= ngood2;
            f = sqrt((gamma - 1.) * (gamma + 1.) / ((gamma_old - 1.) * (gamma_old + 1.)));
            pc[U1] *= f; pc[U2] *= f; pc[U3] *= f;
            i_ret = gamma_calc(pc, g, &gamma);
          }
          if (i_ret) {
            for (l = U1; l <= U3; l++) pc[l] = pold[l];
            gamma_calc(pc, g, &gamma);
            fail(c, F_INTERP_PRIM, 0);
          }
          fail(c, F_USE_INTERP_PRIM, 0);
          if ((!i_ret) && check_gamma(gamma)) fixup_gamma(c, pc, &gamma);
          c->p_gamma[id] = gamma;
        } else {
          if (ngood < ngood_min[c->nsd]) {
            fixup_gamma(c, pc, &c->p_gamma[id]);
            fail(c, F_INTERP_V, 0);
            continue;
          }
          for (l = lo; l <= hi; l++) pc[l] = 0.;
          for (ii = -1; ii <= 1; ii++) for (jj = -1; jj <= 1; jj++) for (kk = -1; kk <= 1; kk++)
            if (pf[o + ii + 3 * (jj + 3 * kk)])
              for (l = lo; l <= hi; l++) pc[l] += pv[IX(c, i + ii, j + jj, k + kk) * NP + l];
          ngood *= 2;
          for (l = lo; l <= hi; l++) pc[l] /= ngood;
          geom_t *g = G(c, i, j, k, 3);
          i_ret = gamma_calc(pc, g, &gamma);
          if (check_gamma(gamma)) {
            gamma_old = gamma; gamma = 0.; ngood2 = 0;
            for (ii = -1; ii <= 1; ii++) for (jj = -1; jj <= 1; jj++) for (kk = -1; kk <= 1; kk++)
              if (pf[o + ii + 3 * (jj + 3 * kk)]) {
                geom_t *g2 = G(c, i + ii, j + jj, k + kk, 3);
                i_ret = gamma_calc(&pv[IX(c, i + ii, j + jj, k + kk) * NP], g2, &f);
                if (!i_ret) { gamma += f; ngood2++; }
              }
            gamma /= ngood2;
            f = sqrt((gamma - 1.) * (gamma + 1.) / ((gamma_old - 1.) * (gamma_old + 1.)));
            pc[U1] *= f; pc[U2] *= f; pc[U3] *= f;
            i_ret = gamma_calc(pc, g, &gamma);
          }
          if (i_ret || check_gamma(gamma)) {
            for (l = U1; l <= U3; l++) pc[l] = pold[l];
            fixup_gamma(c, pc, &c->p_gamma[id]);
            fail(c, F_INTERP_V, 0);
          } else {
            fail(c, F_USE_INTERP_V, 0);
            c->p_gamma[id] = gamma;
          }
        }
      }
}

/* bounds + fixups after each substep, src/step_ch.c:99-120 and 165-180 */
static void post_substep(or_ctx *c, double *pa)
{
  bounds(c, pa);
  if (c->failure_exists) {
    if (c->failure_type[PF_INTERP_V]) fixup_interp(c, pa, PF_INTERP_V);
    if (c->failure_type[PF_INTERP_PRIM]) fixup_interp(c, pa, PF_INTERP_PRIM);
  }
  if (c->bnd_phys_pflag) {
    bounds(c, pa);
    c->bnd_phys_pflag = 0;
  }
}

static void reset_failures(or_ctx *c)
{
  if (c->failure_exists) {
    c->failure_exists = 0;
    c->failure_type[0] = c->failure_type[1] = c->failure_type[2] = 0;
    memset(c->pflag, 0, sizeof(int32_t) * c->ntot);
  }
}

/* timestep(), src/step_ch.c:546-623 (TIMESTEP_ORIGINAL) */
static double timestep(or_ctx *c)
{
  double c1 = c->max_char_speed[1], c2 = c->max_char_speed[2], c3 = c->max_char_speed[3];
  double *dx = c->d.dx;
  double dtsqij = sqrt((1. / 3.) / ((c1 * c1) / (dx[1] * dx[1]) + (c2 * c2) / (dx[2] * dx[2]) + (c3 * c3) / (dx[3] * dx[3])));
  double dtt = c->d.cour * dtsqij;
  if (dtt > SAFE * dx[0]) dtt = SAFE * dx[0];
  if (c->d.t + dtt > (c->d.grid_length[0] + c->d.startx[0])) dtt = c->d.grid_length[0] + c->d.startx[0] - c->d.t;
  return dtt;
}

/* step_ch(), src/step_ch.c:50-234 */
static void step_ch(or_ctx *c)
{
  long n = c->ntot * NP;
  reset_failures(c);
  c->n_substep = 0;
  memcpy(c->p_old, c->p, sizeof(double) * n);
  memcpy(c->ph, c->p, sizeof(double) * n);
  advance(c, c->p, c->p, 0.5 * c->d.dx[0], c->ph);
  post_substep(c, c->ph);
  reset_failures(c);
  c->n_substep = 1;
  advance(c, c->p, c->ph, c->d.dx[0], c->p);
  post_substep(c, c->p);
  c->d.t += c->d.dx[0];
  c->d.dx[0] = timestep(c);
}

/* ------------------------------------------------------------------------- */
or_ctx *or_create(const or_desc *d, const double *geom, const double *conn, const double *cell6, const double *rface)
{
  or_ctx *c = calloc(1, sizeof(or_ctx));
  c->d = *d;
  c->N1 = d->n1; c->N2 = d->n2; c->N3 = d->n3;
  c->N1T = c->N1 + 2 * NG; c->N2T = c->N2 + 2 * NG; c->N3T = c->N3 + 2 * NG;
  c->ntot = (long)c->N1T * c->N2T * c->N3T;
  c->do_recon[0] = c->N1 != 1; c->do_recon[1] = c->N2 != 1; c->do_recon[2] = c->N3 != 1;
  c->nsd = c->do_recon[0] + c->do_recon[1] + c->do_recon[2];
  const int BUF = d->use_flux_ct_para ? NG : 1;
  const int Ns[3] = {c->N1, c->N2, c->N3};
  for (int a = 0; a < 3; a++) {
    if (Ns[a] == 1) { c->r_s[a] = NG; c->r_e[a] = NG; }
    else { c->r_s[a] = NG - BUF; c->r_e[a] = Ns[a] + NG - 1 + BUF; }
  }
  for (int a = 0; a < 4; a++) c->invdx[a] = 1. / d->dx[a];
  long ng = d->metric_dim == 0 ? 1 : 5L * c->N1T * c->N2T;
  c->geom = malloc(sizeof(geom_t) * ng);
  for (long gi = 0; gi < ng; gi++) {
    const double *s = &geom[gi * OR_NGEOM];
    geom_t *t = &c->geom[gi];
    memcpy(t->gcon, s, 16 * 8);
    memcpy(t->gcov, s + 16, 16 * 8);
    t->g = s[32]; t->g_inv = s[33]; t->alpha = s[34];
    t->beta[0] = s[35]; t->beta[1] = s[36]; t->beta[2] = s[37];
    t->ncon[0] = s[38]; t->ncon[1] = s[39]; t->ncon[2] = s[40]; t->ncon[3] = s[41];
  }
  if (d->metric_dim == 2) {
    c->conn = malloc(sizeof(double) * 64 * c->N1 * c->N2);
    memcpy(c->conn, conn, sizeof(double) * 64 * c->N1 * c->N2);
  }
  c->cell6 = malloc(sizeof(double) * 6 * c->ntot);
  memcpy(c->cell6, cell6, sizeof(double) * 6 * c->ntot);
  if (d->rescale_r) {
    for (int a = 0; a < 6; a++) c->rscale[a] = malloc(sizeof(double) * c->N1T);
    for (int i = 0; i < c->N1T; i++) { /* recon.c:1142-1165 */
      double rloc = cell6[IX(c, i, NG, NG) * 6 + 3]; /* x[RR] at CENT (recon.c:1146) */
      double rf2 = rloc * rloc;
      c->rscale[0][i] = sqrt(rf2 * rloc); c->rscale[1][i] = rf2 * rloc; c->rscale[2][i] = rloc;
      rloc = rface[i];
      rf2 = rloc * rloc;
      c->rscale[3][i] = sqrt(rf2 * rloc); c->rscale[4][i] = rf2 * rloc; c->rscale[5][i] = rloc;
    }
  }
  long n = c->ntot;
  c->p = calloc(n * NP, 8); c->ph = calloc(n * NP, 8); c->p_old = calloc(n * NP, 8);
  c->pL = calloc(n * 3 * NP, 8); c->pR = calloc(n * 3 * NP, 8); c->F = calloc(n * 3 * NP, 8);
  for (int a = 0; a < 3; a++) c->emf[a] = calloc(n, 8);
  c->cgf = calloc(n * 6, 8); c->uconL = calloc(n * 6, 8); c->uconR = calloc(n * 6, 8);
  c->U0 = calloc(n * NP, 8); c->Un = calloc(n * NP, 8); c->p_gamma = calloc(n, 8);
  c->pflag = calloc(n, 4);
  c->nfail = calloc(n * OR_NFAIL, 4);
  int mx = c->N1T > c->N2T ? c->N1T : c->N2T;
  mx = mx > c->N3T ? mx : c->N3T;
  c->vec = calloc(mx, 8); c->dq = calloc(mx, 8); c->vL = calloc(mx, 8); c->vR = calloc(mx, 8);
  return c;
}

void or_destroy(or_ctx *c)
{
  if (!c) return;
  free(c->geom); free(c->conn); free(c->cell6); free(c->cool_omega); free(c->cool_temp);
  for (int a = 0; a < 6; a++) free(c->rscale[a]);
  free(c->p); free(c->ph); free(c->p_old); free(c->pL); free(c->pR); free(c->F);
  for (int a = 0; a < 3; a++) free(c->emf[a]);
  free(c->cgf); free(c->uconL); free(c->uconR); free(c->U0); free(c->Un); free(c->p_gamma);
  free(c->pflag); free(c->nfail);
  free(c->vec); free(c->dq); free(c->vL); free(c->vR);
  free(c);
}

void or_set_cooling(or_ctx *c, const double *omega, const double *temp)
{
  free(c->cool_omega);
  free(c->cool_temp);
  c->cool_omega = malloc(sizeof(double) * c->N1T);
  c->cool_temp = malloc(sizeof(double) * c->N1T);
  memcpy(c->cool_omega, omega, sizeof(double) * c->N1T);
  memcpy(c->cool_temp, temp, sizeof(double) * c->N1T);
}

void or_set_prims(or_ctx *c, const double *p_aos, double t, double dt)
{
  memcpy(c->p, p_aos, sizeof(double) * c->ntot * NP);
  c->d.t = t;
  c->d.dx[0] = dt;
  memset(c->nfail, 0, sizeof(int32_t) * c->ntot * OR_NFAIL);
  memset(c->nfailtot, 0, sizeof(c->nfailtot));
}

void or_get_prims(const or_ctx *c, double *p_aos) { memcpy(p_aos, c->p, sizeof(double) * c->ntot * NP); }
void or_get_pflag(const or_ctx *c, int32_t *pf) { memcpy(pf, c->pflag, sizeof(int32_t) * c->ntot); }
void or_get_gamma(const or_ctx *c, double *g) { memcpy(g, c->p_gamma, sizeof(double) * c->ntot); }
void or_get_nfail(const or_ctx *c, int32_t *nf) { memcpy(nf, c->nfail, sizeof(int32_t) * c->ntot * OR_NFAIL); }
void or_get_nfailtot(const or_ctx *c, uint64_t *n) { memcpy(n, c->nfailtot, sizeof(c->nfailtot)); }
void or_get_time(const or_ctx *c, double *t, double *dt, double *m)
{
  *t = c->d.t;
  *dt = c->d.dx[0];
  *m = c->M_tot;
}
long or_ntot(const or_ctx *c) { return c->ntot; }

void or_face_flux(or_ctx *c, int d, double *flux, double *mcs)
{
  memset(c->F, 0, sizeof(double) * c->ntot * 3 * NP);
  memcpy(c->ph, c->p, sizeof(double) * c->ntot * NP);
  reconstruct_fast(c, c->ph);
  numerical_flux(c);
  for (long id = 0; id < c->ntot; id++)
    for (int l = 0; l < NP; l++) flux[id * NP + l] = FX(c, id, d, l);
  *mcs = c->max_char_speed[d + 1];
}

/* dump_ener()'s integrals (diag.c:704-815) after a step: U_tot[l] = dV sum
 * of the last substep's conserved variables over the physical zones, F_tot
 * [d][side][l] = face area times the sum of the last substep's fluxes (after
 * flux_ct) over each boundary face plane; and the largest divb_calc()
 * (diag.c:503-612) over the physical zones. */
static double divb_zone(or_ctx *c, int i, int j, int k)
{
  double det_g[8], b1[8], b2[8], b3[8];
  int id = 0, di, dj, dk;
  for (di = -1; di <= 0; di++)
    for (dj = -1; dj <= 0; dj++)
      for (dk = -1; dk <= 0; dk++) {
        const long o = IX(c, i + di, j + dj, k + dk);
        det_g[id] = G(c, i + di, j + dj, k + dk, 3)->g;
        b1[id] = di == 0 ? c->p[o * NP + B1] : -c->p[o * NP + B1];
        b2[id] = dj == 0 ? c->p[o * NP + B2] : -c->p[o * NP + B2];
        b3[id] = dk == 0 ? c->p[o * NP + B3] : -c->p[o * NP + B3];
        id++;
      }
  double divb = 0., f;
  f = 0.;
  for (id = 0; id < 8; id++) f += b1[id] * det_g[id];
  divb += f * (1. / c->d.dx[1]);
  f = 0.;
  for (id = 0; id < 8; id++) f += b2[id] * det_g[id];
  divb += f * (1. / c->d.dx[2]);
  f = 0.;
  for (id = 0; id < 8; id++) f += b3[id] * det_g[id];
  divb += f * (1. / c->d.dx[3]);
  divb *= 0.25;
  return fabs(divb);
}

void or_totals(or_ctx *c, double *U_tot, double *F_tot, double *divb_max)
{
  int i, j, k, l;
  const int s1 = NG, e1 = c->N1 + NG - 1, s2 = NG, e2 = c->N2 + NG - 1, s3 = NG, e3 = c->N3 + NG - 1;
  const double dV = c->d.dx[1] * c->d.dx[2] * c->d.dx[3];
  for (l = 0; l < NP; l++) U_tot[l] = 0.;
  for (l = 0; l < 48; l++) F_tot[l] = 0.;
  double m = 0.;
  for (i = s1; i <= e1; i++)
    for (j = s2; j <= e2; j++)
      for (k = s3; k <= e3; k++) {
        for (l = 0; l < NP; l++) U_tot[l] += c->Un[IX(c, i, j, k) * NP + l];
        const double v = divb_zone(c, i, j, k);
        if (v > m) m = v;
      }
  for (l = 0; l < NP; l++) U_tot[l] *= dV;
  for (j = s2; j <= e2; j++)
    for (k = s3; k <= e3; k++)
      for (l = 0; l < NP; l++) {
        F_tot[(0 * 2 + 0) * NP + l] += FX(c, IX(c, s1, j, k), 0, l);
        F_tot[(0 * 2 + 1) * NP + l] += FX(c, IX(c, e1 + 1, j, k), 0, l);
      }
  for (i = s1; i <= e1; i++)
    for (k = s3; k <= e3; k++)
      for (l = 0; l < NP; l++) {
        F_tot[(1 * 2 + 0) * NP + l] += FX(c, IX(c, i, s2, k), 1, l);
        F_tot[(1 * 2 + 1) * NP + l] += FX(c, IX(c, i, e2 + 1, k), 1, l);
      }
  for (i = s1; i <= e1; i++)
    for (j = s2; j <= e2; j++)
      for (l = 0; l < NP; l++) {
        F_tot[(2 * 2 + 0) * NP + l] += FX(c, IX(c, i, j, s3), 2, l);
        F_tot[(2 * 2 + 1) * NP + l] += FX(c, IX(c, i, j, e3 + 1), 2, l);
      }
  for (l = 0; l < NP; l++) {
    F_tot[(0 * 2 + 0) * NP + l] *= c->d.dx[2] * c->d.dx[3];
    F_tot[(0 * 2 + 1) * NP + l] *= c->d.dx[2] * c->d.dx[3];
    F_tot[(1 * 2 + 0) * NP + l] *= c->d.dx[1] * c->d.dx[3];
    F_tot[(1 * 2 + 1) * NP + l] *= c->d.dx[1] * c->d.dx[3];
    F_tot[(2 * 2 + 0) * NP + l] *= c->d.dx[1] * c->d.dx[2];
    F_tot[(2 * 2 + 1) * NP + l] *= c->d.dx[1] * c->d.dx[2];
  }
  *divb_max = m;
}

/* init_data()'s fixup(p); bounds(p,0); (init.torus.c:205-215): fixup(),
 * fixup.c:8-33, with fixup1zone(), fixup.c:45-75 (floors, gamma ceiling) */
void or_fixup_bounds(or_ctx *c)
{
  int i, j, k;
  for (i = NG; i < c->N1 + NG; i++)
    for (j = NG; j < c->N2 + NG; j++)
      for (k = NG; k < c->N3 + NG; k++) {
        const geom_t *g = G(c, i, j, k, 3); /* CENT */
        double *pv = &c->p[IX(c, i, j, k) * NP];
        double gamma;
        if (gamma_calc(pv, g, &gamma)) {
          fail(c, F_GAMMA_CALC, 0);
          gamma = 1.;
        }
        fixup_floor(c, pv, IX(c, i, j, k));
        if (check_gamma(gamma)) fixup_gamma(c, pv, &gamma);
      }
  bounds(c, c->p);
}

void or_step(or_ctx *c, int nsteps)
{
  for (int s = 0; s < nsteps; s++) step_ch(c);
}
