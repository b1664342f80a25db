/* hg_driver.c -- the HARM3D driver's side of libharmgpu: compiled into the
 * reference's own build (next to main.c and step_ch.c, with its decs.h) when
 * USE_GPU_STEP is 1.  Five hooks connect it (tests/test_dropin.py applies
 * them to the reference's sources and compares the result):
 *
 *   main.c, after global_init():     hg_gpu_init();        the grid goes to the GPU
 *   step_ch.c, top of step_ch():     if (hg_gpu_step()) return;
 *   main.c, after nstep++ and after
 *   the time loop:                   hg_gpu_sync_host(0 / 1);  p comes back when
 *                                    diag() or restart_write() will read it
 *   diag.c, dump_ener(), after the
 *   flux totals are scaled:          hg_gpu_totals(U_tot, F_tot);  the integrals
 *                                    of the last substep's U and boundary fluxes,
 *                                    summed on the device
 *
 * Everything else of the driver (init.*.c, diag(), restart_write(),
 * check_for_crash()) is unchanged and reads the globals this file keeps
 * current: t, t_old, dx[0], dt_old, nfailtot and M_tot every step, p (and
 * pflag, p_gamma) whenever the host is about to read them.
 *
 * METRIC_GENERAL_DYNAMIC (METRIC_DIM 3) with the Minkowski- or
 * Kerr-Schild-spherical test spacetime is described to the library by
 * hg_set_dynamic_metric(); the library evaluates its geometry itself.
 *
 * USE_COOLING_FUNCTION 1 needs the h_o_r of cooling_func_hr_disk()
 * (phys.c:655, a constant local there): define HG_DROPIN_H_O_R to it. */
#include "decs.h"

#if USE_GPU_STEP
#include <stdlib.h>
#include <string.h>

#include "harmgpu.h"

extern const int mask[]; /* diag.c:31: which output types this build writes */
#if USE_COOLING_FUNCTION == 1
extern double omega_circular_equatorial(double r_loc); /* phys.c */
extern double target_temperature(double r_loc, double h_o_r);
#ifndef HG_DROPIN_H_O_R
#error "USE_COOLING_FUNCTION 1: define HG_DROPIN_H_O_R to cooling_func_hr_disk's h_o_r"
#endif
#endif

static hg_handle *gpu_grid = NULL;

static void hg_check(int rc, const char *what)
{
  if (rc != HG_OK) {
    fprintf(stderr, "libharmgpu: %s: %s\n", what, hg_strerror(rc));
    fail(FAIL_BASIC, 0); /* the reference's fatal-error path (diag.c:458-470) */
  }
}

/* after init()/restart_init() and global_init(): describe the run, hand the
 * geometry, coordinate data and primitives to the GPU */
void hg_gpu_init(void)
{
  int i, j, k, l, ia, ib, ic; /* not a, b, c: a is the global spin */
  hg_grid_desc d;
  memset(&d, 0, sizeof(d));
  d.n1 = N1;
  d.n2 = N2;
  d.n3 = N3;
  d.recon_type = RECON_TYPE_CHOICE;
  d.flux_type = FLUX_TYPE_CHOICE;
  d.use_flux_ct_para = USE_FLUX_CT_PARA;
  d.bc_type = BC_TYPE_CHOICE;
  d.metric_dim = METRIC_DIM;
  d.use_entropy_eq = USE_ENTROPY_EQ;
  d.cooling = USE_COOLING_FUNCTION;
  d.rescale_r = RESCALE_R;
  d.precision = HG_PREC_FP64;
  d.gam = gam;
  d.cour = cour;
  d.t = t;
  d.device = 0;
  for (l = 0; l < NDIM; l++) {
    d.dx[l] = dx[l];
    d.startx[l] = startx[l];
    d.grid_length[l] = GridLength[l];
  }
  hg_check(hg_init(&d, &gpu_grid), "hg_init");

#if METRIC_DIM == 3
  {
    /* METRIC_GENERAL_DYNAMIC: the library evaluates the three time levels
     * and the connection on the device; it takes the spacetime and the
     * COORD_DIAGONAL3 parameters of set_special_coord() */
    hg_dyn_metric m;
    memset(&m, 0, sizeof(m));
#if METRIC_DYNAMIC_TYPE_CHOICE == METRIC_DYNAMIC_MINK_SPHERICAL
    m.spacetime = HG_DYN_MINK_SPHERICAL;
#elif METRIC_DYNAMIC_TYPE_CHOICE == METRIC_DYNAMIC_KS_SPHERICAL
    m.spacetime = HG_DYN_KS_SPHERICAL;
    m.spin = a;
#else
#error "USE_GPU_STEP: this METRIC_DYNAMIC_TYPE_CHOICE has no spacetime in libharmgpu"
#endif
    m.R0 = R0;
    m.h_slope = h_slope;
    m.diag3_factor = diag3_factor;
    m.diag3_exponent = diag3_exponent;
    m.dt_conn = dt_conn;
    hg_check(hg_set_dynamic_metric(gpu_grid, &m), "hg_set_dynamic_metric");
  }
#else
  /* geom_arr[0] is one allocation of N_GEOM structs of 42 doubles
   * (decomp.c:168); conn is a pointer tree with a separate 4-double leaf per
   * [l][a][b] (ALLOC_4D_ARRAY, decomp.c:171), gathered here into one array */
  double *cbuf = (double *)malloc(sizeof(double) * 64 * (N_CONN > 0 ? N_CONN : 1));
  if (!cbuf) fail(FAIL_BASIC, 0);
  for (l = 0; l < N_CONN; l++)
    for (ia = 0; ia < NDIM; ia++)
      for (ib = 0; ib < NDIM; ib++)
        for (ic = 0; ic < NDIM; ic++) cbuf[((l * NDIM + ia) * NDIM + ib) * NDIM + ic] = conn[l][ia][ib][ic];
  hg_check(hg_set_geometry(gpu_grid, (const double *)geom_arr[0], N_GEOM, cbuf, N_CONN), "hg_set_geometry");
  free(cbuf);
#endif

  /* per-cell floors and coordinates at CENT (coord.c:3754-3800) */
  double *cell6 = (double *)malloc(sizeof(double) * 6 * N1TOT * N2TOT * N3TOT);
  double rface[N1TOT];
  if (!cell6) fail(FAIL_BASIC, 0);
  struct of_coord *cd;
  ALL_LOOP {
    get_coord(i, j, k, CENT, 0, cd);
    double *o = cell6 + 6 * ((i * N2TOT + j) * N3TOT + k);
    o[0] = cd->rhoflr;
    o[1] = cd->uuflr;
    o[2] = cd->r;
    o[3] = cd->x[1];
    o[4] = cd->x[2];
    o[5] = cd->x[3];
  }
  for (i = 0; i < N1TOT; i++) { /* x[RR] at FACE1 (rescale_prims_r, recon.c:1142-1165) */
    get_coord(i, N2S, N3S, FACE1, 0, cd);
    rface[i] = cd->x[RR];
  }
  hg_check(hg_set_cell_data(gpu_grid, cell6, RESCALE_R ? rface : NULL), "hg_set_cell_data");
  free(cell6);

#if USE_COOLING_FUNCTION == 1
  {
    /* the tables cooling_func_hr_disk() fills on its first call (phys.c:683-704) */
    double om[N1TOT], tt[N1TOT];
    for (i = 0; i < N1TOT; i++) {
      get_coord(i, N2S, N3S, CENT, 0, cd);
      om[i] = omega_circular_equatorial(cd->x[RR]);
      tt[i] = target_temperature(cd->x[RR], HG_DROPIN_H_O_R);
    }
    hg_check(hg_set_cooling_tables(gpu_grid, om, tt), "hg_set_cooling_tables");
  }
#endif

  hg_check(hg_upload_prims_tree(gpu_grid, p), "hg_upload_prims_tree");
  hg_check(hg_set_time(gpu_grid, t, dx[0]), "hg_set_time");
}

/* one whole step_ch() on the GPU; the globals step_ch() leaves behind
 * (step_ch.c:218-223) are set from its results */
int hg_gpu_step(void)
{
  double tn, dtn;
  hg_check(hg_step(gpu_grid, 1, &tn, &dtn), "hg_step");
  t_old = t;
  t = tn;
  dt_old = dx[0];
  dx[0] = dtn;
  hg_check(hg_get_fail_counts(gpu_grid, nfailtot), "hg_get_fail_counts"); /* check_for_crash() reads it */
  hg_check(hg_get_diag(gpu_grid, &M_tot, NULL), "hg_get_diag");
  return 1;
}

/* Bring p, pflag and p_gamma back when the host is about to read them: the
 * main loop's diag(OUT_EVERY) every 10 steps (diag.c:115-126), diag(i) for the
 * output types this build writes once their time comes, restart_write()
 * every n_restart steps (main.c:87-93), and (force) before the final
 * restart_write() and diag(OUT_FINAL). */
void hg_gpu_sync_host(int force)
{
  int i, j, k, need = force || (nstep % 10) == 0 || (nstep % n_restart) == 0;
  for (i = 0; i < N_OUT_TYPES; i++)
    if (mask[i] && t >= T_out[i]) need = 1;
  if (!need) return;
  hg_check(hg_download_prims_tree(gpu_grid, p), "hg_download_prims_tree");
  int32_t *pf = (int32_t *)malloc(sizeof(int32_t) * N1TOT * N2TOT * N3TOT);
  double *pg = (double *)malloc(sizeof(double) * N1TOT * N2TOT * N3TOT);
  if (!pf || !pg) fail(FAIL_BASIC, 0);
  hg_check(hg_download_pflag(gpu_grid, pf), "hg_download_pflag");
  hg_check(hg_download_gamma(gpu_grid, pg), "hg_download_gamma");
  ALL_LOOP {
    const long o = (i * N2TOT + j) * N3TOT + k;
    pflag[i][j][k] = pf[o];
    p_gamma[i][j][k] = pg[o];
  }
  free(pf);
  free(pg);
}

/* dump_ener()'s integrals (diag.c:745-766) from the device: dV times the sum
 * of the last substep's conserved variables over the physical zones, and the
 * face area times the sum of its fluxes over each physical boundary plane
 * (0 where the boundary is not physical, as dump_ener leaves it).  Sums are
 * per block and then in block order: within rounding of dump_ener's
 * sequential sums. */
void hg_gpu_totals(double *U_tot, double *F_tot)
{
  int d, side, l;
  double u[8], f[48];
  hg_check(hg_get_totals(gpu_grid, u, f, NULL), "hg_get_totals");
  for (l = 0; l < NP; l++) U_tot[l] = u[l];
  for (d = 0; d < NDIM - 1; d++)
    for (side = 0; side < 2; side++)
      for (l = 0; l < NP; l++)
        F_tot[(d * 2 + side) * NP + l] = (bc_pid[d + 1][side] == BC_PHYS) ? f[(d * 2 + side) * 8 + l] : 0.;
}
#endif /* USE_GPU_STEP */
