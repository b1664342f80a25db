/* harmgpu.h -- C ABI of libharmgpu, the B200 (sm_100a) step engine that
 * replaces HARM3D's step_ch()/advance() path.
 *
 * Caller side of the reference (scnastro/coolharm3d, paths relative to src/):
 *   - main.c:81 calls `void step_ch(void)` (step_ch.c:50-234) once per step;
 *     everything flows through globals (p, dx[0], t, pflag, nfail, nfailtot,
 *     p_gamma, M_tot).  A driver built with USE_GPU_STEP calls hg_step()
 *     instead and keeps the primitive variables resident on the GPU between
 *     steps; it downloads them only before diag()/restart_write() write them.
 *   - Geometry (geom_arr, conn: metric.c:4111-4265) and coordinate floors
 *     (coord_arr[].rhoflr/uuflr: coord.c:3792-3796) are computed by the
 *     driver's own init and handed over once with hg_set_geometry() and
 *     hg_set_cell_data(); hg_build_* compute the same tables without the
 *     driver.
 *
 * Conventions: every entry point returns 0 (HG_OK) or a negative HG_ERR_*
 * code; hg_strerror() names it.  A caller maps a negative return to its own
 * fail(FAIL_BASIC,0) (diag.c:458-470).  One handle per grid; a handle is used
 * by one host thread at a time.  Arrays in the reference's layout are
 * N1TOT x N2TOT x N3TOT cells (NG = 3 ghost cells on each side in every
 * direction, N*TOT = N* + 6) with index ((i*N2TOT + j)*N3TOT + k), and, for
 * primitives, the 8 variables innermost: exactly a flattened p[i][j][k][l].
 */
#ifndef HARMGPU_H
#define HARMGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HG_OK 0
#define HG_ERR_CUDA (-1)        /* a CUDA runtime call failed */
#define HG_ERR_BADARG (-2)      /* invalid argument or unsupported switch value */
#define HG_ERR_TIMEOUT (-3)     /* a bounded device-side wait expired */
#define HG_ERR_NOMEM (-4)       /* device memory could not be allocated */
#define HG_ERR_STATE (-5)       /* call out of order (e.g. step before geometry) */
#define HG_ERR_DEVICE (-6)      /* a kernel reported an internal error status */

#define HG_NP 8                 /* NP, macros.h:38 */
#define HG_NG 3                 /* NG, macros.h:39 */
#define HG_NFAIL 15             /* N_NFAIL, macros.h:258 */
#define HG_NGEOM 42             /* doubles per struct of_geom (globals.h:90-98) */

#define HG_PREC_FP64 0          /* every operation in IEEE double, no FMA: bit-identical to the reference */
#define HG_PREC_MIXED 1         /* reconstruction + HLL flux in FP32, everything else FP64
                                   (with fused multiply-adds) */
#define HG_PREC_FP64_FMA 2      /* every operation in IEEE double, multiply-adds fused: within
                                   rounding of HG_PREC_FP64, not bit-identical */

/* Run description: the options.h switches of the path plus init_base() values. */
typedef struct hg_grid_desc {
  int32_t n1, n2, n3;           /* physical zones: N1, N2, N3 (harm_mpi.c:1445 myargs) */
  int32_t recon_type;           /* RECON_TYPE_CHOICE 0..5 (options.h:148-155) */
  int32_t flux_type;            /* FLUX_TYPE_CHOICE: 0 LF, 1 HLLE (options.h:168-172) */
  int32_t use_flux_ct_para;     /* USE_FLUX_CT_PARA (options.h:165) */
  int32_t bc_type;              /* BC_TYPE_CHOICE: 0 CARTESIAN_OUTFLOW, 1 CARTESIAN_PERIODIC,
                                   10 SPHERICAL_OUTFLOW3 (options.h:98-124) */
  int32_t metric_dim;           /* METRIC_DIM: 0 (one geometry for every cell), 2
                                   (axisymmetric tables over i,j) (macros.h:47-53), or 3
                                   (time-dependent metric: hg_set_dynamic_metric) */
  int32_t use_entropy_eq;       /* USE_ENTROPY_EQ (options.h:209) */
  int32_t cooling;              /* USE_COOLING_FUNCTION: 0 or 1 (options.h:192) */
  int32_t rescale_r;            /* RESCALE_R (options.h:267) */
  int32_t precision;            /* HG_PREC_FP64 or HG_PREC_MIXED */
  double gam;                   /* adiabatic index */
  double cour;                  /* Courant number */
  double dx[4];                 /* dx[0] = first time step, dx[1..3] = zone sizes */
  double startx[4];             /* numerical (ghost-inclusive) left edge */
  double grid_length[4];        /* GridLength[0] = final time */
  double t;                     /* initial time */
  int32_t device;               /* CUDA device ordinal */
  int32_t reserved;
} hg_grid_desc;

typedef struct hg_handle hg_handle;

/* Validate the description, select the device and allocate the resident grid.
 * Replaces alloc_grid_arrays() (decomp.c:140-404) for the step's arrays. */
int hg_init(const hg_grid_desc *desc, hg_handle **out);

/* Static geometry: n_geom structs of HG_NGEOM doubles in struct of_geom
 * order (gcon[16], gcov[16], g, g_inv, alpha, beta[3], ncon[4]) and
 * GEOM_ID order (macros.h:592-601): 1 struct for metric_dim 0,
 * 5*N1TOT*N2TOT for metric_dim 2.  conn: n_conn x 64 doubles in CONN_ID
 * order (macros.h:575-586; n_conn = N1*N2 for metric_dim 2, else ignored).
 * Replaces the per-cell reads of geom_arr/conn done by get_geometry(). */
int hg_set_geometry(hg_handle *h, const double *geom, int64_t n_geom, const double *conn, int64_t n_conn);

/* Per-cell centre data in the reference layout, 6 doubles per cell:
 * rhoflr, uuflr, r, x1, x2, x3 (struct of_coord, coord.c:3754-3800);
 * rface[N1TOT]: x[RR] at FACE1 (RESCALE_R only, else NULL).  RESCALE_R
 * scales by x1 (x[RR]) of the row (i, N2S, N3S) and rface, the values
 * rescale_prims_r() reads on its first call (recon.c:1142-1165): pass them
 * as the driver holds them after its init (a setup that leaves x[RR] changed
 * -- init.nz_pn_bbh_disk.c does -- changes the scaling the same way). */
int hg_set_cell_data(hg_handle *h, const double *cell6, const double *rface);

/* USE_COOLING_FUNCTION 1: per radial index i (N1TOT values each) the orbital
 * frequency Omega(r_i) and target temperature T(r_i) that
 * cooling_func_hr_disk() tabulates on its first call (phys.c:683-704,
 * omega_circular_equatorial() and target_temperature()). */
int hg_set_cooling_tables(hg_handle *h, const double *omega, const double *t_target);

/* metric_dim 3: the time-dependent metric path of the reference
 * (METRIC_GENERAL_DYNAMIC, options.h:79; metric.c:3390-3690).  Its geometry
 * is not uploaded: the library evaluates it on the device at the step's
 * three time levels n_beg, n_mid, n_end (set_general_geometry for each,
 * rotated every step as advance_geometry does, metric.c:398-430) and
 * rebuilds the connection before every substep by 4th-order differences of
 * gcov and the time difference of gcov over +-dt_conn (set_general_conn,
 * metric.c:3507-3648, conn.h).  The spacetime and its COORD_DIAGONAL3
 * coordinates (coord.c:270-276, set_special_coord of the setup) are
 * described here.  Spacetimes: HG_DYN_MINK_SPHERICAL and HG_DYN_KS_SPHERICAL,
 * the reference's METRIC_DYNAMIC_MINK_SPHERICAL and _KS_SPHERICAL test
 * spacetimes (options.h:88-90; Kerr-Schild takes the static analytic
 * connection, as the reference does, metric.c:3555-3558, in place of the
 * finite differences), and HG_DYN_PN_BINARY below.  Every direction must be resolved (N > 1); FP64
 * forms only. */
#define HG_DYN_KS_SPHERICAL 0   /* METRIC_DYNAMIC_KS_SPHERICAL (options.h:88): Kerr-Schild, M = 1, spin a */
#define HG_DYN_MINK_SPHERICAL 2
/* HG_DYN_PN_BINARY: two point masses m1, m2 on a quasi-circular orbit in the
 * equatorial plane, in the first post-Newtonian harmonic-gauge metric
 *   g00 = -1 + 2V - 2V^2,  g0i = -4 V_i,  gij = (1 + 2V) delta_ij,
 * V = m1/r1 + m2/r2, V_i = m1 v1^i/r1 + m2 v2^i/r2 (the potentials at their
 * instantaneous point-mass values), taken to the grid's spherical
 * COORD_DIAGONAL3 coordinates; the separation shrinks by the quadrupole
 * formula when inspiral is 1 (Peters 1964), else the orbit is a circle.
 * The reference's own PN metrics (METRIC_DYNAMIC_FULLPN_*, metric.h:105-171)
 * have no bodies in its sources: this spacetime has no counterpart there. */
#define HG_DYN_PN_BINARY 3
typedef struct hg_dyn_metric {
  int32_t spacetime;            /* HG_DYN_* */
  int32_t diag3_exponent;       /* COORD_DIAGONAL3: odd, >= 3 */
  double R0, h_slope, diag3_factor;
  double dt_conn;               /* main.c:569 sets 9e-6 */
  /* HG_DYN_PN_BINARY only */
  double m1, m2;                /* masses, m1 on the +x axis at t = 0 when phase0 = 0 */
  double separation;            /* separation at t = 0 (harmonic coordinates) */
  double phase0;                /* orbital phase at t = 0 */
  int32_t inspiral;             /* 1: quadrupole-formula inspiral; 0: circular orbit */
  int32_t reserved;
  /* HG_DYN_KS_SPHERICAL only */
  double spin;                  /* a, |a| < 1 */
} hg_dyn_metric;
int hg_set_dynamic_metric(hg_handle *h, const hg_dyn_metric *m);
/* The struct of_geom (HG_NGEOM doubles, hg_set_geometry's order) of position
 * pos (0..2 FACE1..FACE3, 3 CENT, 4 CORN) of zone (i, j, k) at time t, as the
 * device evaluates it, computed on the host: for checking the evaluation
 * against the reference's own tables.  The host's elementary functions
 * (exp, sincos, pow) are glibc's, the device's CUDA's. */
int hg_dyn_geometry(const hg_grid_desc *desc, const hg_dyn_metric *m, int32_t pos, int32_t i, int32_t j, int32_t k,
                    double t, double geom[HG_NGEOM]);
/* The same for whole planes i0 .. i0+ni-1 of the grid with ghost zones
 * (every j, k of the reference layout), out[((i-i0)*N2TOT + j)*N3TOT + k]
 * holding HG_NGEOM doubles; host threads.  For setups that turn a
 * 4-velocity into primitives with the grid metric (init.*.c's ucon2pr) and
 * take sqrt(-g) for their fields, as the reference's init_data() reads
 * get_geometry() at t = 0.  No counterpart function in the reference. */
int hg_dyn_geometry_block(const hg_grid_desc *desc, const hg_dyn_metric *m, int32_t pos, double t, int32_t i0,
                          int32_t ni, double *geom);
/* metric_dim 3: the time level `level` (0 n_beg, 1 n_mid, 2 n_end) of the
 * step about to run, as the device evaluated it, in the reference's layout
 * out[(((pos*N1TOT + i)*N2TOT + j)*N3TOT + k)*HG_NGEOM + e] (the geom_arr of
 * METRIC_DIM 3, decomp.c:168) for the positions 0..3 (FACE1..FACE3, CENT;
 * no kernel reads the corner's, so the device does not evaluate it): for
 * checking the device's evaluation. */
int hg_download_dyn_level(hg_handle *h, int32_t level, double *geom);

/* Primitive variables in the reference layout (flattened p[i][j][k][l]).
 * Upload is hg_upload_prims; download is what diag()/restart_write() need. */
int hg_upload_prims(hg_handle *h, const double *p);
int hg_download_prims(hg_handle *h, double *p);
/* Same through the reference's own pointer tree double ****p (decomp.c:148). */
int hg_upload_prims_tree(hg_handle *h, double ****p);
int hg_download_prims_tree(hg_handle *h, double ****p);

/* Set the time and next time step (t, dx[0]); e.g. after restart_init(). */
int hg_set_time(hg_handle *h, double t, double dt);

/* Advance nsteps full RK2 steps: the whole of step_ch() (predictor,
 * boundaries, fixups, corrector, boundaries, fixups, timestep()) on the
 * device.  On return *t and *dt (either may be NULL) hold t and dx[0]. */
int hg_step(hg_handle *h, int32_t nsteps, double *t, double *dt);

/* Failure bookkeeping of fail() (diag.c:159-500): nfailtot[N_NFAIL]
 * accumulated since the last upload, pflag (int32 per cell), p_gamma
 * (double per cell), nfail (int32, [N_NFAIL][cells]). */
int hg_get_fail_counts(hg_handle *h, uint64_t nfailtot[HG_NFAIL]);
int hg_download_pflag(hg_handle *h, int32_t *pflag);
int hg_download_gamma(hg_handle *h, double *p_gamma);
int hg_download_nfail(hg_handle *h, int32_t *nfail);

/* Numerical fluxes of direction dir (0, 1, 2 = x1, x2, x3) of the resident
 * primitives: the HLL/LF fluxes numerical_flux() computes (step_ch.c:636-790,
 * before flux_ct) on every face it computes, at the lower face of each cell,
 * in the reference layout (N1TOT x N2TOT x N3TOT x 8; other faces 0), and
 * the maximum characteristic speed over physical faces (step_ch.c:716-724).
 * diag()'s boundary-flux diagnostics (diag.c:704-815) read these fluxes. */
int hg_face_flux(hg_handle *h, int32_t dir, double *flux, double *max_char_speed);

/* hg_face_flux without any allocation, for callers that cannot allocate
 * device memory: code running while a CUDA graph is being captured (where
 * cudaMalloc is not allowed), hosts whose memory pool already owns the whole
 * device, and real-time loops that must not take the device-wide
 * synchronisation cudaMalloc/cudaFree imply.  No counterpart in the
 * reference.  It needs no handle: prims and flux are device pointers in the
 * reference layout (N1TOT x N2TOT x N3TOT x 8), max_char_speed a device
 * pointer to one double, geom the host struct of a metric_dim 0 geometry,
 * stream a cudaStream_t (NULL: the default stream).  Runs asynchronously on
 * that stream.  Limits: metric_dim 0, no RESCALE_R, every N > 1, and at most
 * 4,194,304 faces in direction dir (HG_ERR_BADARG beyond).  Its scratch is a
 * 256 KiB array inside the library, held on every device that loads the
 * library until exit and shared by all calls: calls that overlap on the GPU
 * (e.g. on two streams) race and must be serialised by the caller.  A call
 * made outside stream capture looks up that array's device address on the
 * current device (allocating nothing); a call made while `stream` is being
 * captured reuses the address of the last such lookup on that device, so
 * make one call on each device before any stream capture begins (and again
 * after a cudaDeviceReset). */
int hg_face_flux_noalloc(const hg_grid_desc *desc, const double *geom, const double *prims, double *flux,
                         double *max_char_speed, int32_t dir, void *stream);

/* Diagnostics of the last step: M_tot (sum of U[RHO] over the domain after
 * the corrector, step_ch.c:402) and the per-direction maximum
 * characteristic speeds that set dx[0] (step_ch.c:716-724). */
int hg_get_diag(hg_handle *h, double *m_tot, double max_char_speed[3]);

/* fixup(p); bounds(p,0); of the setups' init_data() (init.torus.c:205-215):
 * on the resident primitives, the rho/u floors and the gamma ceiling of
 * fixup1zone() over the physical zones (fixup.c:8-75; failures counted with
 * state 0, no zone flagged), then the boundary zones.  Setups call it between
 * uploading initial data and computing fields that read ghost zones. */
int hg_fixup_bounds(hg_handle *h);

/* dump_ener()'s integrals of the last step, computed on the device
 * (diag.c:704-815): U_tot[l] = dV times the sum over the physical zones of
 * the last substep's conserved variables; F_tot[(d*2 + side)*8 + l] = the
 * face area times the sum of the last substep's fluxes over the lower
 * (side 0) and upper (side 1) boundary face planes of direction d, with the
 * flux-CT induction fluxes; and the largest divb_calc() (diag.c:503-612)
 * over the physical zones.  Sums are per block, then over blocks in order:
 * deterministic, within rounding of the reference's sequential sums.  Any
 * output may be NULL.  Meaningful after at least one hg_step. */
int hg_get_totals(hg_handle *h, double U_tot[8], double F_tot[48], double *divb_max);

/* Launch configuration of a grid's kernels: blocks (of 128 threads) per
 * launch for each kernel class, the faces each thread of the strip flux
 * kernels reconstructs in one strip (1..3), and whether x1 faces use strips.  hg_init picks a default;
 * hg_autotune measures candidates on the grid's own state and keeps the
 * fastest per kernel class: it saves the resident state, runs `steps` steps
 * per candidate (per class: 8 block counts, and 3 strip lengths for the
 * flux), puts the state back, and returns the chosen configuration with the
 * device time per step before and after.  grid_fixup sets the entropy
 * faces' and the fixups' launches; the fallback tree's own launch is not
 * configurable (every block the device holds at once, up to the grid's
 * zones).  The results of a step do not depend on the configuration
 * (M_tot's per-block partial sums aside).  No reference counterpart. */
typedef struct hg_launch_config {
  int32_t grid_flux, grid_flux32, grid_emf, grid_update, grid_fixup, grid_bounds;
  int32_t strip_faces;          /* faces per thread of the strip flux kernels, 1..3 */
  int32_t strip_x1;             /* 1: x1 faces in strips too; 0: one x1 face per thread */
} hg_launch_config;
int hg_get_launch_config(hg_handle *h, hg_launch_config *cfg);
int hg_set_launch_config(hg_handle *h, const hg_launch_config *cfg);
int hg_autotune(hg_handle *h, int32_t steps, hg_launch_config *best, double *ms_before, double *ms_after);

/* restart_write() / restart_read() (restart.c:22-94, 205-248) of the
 * resident state: the ASCII rdump file, byte for byte the layout the
 * reference writes ("%28.18e " / "%14d " fields; header t, N1, N2, N3,
 * GridLength[0], nstep, gam, cour, N_out[11], rdump_cnt, dx[0]; then the
 * physical zones' primitives in DUMP_LOOP order, one zone per line).  The
 * caller passes the driver's own counters (nstep, N_out, rdump_cnt; the
 * reader returns them).  The reader checks N1..N3 against the grid, uploads
 * the primitives, sets t, dx[0] and GridLength[0], and fills the ghost zones
 * with the boundaries.  Text is formatted and parsed on host threads. */
#define HG_N_OUT_TYPES 11
int hg_write_rdump(hg_handle *h, const char *path, int32_t nstep, const int32_t n_out[HG_N_OUT_TYPES],
                   int32_t rdump_cnt);
int hg_read_rdump(hg_handle *h, const char *path, int32_t *nstep, int32_t n_out[HG_N_OUT_TYPES],
                  int32_t *rdump_cnt);

/* The device's FP64 peak in TFLOP/s, measured: a kernel of nothing but
 * independent FP64 fused multiply-add chains on every SM (one fma = two
 * operations), best of five timed launches; *ms (may be NULL) gets that
 * launch's duration.  The denominator of the step's FP64 roofline fraction.
 * No reference counterpart. */
int hg_fp64_peak(int32_t device, double *tflops, double *ms);

/* Device time of the last hg_step call in milliseconds (CUDA events). */
int hg_last_step_ms(hg_handle *h, double *ms);

/* Per-kernel timing.  hg_profile(h, 1) makes every following hg_step record a
 * CUDA event on the engine's stream before each kernel; hg_kernel_times()
 * returns, per kernel class (flux, emf, update, fallback, bounds, fixup,
 * misc, geometry -- the time levels and connection of metric_dim 3), the
 * summed milliseconds and the number of launches since the last
 * hg_profile() call.  The reference has no counterpart (it times with
 * gettimeofday around whole routines, macros.h:620-657). */
#define HG_NKCLASS 8
int hg_profile(hg_handle *h, int32_t enable);
int hg_kernel_times(hg_handle *h, double ms[HG_NKCLASS], int64_t launches[HG_NKCLASS]);

/* Batches: resident grids of one device advanced together (no reference
 * counterpart; the reference runs one grid per process).  Each member's step
 * is captured once into a CUDA graph (on the first hg_batch_step after it
 * joins, and again after hg_set_geometry/hg_set_cell_data); one
 * hg_batch_step launches every member's step as independent branches of one
 * graph, so their kernels overlap on the device, and returns each member's
 * t and dx[0] (arrays of hg_batch_size() entries, membership order = order
 * of hg_batch_add, members removed close the gap).  A member is advanced by
 * exactly the kernels hg_step(h, 1, ...) would run: its result is bit for bit
 * the one it gets alone.  Members must have geometry, cell data and
 * primitives (HG_ERR_STATE otherwise) and live on the batch's device; while
 * a batch step runs, no member may be used otherwise.  hg_destroy refuses a
 * grid that is still a member.  HG_ERR_NOMEM if max_grids members are
 * already in; HG_ERR_DEVICE if a member's kernels reported an error. */
/* Free and total memory of a device (cudaMemGetInfo), and the device memory
 * hg_init will allocate for a description: what a server admitting grids by
 * free memory needs.  No reference counterpart. */
int hg_mem_info(int32_t device, uint64_t *free_bytes, uint64_t *total_bytes);
/* Mixed form only (HG_ERR_BADARG otherwise): the number of stored values
 * where the FP32 copy of the state the FP32 flux kernels read differs from
 * the FP64 state rounded to float.  Every step kernel that writes the state
 * writes the copy too, and every host update refreshes it, so this is 0
 * between steps; *first (may be NULL) receives the lowest mismatching
 * offset l * S + o in the stored planes, or -1.  No reference counterpart (a
 * consistency check). */
int hg_check_mirror(hg_handle *h, int64_t *mismatches, int64_t *first);
int hg_grid_bytes(const hg_grid_desc *desc, uint64_t *bytes);

typedef struct hg_batch hg_batch;
int hg_batch_create(int32_t device, int32_t max_grids, hg_batch **out);
int hg_batch_add(hg_batch *b, hg_handle *h);
int hg_batch_remove(hg_batch *b, hg_handle *h);
int hg_batch_size(const hg_batch *b);
int hg_batch_step(hg_batch *b, double *t, double *dt);
void hg_batch_destroy(hg_batch *b);

void hg_destroy(hg_handle *h);
const char *hg_strerror(int code);

/* Host-side geometry builders (the init-time work of calc_all_geom(),
 * metric.c:4111-4265, for the metrics the engine supports).
 * Minkowski Cartesian with COORD_IDENTITY: geom = 1 struct (HG_NGEOM),
 * cell6 = N1TOT*N2TOT*N3TOT*6 with the r-dependent floors RHOMIN r^-1.5,
 * UUMIN r^-2.5 (options.h:233-240). */
int hg_build_geometry_minkowski(const hg_grid_desc *desc, double *geom, double *cell6);

/* Kerr-Schild space-time (M = 1, spin a) in modified Kerr-Schild coordinates
 * COORD_DIAGONAL3 (coord.c:270-276, 3754-3800; metric.c:1168-1258), METRIC_DIM 2:
 *   r = R0 + exp(x1),  th = pi/2 (1 + h_slope f + diag3_factor f^diag3_exponent),
 *   f = 2 seesaw(x2, 0, 1) - 1,  phi = x3.
 * Fills geom (5 * N1TOT * N2TOT structs, GEOM_ID order), conn (N1 * N2 * 64
 * doubles, Gamma^a_bc at zone centres), cell6 (N1TOT*N2TOT*N3TOT*6: floors
 * RHOMIN r^-1.5, UUMIN r^-2.5, r, r, th, phi), rface (N1TOT: r at FACE1) and,
 * when both are non-NULL, the H/R cooling tables cool_omega / cool_temp
 * (N1TOT: omega_circular_equatorial() and target_temperature() of
 * phys.c:805-905 for h_o_r, with the ISCO radius the torus setup computes).
 * The connection is derived from the metric by complex-step differentiation,
 * so the tables agree with the reference's to rounding (relative 1e-12), not
 * bit for bit.  HG_ERR_BADARG for |a| >= 1 or diag3_exponent < 3. */
int hg_build_geometry_ks_mks(const hg_grid_desc *desc, double a, double R0, double h_slope,
                             double diag3_factor, int32_t diag3_exponent, double h_o_r,
                             double *geom, double *conn, double *cell6, double *rface,
                             double *cool_omega, double *cool_temp);

#ifdef __cplusplus
}
#endif
#endif /* HARMGPU_H */
