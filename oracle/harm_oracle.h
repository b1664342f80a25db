/* harm_oracle.h -- CPU restatement of the HARM3D time step (test infrastructure).
 *
 * This is the oracle: a plain-C restatement of the reference's step_ch()/
 * advance() path (src/step_ch.c:50-451 of scnastro/coolharm3d), used only by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, to verify
 * the engine's results.  The product (coolharm3d_b200/) never links or calls
 * it.
 *
 * Parity pin: tests/test_oracle_vs_reference.py runs the reference's own CPU
 * build (oracle/_ref, made by oracle/build_ref.py) and this restatement on
 * the same inputs and requires bit-identical primitives, pflag, p_gamma and
 * failure counters; tests/golden/ holds fixtures made by the reference build.
 *
 * Data layout follows the reference exactly: every grid function spans
 * N1TOT x N2TOT x N3TOT cells (NG = 3 ghosts on each side in every direction,
 * degenerate directions included), index ((i*N2TOT + j)*N3TOT + k), with the
 * NP = 8 primitive variables innermost (src/macros.h:153-160, decomp.c:140).
 */
#ifndef HARM_ORACLE_H
#define HARM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_NP 8
#define OR_NG 3
#define OR_NGEOM 42   /* doubles per struct of_geom: gcon[16] gcov[16] g g_inv alpha beta[3] ncon[4] */
#define OR_NFAIL 15

typedef struct {
  int32_t n1, n2, n3;        /* physical cells per direction */
  int32_t recon_type;        /* RECON_TYPE_CHOICE: 0 MINMOD 1 VANL 2 MC 3 PPM_MM 4 PPM_VL 5 PPM_MC */
  int32_t flux_type;         /* FLUX_TYPE_CHOICE: 0 LF, 1 HLLE */
  int32_t use_flux_ct_para;  /* USE_FLUX_CT_PARA */
  int32_t bc_type;           /* BC_TYPE_CHOICE: 0 cartesian outflow, 1 periodic, 10 spherical outflow3 */
  int32_t metric_dim;        /* METRIC_DIM: 0 (one geometry for all cells) or 2 (tables over i,j) */
  int32_t use_entropy_eq;    /* USE_ENTROPY_EQ */
  int32_t cooling;           /* USE_COOLING_FUNCTION: 0 or 1 */
  int32_t rescale_r;         /* RESCALE_R */
  int32_t pad0;
  double gam, cour;
  double dx[4];              /* dx[0] is the current time step */
  double startx[4];          /* numerical (ghost-inclusive) left edge */
  double grid_length[4];     /* GridLength[0] is the final time */
  double t;
} or_desc;

typedef struct or_ctx or_ctx;

/* geom: NPOS x N1TOT x N2TOT structs (metric_dim 2) or one struct (metric_dim 0);
 * conn: N1 x N2 x 64 doubles (metric_dim 2, may be NULL otherwise);
 * cell6: per cell (rhoflr, uuflr, r, x1, x2, x3) at the cell centre;
 * rface: x[RR] at the FACE1 position for each i (RESCALE_R only, may be NULL). */
or_ctx *or_create(const or_desc *d, const double *geom, const double *conn,
                  const double *cell6, const double *rface);
void or_destroy(or_ctx *c);
/* cooling_func_hr_disk's per-i tables Omega(r_i), T(r_i) (N1TOT each). */
void or_set_cooling(or_ctx *c, const double *omega, const double *temp);
void or_set_prims(or_ctx *c, const double *p_aos, double t, double dt);
void or_get_prims(const or_ctx *c, double *p_aos);
void or_get_pflag(const or_ctx *c, int32_t *pflag);
void or_get_gamma(const or_ctx *c, double *p_gamma);
void or_get_nfail(const or_ctx *c, int32_t *nfail);      /* [OR_NFAIL][NTOT] */
void or_get_nfailtot(const or_ctx *c, uint64_t *nfailtot);
void or_get_time(const or_ctx *c, double *t, double *dt, double *m_tot);
void or_step(or_ctx *c, int nsteps);
/* dump_ener() integrals of the last step and the largest divb_calc():
 * U_tot[8], F_tot[3][2][8] (direction, lower/upper boundary, variable). */
void or_totals(or_ctx *c, double *U_tot, double *F_tot, double *divb_max);
/* fixup(p); bounds(p,0); as the setups' init_data() calls them. */
void or_fixup_bounds(or_ctx *c);
/* reconstruct_fast + numerical_flux of the current primitives: the fluxes of
 * direction d (before flux_ct) in the reference layout, 0 on faces not
 * computed, and max_char_speed[d+1]. */
void or_face_flux(or_ctx *c, int d, double *flux, double *max_char_speed);
long or_ntot(const or_ctx *c);

#ifdef __cplusplus
}
#endif
#endif
