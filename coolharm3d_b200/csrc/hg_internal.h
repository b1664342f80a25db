// hg_internal.h -- shared definitions of the libharmgpu engine (host + device).
//
// Device layout (HBM): structure of arrays.  Every grid function is stored as
// planes of T0*T1*T2 doubles, x1 (index i) fastest, so warps that map lanes to
// consecutive i read coalesced 256-byte segments for stencils along any of the
// three directions.  A direction with a single physical zone (N == 1) is
// "degenerate": the reference keeps NG ghost copies of that zone (recon.c:
// 1050-1075, bounds.c), which are bit-identical to the zone itself, so here it
// is stored once (T = 1, stride 0) and every index along it maps to that zone.
// Indices used in kernels are the reference's own (ghost-inclusive, 0..N+5).
#pragma once
#include <cstdint>

#define HG_NPR 8
#define HG_NGH 3
#define HG_NF 15
#define HG_NPOS 5

namespace hg {

enum { RHO = 0, UU, U1, U2, U3, B1, B2, B3 };

// nfail[] slots (macros.h:243-258)
enum { NF_FLOOR = 0, NF_TMAX, NF_GAMMA_MAX, NF_GAMMA_CALC, NF_USE_FULL_INV, NF_USE_EE, NF_UTOPRIM,
       NF_UTOPRIM_EE, NF_USE_INTERP_PRIM, NF_USE_INTERP_V, NF_INTERP_PRIM, NF_INTERP_V };
enum { PF_NONE = 0, PF_INTERP_V = 1, PF_INTERP_PRIM = 2 };

// planes of the FP32 face geometry: gcov[16], gcon00, gcon0j (j=1..3),
// gconjj (j=1..3), ncon0, beta[3], sqrt(-g)
#define HG_GF 28

struct Geom {
  double gcon[4][4];
  double gcov[4][4];
  double g, g_inv, alpha;
  double beta[3];
  double ncon[4];
  // accessors shared with table-backed geometry (hg_phys.cuh GRef)
  __host__ __device__ double cov(int a, int b) const { return gcov[a][b]; }
  __host__ __device__ double con(int a, int b) const { return gcon[a][b]; }
  __host__ __device__ double nc(int a) const { return ncon[a]; }
  __host__ __device__ double bet(int a) const { return beta[a]; }
  __host__ __device__ double det() const { return g; }
};

// metric_dim 3 (the time-dependent metric path): the spacetime and the
// COORD_DIAGONAL3 coordinate parameters its geometry is evaluated from.
struct DynMetric {
  int spacetime;       // HG_DYN_* of harmgpu.h
  int diag3_exponent;
  double R0, h_slope, diag3_factor;
  double dt_conn;      // half-width of the connection's time difference (main.c:569)
  double m1, m2, sep, phase0;  // HG_DYN_PN_BINARY: the binary
  int inspiral;
  double spin;                 // HG_DYN_KS_SPHERICAL: a (M = 1)
};

// Device-resident scalars of one grid (t, dx[0], reductions, failure flags).
struct DevScalars {
  double t, dt;
  unsigned long long maxs[4];       // bit patterns of max_char_speed[1..3] (non-negative doubles)
  unsigned long long nfailtot[16];  // nfailtot[N_NFAIL]
  int failure_exists;
  int ftype[3];                     // failure_type[N_PFLAG_TYPES]
  int bnd_phys;                     // boundary_phys_pflag
  int q_count;                      // cells queued for the inversion fallback tree
  int fl_count;                     // cells flagged for interpolation
  int err;                          // internal error status (queue overflow ...)
  double m_tot;
  double last_maxs[4];              // max_char_speed of the last corrector, as doubles
  int lev[3];                       // metric_dim 3: geomL buffers of n_beg, n_mid, n_end
};

// Everything a kernel needs, passed by value.
struct GridDev {
  int N[3];          // physical zones
  int T[3];          // stored extent per direction (N+6, or 1 when degenerate)
  int deg[3];        // 1 if N == 1
  int st[3];         // stride per direction (0 when degenerate); planes hold < 2^31 entries
  long S;            // plane size
  int NE[3];         // last physical index N+2
  int recon, flux, ct_para, bc, mdim, use_ee, cooling, rescale, nsd;
  int prec;                  // HG_PREC_FP64 or HG_PREC_MIXED (FP32 face fluxes)
  // HG_PREC_MIXED only: FP32 copy of the substep's input primitives (8
  // planes of S), FP32 geometry of the faces (HG_GF planes of gS, metric_dim
  // 2) and FP32 RESCALE_R factors (12 planes of T0)
  float *p32, *geomF, *rsc32;
  double *Uc;                // conserved variables after the update (8 planes of S)
  double *q_F;               // entropy face fluxes of the queued zones (6 per queue slot)
  double gam, cour;
  double dx[4], invdx[4];
  double startx[4], grid_length[4];
  // state
  double *p, *ph;            // 8 planes each
  double *F[3];              // 8 planes each, face index = lower face of the cell
  double *emf[3];            // corner EMFs
  double *p_gamma;
  int *pflag;
  unsigned int *nfail;       // HG_NF planes
  double *floors;            // 2 planes: rhoflr, uuflr
  double *geomT;             // metric_dim 2: 42 planes of HG_NPOS*T0*T1, index (pos*T1 + j)*T0 + i
  long gS;                   // geometry plane size
  double *conn;              // metric_dim 2: 64 planes of T0*T1 (physical i,j only used)
  double *rsc;               // RESCALE_R: 12 planes of T0: rscale[0..5], 1/rscale[0..5]
  double *cool;              // cooling 1: 2 planes of T0: Omega(r_i), T(r_i)
  DevScalars *sc;
  unsigned long long *q_idx; // fallback queue: packed (i,j,k)
  double *q_U;               // 8 doubles per queued cell
  unsigned long long *fl_idx;// interpolation list: packed (i,j,k)
  long capacity;             // N0*N1*N2
  double *blk;               // per-block partial sums of M_tot
  Geom g0;                   // metric_dim 0 geometry
  // metric_dim 3: three time levels of geometry, each HG_DYN_PLANES planes
  // of gS3 = 5*S doubles (index pos*S + zone offset), filled by
  // k_geom_level; the connection of the current substep, HG_CONN3_PLANES
  // planes of S (k_conn_dyn)
  double *geomL[3];
  long gS3;
  double *conn3;
  DynMetric dyn;
  // metric_dim 3: per-axis coordinate tables at faces and centres (r, dr/dx1,
  // th, dth/dx2, sin th, cos th, sin phi, cos phi), filled on the host with
  // the platform's libm (dyn_coord_tables, hg_dyn.cuh)
  double *ctab;
  // metric_dim 3, mixed form: per level the FP32 face geometry of FACE1..3
  // (HG_GF planes of 3*S floats, index d*S + zone offset), written by
  // k_geom_level beside geomL
  float *geomF3[3];
};

// metric_dim 3 level tables: the geometry the engine evaluates is symmetric
// (gcov[a][b] and gcov[b][a] are the same double), so a struct of_geom is
// stored as the 10 entries a <= b of gcon and of gcov, g, g_inv, alpha,
// beta[3] and ncon[0]: 27 planes in place of 42.  ncon[1..3] = -alpha
// gcon[0][i] are formed on reading with dyn_geom's own operations.
#define HG_DYN_PLANES 27
// positions kept per level: FACE1, FACE2, FACE3, CENT (no kernel reads the
// corner position's geometry)
#define HG_DYN_NPOS 4
#define HG_DP_GCON 0
#define HG_DP_GCOV 10
#define HG_DP_G 20
#define HG_DP_GINV 21
#define HG_DP_ALPHA 22
#define HG_DP_BETA 23
#define HG_DP_NCON0 26
__host__ __device__ __forceinline__ int dyn_sym(int a, int b)
{
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  return lo * 4 - (lo * (lo - 1)) / 2 + (hi - lo);  // (0,0)..(0,3) 0..3, (1,1)..(1,3) 4..6, (2,2) 7, (2,3) 8, (3,3) 9
}

// metric_dim 3 connection: conn[a][b][c] = conn[a][c][b] to the bit (the
// two swapped terms of DGCOV_TO_CONN add in the other order), so conn3
// keeps the 40 entries b <= c, plane a*10 + dyn_sym(b, c).
#define HG_CONN3_PLANES 40

// Fixed grid sizes of the step's kernels (grid-stride loops).
struct LaunchCfg {
  int grid_flux, grid_emf, grid_upd, grid_fix, grid_bnd;
  int grid_flux32;  // FP32 flux kernel of the mixed form (more resident blocks)
  int strip_nf;     // faces per thread of the strip flux kernels (1..3)
  int strip_x1;     // x1 faces in strips too (else one face per thread)
  int grid_fb;      // k_fallback: every block the device holds at once (set by hg_init)
};
#define HG_BLK_CAP 65536  // largest grid of any kernel (the per-block M_tot partials are sized for it)

// Kernel classes timed by the optional event recorder.
enum { KC_FLUX = 0, KC_EMF, KC_UPDATE, KC_FALLBACK, KC_BOUNDS, KC_FIXUP, KC_MISC, KC_GEOM, KC_END, KC_N };

// Optional CUDA-event recorder: an event is recorded on the launch stream
// before every kernel (tagged with its class) and one after the last.
struct EventRec {
  void **ev;   // cudaEvent_t pool
  int *cls;
  int n, cap;
};

__host__ __device__ inline unsigned long long pack_ijk(int i, int j, int k)
{
  return (unsigned long long)i | ((unsigned long long)j << 21) | ((unsigned long long)k << 42);
}
__host__ __device__ inline void unpack_ijk(unsigned long long v, int &i, int &j, int &k)
{
  i = (int)(v & 0x1FFFFF);
  j = (int)((v >> 21) & 0x1FFFFF);
  k = (int)((v >> 42) & 0x1FFFFF);
}

// hg_geometry.cu: the Kerr-Schild connection rows of a COORD_DIAGONAL3 grid
void ks_conn_rows(double a, double R0, double h_slope, double diag3_factor, int diag3_exponent, const double *startx,
                  const double *dx, int n1, int n2, double *out);

}  // namespace hg
