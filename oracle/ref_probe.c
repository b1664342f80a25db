/* ref_probe.c -- harness hook linked into the reference build (oracle/_ref).
 *
 * Test infrastructure only.  oracle/build_ref.py compiles the reference's
 * step_ch.c with -Dstep_ch=ref_step_ch, so the reference's own main() loop
 * (src/main.c:64-115) calls the step_ch() defined here, which wraps the real
 * step (src/step_ch.c:50-234) and adds, driven by environment variables:
 *
 *   HARM_PROBE_LOAD=<file>     before the first step, replace p[][][][] (all
 *                              cells, ghosts included), t and dx[0] with the
 *                              contents of a state file (format below)
 *   HARM_PROBE_OUT=<prefix>    write <prefix>.<nstep>.bin after every dumped step
 *   HARM_PROBE_DUMP=a,b,...    steps after which to dump (0 = the state before
 *                              the first step); default: only the last step
 *   HARM_PROBE_MAXSTEPS=N      stop (exit 0) after N steps
 *   HARM_PROBE_TIME=1          print one line "probe_time steps=<n> seconds=<s>
 *                              cells=<NCELLS>" timing only the step calls
 *   HARM_PROBE_TIME_SKIP=k     leave the first k steps out of that timing
 *                              (warm-up: first-call set-up such as the
 *                              cooling tables of phys.c:683-704)
 *   HARM_PROBE_FINAL=1         write <prefix>.<nstep>.bin after the step that
 *                              reaches t >= GridLength[0] (where main()'s loop,
 *                              main.c:64, ends the run) and exit 0
 *
 * State file (native little-endian):
 *   char magic[4]="HGST"; int32 version=1;
 *   int32 N1,N2,N3,NG,NP; double t, dt, M_tot; int32 nstep;
 *   uint64 nfailtot[N_NFAIL];
 *   double p[N1TOT][N2TOT][N3TOT][NP];   (the reference's own index order)
 *   int32  pflag[N1TOT][N2TOT][N3TOT];
 *   double p_gamma[N1TOT][N2TOT][N3TOT];
 *   int32  nfail[N_NFAIL][N1TOT][N2TOT][N3TOT];
 * A load file needs the header and p only.
 */
#include "decs.h"
#include <stdint.h>
#include <time.h>

extern void ref_step_ch(void);
extern double omega_circular_equatorial(double r_loc);
extern double target_temperature(double r_loc, double h_o_r);

static int probe_started = 0;
static long probe_maxsteps = -1;
static double probe_seconds = 0.;
static long probe_steps = 0;
static int probe_time = 0;
static long probe_skip = 0;

static int should_dump(int n)
{
  const char *s = getenv("HARM_PROBE_DUMP");
  if (!s) return 0;
  char buf[4096];
  strncpy(buf, s, sizeof(buf) - 1);
  buf[sizeof(buf) - 1] = 0;
  for (char *tok = strtok(buf, ","); tok; tok = strtok(NULL, ",")) {
    if (atoi(tok) == n) return 1;
  }
  return 0;
}

static void dump_state(int n)
{
  const char *pre = getenv("HARM_PROBE_OUT");
  if (!pre) return;
  char fname[4200];
  snprintf(fname, sizeof(fname), "%s.%d.bin", pre, n);
  FILE *f = fopen(fname, "wb");
  if (!f) { fprintf(stderr, "probe: cannot open %s\n", fname); exit(3); }
  int32_t hdr[6] = {1, N1, N2, N3, NG, NP};
  fwrite("HGST", 1, 4, f);
  fwrite(hdr, sizeof(int32_t), 6, f);
  double d3[3] = {t, dx[0], M_tot};
  fwrite(d3, sizeof(double), 3, f);
  int32_t ns = nstep;
  fwrite(&ns, sizeof(int32_t), 1, f);
  for (int l = 0; l < N_NFAIL; l++) { uint64_t v = nfailtot[l]; fwrite(&v, 8, 1, f); }
  int i, j, k;
  ALL_LOOP fwrite(p[i][j][k], sizeof(double), NP, f);
  ALL_LOOP { int32_t v = pflag[i][j][k]; fwrite(&v, 4, 1, f); }
  ALL_LOOP fwrite(&p_gamma[i][j][k], sizeof(double), 1, f);
  for (int l = 0; l < N_NFAIL; l++) ALL_LOOP { int32_t v = nfail[l][i][j][k]; fwrite(&v, 4, 1, f); }
  fclose(f);
}

static void load_state(const char *fname)
{
  FILE *f = fopen(fname, "rb");
  if (!f) { fprintf(stderr, "probe: cannot open %s\n", fname); exit(3); }
  char magic[4];
  int32_t hdr[6];
  double d3[3];
  int32_t ns;
  uint64_t nf[N_NFAIL];
  if (fread(magic, 1, 4, f) != 4 || memcmp(magic, "HGST", 4) ||
      fread(hdr, 4, 6, f) != 6 || fread(d3, 8, 3, f) != 3 || fread(&ns, 4, 1, f) != 1 ||
      fread(nf, 8, N_NFAIL, f) != N_NFAIL) {
    fprintf(stderr, "probe: bad header in %s\n", fname); exit(3);
  }
  if (hdr[1] != N1 || hdr[2] != N2 || hdr[3] != N3 || hdr[4] != NG || hdr[5] != NP) {
    fprintf(stderr, "probe: grid mismatch in %s\n", fname); exit(3);
  }
  int i, j, k, l;
  ALL_LOOP {
    if (fread(p[i][j][k], sizeof(double), NP, f) != NP) {
      fprintf(stderr, "probe: short file %s\n", fname); exit(3);
    }
  }
  fclose(f);
  t = d3[0];
  dx[0] = d3[1];
  for (l = 0; l < N_NFAIL; l++) nfailtot[l] = 0;
  for (l = 0; l < N_NFAIL; l++) ALL_LOOP nfail[l][i][j][k] = 0;
}

/* HARM_PROBE_GEOM=<file>: after init, write the run parameters and the static
 * geometry tables:
 *   char magic[4]="HGGM"; double gam, cour, GridLength[4], startx[4], dx[4];
 *   int32 N_GEOM, N_CONN; then N_GEOM x 42 doubles (struct of_geom order:
 *   gcon[16], gcov[16], g, g_inv, alpha, beta[3], ncon[4]) of time level 0,
 *   N_CONN x 64 doubles of conn[][][][], and per cell (ALL_LOOP order) the
 *   CENT coordinate data: rhoflr, uuflr, r, x[1], x[2], x[3]; then per i:
 *   x[RR] at FACE1, Omega(r_i), T(r_i) (3 doubles). */
static void dump_geom(const char *fname)
{
  FILE *f = fopen(fname, "wb");
  if (!f) { fprintf(stderr, "probe: cannot open %s\n", fname); exit(3); }
  fwrite("HGGM", 1, 4, f);
  double prm[14] = {gam, cour, GridLength[0], GridLength[1], GridLength[2], GridLength[3],
                    startx[0], startx[1], startx[2], startx[3], dx[0], dx[1], dx[2], dx[3]};
  fwrite(prm, 8, 14, f);
  int32_t n[2] = {N_GEOM, N_CONN};
  fwrite(n, 4, 2, f);
  for (long g = 0; g < N_GEOM; g++) {
    struct of_geom *gm = &geom_arr[0][g];
    fwrite(gm->gcon, 8, 16, f);
    fwrite(gm->gcov, 8, 16, f);
    fwrite(&gm->g, 8, 1, f);
    fwrite(&gm->g_inv, 8, 1, f);
    fwrite(&gm->alpha, 8, 1, f);
    fwrite(gm->beta, 8, 3, f);
    fwrite(gm->ncon, 8, 4, f);
  }
  for (long l = 0; l < N_CONN; l++) {
    int a, b, c;
    for (a = 0; a < NDIM; a++) for (b = 0; b < NDIM; b++) for (c = 0; c < NDIM; c++)
      fwrite(&conn[l][a][b][c], 8, 1, f);
  }
  int i, j, k;
  ALL_LOOP {
    struct of_coord *cd;
    get_coord(i, j, k, CENT, 0, cd);
    double v[6] = {cd->rhoflr, cd->uuflr, cd->r, cd->x[1], cd->x[2], cd->x[3]};
    fwrite(v, 8, 6, f);
  }
  /* per radial index: x[RR] at FACE1 (rescale_prims_r, recon.c:1142-1165) and
   * the H/R cooling tables of cooling_func_hr_disk (phys.c:683-704), for the
   * h_o_r given in HARM_PROBE_HOR (0 when not given) */
  const char *hs = getenv("HARM_PROBE_HOR");
  double hor = hs ? atof(hs) : 0.;
  for (i = 0; i < N1TOT; i++) {
    struct of_coord *cd;
    get_coord(i, N2S, N3S, FACE1, 0, cd);
    double rf = cd->x[RR];
    get_coord(i, N2S, N3S, CENT, 0, cd);
    double v[3] = {rf, 0., 0.};
    if (hor > 0.) {
      v[1] = omega_circular_equatorial(cd->x[RR]);
      v[2] = target_temperature(cd->x[RR], hor);
    }
    fwrite(v, 8, 3, f);
  }
  fclose(f);
}

static double now_s(void)
{
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void probe_finish(void)
{
  if (probe_time) {
    printf("probe_time steps=%ld seconds=%.9f cells=%ld\n", probe_steps - (probe_skip < probe_steps ? probe_skip : probe_steps),
           probe_seconds, (long)NCELLS);
    fflush(stdout);
  }
}

void step_ch(void)
{
  if (!probe_started) {
    probe_started = 1;
    const char *gf = getenv("HARM_PROBE_GEOM");
    if (gf) dump_geom(gf);
    const char *ld = getenv("HARM_PROBE_LOAD");
    if (ld) load_state(ld);
    const char *ms = getenv("HARM_PROBE_MAXSTEPS");
    if (ms) probe_maxsteps = atol(ms);
    probe_time = getenv("HARM_PROBE_TIME") != NULL;
    const char *sk = getenv("HARM_PROBE_TIME_SKIP");
    if (sk) probe_skip = atol(sk);
    if (should_dump(0)) dump_state(0);
  }
  const int timed = probe_time && probe_steps >= probe_skip;
  double t0 = timed ? now_s() : 0.;
  ref_step_ch();
  if (timed) probe_seconds += now_s() - t0;
  probe_steps++;
  /* main() increments nstep after this returns; report the step count done */
  int done = nstep + 1;
  int last = (probe_maxsteps > 0 && probe_steps >= probe_maxsteps);
  if (getenv("HARM_PROBE_FINAL") && t >= GridLength[0]) {
    int save = nstep;
    nstep = done;
    dump_state(done);
    nstep = save;
    probe_finish();
    exit(0);
  }
  if (should_dump(done) || (last && getenv("HARM_PROBE_OUT") && !getenv("HARM_PROBE_DUMP"))) {
    int save = nstep;
    nstep = done;
    dump_state(done);
    nstep = save;
  }
  if (last) {
    probe_finish();
    exit(0);
  }
}
