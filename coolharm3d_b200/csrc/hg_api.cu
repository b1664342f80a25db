// hg_api.cu -- host side of libharmgpu: the C ABI declared in include/harmgpu.h.
//
// Owns the device-resident grid of one simulation, converts between the
// reference's array layout (flattened p[i][j][k][l]) and the engine's
// structure-of-arrays layout, and launches the step (hg_kernels.cu).
#include <cuda.h>  // CUpointer_attribute (queried through the runtime's driver entry point)
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "harmgpu.h"
#include "hg_internal.h"
#include "hg_dyn.cuh"

namespace hg {
void launch_step(const GridDev &G, const LaunchCfg &L, cudaStream_t s, EventRec *R);
void *gather_times_kernel();
void launch_to_f32(const GridDev &G, int grid, cudaStream_t s, const double *src);
void launch_mirror_check(const GridDev &G, int grid, cudaStream_t s, const double *src, unsigned long long *count);
void launch_face_flux(const GridDev &G, const LaunchCfg &L, cudaStream_t s, int d);
void launch_fixup_bounds(const GridDev &G, const LaunchCfg &L, cudaStream_t s);
void launch_bounds_only(const GridDev &G, const LaunchCfg &L, cudaStream_t s);
cudaError_t prepare_kernels();
int fallback_blocks_per_sm(bool rs);
void launch_geom_levels(const GridDev &G, const LaunchCfg &L, cudaStream_t s);
void launch_conn_broadcast(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *rows);
void launch_totals(const GridDev &G, const LaunchCfg &L, cudaStream_t s, double *part, double *out);
void launch_ref_to_planes(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *ref, int NT1, int NT2,
                          double *out);
void launch_planes_to_ref(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *in, int NT0, int NT1,
                          int NT2, double *ref);
}  // namespace hg

// The same step kernels built with contracted multiply-adds
// (hg_kernels.cu compiled with HG_FMA_BUILD): HG_PREC_FP64_FMA.
namespace hg_fma {
void launch_step(const hg::GridDev &G, const hg::LaunchCfg &L, cudaStream_t s, hg::EventRec *R);
void launch_geom_levels(const hg::GridDev &G, const hg::LaunchCfg &L, cudaStream_t s);
void launch_face_flux(const hg::GridDev &G, const hg::LaunchCfg &L, cudaStream_t s, int d);
cudaError_t prepare_kernels();
int fallback_blocks_per_sm(bool rs);
}  // namespace hg_fma

// One step's launch sequence of the grid's precision form.  The plain FP64
// form runs the kernels built without contracted multiply-adds
// (bit-identical to the reference); the FMA form and the mixed form, whose
// FP32 fluxes are not bit-identical anyway, run the build with fused
// multiply-adds for their FP64 kernels.
static bool fma_kernels(const hg::GridDev &G) { return G.prec == HG_PREC_FP64_FMA || G.prec == HG_PREC_MIXED; }

static void launch_grid_step(const hg::GridDev &G, const hg::LaunchCfg &L, cudaStream_t s, hg::EventRec *R)
{
  if (fma_kernels(G)) hg_fma::launch_step(G, L, s, R);
  else hg::launch_step(G, L, s, R);
}

using hg::GridDev;

#define HG_XCH_THREADS 8              // host threads of one transfer
#define HG_XCH (2 * HG_XCH_THREADS)   // pinned staging slots, two per thread
#define HG_XCH_BYTES (4L << 20)       // bytes per transfer chunk (a multiple of 64)

struct hg_handle {
  hg_grid_desc d;
  GridDev G;
  hg::LaunchCfg L;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  float last_ms = 0.f;
  bool have_geom = false, have_cells = false, have_prims = false, have_cool = false;
  std::vector<void *> allocs;
  double *h_stage = nullptr;  // pinned transfer chunks (HG_XCH x HG_XCH_BYTES)
  cudaEvent_t xev[HG_XCH] = {};  // DMA completion of each transfer chunk
  double *d_ref = nullptr;    // device buffer in the reference layout (host <-> device transfers)
  cudaGraph_t step_graph = nullptr;  // one hg_step(1) captured (batches, and hg_step itself)
  cudaGraphExec_t step_exec = nullptr;  // step_graph instantiated for hg_step
  bool exec_stale = true;
  bool graph_dirty = true;           // the capture predates a change of the kernels' arguments
  uint64_t capture_gen = 0;          // number of captures of step_graph so far (batches compare it)
  bool levels_stale = false;         // metric_dim 3: the time levels predate t, dx[0] or the metric
  double *d_tot = nullptr;           // hg_get_totals: per-block partials and the result
  int batch_refs = 0;                // batches this grid belongs to
  long ntot_ref = 0;          // N1TOT*N2TOT*N3TOT of the reference layout
  int NT[3] = {0, 0, 0};      // reference extents
  // per-kernel-class timing (hg_profile)
  bool prof = false;
  std::vector<cudaEvent_t> pev;
  std::vector<int> pcls;
  double kc_ms[hg::KC_N] = {0};
  long long kc_n[hg::KC_N] = {0};
};

#define HG_CK(call)                                                                   \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      fprintf(stderr, "libharmgpu: %s failed: %s\n", #call, cudaGetErrorString(e_)); \
      return HG_ERR_CUDA;                                                             \
    }                                                                                 \
  } while (0)

// a copy on the grid's stream, complete on return
static cudaError_t copy_sync(hg_handle *h, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind)
{
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  return e;
}

// address of a field of the device-resident DevScalars (no host dereference)
static void *sc_field(const GridDev &G, size_t off) { return (char *)G.sc + off; }

// Every copy and memset of a grid goes through the grid's own stream: the
// stream is non-blocking, so work on the legacy default stream (plain
// cudaMemcpy / cudaMemset) would not be ordered before its kernels.
static int dev_alloc(hg_handle *h, void **p, size_t bytes)
{
  if (cudaMalloc(p, bytes) != cudaSuccess) {
    cudaGetLastError();
    return HG_ERR_NOMEM;
  }
  if (cudaMemsetAsync(*p, 0, bytes, h->stream) != cudaSuccess) {
    cudaFree(*p);
    return HG_ERR_CUDA;
  }
  h->allocs.push_back(*p);
  return HG_OK;
}

extern "C" const char *hg_strerror(int code)
{
  switch (code) {
    case HG_OK: return "ok";
    case HG_ERR_CUDA: return "CUDA runtime error";
    case HG_ERR_BADARG: return "invalid argument or unsupported switch value";
    case HG_ERR_TIMEOUT: return "device-side wait timed out";
    case HG_ERR_NOMEM: return "out of device memory";
    case HG_ERR_STATE: return "call out of order";
    case HG_ERR_DEVICE: return "kernel reported an internal error";
    default: return "unknown error";
  }
}

static int validate(const hg_grid_desc *d)
{
  if (!d) return HG_ERR_BADARG;
  if (d->n1 < 1 || d->n2 < 1 || d->n3 < 1) return HG_ERR_BADARG;
  if (d->n1 + 2 * HG_NGH >= (1 << 21) || d->n2 + 2 * HG_NGH >= (1 << 21) || d->n3 + 2 * HG_NGH >= (1 << 21))
    return HG_ERR_BADARG;
  // the kernels index zones and faces with 32-bit arithmetic: every plane
  // must hold fewer than 2^31 entries (2^31 zones would need ~1 TB of HBM)
  if ((long long)(d->n1 + 2 * HG_NGH) * (d->n2 + 2 * HG_NGH) * (d->n3 + 2 * HG_NGH) >= (1LL << 31))
    return HG_ERR_BADARG;
  if (d->recon_type < 0 || d->recon_type > 5) return HG_ERR_BADARG;
  if (d->flux_type != 0 && d->flux_type != 1) return HG_ERR_BADARG;
  if (d->bc_type != 0 && d->bc_type != 1 && d->bc_type != 10) return HG_ERR_BADARG;
  // the spherical boundaries need the radial and polar directions resolved
  if (d->bc_type == 10 && (d->n1 == 1 || d->n2 == 1)) return HG_ERR_BADARG;
  if (d->metric_dim != 0 && d->metric_dim != 2 && d->metric_dim != 3) return HG_ERR_BADARG;
  // metric_dim 3 (time-dependent metric): every direction resolved, FP64 forms
  if (d->metric_dim == 3 && (d->n1 == 1 || d->n2 == 1 || d->n3 == 1))
    return HG_ERR_BADARG;
  if (d->cooling != 0 && d->cooling != 1) return HG_ERR_BADARG;
  if (d->precision != HG_PREC_FP64 && d->precision != HG_PREC_MIXED && d->precision != HG_PREC_FP64_FMA)
    return HG_ERR_BADARG;
  // the tables of METRIC_DIM 2 vary with i and j: those directions must be resolved
  if (d->metric_dim == 2 && (d->n1 == 1 || d->n2 == 1)) return HG_ERR_BADARG;
  if (d->rescale_r && d->n1 == 1) return HG_ERR_BADARG;
  if (!(d->gam > 1.) || !(d->cour > 0.)) return HG_ERR_BADARG;
  for (int a = 1; a < 4; a++)
    if (!(d->dx[a] > 0.)) return HG_ERR_BADARG;
  return HG_OK;
}

extern "C" int hg_init(const hg_grid_desc *desc, hg_handle **out)
{
  if (!out) return HG_ERR_BADARG;
  *out = nullptr;
  int rc = validate(desc);
  if (rc) return rc;
  HG_CK(cudaSetDevice(desc->device));
  hg_handle *h = new (std::nothrow) hg_handle();
  if (!h) return HG_ERR_NOMEM;
  h->d = *desc;
  GridDev &G = h->G;
  memset(&G, 0, sizeof(G));
  const int n[3] = {desc->n1, desc->n2, desc->n3};
  long st = 1;
  for (int a = 0; a < 3; a++) {
    G.N[a] = n[a];
    G.deg[a] = (n[a] == 1);
    G.T[a] = G.deg[a] ? 1 : n[a] + 2 * HG_NGH;
    G.NE[a] = n[a] + HG_NGH - 1;
    h->NT[a] = n[a] + 2 * HG_NGH;
  }
  for (int a = 0; a < 3; a++) {
    G.st[a] = G.deg[a] ? 0 : st;
    st *= G.T[a];
  }
  G.S = st;
  h->ntot_ref = (long)h->NT[0] * h->NT[1] * h->NT[2];
  G.recon = desc->recon_type;
  G.flux = desc->flux_type;
  G.prec = desc->precision;
  G.ct_para = desc->use_flux_ct_para;
  G.bc = desc->bc_type;
  G.mdim = desc->metric_dim;
  G.use_ee = desc->use_entropy_eq;
  G.cooling = desc->cooling;
  G.rescale = desc->rescale_r;
  G.nsd = (n[0] > 1) + (n[1] > 1) + (n[2] > 1);
  G.gam = desc->gam;
  G.cour = desc->cour;
  for (int a = 0; a < 4; a++) {
    G.dx[a] = desc->dx[a];
    G.invdx[a] = 1. / desc->dx[a];
    G.startx[a] = desc->startx[a];
    G.grid_length[a] = desc->grid_length[a];
  }
  G.capacity = (long)n[0] * n[1] * n[2];
  const size_t S8 = sizeof(double) * G.S;
#define ALLOC(ptr, bytes)                                     \
  do {                                                        \
    void *q_ = nullptr;                                       \
    if ((rc = dev_alloc(h, &q_, (bytes))) != HG_OK) goto fail; \
    ptr = (decltype(ptr))q_;                                  \
  } while (0)
  if (hg::prepare_kernels() != cudaSuccess || hg_fma::prepare_kernels() != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    delete h;
    return HG_ERR_CUDA;
  }
  {
    ALLOC(G.p, S8 * HG_NPR);
    ALLOC(G.ph, S8 * HG_NPR);
    ALLOC(G.Uc, S8 * HG_NPR);
    for (int d = 0; d < 3; d++) ALLOC(G.F[d], S8 * HG_NPR);
    for (int d = 0; d < 3; d++) ALLOC(G.emf[d], S8);
    ALLOC(G.p_gamma, S8);
    ALLOC(G.pflag, sizeof(int) * G.S);
    ALLOC(G.nfail, sizeof(unsigned int) * G.S * HG_NF);
    ALLOC(G.floors, S8 * 2);
    ALLOC(G.sc, sizeof(hg::DevScalars));
    ALLOC(G.q_idx, sizeof(unsigned long long) * G.capacity);
    ALLOC(G.q_U, sizeof(double) * HG_NPR * G.capacity);
    if (G.use_ee) ALLOC(G.q_F, sizeof(double) * 6 * G.capacity);
    ALLOC(G.fl_idx, sizeof(unsigned long long) * G.capacity);
    if (G.mdim == 2) {
      G.gS = (long)HG_NPOS * G.T[0] * G.T[1];
      ALLOC(G.geomT, sizeof(double) * 42 * G.gS);
      ALLOC(G.conn, sizeof(double) * 64 * G.T[0] * G.T[1]);
    }
    if (G.mdim == 3) {  // three time levels of 42 planes of 5 positions, the substep's connection
      G.gS3 = (long)HG_DYN_NPOS * G.S;
      for (int l = 0; l < 3; l++) ALLOC(G.geomL[l], sizeof(double) * HG_DYN_PLANES * G.gS3);
      ALLOC(G.conn3, sizeof(double) * HG_CONN3_PLANES * G.S);
      ALLOC(G.ctab, sizeof(double) * hg::dyn_tab_layout(G.T).total);
    }
    if (G.rescale) ALLOC(G.rsc, sizeof(double) * 12 * G.T[0]);
    if (G.prec == HG_PREC_MIXED) {
      ALLOC(G.p32, sizeof(float) * HG_NPR * G.S);
      if (G.mdim == 2) ALLOC(G.geomF, sizeof(float) * HG_GF * G.gS);
      if (G.mdim == 3)
        for (int l = 0; l < 3; l++) ALLOC(G.geomF3[l], sizeof(float) * HG_GF * 3 * G.S);
      if (G.rescale) ALLOC(G.rsc32, sizeof(float) * 12 * G.T[0]);
    }
    if (G.cooling) ALLOC(G.cool, sizeof(double) * 2 * G.T[0]);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, desc->device);
    auto grid_for = [&](long work, int per_sm) {
      long g = (work + 127) / 128;
      long cap = (long)sms * per_sm;
      if (g > cap) g = cap;
      if (g > HG_BLK_CAP) g = HG_BLK_CAP;
      if (g < 1) g = 1;
      return (int)g;
    };
    long faces = (long)G.T[0] * G.T[1] * G.T[2];
    // defaults from hg_autotune on the 192x192x128 torus: many short-lived
    // blocks for the stencil and update kernels, few for the sparse lists
    h->L.grid_flux = grid_for(faces, 64);
    h->L.grid_flux32 = grid_for(faces, 96);
    h->L.grid_emf = grid_for(faces, 64);
    h->L.grid_upd = grid_for(G.capacity, 128);
    h->L.grid_fix = grid_for(G.capacity, 2);
    h->L.grid_bnd = grid_for(faces - G.capacity, 16);
    h->L.strip_nf = 2;  // 2-face strips in all three directions (with these
    h->L.strip_x1 = 1;  // block counts, the torus's fastest)
    {  // the fallback tree: every block the device holds at once, no more
       // than the grid's zones need (small grids in a batch launch few)
      const int fb = fma_kernels(G) ? hg_fma::fallback_blocks_per_sm(G.rescale != 0)
                                    : hg::fallback_blocks_per_sm(G.rescale != 0);
      h->L.grid_fb = grid_for(G.capacity, fb);
    }
    ALLOC(G.blk, sizeof(double) * HG_BLK_CAP);
    if (cudaMallocHost((void **)&h->h_stage, (size_t)HG_XCH * HG_XCH_BYTES) != cudaSuccess) {
      cudaGetLastError();
      rc = HG_ERR_NOMEM;
      goto fail;
    }
    if (cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
      rc = HG_ERR_CUDA;
      goto fail;
    }
    for (int x = 0; x < HG_XCH; x++)
      if (cudaEventCreateWithFlags(&h->xev[x], cudaEventDisableTiming) != cudaSuccess) {
        rc = HG_ERR_CUDA;
        goto fail;
      }
    hg::DevScalars sc0;
    memset(&sc0, 0, sizeof(sc0));
    sc0.t = desc->t;
    sc0.dt = desc->dx[0];
    sc0.lev[0] = 0;  // n_beg, n_mid, n_end (init_general_metric, metric.c:3676-3679)
    sc0.lev[1] = 1;
    sc0.lev[2] = 2;
    if (copy_sync(h, G.sc, &sc0, sizeof(sc0), cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = HG_ERR_CUDA;
      goto fail;
    }
  }
#undef ALLOC
  *out = h;
  return HG_OK;
fail:
  hg_destroy(h);
  return rc;
}

extern "C" void hg_destroy(hg_handle *h)
{
  if (!h) return;
  if (h->batch_refs > 0) {
    fprintf(stderr, "libharmgpu: hg_destroy on a grid that is still in a batch; hg_batch_remove it first\n");
    return;
  }
  cudaSetDevice(h->d.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (cudaEvent_t e : h->pev) cudaEventDestroy(e);
  for (void *p : h->allocs) cudaFree(p);
  if (h->h_stage) cudaFreeHost(h->h_stage);
  if (h->step_exec) cudaGraphExecDestroy(h->step_exec);
  if (h->step_graph) cudaGraphDestroy(h->step_graph);
  for (int x = 0; x < HG_XCH; x++)
    if (h->xev[x]) cudaEventDestroy(h->xev[x]);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

extern "C" int hg_set_geometry(hg_handle *h, const double *geom, int64_t n_geom, const double *conn, int64_t n_conn)
{
  if (!h || !geom) return HG_ERR_BADARG;
  if (h->G.mdim == 3) return HG_ERR_BADARG;  // its geometry comes from hg_set_dynamic_metric
  h->graph_dirty = true;
  GridDev &G = h->G;
  HG_CK(cudaSetDevice(h->d.device));
  if (G.mdim == 0) {
    if (n_geom < 1) return HG_ERR_BADARG;
    hg::Geom &g = G.g0;
    memcpy(g.gcon, geom, 16 * 8);
    memcpy(g.gcov, geom + 16, 16 * 8);
    g.g = geom[32];
    g.g_inv = geom[33];
    g.alpha = geom[34];
    for (int a = 0; a < 3; a++) g.beta[a] = geom[35 + a];
    for (int a = 0; a < 4; a++) g.ncon[a] = geom[38 + a];
  } else {
    const int N1T = h->NT[0], N2T = h->NT[1];
    if (n_geom != (int64_t)HG_NPOS * N1T * N2T || !conn || n_conn != (int64_t)G.N[0] * G.N[1]) return HG_ERR_BADARG;
    std::vector<double> t((size_t)42 * G.gS);
    for (int pos = 0; pos < HG_NPOS; pos++)
      for (int i = 0; i < N1T; i++)
        for (int j = 0; j < N2T; j++) {
          const double *s = geom + 42L * (j + (long)N2T * (i + (long)N1T * pos));  // GEOM_ID
          const long o = ((long)pos * G.T[1] + j) * G.T[0] + i;
          for (int f = 0; f < 42; f++) t[f * G.gS + o] = s[f];
        }
    HG_CK(copy_sync(h, G.geomT, t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice));
    if (G.geomF) {  // the mixed form's FP32 face geometry
      std::vector<float> f((size_t)HG_GF * G.gS);
      for (long o = 0; o < G.gS; o++) {
        for (int a = 0; a < 16; a++) f[a * G.gS + o] = (float)t[(16 + a) * G.gS + o];
        f[16 * G.gS + o] = (float)t[0 * G.gS + o];
        for (int j = 1; j <= 3; j++) {
          f[(16 + j) * G.gS + o] = (float)t[j * G.gS + o];
          f[(19 + j) * G.gS + o] = (float)t[(j * 4 + j) * G.gS + o];
        }
        f[23 * G.gS + o] = (float)t[38 * G.gS + o];
        for (int a = 0; a < 3; a++) f[(24 + a) * G.gS + o] = (float)t[(35 + a) * G.gS + o];
        f[27 * G.gS + o] = (float)t[32 * G.gS + o];
      }
      HG_CK(copy_sync(h, G.geomF, f.data(), sizeof(float) * f.size(), cudaMemcpyHostToDevice));
    }
    const long cS = (long)G.T[0] * G.T[1];
    std::vector<double> c((size_t)64 * cS, 0.);
    for (int i = 0; i < G.N[0]; i++)
      for (int j = 0; j < G.N[1]; j++) {
        const double *s = conn + 64L * (j + (long)G.N[1] * i);  // CONN_ID
        const long o = (long)(j + HG_NGH) * G.T[0] + (i + HG_NGH);
        for (int f = 0; f < 64; f++) c[f * cS + o] = s[f];
      }
    HG_CK(copy_sync(h, G.conn, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice));
  }
  h->have_geom = true;
  return HG_OK;
}

// ref index of the stored zone along direction a for stored index x
static inline int ref_of(const GridDev &G, int a, int x) { return G.deg[a] ? HG_NGH : x; }

extern "C" int hg_set_cell_data(hg_handle *h, const double *cell6, const double *rface)
{
  if (!h || !cell6) return HG_ERR_BADARG;
  h->graph_dirty = true;
  GridDev &G = h->G;
  HG_CK(cudaSetDevice(h->d.device));
  const int N2T = h->NT[1], N3T = h->NT[2];
  std::vector<double> fl((size_t)2 * G.S);
  for (int k = 0; k < G.T[2]; k++)
    for (int j = 0; j < G.T[1]; j++)
      for (int i = 0; i < G.T[0]; i++) {
        const long r = ((long)ref_of(G, 0, i) * N2T + ref_of(G, 1, j)) * N3T + ref_of(G, 2, k);
        const long o = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
        fl[o] = cell6[r * 6 + 0];
        fl[G.S + o] = cell6[r * 6 + 1];
      }
  HG_CK(copy_sync(h, G.floors, fl.data(), sizeof(double) * fl.size(), cudaMemcpyHostToDevice));
  if (G.rescale) {
    if (!rface) return HG_ERR_BADARG;
    const int T0 = G.T[0];
    std::vector<double> r((size_t)12 * T0);
    // rescale_prims_r(), recon.c:1142-1165: x[RR] (the x1 column) of the
    // zone centres of the row (i, N2S, N3S), as that row reads on its first call
    for (int i = 0; i < T0; i++) {
      double rloc = cell6[(((long)i * N2T + HG_NGH) * N3T + HG_NGH) * 6 + 3];
      double rf2 = rloc * rloc;
      r[0 * T0 + i] = sqrt(rf2 * rloc);
      r[1 * T0 + i] = rf2 * rloc;
      r[2 * T0 + i] = rloc;
      rloc = rface[i];
      rf2 = rloc * rloc;
      r[3 * T0 + i] = sqrt(rf2 * rloc);
      r[4 * T0 + i] = rf2 * rloc;
      r[5 * T0 + i] = rloc;
      for (int a = 0; a < 6; a++) r[(6 + a) * T0 + i] = 1 / r[a * T0 + i];
    }
    HG_CK(copy_sync(h, G.rsc, r.data(), sizeof(double) * r.size(), cudaMemcpyHostToDevice));
    if (G.rsc32) {
      std::vector<float> r32(r.begin(), r.end());
      HG_CK(copy_sync(h, G.rsc32, r32.data(), sizeof(float) * r32.size(), cudaMemcpyHostToDevice));
    }
  }
  h->have_cells = true;
  return HG_OK;
}

extern "C" int hg_set_cooling_tables(hg_handle *h, const double *omega, const double *t_target)
{
  if (!h || !omega || !t_target) return HG_ERR_BADARG;
  if (!h->G.cooling) return HG_ERR_STATE;
  HG_CK(cudaSetDevice(h->d.device));
  const int T0 = h->G.T[0];
  std::vector<double> c((size_t)2 * T0);
  for (int i = 0; i < T0; i++) {
    c[i] = omega[i];
    c[T0 + i] = t_target[i];
  }
  HG_CK(copy_sync(h, h->G.cool, c.data(), sizeof(double) * c.size(), cudaMemcpyHostToDevice));
  h->have_cool = true;
  return HG_OK;
}

// Host <-> device transfer of the primitives in the reference layout.  The
// reference-ordered array (N1TOT*N2TOT*N3TOT zones of 8 doubles) moves as a
// byte stream of HG_XCH_BYTES chunks through pinned staging slots: up to
// HG_XCH_THREADS host threads each copy their share of chunks between the
// caller's memory and two slots of their own, so host copies overlap one
// another and the DMA of the other chunks.  On the device the stream lands
// in a buffer in the same layout, and a kernel converts it to or from the
// resident planes.  That buffer is a buffer of its own, allocated on the
// first transfer: the flux planes are not free between steps, because
// hg_get_totals (dump_ener's boundary-flux integrals) reads the last
// substep's fluxes after the driver has brought the primitives back.
static double *ref_buffer(hg_handle *h)
{
  if (!h->d_ref) {
    void *q = nullptr;
    if (dev_alloc(h, &q, sizeof(double) * HG_NPR * h->ntot_ref) != HG_OK) return nullptr;
    h->d_ref = (double *)q;
  }
  return h->d_ref;
}

// Runs work(w, nw) on nw = min(HG_XCH_THREADS, chunks) threads (the calling
// thread is worker 0); returns the first non-success status.
template <class W>
static cudaError_t run_workers(long nch, W work)
{
  const int nw = (int)std::max<long>(1, std::min<long>(nch, HG_XCH_THREADS));
  std::vector<cudaError_t> st(nw, cudaSuccess);
  std::vector<std::thread> th;
  int started = 1;
  for (int w = 1; w < nw; w++, started++) {
    try {
      th.emplace_back([&st, &work, w, nw] { st[w] = work(w, nw); });
    } catch (...) {
      break;
    }
  }
  // worker 0 takes its own chunks and those of any worker not started
  st[0] = work(0, nw);
  for (int w = started; w < nw; w++) st[w] = work(w, nw);
  for (auto &t : th) t.join();
  for (cudaError_t e : st)
    if (e != cudaSuccess) return e;
  return cudaSuccess;
}

// cuPointerGetAttribute through the runtime's driver entry point (no link
// against libcuda); null if the driver does not provide it.
typedef CUresult (*hg_ptr_attr_fn)(void *, CUpointer_attribute, CUdeviceptr);
static hg_ptr_attr_fn ptr_attr_fn()
{
  static hg_ptr_attr_fn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (hg_ptr_attr_fn)f;
    cudaGetLastError();
  });
  return fn;
}

// True if the whole range [p, p + bytes) lies in ONE page-locked host
// allocation (cudaHostAlloc or cudaHostRegister): the DMA engines can then
// read or write the caller's buffer directly, with no staging copy on the
// host.  Both ends must be page-locked and carry the same allocation id, so
// a range spanning two page-locked allocations with pageable memory between
// them takes the staged path.
static bool host_pinned(const void *p, size_t bytes)
{
  cudaPointerAttributes a, b;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess ||
      cudaPointerGetAttributes(&b, (const char *)p + bytes - 1) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type != cudaMemoryTypeHost || b.type != cudaMemoryTypeHost) return false;
  hg_ptr_attr_fn fn = ptr_attr_fn();
  unsigned long long ida = 0, idb = 0;
  if (!fn || fn(&ida, CU_POINTER_ATTRIBUTE_BUFFER_ID, (CUdeviceptr)p) != CUDA_SUCCESS ||
      fn(&idb, CU_POINTER_ATTRIBUTE_BUFFER_ID, (CUdeviceptr)((const char *)p + bytes - 1)) != CUDA_SUCCESS)
    return false;
  return ida == idb;
}

// FILL(dst, first zone, zones) writes that many zones of the reference order;
// with a page-locked `direct` source the reference-order array is copied by
// one DMA instead.
template <class FILL>
static int upload_impl(hg_handle *h, FILL fill, const double *direct = nullptr)
{
  GridDev &G = h->G;
  HG_CK(cudaSetDevice(h->d.device));
  double *dref = ref_buffer(h);
  if (!dref) return HG_ERR_NOMEM;
  const long zc = HG_XCH_BYTES / (sizeof(double) * HG_NPR);  // zones per chunk
  const long nch = direct ? 0 : (h->ntot_ref + zc - 1) / zc;
  const int dev = h->d.device;
  if (direct)
    HG_CK(cudaMemcpyAsync(dref, direct, sizeof(double) * HG_NPR * h->ntot_ref, cudaMemcpyHostToDevice, h->stream));
  else HG_CK(run_workers(nch, [&](int w, int nw) -> cudaError_t {
    cudaError_t e = cudaSetDevice(dev);
    long n = 0;
    for (long c = w; c < nch && e == cudaSuccess; c += nw, n++) {
      const int slot = 2 * w + (int)(n & 1);
      const long z0 = c * zc, nz = std::min(zc, h->ntot_ref - z0);
      double *hb = h->h_stage + (long)slot * zc * HG_NPR;
      if (n >= 2) e = cudaEventSynchronize(h->xev[slot]);
      if (e != cudaSuccess) break;
      fill(hb, z0, nz);
      e = cudaMemcpyAsync(dref + z0 * HG_NPR, hb, sizeof(double) * HG_NPR * nz, cudaMemcpyHostToDevice, h->stream);
      if (e == cudaSuccess) e = cudaEventRecord(h->xev[slot], h->stream);
    }
    return e;
  }));
  hg::launch_ref_to_planes(G, h->L, h->stream, dref, h->NT[1], h->NT[2], G.p);
  HG_CK(cudaGetLastError());
  HG_CK(cudaMemsetAsync(G.nfail, 0, sizeof(unsigned int) * HG_NF * G.S, h->stream));
  HG_CK(cudaMemsetAsync(G.pflag, 0, sizeof(int) * G.S, h->stream));
  HG_CK(cudaMemsetAsync(sc_field(G, offsetof(hg::DevScalars, nfailtot)), 0, sizeof(unsigned long long) * 16, h->stream));
  HG_CK(cudaStreamSynchronize(h->stream));
  h->have_prims = true;
  return HG_OK;
}

// DRAIN(src, first zone, zones) reads that many zones of the reference order;
// a page-locked `direct` destination receives the array by one DMA instead.
template <class DRAIN>
static int download_impl(hg_handle *h, DRAIN drain, double *direct = nullptr)
{
  GridDev &G = h->G;
  HG_CK(cudaSetDevice(h->d.device));
  double *dref = ref_buffer(h);
  if (!dref) return HG_ERR_NOMEM;
  hg::launch_planes_to_ref(G, h->L, h->stream, G.p, h->NT[0], h->NT[1], h->NT[2], dref);
  HG_CK(cudaGetLastError());
  if (direct) {
    HG_CK(cudaMemcpyAsync(direct, dref, sizeof(double) * HG_NPR * h->ntot_ref, cudaMemcpyDeviceToHost, h->stream));
    HG_CK(cudaStreamSynchronize(h->stream));
    return HG_OK;
  }
  const long zc = HG_XCH_BYTES / (sizeof(double) * HG_NPR);
  const long nch = (h->ntot_ref + zc - 1) / zc;
  const int dev = h->d.device;
  HG_CK(run_workers(nch, [&](int w, int nw) -> cudaError_t {
    cudaError_t e = cudaSetDevice(dev);
    // two chunks in flight per worker: issue c, then drain c - nw
    long prev = -1;
    int n = 0;
    for (long c = w; e == cudaSuccess; c += nw, n++) {
      if (c < nch) {
        const int slot = 2 * w + (n & 1);
        const long z0 = c * zc, nz = std::min(zc, h->ntot_ref - z0);
        e = cudaMemcpyAsync(h->h_stage + (long)slot * zc * HG_NPR, dref + z0 * HG_NPR, sizeof(double) * HG_NPR * nz,
                            cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaEventRecord(h->xev[slot], h->stream);
        if (e != cudaSuccess) break;
      }
      if (prev >= 0) {
        const int slot = 2 * w + ((n - 1) & 1);
        const long z0 = prev * zc, nz = std::min(zc, h->ntot_ref - z0);
        e = cudaEventSynchronize(h->xev[slot]);
        if (e != cudaSuccess) break;
        drain(h->h_stage + (long)slot * zc * HG_NPR, z0, nz);
      }
      if (c >= nch) break;
      prev = c;
    }
    return e;
  }));
  return HG_OK;
}

extern "C" int hg_upload_prims(hg_handle *h, const double *p)
{
  if (!h || !p) return HG_ERR_BADARG;
  HG_CK(cudaSetDevice(h->d.device));
  const bool pinned = host_pinned(p, sizeof(double) * HG_NPR * h->ntot_ref);
  return upload_impl(
      h, [&](double *dst, long z0, long nz) { memcpy(dst, p + z0 * HG_NPR, sizeof(double) * HG_NPR * nz); },
      pinned ? p : nullptr);
}

extern "C" int hg_download_prims(hg_handle *h, double *p)
{
  if (!h || !p) return HG_ERR_BADARG;
  HG_CK(cudaSetDevice(h->d.device));
  const bool pinned = host_pinned(p, sizeof(double) * HG_NPR * h->ntot_ref);
  return download_impl(
      h, [&](const double *src, long z0, long nz) { memcpy(p + z0 * HG_NPR, src, sizeof(double) * HG_NPR * nz); },
      pinned ? p : nullptr);
}

// zone z of the reference order -> (i, j, k)
static inline void ref_ijk(const hg_handle *h, long z, int &i, int &j, int &k)
{
  k = (int)(z % h->NT[2]);
  j = (int)((z / h->NT[2]) % h->NT[1]);
  i = (int)(z / ((long)h->NT[2] * h->NT[1]));
}

extern "C" int hg_upload_prims_tree(hg_handle *h, double ****p)
{
  if (!h || !p) return HG_ERR_BADARG;
  return upload_impl(h, [&](double *dst, long z0, long nz) {
    for (long z = 0; z < nz; z++) {
      int i, j, k;
      ref_ijk(h, z0 + z, i, j, k);
      memcpy(dst + z * HG_NPR, p[i][j][k], sizeof(double) * HG_NPR);
    }
  });
}

extern "C" int hg_download_prims_tree(hg_handle *h, double ****p)
{
  if (!h || !p) return HG_ERR_BADARG;
  return download_impl(h, [&](const double *src, long z0, long nz) {
    for (long z = 0; z < nz; z++) {
      int i, j, k;
      ref_ijk(h, z0 + z, i, j, k);
      memcpy(p[i][j][k], src + z * HG_NPR, sizeof(double) * HG_NPR);
    }
  });
}

extern "C" int hg_set_time(hg_handle *h, double t, double dt)
{
  if (!h) return HG_ERR_BADARG;
  HG_CK(cudaSetDevice(h->d.device));
  double v[2] = {t, dt};
  HG_CK(copy_sync(h, sc_field(h->G, offsetof(hg::DevScalars, t)), v, sizeof(v), cudaMemcpyHostToDevice));
  if (h->G.mdim == 3) h->levels_stale = true;
  return HG_OK;
}

// metric_dim 3: (re)fill the three time levels at the device's t and dx[0]
// after the metric, t or dx[0] changed (init_general_metric, metric.c:3664)
static int refresh_levels(hg_handle *h)
{
  if (h->G.mdim != 3 || !h->levels_stale) return HG_OK;
  if (fma_kernels(h->G)) hg_fma::launch_geom_levels(h->G, h->L, h->stream);  // the build the steps use
  else hg::launch_geom_levels(h->G, h->L, h->stream);
  HG_CK(cudaGetLastError());
  h->levels_stale = false;
  return HG_OK;
}

static int capture_step(hg_handle *h);

static int step_exec_ready(hg_handle *h)
{
  const bool recaptured = !h->step_graph || h->graph_dirty;
  int rc = capture_step(h);
  if (rc != HG_OK) return rc;
  if (h->step_exec && !recaptured && !h->exec_stale) return HG_OK;
  if (h->step_exec) {
    cudaGraphExecDestroy(h->step_exec);
    h->step_exec = nullptr;
  }
  HG_CK(cudaGraphInstantiate(&h->step_exec, h->step_graph, 0));
  h->exec_stale = false;
  return HG_OK;
}

extern "C" int hg_step(hg_handle *h, int32_t nsteps, double *t, double *dt)
{
  if (!h || nsteps < 0) return HG_ERR_BADARG;
  if (!h->have_geom || !h->have_cells || !h->have_prims) return HG_ERR_STATE;
  if (h->G.cooling && !h->have_cool) return HG_ERR_STATE;
  HG_CK(cudaSetDevice(h->d.device));
  hg::EventRec rec, *R = nullptr;
  if (h->prof) {
    const size_t need = (size_t)40 * (nsteps > 0 ? nsteps : 1);
    while (h->pev.size() < need) {
      cudaEvent_t e;
      HG_CK(cudaEventCreate(&e));
      h->pev.push_back(e);
    }
    h->pcls.resize(h->pev.size());
    rec.ev = (void **)h->pev.data();
    rec.cls = h->pcls.data();
    rec.n = 0;
    rec.cap = (int)h->pev.size();
    R = &rec;
  }
  // Without per-kernel events the step runs as one CUDA graph launch (the
  // same kernels with the same arguments, captured once), which takes the
  // host's launch cost of small grids off the step.
  if (!R && nsteps > 0) {
    int rc = step_exec_ready(h);
    if (rc != HG_OK) return rc;
  }
  {
    int rc = refresh_levels(h);
    if (rc != HG_OK) return rc;
  }
  HG_CK(cudaEventRecord(h->ev0, h->stream));
  for (int s = 0; s < nsteps; s++) {
    if (R) launch_grid_step(h->G, h->L, h->stream, R);
    else HG_CK(cudaGraphLaunch(h->step_exec, h->stream));
  }
  HG_CK(cudaGetLastError());
  HG_CK(cudaEventRecord(h->ev1, h->stream));
  HG_CK(cudaEventSynchronize(h->ev1));
  HG_CK(cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
  if (R) {
    for (int e = 0; e + 1 < R->n; e++) {
      float ms = 0.f;
      HG_CK(cudaEventElapsedTime(&ms, h->pev[e], h->pev[e + 1]));
      const int c = R->cls[e];
      if (c >= 0 && c < hg::KC_END) {
        h->kc_ms[c] += ms;
        h->kc_n[c] += 1;
      }
    }
  }
  hg::DevScalars sc;
  HG_CK(copy_sync(h, &sc, h->G.sc, sizeof(sc), cudaMemcpyDeviceToHost));
  if (sc.err) return HG_ERR_DEVICE;
  if (t) *t = sc.t;
  if (dt) *dt = sc.dt;
  return HG_OK;
}

static int dyn_from_abi(const hg_dyn_metric *m, hg::DynMetric &dm)
{
  if (!m ||
      (m->spacetime != HG_DYN_MINK_SPHERICAL && m->spacetime != HG_DYN_PN_BINARY &&
       m->spacetime != HG_DYN_KS_SPHERICAL) ||
      m->diag3_exponent < 3 || !(m->dt_conn > 0.))
    return HG_ERR_BADARG;
  if (m->spacetime == HG_DYN_KS_SPHERICAL && !(fabs(m->spin) < 1.)) return HG_ERR_BADARG;
  dm.spin = m->spin;
  if (m->spacetime == HG_DYN_PN_BINARY &&
      (!(m->m1 > 0.) || !(m->m2 > 0.) || !(m->separation > 0.) || (m->inspiral != 0 && m->inspiral != 1)))
    return HG_ERR_BADARG;
  dm.m1 = m->m1;
  dm.m2 = m->m2;
  dm.sep = m->separation;
  dm.phase0 = m->phase0;
  dm.inspiral = m->inspiral;
  dm.spacetime = m->spacetime;
  dm.diag3_exponent = m->diag3_exponent;
  dm.R0 = m->R0;
  dm.h_slope = m->h_slope;
  dm.diag3_factor = m->diag3_factor;
  dm.dt_conn = m->dt_conn;
  return HG_OK;
}

extern "C" int hg_set_dynamic_metric(hg_handle *h, const hg_dyn_metric *m)
{
  if (!h || h->G.mdim != 3) return HG_ERR_BADARG;
  int rc = dyn_from_abi(m, h->G.dyn);
  if (rc != HG_OK) return rc;
  HG_CK(cudaSetDevice(h->d.device));
  {  // the coordinates' per-axis tables (the device reads, never evaluates, them)
    GridDev Gh = h->G;
    std::vector<double> tab((size_t)hg::dyn_tab_layout(Gh.T).total);
    Gh.ctab = tab.data();
    hg::dyn_coord_tables(Gh, tab.data());
    HG_CK(copy_sync(h, h->G.ctab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
  }
  if (h->G.dyn.spacetime == HG_DYN_KS_SPHERICAL) {
    // the static analytic connection of the Kerr-Schild test spacetime
    // (metric.c:3555-3558), the same in every phi layer: rows per (i, j),
    // spread over k on the device
    const hg::DynMetric &dm = h->G.dyn;
    const int n1 = h->G.N[0], n2 = h->G.N[1];
    std::vector<double> rows((size_t)64 * n1 * n2);
    hg::ks_conn_rows(dm.spin, dm.R0, dm.h_slope, dm.diag3_factor, dm.diag3_exponent, h->d.startx, h->d.dx, n1, n2,
                     rows.data());
    void *drows = nullptr;  // set-up-time staging of the rows, freed below
    if (cudaMalloc(&drows, sizeof(double) * rows.size()) != cudaSuccess) {
      cudaGetLastError();
      return HG_ERR_NOMEM;
    }
    cudaError_t e = cudaMemcpyAsync(drows, rows.data(), sizeof(double) * rows.size(), cudaMemcpyHostToDevice,
                                    h->stream);
    if (e == cudaSuccess) {
      hg::launch_conn_broadcast(h->G, h->L, h->stream, (const double *)drows);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(drows);
    HG_CK(e);
  }
  const int lev[3] = {0, 1, 2};  // n_beg, n_mid, n_end (init_general_metric, metric.c:3676-3679)
  HG_CK(copy_sync(h, sc_field(h->G, offsetof(hg::DevScalars, lev)), lev, sizeof(lev), cudaMemcpyHostToDevice));
  h->levels_stale = true;
  h->graph_dirty = true;  // the metric's parameters are kernel arguments
  h->have_geom = true;
  return HG_OK;
}

extern "C" int hg_dyn_geometry(const hg_grid_desc *d, const hg_dyn_metric *m, int32_t pos, int32_t i, int32_t j,
                               int32_t k, double t, double geom[HG_NGEOM])
{
  if (!d || !geom || pos < 0 || pos > 4) return HG_ERR_BADARG;
  GridDev G;
  memset(&G, 0, sizeof(G));
  int rc = dyn_from_abi(m, G.dyn);
  if (rc != HG_OK) return rc;
  for (int a = 0; a < 4; a++) {
    G.startx[a] = d->startx[a];
    G.dx[a] = d->dx[a];
  }
  G.T[0] = d->n1 + 2 * HG_NGH;
  G.T[1] = d->n2 + 2 * HG_NGH;
  G.T[2] = d->n3 + 2 * HG_NGH;
  if (i < 0 || j < 0 || k < 0 || i >= G.T[0] || j >= G.T[1] || k >= G.T[2]) return HG_ERR_BADARG;
  std::vector<double> tab((size_t)hg::dyn_tab_layout(G.T).total);
  hg::dyn_coord_tables(G, tab.data());
  G.ctab = tab.data();
  hg::Geom g;
  hg::dyn_geom(G, pos, i, j, k, t, g);
  memcpy(geom, g.gcon, 16 * 8);
  memcpy(geom + 16, g.gcov, 16 * 8);
  geom[32] = g.g;
  geom[33] = g.g_inv;
  geom[34] = g.alpha;
  for (int a = 0; a < 3; a++) geom[35 + a] = g.beta[a];
  for (int a = 0; a < 4; a++) geom[38 + a] = g.ncon[a];
  return HG_OK;
}

extern "C" int hg_download_dyn_level(hg_handle *h, int32_t level, double *geom)
{
  if (!h || !geom || h->G.mdim != 3 || level < 0 || level > 2) return HG_ERR_BADARG;
  if (!h->have_geom) return HG_ERR_STATE;
  HG_CK(cudaSetDevice(h->d.device));
  int rc = refresh_levels(h);
  if (rc != HG_OK) return rc;
  int lev[3];
  HG_CK(copy_sync(h, lev, sc_field(h->G, offsetof(hg::DevScalars, lev)), sizeof(lev), cudaMemcpyDeviceToHost));
  const GridDev &G = h->G;
  std::vector<double> buf((size_t)HG_DYN_PLANES * G.gS3);
  HG_CK(copy_sync(h, buf.data(), G.geomL[lev[level]], sizeof(double) * buf.size(), cudaMemcpyDeviceToHost));
  const long T0 = G.T[0], T1 = G.T[1], T2 = G.T[2];
  for (int pos = 0; pos < HG_DYN_NPOS; pos++)
    for (long i = 0; i < T0; i++)
      for (long j = 0; j < T1; j++)
        for (long k = 0; k < T2; k++) {
          const long src = (long)pos * G.S + i * G.st[0] + j * G.st[1] + k * G.st[2];
          auto at = [&](int plane) { return buf[(size_t)plane * G.gS3 + src]; };
          double *o = geom + ((((long)pos * T0 + i) * T1 + j) * T2 + k) * HG_NGEOM;
          for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
              o[a * 4 + b] = at(HG_DP_GCON + hg::dyn_sym(a, b));
              o[16 + a * 4 + b] = at(HG_DP_GCOV + hg::dyn_sym(a, b));
            }
          o[32] = at(HG_DP_G);
          o[33] = at(HG_DP_GINV);
          o[34] = at(HG_DP_ALPHA);
          for (int a = 0; a < 3; a++) o[35 + a] = at(HG_DP_BETA + a);
          o[38] = at(HG_DP_NCON0);
          for (int a = 1; a < 4; a++) o[38 + a] = -o[34] * o[a];
        }
  return HG_OK;
}

extern "C" int hg_dyn_geometry_block(const hg_grid_desc *d, const hg_dyn_metric *m, int32_t pos, double t,
                                     int32_t i0, int32_t ni, double *geom)
{
  if (!d || !geom || pos < 0 || pos > 4 || ni < 0) return HG_ERR_BADARG;
  const int T0 = d->n1 + 2 * HG_NGH, T1 = d->n2 + 2 * HG_NGH, T2 = d->n3 + 2 * HG_NGH;
  if (i0 < 0 || i0 + ni > T0) return HG_ERR_BADARG;
  GridDev G;
  memset(&G, 0, sizeof(G));
  int rc = dyn_from_abi(m, G.dyn);
  if (rc != HG_OK) return rc;
  for (int a = 0; a < 4; a++) {
    G.startx[a] = d->startx[a];
    G.dx[a] = d->dx[a];
  }
  G.T[0] = T0;
  G.T[1] = T1;
  G.T[2] = T2;
  std::vector<double> tab((size_t)hg::dyn_tab_layout(G.T).total);
  hg::dyn_coord_tables(G, tab.data());
  G.ctab = tab.data();
  const long rows = (long)ni * T1;
  const int nw = (int)std::max<long>(1, std::min<long>(rows, std::max(1u, std::thread::hardware_concurrency())));
  auto work = [&](int w) {
    for (long r = w; r < rows; r += nw) {
      const int i = i0 + (int)(r / T1), j = (int)(r % T1);
      for (int k = 0; k < T2; k++) {
        hg::Geom g;
        hg::dyn_geom(G, pos, i, j, k, t, g);
        double *o = geom + ((r * T2) + k) * HG_NGEOM;
        memcpy(o, g.gcon, 16 * 8);
        memcpy(o + 16, g.gcov, 16 * 8);
        o[32] = g.g;
        o[33] = g.g_inv;
        o[34] = g.alpha;
        for (int a = 0; a < 3; a++) o[35 + a] = g.beta[a];
        for (int a = 0; a < 4; a++) o[38 + a] = g.ncon[a];
      }
    }
  };
  std::vector<std::thread> th;
  for (int w = 1; w < nw; w++) th.emplace_back(work, w);
  work(0);
  for (auto &x : th) x.join();
  return HG_OK;
}

extern "C" int hg_fixup_bounds(hg_handle *h)
{
  if (!h) return HG_ERR_BADARG;
  if (!h->have_geom || !h->have_cells || !h->have_prims) return HG_ERR_STATE;
  HG_CK(cudaSetDevice(h->d.device));
  int rc = refresh_levels(h);
  if (rc != HG_OK) return rc;
  hg::launch_fixup_bounds(h->G, h->L, h->stream);
  HG_CK(cudaGetLastError());
  HG_CK(cudaStreamSynchronize(h->stream));
  return HG_OK;
}

extern "C" int hg_face_flux(hg_handle *h, int32_t dir, double *flux, double *max_char_speed)
{
  if (!h || dir < 0 || dir > 2 || !flux) return HG_ERR_BADARG;
  if (!h->have_geom || !h->have_cells || !h->have_prims) return HG_ERR_STATE;
  GridDev &G = h->G;
  HG_CK(cudaSetDevice(h->d.device));
  HG_CK(cudaMemsetAsync(G.F[dir], 0, sizeof(double) * HG_NPR * G.S, h->stream));
  {
    int rc = refresh_levels(h);
    if (rc != HG_OK) return rc;
  }
  if (fma_kernels(G)) hg_fma::launch_face_flux(G, h->L, h->stream, dir);
  else hg::launch_face_flux(G, h->L, h->stream, dir);
  HG_CK(cudaGetLastError());
  HG_CK(cudaStreamSynchronize(h->stream));
  // per-cell planes -> reference layout with the variable index innermost
  std::vector<double> tmp((size_t)HG_NPR * G.S);
  HG_CK(copy_sync(h, tmp.data(), G.F[dir], sizeof(double) * tmp.size(), cudaMemcpyDeviceToHost));
  // faces numerical_flux() computes (step_ch.c:668-675), in reference indices
  int lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    if (a == dir) {
      lo[a] = HG_NGH;
      hi[a] = G.NE[a] + 1;
    } else if (G.ct_para) {
      lo[a] = 0;
      hi[a] = G.NE[a] + HG_NGH;
    } else {
      lo[a] = HG_NGH - 1;
      hi[a] = G.NE[a] + 1;
    }
  }
  for (int i = 0; i < h->NT[0]; i++)
    for (int j = 0; j < h->NT[1]; j++)
      for (int k = 0; k < h->NT[2]; k++) {
        const long o = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
        double *dst = flux + (((long)i * h->NT[1] + j) * h->NT[2] + k) * HG_NPR;
        const bool in = i >= lo[0] && i <= hi[0] && j >= lo[1] && j <= hi[1] && k >= lo[2] && k <= hi[2];
        for (int l = 0; l < HG_NPR; l++) dst[l] = in ? tmp[l * G.S + o] : 0.;
      }
  if (max_char_speed) {
    unsigned long long m;
    HG_CK(copy_sync(h, &m, sc_field(G, offsetof(hg::DevScalars, maxs) + sizeof(unsigned long long) * (dir + 1)),
                     sizeof(m), cudaMemcpyDeviceToHost));
    memcpy(max_char_speed, &m, sizeof(double));
  }
  return HG_OK;
}

extern "C" int hg_get_fail_counts(hg_handle *h, uint64_t nfailtot[HG_NFAIL])
{
  if (!h || !nfailtot) return HG_ERR_BADARG;
  HG_CK(cudaSetDevice(h->d.device));
  unsigned long long v[16];
  HG_CK(copy_sync(h, v, sc_field(h->G, offsetof(hg::DevScalars, nfailtot)), sizeof(v), cudaMemcpyDeviceToHost));
  for (int l = 0; l < HG_NFAIL; l++) nfailtot[l] = v[l];
  return HG_OK;
}

template <class T>
static int download_cellwise(hg_handle *h, const T *dsrc, T *out, int planes)
{
  GridDev &G = h->G;
  HG_CK(cudaSetDevice(h->d.device));
  std::vector<T> tmp((size_t)planes * G.S);
  HG_CK(copy_sync(h, tmp.data(), dsrc, sizeof(T) * tmp.size(), cudaMemcpyDeviceToHost));
  const long nref = h->ntot_ref;
  for (int pl = 0; pl < planes; pl++)
    for (int i = 0; i < h->NT[0]; i++)
      for (int j = 0; j < h->NT[1]; j++)
        for (int k = 0; k < h->NT[2]; k++) {
          const long o = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
          out[pl * nref + ((long)i * h->NT[1] + j) * h->NT[2] + k] = tmp[pl * G.S + o];
        }
  return HG_OK;
}

extern "C" int hg_download_pflag(hg_handle *h, int32_t *pflag)
{
  if (!h || !pflag) return HG_ERR_BADARG;
  return download_cellwise<int>(h, h->G.pflag, pflag, 1);
}

extern "C" int hg_download_gamma(hg_handle *h, double *g)
{
  if (!h || !g) return HG_ERR_BADARG;
  return download_cellwise<double>(h, h->G.p_gamma, g, 1);
}

extern "C" int hg_download_nfail(hg_handle *h, int32_t *nfail)
{
  if (!h || !nfail) return HG_ERR_BADARG;
  return download_cellwise<int>(h, (const int *)h->G.nfail, nfail, HG_NF);
}

extern "C" int hg_get_diag(hg_handle *h, double *m_tot, double mcs[3])
{
  if (!h) return HG_ERR_BADARG;
  HG_CK(cudaSetDevice(h->d.device));
  hg::DevScalars sc;
  HG_CK(copy_sync(h, &sc, h->G.sc, sizeof(sc), cudaMemcpyDeviceToHost));
  if (m_tot) *m_tot = sc.m_tot;
  if (mcs)
    for (int a = 0; a < 3; a++) mcs[a] = sc.last_maxs[a + 1];
  return HG_OK;
}

extern "C" int hg_profile(hg_handle *h, int32_t enable)
{
  if (!h) return HG_ERR_BADARG;
  h->prof = enable != 0;
  for (int c = 0; c < hg::KC_N; c++) {
    h->kc_ms[c] = 0.;
    h->kc_n[c] = 0;
  }
  return HG_OK;
}

extern "C" int hg_kernel_times(hg_handle *h, double ms[HG_NKCLASS], int64_t launches[HG_NKCLASS])
{
  if (!h || !ms || !launches) return HG_ERR_BADARG;
  for (int c = 0; c < HG_NKCLASS; c++) {
    ms[c] = h->kc_ms[c];
    launches[c] = h->kc_n[c];
  }
  return HG_OK;
}

extern "C" int hg_last_step_ms(hg_handle *h, double *ms)
{
  if (!h || !ms) return HG_ERR_BADARG;
  *ms = h->last_ms;
  return HG_OK;
}

// calc_all_geom() for METRIC_MINK_CARTESIAN / COORD_IDENTITY (metric.c:4130-4140,
// 4235-4247) and coord_of_xp()'s floors (coord.c:3775-3796, FLOOR_STATIC).
extern "C" int hg_build_geometry_minkowski(const hg_grid_desc *d, double *geom, double *cell6)
{
  if (!d || !geom || !cell6) return HG_ERR_BADARG;
  for (int f = 0; f < 42; f++) geom[f] = 0.;
  geom[0] = -1.; geom[5] = 1.; geom[10] = 1.; geom[15] = 1.;           // gcon
  geom[16] = -1.; geom[21] = 1.; geom[26] = 1.; geom[31] = 1.;         // gcov
  geom[32] = 1.;                                                       // g
  geom[33] = 1. / geom[32];                                            // g_inv
  geom[38] = sqrt(-geom[0]);                                           // ncon[0] = 1/alpha
  geom[34] = 1. / geom[38];                                            // alpha
  for (int a = 1; a < 4; a++) geom[38 + a] = -geom[34] * geom[a];      // ncon[1..3]
  for (int a = 0; a < 3; a++) geom[35 + a] = -geom[a + 1] / geom[0];   // beta
  const double RHOMIN = 2.e-10, UUMIN = 2.e-12, RHOPOWER = -1.5, UUPOWER = -2.5;
  const int N1T = d->n1 + 6, N2T = d->n2 + 6, N3T = d->n3 + 6;
  for (int i = 0; i < N1T; i++)
    for (int j = 0; j < N2T; j++)
      for (int k = 0; k < N3T; k++) {
        const double x1 = d->startx[1] + (i + 0.5) * d->dx[1];
        const double x2 = d->startx[2] + (j + 0.5) * d->dx[2];
        const double x3 = d->startx[3] + (k + 0.5) * d->dx[3];
        const double r = sqrt(x1 * x1 + x2 * x2 + x3 * x3);
        double *c = cell6 + (((long)i * N2T + j) * N3T + k) * 6;
        c[0] = RHOMIN * pow(r, RHOPOWER);
        c[1] = UUMIN * pow(r, UUPOWER);
        c[2] = r;
        c[3] = x1;
        c[4] = x2;
        c[5] = x3;
      }
  return HG_OK;
}

// ===========================================================================
// Batches: several resident grids of one device advanced together.  Each
// member's step (the launch sequence of hg_step) is captured once into a
// CUDA graph; the batch graph holds every member's graph as an independent
// child node, so one graph launch runs all members' kernels concurrently,
// followed by one kernel that gathers every member's t, dx[0] and error
// status for a single small copy to the host.  The batch graph is rebuilt
// when the membership changes or a member's captured step goes stale.
// ===========================================================================
struct hg_batch {
  int device = 0, cap = 0;
  std::vector<hg_handle *> members;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool dirty = true;
  std::vector<uint64_t> gens;       // each member's capture_gen when the batch graph was built
  hg::DevScalars **d_sc = nullptr;  // device array of the members' DevScalars pointers
  double *d_out = nullptr;          // 3 doubles per member: t, dt, err
  double *h_out = nullptr;          // pinned copy
};

static int capture_step(hg_handle *h)
{
  if (h->step_graph && !h->graph_dirty) return HG_OK;
  if (h->step_graph) {
    cudaGraphDestroy(h->step_graph);
    h->step_graph = nullptr;
  }
  HG_CK(cudaSetDevice(h->d.device));
  HG_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  launch_grid_step(h->G, h->L, h->stream, nullptr);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  HG_CK(e);
  HG_CK(cudaGetLastError());
  h->step_graph = g;
  h->graph_dirty = false;
  h->exec_stale = true;
  h->capture_gen++;
  return HG_OK;
}

static int batch_rebuild(hg_batch *b)
{
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  const int n = (int)b->members.size();
  if (n == 0) {
    b->dirty = false;
    return HG_OK;
  }
  std::vector<hg::DevScalars *> sc(n);
  b->gens.assign(n, 0);
  for (int m = 0; m < n; m++) {
    int rc = capture_step(b->members[m]);
    if (rc != HG_OK) return rc;
    sc[m] = b->members[m]->G.sc;
    b->gens[m] = b->members[m]->capture_gen;
  }
  HG_CK(cudaSetDevice(b->device));
  HG_CK(cudaMemcpyAsync(b->d_sc, sc.data(), sizeof(void *) * n, cudaMemcpyHostToDevice, b->stream));
  HG_CK(cudaStreamSynchronize(b->stream));
  cudaGraph_t g = nullptr;
  HG_CK(cudaGraphCreate(&g, 0));
  std::vector<cudaGraphNode_t> kids(n);
  cudaError_t e = cudaSuccess;
  for (int m = 0; m < n && e == cudaSuccess; m++)
    e = cudaGraphAddChildGraphNode(&kids[m], g, nullptr, 0, b->members[m]->step_graph);
  if (e == cudaSuccess) {
    hg::DevScalars **scp = b->d_sc;
    int nn = n;
    double *out = b->d_out;
    void *args[] = {&scp, &nn, &out};
    cudaKernelNodeParams kp = {};
    kp.func = hg::gather_times_kernel();
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(128);
    kp.kernelParams = args;
    cudaGraphNode_t gather;
    e = cudaGraphAddKernelNode(&gather, g, kids.data(), n, &kp);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  HG_CK(e);
  b->dirty = false;
  return HG_OK;
}

extern "C" int hg_batch_create(int32_t device, int32_t max_grids, hg_batch **out)
{
  if (!out || max_grids < 1 || max_grids > 4096) return HG_ERR_BADARG;
  *out = nullptr;
  HG_CK(cudaSetDevice(device));
  hg_batch *b = new (std::nothrow) hg_batch;
  if (!b) return HG_ERR_NOMEM;
  b->device = device;
  b->cap = max_grids;
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc((void **)&b->d_sc, sizeof(void *) * max_grids) != cudaSuccess ||
      cudaMalloc((void **)&b->d_out, sizeof(double) * 3 * max_grids) != cudaSuccess ||
      cudaMallocHost((void **)&b->h_out, sizeof(double) * 3 * max_grids) != cudaSuccess) {
    cudaGetLastError();
    hg_batch_destroy(b);
    return HG_ERR_NOMEM;
  }
  *out = b;
  return HG_OK;
}

extern "C" int hg_batch_add(hg_batch *b, hg_handle *h)
{
  if (!b || !h || h->d.device != b->device) return HG_ERR_BADARG;
  if (!h->have_geom || !h->have_cells || !h->have_prims || (h->G.cooling && !h->have_cool)) return HG_ERR_STATE;
  for (hg_handle *m : b->members)
    if (m == h) return HG_ERR_BADARG;
  if ((int)b->members.size() >= b->cap) return HG_ERR_NOMEM;
  b->members.push_back(h);
  h->batch_refs++;
  b->dirty = true;
  return HG_OK;
}

extern "C" int hg_batch_remove(hg_batch *b, hg_handle *h)
{
  if (!b || !h) return HG_ERR_BADARG;
  for (size_t m = 0; m < b->members.size(); m++)
    if (b->members[m] == h) {
      b->members.erase(b->members.begin() + m);
      h->batch_refs--;
      b->dirty = true;
      return HG_OK;
    }
  return HG_ERR_BADARG;
}

extern "C" int hg_batch_size(const hg_batch *b) { return b ? (int)b->members.size() : HG_ERR_BADARG; }

extern "C" int hg_batch_step(hg_batch *b, double *t, double *dt)
{
  if (!b) return HG_ERR_BADARG;
  HG_CK(cudaSetDevice(b->device));
  // A member recaptured since the batch graph was built (a solo hg_step after
  // hg_set_geometry, hg_set_launch_config, hg_read_rdump, ...) holds new
  // kernel arguments that the batch's copy of its old graph lacks.
  for (size_t m = 0; m < b->members.size(); m++)
    if (b->members[m]->graph_dirty || m >= b->gens.size() || b->gens[m] != b->members[m]->capture_gen)
      b->dirty = true;
  if (b->dirty) {
    int rc = batch_rebuild(b);
    if (rc != HG_OK) return rc;
  }
  const int n = (int)b->members.size();
  if (n == 0) return HG_OK;
  for (hg_handle *m : b->members) {  // metric_dim 3 members whose time levels are not yet filled
    int rc = refresh_levels(m);
    if (rc != HG_OK) return rc;
  }
  // work the members queued on their own streams (uploads, set_time) comes first
  for (hg_handle *m : b->members) HG_CK(cudaStreamSynchronize(m->stream));
  HG_CK(cudaGraphLaunch(b->exec, b->stream));
  HG_CK(cudaMemcpyAsync(b->h_out, b->d_out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, b->stream));
  HG_CK(cudaStreamSynchronize(b->stream));
  int rc = HG_OK;
  for (int m = 0; m < n; m++) {
    if (t) t[m] = b->h_out[3 * m];
    if (dt) dt[m] = b->h_out[3 * m + 1];
    if (b->h_out[3 * m + 2] != 0.) rc = HG_ERR_DEVICE;
  }
  return rc;
}

extern "C" void hg_batch_destroy(hg_batch *b)
{
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (hg_handle *m : b->members) m->batch_refs--;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->d_sc) cudaFree(b->d_sc);
  if (b->d_out) cudaFree(b->d_out);
  if (b->h_out) cudaFreeHost(b->h_out);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

// ---------------------------------------------------------------------------
extern "C" int hg_check_mirror(hg_handle *h, int64_t *mismatches, int64_t *first)
{
  if (!h || !mismatches) return HG_ERR_BADARG;
  if (!h->G.p32) return HG_ERR_BADARG;  // the FP64 form keeps no FP32 copy
  HG_CK(cudaSetDevice(h->d.device));
  unsigned long long *d = nullptr, n[2] = {0ull, ~0ull};
  HG_CK(cudaMallocAsync((void **)&d, sizeof(n), h->stream));
  HG_CK(cudaMemcpyAsync(d, n, sizeof(n), cudaMemcpyHostToDevice, h->stream));
  hg::launch_mirror_check(h->G, h->L.grid_upd, h->stream, h->G.p, d);
  HG_CK(cudaGetLastError());
  HG_CK(cudaMemcpyAsync(n, d, sizeof(n), cudaMemcpyDeviceToHost, h->stream));
  HG_CK(cudaFreeAsync(d, h->stream));
  HG_CK(cudaStreamSynchronize(h->stream));
  *mismatches = (int64_t)n[0];
  if (first) *first = n[0] ? (int64_t)n[1] : -1;
  return HG_OK;
}

extern "C" int hg_mem_info(int32_t device, uint64_t *free_bytes, uint64_t *total_bytes)
{
  size_t f = 0, t = 0;
  HG_CK(cudaSetDevice(device));
  HG_CK(cudaMemGetInfo(&f, &t));
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return HG_OK;
}

// The device memory hg_init allocates for a description (the same planes
// and tables), plus the reference-layout transfer buffer a grid with a
// one-zone direction adds on its first transfer.
extern "C" int hg_grid_bytes(const hg_grid_desc *d, uint64_t *bytes)
{
  if (!d || !bytes) return HG_ERR_BADARG;
  int rc = validate(d);
  if (rc) return rc;
  const long n[3] = {d->n1, d->n2, d->n3};
  long T[3], S = 1, NT = 1;
  for (int a = 0; a < 3; a++) {
    T[a] = n[a] == 1 ? 1 : n[a] + 2 * HG_NGH;
    S *= T[a];
    NT *= n[a] + 2 * HG_NGH;
  }
  const long cap = n[0] * n[1] * n[2];
  const long gS = (long)HG_NPOS * T[0] * T[1];
  uint64_t b = 0;
  b += 8ull * HG_NPR * S * 6;                 // p, ph, Uc, F[3]
  b += 8ull * S * 3 + 8ull * S + 4ull * S;    // emf[3], p_gamma, pflag
  b += 4ull * S * HG_NF + 8ull * S * 2;       // nfail, floors
  b += sizeof(hg::DevScalars) + 8ull * cap * (2 + HG_NPR);  // scalars, queue, flagged list
  if (d->use_entropy_eq) b += 8ull * 6 * cap;                 // entropy face fluxes of the queue
  if (d->metric_dim == 2) b += 8ull * 42 * gS + 8ull * 64 * T[0] * T[1];
  if (d->metric_dim == 3) b += 3ull * 8 * HG_DYN_PLANES * HG_DYN_NPOS * S + 8ull * HG_CONN3_PLANES * S + 8ull * (4 * T[0] + 8 * T[1] + 4 * T[2]);  // coordinate tables
  if (d->rescale_r) b += 8ull * 12 * T[0];
  if (d->cooling) b += 8ull * 2 * T[0];
  if (d->precision == HG_PREC_MIXED) {
    b += 4ull * HG_NPR * S;
    if (d->metric_dim == 2) b += 4ull * HG_GF * gS;
    if (d->metric_dim == 3) b += 3ull * 4 * HG_GF * 3 * S;  // FP32 face geometry of the three levels
    if (d->rescale_r) b += 4ull * 12 * T[0];
  }
  b += 8ull * 148 * 8;                        // per-block partials
  b += 8ull * HG_NPR * NT;                    // transfer buffer in the reference layout
  *bytes = b;
  return HG_OK;
}

extern "C" int hg_get_totals(hg_handle *h, double U_tot[8], double F_tot[48], double *divb_max)
{
  if (!h) return HG_ERR_BADARG;
  if (!h->have_geom || !h->have_cells || !h->have_prims) return HG_ERR_STATE;
  HG_CK(cudaSetDevice(h->d.device));
  if (!h->d_tot) {
    void *q = nullptr;
    int rc = dev_alloc(h, &q, sizeof(double) * 57 * (2048 + 1));
    if (rc != HG_OK) return rc;
    h->d_tot = (double *)q;
  }
  double *out = h->d_tot + 57L * 2048;
  {
    int rc = refresh_levels(h);
    if (rc != HG_OK) return rc;
  }
  hg::launch_totals(h->G, h->L, h->stream, h->d_tot, out);
  HG_CK(cudaGetLastError());
  double v[57];
  HG_CK(copy_sync(h, v, out, sizeof(v), cudaMemcpyDeviceToHost));
  if (U_tot) memcpy(U_tot, v, 8 * sizeof(double));
  if (F_tot) memcpy(F_tot, v + 8, 48 * sizeof(double));
  if (divb_max) *divb_max = v[56];
  return HG_OK;
}

// ===========================================================================
// Launch configuration and its autotuner.
// ===========================================================================
static bool config_ok(const hg_launch_config *c)
{
  const int32_t g[6] = {c->grid_flux, c->grid_flux32, c->grid_emf, c->grid_update, c->grid_fixup, c->grid_bounds};
  for (int a = 0; a < 6; a++)
    if (g[a] < 1 || g[a] > HG_BLK_CAP) return false;
  return c->strip_faces >= 1 && c->strip_faces <= 3 && (c->strip_x1 == 0 || c->strip_x1 == 1);
}

extern "C" int hg_get_launch_config(hg_handle *h, hg_launch_config *c)
{
  if (!h || !c) return HG_ERR_BADARG;
  const hg::LaunchCfg &L = h->L;
  *c = hg_launch_config{L.grid_flux, L.grid_flux32, L.grid_emf, L.grid_upd, L.grid_fix, L.grid_bnd, L.strip_nf,
                        L.strip_x1};
  return HG_OK;
}

extern "C" int hg_set_launch_config(hg_handle *h, const hg_launch_config *c)
{
  if (!h || !c || !config_ok(c)) return HG_ERR_BADARG;
  hg::LaunchCfg &L = h->L;
  L.grid_flux = c->grid_flux;
  L.grid_flux32 = c->grid_flux32;
  L.grid_emf = c->grid_emf;
  L.grid_upd = c->grid_update;
  L.grid_fix = c->grid_fixup;
  L.grid_bnd = c->grid_bounds;
  L.strip_nf = c->strip_faces;
  L.strip_x1 = c->strip_x1;
  h->graph_dirty = true;
  return HG_OK;
}

// The resident state a step changes, saved and put back around trial steps.
struct Snapshot {
  double *p = nullptr, *gam = nullptr;
  int *pflag = nullptr;
  unsigned int *nfail = nullptr;
  hg::DevScalars *sc = nullptr;
};

static int snap(hg_handle *h, Snapshot &s, bool save)
{
  GridDev &G = h->G;
  const size_t S8 = sizeof(double) * G.S;
  if (save) {
    if (cudaMalloc(&s.p, S8 * HG_NPR) != cudaSuccess || cudaMalloc(&s.gam, S8) != cudaSuccess ||
        cudaMalloc(&s.pflag, sizeof(int) * G.S) != cudaSuccess ||
        cudaMalloc(&s.nfail, sizeof(unsigned int) * G.S * HG_NF) != cudaSuccess ||
        cudaMalloc(&s.sc, sizeof(hg::DevScalars)) != cudaSuccess) {
      cudaGetLastError();
      return HG_ERR_NOMEM;
    }
  }
  auto cp = [&](void *a, void *b, size_t n) {  // save: device -> snapshot; else snapshot -> device
    return save ? cudaMemcpyAsync(a, b, n, cudaMemcpyDeviceToDevice, h->stream)
                : cudaMemcpyAsync(b, a, n, cudaMemcpyDeviceToDevice, h->stream);
  };
  HG_CK(cp(s.p, G.p, S8 * HG_NPR));
  HG_CK(cp(s.gam, G.p_gamma, S8));
  HG_CK(cp(s.pflag, G.pflag, sizeof(int) * G.S));
  HG_CK(cp(s.nfail, G.nfail, sizeof(unsigned int) * G.S * HG_NF));
  HG_CK(cp(s.sc, G.sc, sizeof(hg::DevScalars)));
  if (!save && G.p32) hg::launch_to_f32(G, h->L.grid_upd, h->stream, G.p);  // the FP32 copy of the restored state
  if (!save && G.mdim == 3) h->levels_stale = true;  // the time levels moved on with the candidates' steps
  HG_CK(cudaGetLastError());
  HG_CK(cudaStreamSynchronize(h->stream));
  return HG_OK;
}

static void snap_free(Snapshot &s)
{
  cudaFree(s.p);
  cudaFree(s.gam);
  cudaFree(s.pflag);
  cudaFree(s.nfail);
  cudaFree(s.sc);
}

// Per-class device time of `steps` steps from the snapshot under L.
static int trial(hg_handle *h, Snapshot &s, int steps, double ms[HG_NKCLASS])
{
  int rc = snap(h, s, false);
  if (rc != HG_OK) return rc;
  const bool prof = h->prof;
  h->prof = true;
  for (int c = 0; c < HG_NKCLASS; c++) {
    h->kc_ms[c] = 0.;
    h->kc_n[c] = 0;
  }
  rc = hg_step(h, steps, nullptr, nullptr);
  h->prof = prof;
  for (int c = 0; c < HG_NKCLASS; c++) ms[c] = h->kc_ms[c];
  return rc;
}

extern "C" int hg_autotune(hg_handle *h, int32_t steps, hg_launch_config *best, double *ms_before, double *ms_after)
{
  if (!h || steps < 1) return HG_ERR_BADARG;
  if (!h->have_geom || !h->have_cells || !h->have_prims || (h->G.cooling && !h->have_cool)) return HG_ERR_STATE;
  HG_CK(cudaSetDevice(h->d.device));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->d.device);
  GridDev &G = h->G;
  const long faces = (long)G.T[0] * G.T[1] * G.T[2];
  auto grid_for = [&](long work, int per_sm) {
    long g = (work + 127) / 128, cap = (long)sms * per_sm;
    g = g > cap ? cap : g;
    g = g > HG_BLK_CAP ? HG_BLK_CAP : g;
    return (int)(g < 1 ? 1 : g);
  };
  const double sv_ms[HG_NKCLASS] = {0};
  double sv_kc[HG_NKCLASS];
  long long sv_kn[HG_NKCLASS];
  memcpy(sv_kc, h->kc_ms, sizeof(sv_kc));
  memcpy(sv_kn, h->kc_n, sizeof(sv_kn));
  (void)sv_ms;
  Snapshot s;
  int rc = snap(h, s, true);
  if (rc != HG_OK) {
    snap_free(s);
    return rc;
  }
  const hg::LaunchCfg start = h->L;
  double ms[HG_NKCLASS];
  auto total = [&](const double *m) {
    double t = 0.;
    for (int c = 0; c < HG_NKCLASS; c++) t += m[c];
    return t;
  };
  rc = trial(h, s, steps, ms);  // first run pays one-time costs
  if (rc == HG_OK) rc = trial(h, s, steps, ms);
  const double t0 = total(ms);
  hg::LaunchCfg L = start;
  // one kernel class at a time, every candidate from the same state
  const int mults[8] = {2, 4, 8, 16, 32, 64, 128, 1 << 20};  // blocks per SM; the last: one item per thread
  auto pick = [&](int cls, auto apply) {
    double bt = 1e300;
    hg::LaunchCfg bl = L;
    for (int a = 0; a < 8 && rc == HG_OK; a++)
      for (int nf = 1; nf <= 6 && rc == HG_OK; nf++) {  // nf 4..6: strips of nf-3 faces, x1 in strips
        hg::LaunchCfg c = L;
        if (!apply(c, mults[a], nf)) continue;
        h->L = c;
        rc = trial(h, s, steps, ms);
        if (rc == HG_OK && ms[cls] < bt) {
          bt = ms[cls];
          bl = c;
        }
      }
    L = bl;
  };
  pick(hg::KC_FLUX, [&](hg::LaunchCfg &c, int m, int nf) {
    c.grid_flux = grid_for(faces, m);
    c.grid_flux32 = grid_for(faces, m + m / 2);
    c.strip_nf = nf > 3 ? nf - 3 : nf;
    c.strip_x1 = nf > 3;
    return true;
  });
  pick(hg::KC_EMF, [&](hg::LaunchCfg &c, int m, int nf) {
    c.grid_emf = grid_for(faces, m);
    return nf == 1;
  });
  pick(hg::KC_UPDATE, [&](hg::LaunchCfg &c, int m, int nf) {
    c.grid_upd = grid_for(G.capacity, m);
    return nf == 1;
  });
  pick(hg::KC_FALLBACK, [&](hg::LaunchCfg &c, int m, int nf) {
    c.grid_fix = grid_for(G.capacity, m / 2);
    return nf == 1;
  });
  pick(hg::KC_BOUNDS, [&](hg::LaunchCfg &c, int m, int nf) {
    c.grid_bnd = grid_for(faces - G.capacity, m);
    return nf == 1;
  });
  double t1 = t0;
  if (rc == HG_OK) {
    h->L = L;
    rc = trial(h, s, steps, ms);
    t1 = total(ms);
    if (rc == HG_OK && t1 > t0) {  // keep the starting configuration if nothing beat it
      h->L = start;
      t1 = t0;
    }
  } else {
    h->L = start;
  }
  const int rc2 = snap(h, s, false);
  snap_free(s);
  memcpy(h->kc_ms, sv_kc, sizeof(sv_kc));
  memcpy(h->kc_n, sv_kn, sizeof(sv_kn));
  h->graph_dirty = true;
  if (rc != HG_OK) return rc;
  if (rc2 != HG_OK) return rc2;
  if (best) hg_get_launch_config(h, best);
  if (ms_before) *ms_before = t0 / steps;
  if (ms_after) *ms_after = t1 / steps;
  return HG_OK;
}

// ===========================================================================
// restart_write() / restart_read() of the reference (restart.c:22-94,
// 205-248): the ASCII rdump file of the resident state.  Header: t, N1, N2,
// N3, GridLength[0], nstep, gam, cour, N_out[N_OUT_TYPES], rdump_cnt, dx[0]
// ("%28.18e " for doubles, "%14d " for integers), a newline, then the
// primitives of the physical zones in DUMP_LOOP order (i, j, k), eight
// "%28.18e " fields and a newline per zone.  19 significant digits: every
// double reads back exactly.  The download lands in host memory once; the
// text of consecutive blocks of zones is formatted on HG_XCH_THREADS host
// threads and written in order.
// ===========================================================================
extern "C" int hg_write_rdump(hg_handle *h, const char *path, int32_t nstep, const int32_t n_out[HG_N_OUT_TYPES],
                              int32_t rdump_cnt)
{
  if (!h || !path || !n_out) return HG_ERR_BADARG;
  if (!h->have_prims) return HG_ERR_STATE;
  std::vector<double> p((size_t)h->ntot_ref * HG_NPR);
  int rc = hg_download_prims(h, p.data());
  if (rc != HG_OK) return rc;
  hg::DevScalars sc;
  HG_CK(copy_sync(h, &sc, h->G.sc, sizeof(sc), cudaMemcpyDeviceToHost));
  FILE *fp = fopen(path, "wt");
  if (!fp) return HG_ERR_BADARG;
  fprintf(fp, "%28.18e ", sc.t);
  fprintf(fp, "%14d ", h->d.n1);
  fprintf(fp, "%14d ", h->d.n2);
  fprintf(fp, "%14d ", h->d.n3);
  fprintf(fp, "%28.18e ", h->d.grid_length[0]);
  fprintf(fp, "%14d ", nstep);
  fprintf(fp, "%28.18e ", h->d.gam);
  fprintf(fp, "%28.18e ", h->d.cour);
  for (int i = 0; i < HG_N_OUT_TYPES; i++) fprintf(fp, "%14d ", n_out[i]);
  fprintf(fp, "%14d ", rdump_cnt);
  fprintf(fp, "%28.18e ", sc.dt);
  fprintf(fp, "\n");
  const long n1 = h->d.n1, n2 = h->d.n2, n3 = h->d.n3, zones = n1 * n2 * n3;
  const int N2T = h->NT[1], N3T = h->NT[2];
  const long per = 1 << 15;  // zones per formatting task
  const int nth = HG_XCH_THREADS;
  std::vector<std::string> buf(nth);
  bool ok = true;
  for (long z0 = 0; z0 < zones && ok; z0 += per * nth) {
    std::vector<std::thread> th;
    for (int w = 0; w < nth; w++) {
      const long a = z0 + w * per, b = std::min(zones, a + per);
      buf[w].clear();
      if (a >= b) continue;
      auto job = [&, w, a, b] {
        std::string &o = buf[w];
        o.reserve((size_t)(b - a) * (HG_NPR * 29 + 1));
        char line[HG_NPR * 40 + 2];
        for (long z = a; z < b; z++) {
          const long i = z / (n2 * n3) + HG_NG, j = (z / n3) % n2 + HG_NG, k = z % n3 + HG_NG;
          const double *v = p.data() + ((i * N2T + j) * N3T + k) * HG_NPR;
          int len = 0;
          for (int l = 0; l < HG_NPR; l++) len += snprintf(line + len, sizeof(line) - len, "%28.18e ", v[l]);
          line[len++] = '\n';
          o.append(line, len);
        }
      };
      try {
        th.emplace_back(job);
      } catch (...) {
        job();
      }
    }
    for (auto &t : th) t.join();
    for (int w = 0; w < nth && ok; w++)
      if (!buf[w].empty() && fwrite(buf[w].data(), 1, buf[w].size(), fp) != buf[w].size()) ok = false;
  }
  if (fclose(fp) != 0) ok = false;
  return ok ? HG_OK : HG_ERR_BADARG;
}

extern "C" int hg_read_rdump(hg_handle *h, const char *path, int32_t *nstep, int32_t n_out[HG_N_OUT_TYPES],
                             int32_t *rdump_cnt)
{
  if (!h || !path) return HG_ERR_BADARG;
  FILE *fp = fopen(path, "rt");
  if (!fp) return HG_ERR_BADARG;
  double t, gl0, gam, cour, dt;
  int n1, n2, n3, ns, rc_ = 0, no[HG_N_OUT_TYPES];
  bool ok = fscanf(fp, "%lf %d %d %d %lf %d %lf %lf", &t, &n1, &n2, &n3, &gl0, &ns, &gam, &cour) == 8;
  for (int i = 0; i < HG_N_OUT_TYPES && ok; i++) ok = fscanf(fp, "%d", &no[i]) == 1;
  ok = ok && fscanf(fp, "%d %lf", &rc_, &dt) == 2;
  if (!ok || n1 != h->d.n1 || n2 != h->d.n2 || n3 != h->d.n3) {
    fclose(fp);
    return HG_ERR_BADARG;
  }
  // the body: parse the rest of the file in parallel, one zone per line
  const long here = ftell(fp);
  fseek(fp, 0, SEEK_END);
  const long end = ftell(fp);
  fseek(fp, here, SEEK_SET);
  std::string text((size_t)(end - here), '\0');
  ok = fread(&text[0], 1, text.size(), fp) == text.size();
  fclose(fp);
  if (!ok) return HG_ERR_BADARG;
  const long n1l = n1, n2l = n2, n3l = n3, zones = n1l * n2l * n3l;
  std::vector<long> starts;  // offset of each zone's line
  starts.reserve(zones + 1);
  size_t pos = text.find('\n');
  while (pos != std::string::npos && (long)starts.size() < zones) {
    starts.push_back((long)pos + 1);
    pos = text.find('\n', pos + 1);
  }
  if ((long)starts.size() < zones) return HG_ERR_BADARG;
  std::vector<double> p((size_t)h->ntot_ref * HG_NPR, 0.);
  const int N2T = h->NT[1], N3T = h->NT[2];
  const int nth = HG_XCH_THREADS;
  std::vector<int> bad(nth, 0);
  std::vector<std::thread> th;
  for (int w = 0; w < nth; w++) {
    auto job = [&, w] {
      for (long z = w; z < zones; z += nth) {
        const char *c = text.c_str() + starts[z];
        const long i = z / (n2l * n3l) + HG_NG, j = (z / n3l) % n2l + HG_NG, k = z % n3l + HG_NG;
        double *v = p.data() + ((i * N2T + j) * N3T + k) * HG_NPR;
        for (int l = 0; l < HG_NPR; l++) {
          char *e;
          v[l] = strtod(c, &e);
          if (e == c) bad[w] = 1;
          c = e;
        }
      }
    };
    try {
      th.emplace_back(job);
    } catch (...) {
      job();
    }
  }
  for (auto &t2 : th) t2.join();
  for (int b : bad)
    if (b) return HG_ERR_BADARG;
  // ghost zones are filled by the boundaries, as after restart_init()
  int rc = hg_upload_prims(h, p.data());
  if (rc == HG_OK) rc = hg_set_time(h, t, dt);
  if (rc == HG_OK) {
    h->G.grid_length[0] = gl0;
    h->d.grid_length[0] = gl0;
    h->graph_dirty = true;
    hg::launch_bounds_only(h->G, h->L, h->stream);
    HG_CK(cudaGetLastError());
    HG_CK(cudaStreamSynchronize(h->stream));
  }
  if (rc != HG_OK) return rc;
  if (nstep) *nstep = ns;
  if (n_out)
    for (int i = 0; i < HG_N_OUT_TYPES; i++) n_out[i] = no[i];
  if (rdump_cnt) *rdump_cnt = rc_;
  return HG_OK;
}
