// hg_mixed.cu -- the FP32 flux kernel of the mixed-precision form
// (hg_grid_desc.precision = HG_PREC_MIXED).
//
// Reconstruction (reconstruct_fast, recon.c:894-1103, with rescale_prims_r
// for RESCALE_R), the face states (get_state), the characteristic speeds
// (vchar_fast) and the HLL/LF flux (numerical_flux, step_ch.c:636-790) run
// in FP32: each substep first rounds its input primitives to an FP32 copy
// (k_to_f32), the face geometry comes from an FP32 table made once, and the
// fluxes are widened to double on store.  Everything after the
// flux -- flux-CT EMFs and the induction update, the geometric and cooling
// source terms, the conserved update, con-to-prim and the fixups -- stays in
// the FP64 kernels, so the state is FP64 and only the face fluxes carry FP32
// rounding.
//
// This file is compiled with fused multiply-add enabled (the FP64 kernels
// are not): the FP32 path is not bit-matched to the reference, and FMA is
// both faster and more accurate.
#include <cuda_runtime.h>

#include "hg_common.cuh"

namespace hg {

#ifndef HG_FLUX32_MINB
// blocks of 128 per SM for the FP32 flux kernels: 7 (72 registers, a few
// dozen bytes of spills in the strip kernels) took the mixed torus step
// from 4.18 to 4.15 ms against 6 (80 registers); 8 (64 registers) changed
// results in the shock tube, where U3 and B3 must stay exactly zero
#define HG_FLUX32_MINB 7
#endif

// The face's geometry in float: the entries get_state and vchar_fast read
// (gcov, three gcon entries, ncon^0, beta, sqrt(-g)).
struct GeomF {
  float gcov[4][4];
  float gcon00, gcon0d, gcondd;
  float ncon0, beta[3], g;
  __device__ float cov(int a, int b) const { return gcov[a][b]; }
  __device__ float con(int a, int b) const { return a == 0 ? (b == 0 ? gcon00 : gcon0d) : gcondd; }
  __device__ float nc(int) const { return ncon0; }
  __device__ float bet(int a) const { return beta[a]; }
  __device__ float det() const { return g; }
};

// metric_dim 0: the one geometry of the grid, rounded; metric_dim 2: the
// FP32 table built by hg_set_geometry (HG_GF planes, see hg_internal.h)
template <int MDIM>
__device__ __forceinline__ void geom_f32(const GridDev &G, int d, int i, int j, GeomF &f, int k = 0, int slot = 0)
{
  const int js = d + 1;
  if (MDIM == 0) {
    const Geom &g = G.g0;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) f.gcov[a][b] = (float)g.gcov[a][b];
    f.gcon00 = (float)g.gcon[0][0];
    f.gcon0d = (float)g.gcon[0][js];
    f.gcondd = (float)g.gcon[js][js];
    f.ncon0 = (float)g.ncon[0];
    f.beta[0] = (float)g.beta[0];
    f.beta[1] = (float)g.beta[1];
    f.beta[2] = (float)g.beta[2];
    f.g = (float)g.g;
  } else {
    const float *t;
    long s;
    if (MDIM == 3) {  // the level's table, written by k_geom_level
      const int L = G.sc->lev[slot];
      t = (L == 0 ? G.geomF3[0] : L == 1 ? G.geomF3[1] : G.geomF3[2]) + (long)d * G.S + off3(G, i, j, k);
      s = 3 * (long)G.S;
    } else {
      const int ii = G.deg[0] ? 0 : i, jj = G.deg[1] ? 0 : j;
      t = G.geomF + ((long)d * G.T[1] + jj) * G.T[0] + ii;
      s = G.gS;
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++) f.gcov[a][b] = __ldg(t + (a * 4 + b) * s);
    f.gcon00 = __ldg(t + 16 * s);
    f.gcon0d = __ldg(t + (16 + js) * s);
    f.gcondd = __ldg(t + (19 + js) * s);
    f.ncon0 = __ldg(t + 23 * s);
    f.beta[0] = __ldg(t + 24 * s);
    f.beta[1] = __ldg(t + 25 * s);
    f.beta[2] = __ldg(t + 26 * s);
    f.g = __ldg(t + 27 * s);
  }
}

// Left/right FP32 states of face (i,j,k) in direction d from the FP32 copy
// of the primitives; RESCALE_R scales the x1 stencil by the per-zone
// factors of rescale_prims_r and the face values back by the FACE1 factors.
template <bool RS>
__device__ __forceinline__ void face_prims_f32(const GridDev &G, int d, int i, int j, int k, float *pl, float *pr)
{
  const long o = off3(G, i, j, k);
  const float *ph = G.p32;
  if (G.deg[d]) {
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) pl[l] = pr[l] = __ldg(ph + l * G.S + o);
    return;
  }
  const int st = G.st[d];
#pragma unroll
  for (int l = 0; l < HG_NPR; l++) {
    float y[6];
    const float *b = ph + l * G.S + o - 3 * st;
#pragma unroll
    for (int m = 0; m < 6; m++) y[m] = __ldg(b + m * st);
    if (RS && d == 0) {
      const int t = rs_type(l);
#pragma unroll
      for (int m = 0; m < 6; m++) y[m] *= __ldg(G.rsc32 + t * G.T[0] + i - 3 + m);
    }
    recon_face(G.recon, y, &pl[l], &pr[l]);
    if (RS && d == 0) {
      const float f = __ldg(G.rsc32 + (9 + rs_type(l)) * G.T[0] + i);
      pl[l] *= f;
      pr[l] *= f;
    }
  }
}

// FP32 copy of the substep's input primitives (all 8 planes, ghosts included)
__global__ void __launch_bounds__(HG_BLK) k_to_f32(GridDev G, const double *__restrict__ src)
{
  const long total = (long)HG_NPR * G.S;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += stride) G.p32[t] = (float)src[t];
}

void launch_to_f32(const GridDev &G, int grid, cudaStream_t s, const double *src)
{
  k_to_f32<<<grid, HG_BLK, 0, s>>>(G, src);
}

// Stored values where the FP32 copy differs from the state rounded to float
// (hg_check_mirror): zero after every step and every host update.
// count[0]: mismatches, count[1]: the lowest mismatching offset (l * S + o).
// Compared as FP32 values in this flush-to-zero unit, as the FP32 flux
// kernels read them: a subnormal written by an FP64 kernel's conversion
// equals the zero this unit's conversion gives.
__global__ void __launch_bounds__(HG_BLK) k_mirror_check(GridDev G, const double *__restrict__ src,
                                                        unsigned long long *count)
{
  const long total = (long)HG_NPR * G.S;
  const long stride = (long)gridDim.x * blockDim.x;
  unsigned long long n = 0, first = ~0ull;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += stride)
    if (G.p32[t] != (float)src[t]) {
      n++;
      if ((unsigned long long)t < first) first = (unsigned long long)t;
    }
  if (n) {
    atomicAdd(count, n);
    atomicMin(count + 1, first);
  }
}

void launch_mirror_check(const GridDev &G, int grid, cudaStream_t s, const double *src, unsigned long long *count)
{
  k_mirror_check<<<grid, HG_BLK, 0, s>>>(G, src, count);
}

template <bool RS, int MDIM, int d>
__global__ void __launch_bounds__(HG_BLK, HG_FLUX32_MINB) k_flux_f32(const __grid_constant__ GridDev G, int lo0,
                                                                    int lo1, int lo2, int n0, int n1, int n2,
                                                                    unsigned int mult, int slot)
{
  const unsigned total = (unsigned)n0 * n1 * n2;  // < 2^31 (hg_init)
  const int dim = d + 1;
  const float gam = (float)G.gam;
  double vmax = 0.;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned tq = t / (unsigned)n0;
    const int i = lo0 + (int)(t - tq * (unsigned)n0);
    const int j = lo1 + (int)(tq % (unsigned)n1);
    const int k = lo2 + (int)(tq / (unsigned)n1);
    const long o = off3(G, i, j, k);
    float pl[HG_NPR], pr[HG_NPR];
    face_prims_f32<RS>(G, d, i, j, k, pl, pr);
    GeomF g;
    geom_f32<MDIM>(G, d, i, j, g, k, slot);
    StateT<float> ql, qr;
    if (get_state(pl, g, gam, ql)) book_face(G, i, j, k, mult);
    if (get_state(pr, g, gam, qr)) book_face(G, i, j, k, mult);
    float cmaxl, cminl, cmaxr, cminr;
    vchar_fast(ql, g, dim, gam, &cmaxl, &cminl);
    vchar_fast(qr, g, dim, gam, &cmaxr, &cminr);
    const float cmax = fabsf(fmaxf(fmaxf(0.f, cmaxl), cmaxr));
    const float cmin = fabsf(fmaxf(fmaxf(0.f, -cminl), -cminr));
    const float ctop = fmaxf(cmin, cmax);
    const float gg = g.g;
    double *Fd = G.F[d];
    if (G.flux == 1) {
      const float inv = 1.f / (cmax + cmin + (float)HG_SMALL);
      const float cc = cmax * cmin;
#pragma unroll
      for (int l = 0; l < HG_NPR; l++) {
        const float Ul = flux_comp(pl, ql, 0, gg, l), Ur = flux_comp(pr, qr, 0, gg, l);
        const float Fl = flux_comp(pl, ql, dim, gg, l), Fr = flux_comp(pr, qr, dim, gg, l);
        Fd[l * G.S + o] = (double)((cmax * Fl + cmin * Fr - cc * (Ur - Ul)) * inv);
      }
    } else {
#pragma unroll
      for (int l = 0; l < HG_NPR; l++) {
        const float Ul = flux_comp(pl, ql, 0, gg, l), Ur = flux_comp(pr, qr, 0, gg, l);
        const float Fl = flux_comp(pl, ql, dim, gg, l), Fr = flux_comp(pr, qr, dim, gg, l);
        Fd[l * G.S + o] = (double)(0.5f * (Fl + Fr - ctop * (Ur - Ul)));
      }
    }
    if (d == 0 && G.bc == 10) {  // fix_flux(), bounds.c:2263-2275
      double *fr = G.F[0] + RHO * G.S + o;
      if (i == HG_NGH && *fr > 0) *fr = 0.;
      if (i == G.NE[0] + 1 && *fr < 0) *fr = 0.;
    }
    if (i >= HG_NGH && i <= G.NE[0] && j >= HG_NGH && j <= G.NE[1] && k >= HG_NGH && k <= G.NE[2])
      if ((double)ctop > vmax) vmax = (double)ctop;
  }
  block_max_atomic(vmax, &G.sc->maxs[d + 1]);
}

// Strips of NF consecutive faces along a strided direction (x2, x3), lanes
// along x1: each zone's PPM edges are formed once per strip (the FP64
// k_flux_strip's scheme); the strip's face states wait in shared memory.

// X1 with RESCALE_R: zones scaled by their factors before, face states by
// their faces' factors after the reconstruction (FP32 copies of the tables).
template <bool RS, bool X1, int NF>
__device__ __forceinline__ void strip_recon_f32(const GridDev &G, const float *__restrict__ col, int st, int l, int i,
                                                int nf, float *sm, int bl, int br, int tx)
{
  const int rt = G.recon;
  float y[NF + 5];
#pragma unroll
  for (int c = 0; c < NF + 5; c++) {
    const int cc = c <= 4 ? c : min(c, nf + 4);  // nf >= 1: zones 0..4 always exist
    float v = __ldg(col + cc * st);
    if (RS && X1) v *= __ldg(G.rsc32 + rs_type(l) * G.T[0] + i - 3 + cc);
    y[c] = v;
  }
  float rnv[NF + 3], lnv[NF + 3];
  if (rt >= 3) {
    float q[NF + 4];
#pragma unroll
    for (int c = 1; c <= NF + 3; c++) q[c] = slope_vect(rt, y[c] - y[c - 1], y[c + 1] - y[c]);
    float I[NF + 3];
#pragma unroll
    for (int c = 1; c <= NF + 2; c++) I[c] = 0.5f * (y[c + 1] + y[c]) - float(HG_PPM_FACTOR) * (q[c + 1] - q[c]);
#pragma unroll
    for (int c = 2; c <= NF + 2; c++) para_cell(y[c], I[c - 1], I[c], &lnv[c], &rnv[c]);
  } else {
#pragma unroll
    for (int c = 2; c <= NF + 2; c++) {
      const float dq = 0.5f * linear_recon(rt, y[c - 1], y[c], y[c + 1]);
      rnv[c] = y[c] + dq;
      lnv[c] = y[c] - dq;
    }
  }
#pragma unroll
  for (int c = 2; c <= NF + 2; c++) {
    float rn = rnv[c], ln = lnv[c];
    if (RS && X1) {
      const float *f = G.rsc32 + (9 + rs_type(l)) * G.T[0] + i;
      if (c - 2 < NF) rn *= __ldg(f + (c - 2 < nf ? c - 2 : nf - 1));
      if (c - 3 >= 0) ln *= __ldg(f + (c - 3 < nf ? c - 3 : nf - 1));
    }
    if (c - 2 < NF) sm[(bl + c - 2) * HG_BLK + tx] = rn;
    if (c - 3 >= 0) sm[(br + c - 3) * HG_BLK + tx] = ln;
  }
}

// HLL/LF flux of one face from FP32 states; returns ctop
template <int MDIM, int d>
__device__ __forceinline__ float face_flux_f32(const GridDev &G, const float *pl, const float *pr, int i, int j, int k,
                                               unsigned int mult, long o, int slot)
{
  const int dim = d + 1;
  const float gam = (float)G.gam;
  GeomF g;
  geom_f32<MDIM>(G, d, i, j, g, k, slot);
  StateT<float> ql, qr;
  if (get_state(pl, g, gam, ql)) book_face(G, i, j, k, mult);
  if (get_state(pr, g, gam, qr)) book_face(G, i, j, k, mult);
  float cmaxl, cminl, cmaxr, cminr;
  vchar_fast(ql, g, dim, gam, &cmaxl, &cminl);
  vchar_fast(qr, g, dim, gam, &cmaxr, &cminr);
  const float cmax = fabsf(fmaxf(fmaxf(0.f, cmaxl), cmaxr));
  const float cmin = fabsf(fmaxf(fmaxf(0.f, -cminl), -cminr));
  const float ctop = fmaxf(cmin, cmax);
  const float gg = g.g;
  double *Fd = G.F[d];
  if (G.flux == 1) {
    const float inv = 1.f / (cmax + cmin + (float)HG_SMALL);
    const float cc = cmax * cmin;
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) {
      const float Ul = flux_comp(pl, ql, 0, gg, l), Ur = flux_comp(pr, qr, 0, gg, l);
      const float Fl = flux_comp(pl, ql, dim, gg, l), Fr = flux_comp(pr, qr, dim, gg, l);
      Fd[l * G.S + o] = (double)((cmax * Fl + cmin * Fr - cc * (Ur - Ul)) * inv);
    }
  } else {
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) {
      const float Ul = flux_comp(pl, ql, 0, gg, l), Ur = flux_comp(pr, qr, 0, gg, l);
      const float Fl = flux_comp(pl, ql, dim, gg, l), Fr = flux_comp(pr, qr, dim, gg, l);
      Fd[l * G.S + o] = (double)(0.5f * (Fl + Fr - ctop * (Ur - Ul)));
    }
  }
  return ctop;
}

template <bool RS, int MDIM, int d, int NF>
__global__ void __launch_bounds__(HG_BLK, HG_FLUX32_MINB) k_flux_strip_f32(const __grid_constant__ GridDev G, int lo0,
                                                                          int lo1, int lo2, int n0, int n1, int n2,
                                                                          unsigned int mult, int slot)
{
  __shared__ float sm[16 * NF * HG_BLK];
  const int tx = threadIdx.x;
  const int nd = (d == 0) ? n0 : (d == 1) ? n1 : n2;
  const int nseg = (nd + NF - 1) / NF;
  const unsigned total = (unsigned)nseg * (d == 0 ? n1 * n2 : d == 1 ? n0 * n2 : n0 * n1);  // < 2^31 (hg_init)
  const int st = G.st[d];
  double vmax = 0.;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int seg, i0, j0, k0;
    if (d == 0) {  // consecutive lanes on consecutive strips of a line
      const unsigned rest = t / (unsigned)nseg;
      seg = (int)(t - rest * (unsigned)nseg);
      i0 = lo0 + seg * NF;
      j0 = lo1 + (int)(rest % (unsigned)n1);
      k0 = lo2 + (int)(rest / (unsigned)n1);
    } else {  // lanes along x1
      const unsigned rest = t / (unsigned)n0;
      i0 = lo0 + (int)(t - rest * (unsigned)n0);
      const unsigned other = rest / (unsigned)nseg;
      seg = (int)(rest - other * (unsigned)nseg);
      j0 = (d == 1) ? lo1 + seg * NF : lo1 + other;
      k0 = (d == 1) ? lo2 + other : lo2 + seg * NF;
    }
    const int nf = min(NF, nd - seg * NF);
    const long o0 = off3(G, i0, j0, k0);
#pragma unroll 1  // one copy of the reconstruction code: the kernel fits the instruction cache
    for (int l = 0; l < HG_NPR; l++)
      strip_recon_f32<RS, d == 0, NF>(G, G.p32 + l * G.S + o0 - 3 * st, st, l, i0, nf, sm, 2 * NF * l,
                                      2 * NF * l + NF, tx);
    for (int s = 0; s < nf; s++) {
      const int i = (d == 0) ? i0 + s : i0;
      const int j = (d == 1) ? j0 + s : j0, k = (d == 2) ? k0 + s : k0;
      float pl[HG_NPR], pr[HG_NPR];
#pragma unroll
      for (int l = 0; l < HG_NPR; l++) {
        pl[l] = sm[(2 * NF * l + s) * HG_BLK + tx];
        pr[l] = sm[(2 * NF * l + NF + s) * HG_BLK + tx];
      }
      const long o = o0 + s * st;
      const float ctop = face_flux_f32<MDIM, d>(G, pl, pr, i, j, k, mult, o, slot);
      if (d == 0 && G.bc == 10) {  // fix_flux(), bounds.c:2263-2275
        double *fr = G.F[0] + RHO * G.S + o;
        if (i == HG_NGH && *fr > 0) *fr = 0.;
        if (i == G.NE[0] + 1 && *fr < 0) *fr = 0.;
      }
      if (i >= HG_NGH && i <= G.NE[0] && j >= HG_NGH && j <= G.NE[1] && k >= HG_NGH && k <= G.NE[2])
        if ((double)ctop > vmax) vmax = (double)ctop;
    }
  }
  block_max_atomic(vmax, &G.sc->maxs[d + 1]);
}

template <bool RS, int MDIM, int d>
static void launch_strip32(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const int *lo, const int *n,
                           unsigned int mult, int slot)
{
#define HG_S32N(NF) \
  k_flux_strip_f32<RS, MDIM, d, NF><<<L.grid_flux32, HG_BLK, 0, s>>>(G, lo[0], lo[1], lo[2], n[0], n[1], n[2], mult, \
                                                                     slot)
  if (L.strip_nf <= 1) HG_S32N(1);
  else if (L.strip_nf == 2) HG_S32N(2);
  else HG_S32N(3);
#undef HG_S32N
}

void launch_flux_f32(const GridDev &G, const LaunchCfg &L, cudaStream_t s, int d, const int *lo, const int *n,
                     unsigned int mult, int slot)
{
  const int grid = L.grid_flux32;
#define HG_F32(RSV, MD, DD) \
  k_flux_f32<RSV, MD, DD><<<grid, HG_BLK, 0, s>>>(G, lo[0], lo[1], lo[2], n[0], n[1], n[2], mult, slot)
#define HG_F32_D(RSV, MD) \
  if (d == 0) { if (G.deg[0] || !L.strip_x1) HG_F32(RSV, MD, 0); else launch_strip32<RSV, MD, 0>(G, L, s, lo, n, mult, slot); } \
  else if (d == 1) { if (G.deg[1]) HG_F32(RSV, MD, 1); else launch_strip32<RSV, MD, 1>(G, L, s, lo, n, mult, slot); } \
  else { if (G.deg[2]) HG_F32(RSV, MD, 2); else launch_strip32<RSV, MD, 2>(G, L, s, lo, n, mult, slot); }
  if (G.mdim == 0) {
    if (G.rescale) { HG_F32_D(true, 0) }
    else { HG_F32_D(false, 0) }
  } else if (G.mdim == 3) {
    if (G.rescale) { HG_F32_D(true, 3) }
    else { HG_F32_D(false, 3) }
  } else {
    if (G.rescale) { HG_F32_D(true, 2) }
    else { HG_F32_D(false, 2) }
  }
#undef HG_F32_D
#undef HG_F32
}

}  // namespace hg
