// hg_kernels.cu -- sm_100a kernels of one HARM3D time step (step_ch.c:50-234).
//
// Per substep (predictor with Dt/2, corrector with Dt):
//   k_begin     reset the substep's reductions and failure flags
//   k_flux x3   one kernel per direction: reconstruction of the six-zone
//               stencil of each face (reconstruct_fast, recon.c:894-1103)
//               fused with get_state/primtoflux/vchar_fast and the HLL or LF
//               flux (numerical_flux, step_ch.c:636-790); the maximum
//               characteristic speed is reduced per block into one atomic
//   k_emf       corner EMFs of flux_ct_para_fast2 / flux_ct (flux_ct.c)
//   k_update_cons  conserved update with the geometric source and the CT
//               corrected induction fluxes (advance, step_ch.c:312-370)
//   k_update_c2p   the 2D Newton inversion (step_ch.c:371-399); zones that
//               need the rest of the recover_primitives() tree are queued
//   k_fallback  Utoprim_1d / entropy fix / floors for the queued zones
//   k_bounds    ghost zones (bounds.c) and pflag ghosts
//   k_fixup     fixup_interp_v / fixup_interp_prim over the flagged zones
//   k_bounds    again if a flagged zone touched a physical boundary
// then k_timestep (timestep(), step_ch.c:546-623) on one block.
// All loops are grid-stride loops over a fixed grid so that reductions are
// per block and deterministic.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "harmgpu.h"
#include "hg_common.cuh"
#include "hg_dyn.cuh"
#include "hg_fallback.cuh"

// This file is compiled twice.  Plain: into namespace hg with no multiply-add
// contracted (-fmad=false), every FP64 operation rounded as in the
// reference's build (HG_PREC_FP64, bit-identical results).  With HG_FMA_BUILD
// and -fmad=true: the same kernels and launch sequence into namespace hg_fma,
// where the compiler fuses multiply-adds (HG_PREC_FP64_FMA: fewer FP64
// instructions, results within rounding of the plain form).  Types and the
// device functions of the headers are shared through namespace hg.
#ifdef HG_FMA_BUILD
#define HG_KNS hg_fma
#else
#define HG_KNS hg
#endif

namespace hg {
// the FP32 flux kernels of the mixed form (hg_mixed.cu)
void launch_flux_f32(const GridDev &G, const LaunchCfg &L, cudaStream_t s, int d, const int *lo, const int *n,
                     unsigned int mult, int slot);
void launch_to_f32(const GridDev &G, int grid, cudaStream_t s, const double *src);
}  // namespace hg

namespace HG_KNS {
using namespace hg;

// register caps (minimum resident blocks of 128 threads per SM), measured on
// the 192x192x128 torus: the flux kernels at 3 blocks (168 registers, no
// spills; at 4 blocks, 128 registers, they spilled ~3e6 local-load sectors
// per launch: 6.36 against 6.70 ms per step); the corrector's conserved
// update at 3 blocks (168 registers; 4 blocks spill 264 bytes), the
// predictor's at 4 (128 registers without spills); the inversion at 5 (96
// registers, 112 bytes of spill stores) -- those two: 6.31 -> 6.24 ms per
// step, the mixed form 4.25 -> 4.16
#ifndef HG_CONS_MINB
#define HG_CONS_MINB 3
#endif
#ifndef HG_CONS0_MINB
#define HG_CONS0_MINB 4
#endif
#ifndef HG_C2P_MINB
#define HG_C2P_MINB 5
#endif
#ifndef HG_FLUX_MINB
#define HG_FLUX_MINB 3
#endif
#ifndef HG_EE_MINB
#define HG_EE_MINB 4
#endif

// (x * rscale) * (1/rscale): the value rescale_prims_r() leaves in p_h after
// it scaled and unscaled it around the x1 reconstruction (recon.c:1168-1200).
__device__ __forceinline__ double rs_roundtrip(const GridDev &G, double x, int l, int i)
{
  const int t = rs_type(l);
  return (x * G.rsc[t * G.T[0] + i]) * G.rsc[(6 + t) * G.T[0] + i];
}

__device__ __forceinline__ double block_sum(double v)
{
  __shared__ double red[HG_BLK / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.;
  if (threadIdx.x == 0)
    for (int w = 0; w < HG_BLK / 32; w++) s += red[w];
  __syncthreads();
  return s;
}

__device__ __forceinline__ unsigned int block_count(unsigned int v)
{
  __shared__ unsigned int red[HG_BLK / 32];
  v = __reduce_add_sync(0xffffffffu, v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  unsigned int s = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < HG_BLK / 32; w++) s += red[w];
  __syncthreads();
  return s;
}

// fail() bookkeeping (diag.c:159-330) for the rare branches: per-zone nfail
// counter and the global total, both atomic.
__device__ __forceinline__ void book(const GridDev &G, int nf, int i, int j, int k)
{
  atomicAdd(&G.nfail[nf * G.S + off3(G, i, j, k)], 1u);
  atomicAdd(&G.sc->nfailtot[nf], 1ull);
}

// fail(type, state != 0): pflag, failure flags, boundary flag
// (check_boundary_pflag, harm_mpi.c:1388-1426) and the interpolation list.
__device__ __forceinline__ void flag_zone(const GridDev &G, int pf, int i, int j, int k)
{
  G.pflag[off3(G, i, j, k)] = pf;
  G.sc->failure_exists = 1;
  G.sc->ftype[pf] = 1;
  const int n0 = G.N[0] + HG_NGH - 1, n1 = G.N[1] + HG_NGH - 1, n2 = G.N[2] + HG_NGH - 1;
  if (i < 2 * HG_NGH || i > n0 - HG_NGH || j < 2 * HG_NGH || j > n1 - HG_NGH || k < 2 * HG_NGH || k > n2 - HG_NGH)
    G.sc->bnd_phys = 1;
  const int slot = atomicAdd(&G.sc->fl_count, 1);
  if (slot < G.capacity) G.fl_idx[slot] = pack_ijk(i, j, k);
  else G.sc->err = 1;
}

// Left/right primitive states of face (i,j,k) in direction d (p_L[i][j][k][d],
// p_R[i][j][k][d] of reconstruct_fast).
template <bool RS>
__device__ __forceinline__ void face_prims(const GridDev &G, const double *__restrict__ ph, int d, int i, int j,
                                           int k, double *pl, double *pr)
{
  const long o = off3(G, i, j, k);
  if (G.deg[d]) {
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) {
      double v = __ldg(ph + l * G.S + o);
      if (RS) v = rs_roundtrip(G, v, l, i);
      pl[l] = pr[l] = v;
    }
    return;
  }
  const int st = G.st[d];
#pragma unroll
  for (int l = 0; l < HG_NPR; l++) {
    double y[6];
    const double *b = ph + l * G.S + o - 3 * st;
#pragma unroll
    for (int m = 0; m < 6; m++) y[m] = __ldg(b + m * st);
    if (RS) {
      const int t = rs_type(l);
      if (d == 0) {
#pragma unroll
        for (int m = 0; m < 6; m++) y[m] *= G.rsc[t * G.T[0] + i - 3 + m];
      } else {
#pragma unroll
        for (int m = 0; m < 6; m++) y[m] = rs_roundtrip(G, y[m], l, i);
      }
    }
    recon_face(G.recon, y, &pl[l], &pr[l]);
    if (RS && d == 0) {
      const double f = G.rsc[(9 + rs_type(l)) * G.T[0] + i];
      pl[l] *= f;
      pr[l] *= f;
    }
  }
}

// ---------------------------------------------------------------------------
// k_flux: F[d] on faces [lo, lo+n) (reference indices).
// HLL/LF flux of a face from its two states; writes the 8 components and
// returns ctop.  Component by component, so no 32-value temporaries.
__device__ __forceinline__ double face_flux(const GridDev &G, const double *pl, const double *pr, const Geom &g, int d,
                                            int i, int j, int k, unsigned int mult, double *__restrict__ Fd, long o)
{
  const int dim = d + 1;
  State ql, qr;
  if (get_state(pl, g, G.gam, ql)) book_face(G, i, j, k, mult);
  if (get_state(pr, g, G.gam, qr)) book_face(G, i, j, k, mult);
  double cmaxl, cminl, cmaxr, cminr;
  vchar_fast(ql, g, dim, G.gam, &cmaxl, &cminl);
  vchar_fast(qr, g, dim, G.gam, &cmaxr, &cminr);
  const double a0 = 0. > cmaxl ? 0. : cmaxl;
  const double cmax = fabs(a0 > cmaxr ? a0 : cmaxr);
  const double a1 = 0. > -cminl ? 0. : -cminl;
  const double cmin = fabs(a1 > -cminr ? a1 : -cminr);
  const double ctop = cmin > cmax ? cmin : cmax;
  const double gg = g.g;
  if (G.flux == 1) {
    const double den = cmax + cmin + HG_SMALL;
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) {
      const double Ul = flux_comp(pl, ql, 0, gg, l), Ur = flux_comp(pr, qr, 0, gg, l);
      const double Fl = flux_comp(pl, ql, dim, gg, l), Fr = flux_comp(pr, qr, dim, gg, l);
      Fd[l * G.S + o] = (cmax * Fl + cmin * Fr - cmax * cmin * (Ur - Ul)) / den;
    }
  } else {
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) {
      const double Ul = flux_comp(pl, ql, 0, gg, l), Ur = flux_comp(pr, qr, 0, gg, l);
      const double Fl = flux_comp(pl, ql, dim, gg, l), Fr = flux_comp(pr, qr, dim, gg, l);
      Fd[l * G.S + o] = 0.5 * (Fl + Fr - ctop * (Ur - Ul));
    }
  }
  return ctop;
}

// ---------------------------------------------------------------------------
// k_flux: F[d] on faces [lo, lo+n) (reference indices), one thread per face.
template <bool RS, int MDIM, int d>
__global__ void __launch_bounds__(HG_BLK, HG_FLUX_MINB) k_flux(const __grid_constant__ GridDev G, const double *__restrict__ ph,
                                                 int lo0, int lo1, int lo2, int n0, int n1, int n2, unsigned int mult,
                                                 int slot)
{
  const unsigned total = (unsigned)n0 * n1 * n2;  // < 2^31 (hg_init)
  double vmax = 0.;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned tq = t / (unsigned)n0;
    const int i = lo0 + (int)(t - tq * (unsigned)n0);
    const int j = lo1 + (int)(tq % (unsigned)n1);
    const int k = lo2 + (int)(tq / (unsigned)n1);
    double pl[HG_NPR], pr[HG_NPR];
    face_prims<RS>(G, ph, d, i, j, k, pl, pr);
    double ctop;
    const long o = off3(G, i, j, k);
    if (MDIM == 0) {
      ctop = face_flux(G, pl, pr, G.g0, d, i, j, k, mult, G.F[d], o);
    } else {
      Geom g;
      load_geom(G, d, i, j, g, k, slot);
      ctop = face_flux(G, pl, pr, g, d, i, j, k, mult, G.F[d], o);
    }
    if (d == 0 && G.bc == 10) {  // fix_flux(), bounds.c:2263-2275: no mass inflow through r_in, r_out
      double *fr = G.F[0] + RHO * G.S + o;
      if (i == HG_NGH && *fr > 0) *fr = 0.;
      if (i == G.NE[0] + 1 && *fr < 0) *fr = 0.;
    }
    if (i >= HG_NGH && i <= G.NE[0] && j >= HG_NGH && j <= G.NE[1] && k >= HG_NGH && k <= G.NE[2])
      if (ctop > vmax) vmax = ctop;
  }
  block_max_atomic(vmax, &G.sc->maxs[d + 1]);
}

// ---------------------------------------------------------------------------
// k_flux_strip: the faces of a strided direction d (x2 or x3) in strips of
// NF consecutive faces along d, one strip per thread, lanes along x1.  The
// thread marches along its strip once per variable, so each zone's slope,
// interface value and PPM edges are computed once per strip instead of once
// for each of the faces that read them (reconstruct_fast computes them once
// per zone as well).  The face states wait in shared memory, each thread in
// its own column, until the strip's fluxes are formed.  Every face value is
// produced by the same operations on the same inputs as in face_prims.
#ifndef HG_STRIP_NF
#define HG_STRIP_NF 2
#endif

// Face states of NF faces f0 .. f0+NF-1 along d from zones f0-3 .. f0+NF+1
// of one variable; zones past the strip's nf faces are clamped (their
// results are not used).  pl -> sm[bl + s], pr -> sm[br + s].
// X1: a strip along x1, where RESCALE_R scales each zone by its own factor
// before the reconstruction and each face state by its face's factor after
// it (face_prims<RS>, d = 0); along x2, x3 every value takes the
// scale/unscale round trip of its zone i.
template <bool RS, bool X1, int NF>
__device__ __forceinline__ void strip_recon(const GridDev &G, const double *__restrict__ col, int st, int l, int i,
                                            int nf, double *sm, int bl, int br, int tx)
{
  const int rt = G.recon;
  double y[NF + 5];
#pragma unroll
  for (int c = 0; c < NF + 5; c++) {
    const int cc = c <= 4 ? c : min(c, nf + 4);  // nf >= 1: zones 0..4 always exist
    double v = __ldg(col + cc * st);
    if (RS && !X1) v = rs_roundtrip(G, v, l, i);
    if (RS && X1) v *= G.rsc[rs_type(l) * G.T[0] + i - 3 + cc];
    y[c] = v;
  }
  if (rt >= 3) {
    double q[NF + 4];  // q[c]: slope of zone c, c = 1 .. NF+3
#pragma unroll
    for (int c = 1; c <= NF + 3; c++) q[c] = slope_vect(rt, y[c] - y[c - 1], y[c + 1] - y[c]);
    double I[NF + 3];  // I[c]: value at the interface of zones c and c+1, c = 1 .. NF+2
#pragma unroll
    for (int c = 1; c <= NF + 2; c++) I[c] = 0.5 * (y[c + 1] + y[c]) - HG_PPM_FACTOR * (q[c + 1] - q[c]);
    // zones c = 2 .. NF+2: face s = c - 2 takes the right edge of zone c
    // (its left state), face s = c - 3 the left edge (its right state)
#pragma unroll
    for (int c = 2; c <= NF + 2; c++) {
      double ln, rn;
      para_cell(y[c], I[c - 1], I[c], &ln, &rn);
      if (RS && X1) {  // the FACE1 factors of the faces these edges belong to
        const int t9 = (9 + rs_type(l)) * G.T[0] + i;
        if (c - 2 < NF) rn *= G.rsc[t9 + (c - 2 < nf ? c - 2 : nf - 1)];
        if (c - 3 >= 0) ln *= G.rsc[t9 + (c - 3 < nf ? c - 3 : nf - 1)];
      }
      if (c - 2 < NF) sm[(bl + c - 2) * HG_BLK + tx] = rn;
      if (c - 3 >= 0) sm[(br + c - 3) * HG_BLK + tx] = ln;
    }
  } else {
#pragma unroll
    for (int c = 2; c <= NF + 2; c++) {
      const double dq = 0.5 * linear_recon(rt, y[c - 1], y[c], y[c + 1]);
      double rn = y[c] + dq, ln = y[c] - dq;
      if (RS && X1) {
        const int t9 = (9 + rs_type(l)) * G.T[0] + i;
        if (c - 2 < NF) rn *= G.rsc[t9 + (c - 2 < nf ? c - 2 : nf - 1)];
        if (c - 3 >= 0) ln *= G.rsc[t9 + (c - 3 < nf ? c - 3 : nf - 1)];
      }
      if (c - 2 < NF) sm[(bl + c - 2) * HG_BLK + tx] = rn;
      if (c - 3 >= 0) sm[(br + c - 3) * HG_BLK + tx] = ln;
    }
  }
}

template <bool RS, int MDIM, int d, int NF>
__global__ void __launch_bounds__(HG_BLK, HG_FLUX_MINB) k_flux_strip(const __grid_constant__ GridDev G,
                                                                   const double *__restrict__ ph, int lo0, int lo1,
                                                                   int lo2, int n0, int n1, int n2, unsigned int mult,
                                                                   int slot)
{
  extern __shared__ double sm[];  // 16 * NF * HG_BLK doubles: the strip's face states
  const int tx = threadIdx.x;
  // x2, x3: lanes along x1, one strip per thread along d; x1: consecutive
  // lanes take consecutive strips of the same line
  const int nd = (d == 0) ? n0 : (d == 1) ? n1 : n2;
  const int nseg = (nd + NF - 1) / NF;
  const unsigned total = (unsigned)nseg * (d == 0 ? n1 * n2 : d == 1 ? n0 * n2 : n0 * n1);  // < 2^31 (hg_init)
  const int st = G.st[d];
  double vmax = 0.;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int seg, i0, j0, k0;
    if (d == 0) {
      const unsigned rest = t / (unsigned)nseg;
      seg = (int)(t - rest * (unsigned)nseg);
      i0 = lo0 + seg * NF;
      j0 = lo1 + (int)(rest % (unsigned)n1);
      k0 = lo2 + (int)(rest / (unsigned)n1);
    } else {
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
      strip_recon<RS, d == 0, NF>(G, ph + l * G.S + o0 - 3 * st, st, l, i0, nf, sm, 2 * NF * l, 2 * NF * l + NF, tx);
    for (int s = 0; s < nf; s++) {
      const int i = (d == 0) ? i0 + s : i0;
      const int j = (d == 1) ? j0 + s : j0, k = (d == 2) ? k0 + s : k0;
      double pl[HG_NPR], pr[HG_NPR];
#pragma unroll
      for (int l = 0; l < HG_NPR; l++) {
        pl[l] = sm[(2 * NF * l + s) * HG_BLK + tx];
        pr[l] = sm[(2 * NF * l + NF + s) * HG_BLK + tx];
      }
      const long o = o0 + s * st;
      double ctop;
      if (MDIM == 0) {
        ctop = face_flux(G, pl, pr, G.g0, d, i, j, k, mult, G.F[d], o);
      } else {
        Geom g;
        load_geom(G, d, i, j, g, k, slot);  // metric_dim 3: time level `slot`
        ctop = face_flux(G, pl, pr, g, d, i, j, k, mult, G.F[d], o);
      }
      if (d == 0 && G.bc == 10) {  // fix_flux(), bounds.c:2263-2275: no mass inflow through r_in, r_out
        double *fr = G.F[0] + RHO * G.S + o;
        if (i == HG_NGH && *fr > 0) *fr = 0.;
        if (i == G.NE[0] + 1 && *fr < 0) *fr = 0.;
      }
      if (i >= HG_NGH && i <= G.NE[0] && j >= HG_NGH && j <= G.NE[1] && k >= HG_NGH && k <= G.NE[2])
        if (ctop > vmax) vmax = ctop;
    }
  }
  block_max_atomic(vmax, &G.sc->maxs[d + 1]);
}

// ---------------------------------------------------------------------------
// k_emf: corner EMFs at [lo, lo+n).
// Right edge of zone c-1 and left edge of zone c on a line through the corner
// (flux_ct.c:782-900 accumulate exactly these two into each corner).
__device__ __forceinline__ void line_edges(const GridDev &G, const double *__restrict__ f, long o, int a, double *rprev,
                                           double *lcur)
{
  if (G.deg[a]) {
    *rprev = *lcur = __ldg(f + o);
    return;
  }
  const int st = G.st[a];
  double y[6];
#pragma unroll
  for (int m = 0; m < 6; m++) y[m] = __ldg(f + o + (m - 3) * st);
  ppm_face(G.recon, y, rprev, lcur);
}

__global__ void __launch_bounds__(HG_BLK) k_emf(GridDev G, int lo0, int lo1, int lo2, int n0, int n1, int n2)
{
  const unsigned total = (unsigned)n0 * n1 * n2;  // < 2^31 (hg_init)
  const double *F0 = G.F[0], *F1 = G.F[1], *F2 = G.F[2];
  const long S = G.S;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned tq = t / (unsigned)n0;
    const int i = lo0 + (int)(t - tq * (unsigned)n0);
    const int j = lo1 + (int)(tq % (unsigned)n1);
    const int k = lo2 + (int)(tq / (unsigned)n1);
    const long o = off3(G, i, j, k);
    double e0, e1, e2;
    if (G.ct_para) {
      double r, l, r2, l2;
      line_edges(G, F1 + B3 * S, o, 2, &r, &l);
      line_edges(G, F2 + B2 * S, o, 1, &r2, &l2);
      e0 = (((0. + r) + l) - r2) - l2;
      line_edges(G, F2 + B1 * S, o, 0, &r, &l);
      line_edges(G, F0 + B3 * S, o, 2, &r2, &l2);
      e1 = (((0. + r) + l) - r2) - l2;
      line_edges(G, F0 + B2 * S, o, 1, &r, &l);
      line_edges(G, F1 + B1 * S, o, 0, &r2, &l2);
      e2 = (((0. + r) + l) - r2) - l2;
    } else {  // flux_ct.c:33-41
      const long oi = off3(G, i - 1, j, k), oj = off3(G, i, j - 1, k), ok = off3(G, i, j, k - 1);
      e0 = 0.25 * (F1[B3 * S + o] + F1[B3 * S + ok] - F2[B2 * S + o] - F2[B2 * S + oj]);
      e1 = 0.25 * (F2[B1 * S + o] + F2[B1 * S + oi] - F0[B3 * S + o] - F0[B3 * S + ok]);
      e2 = 0.25 * (F0[B2 * S + o] + F0[B2 * S + oj] - F1[B1 * S + o] - F1[B1 * S + oi]);
    }
    G.emf[0][o] = e0;
    G.emf[1][o] = e1;
    G.emf[2][o] = e2;
  }
}

// ---------------------------------------------------------------------------
// source(), phys.c:121-187 (cooling off): T^mu_kappa Gamma^kappa_nu mu for
// METRIC_DIM 2 (U1, U2 only), times sqrt(-g).  Returns 1 on a gamma failure.
// With PRE the state of ph is given (qpre, and badpre the result of its
// gamma_calc): the predictor's sources are evaluated at p_i, whose state the
// conserved variables already needed.
template <bool PRE>
__device__ __forceinline__ int source_terms(const GridDev &G, const double *ph, const Geom &g, int i, int j, int k,
                                            double *dU, const State &qpre, int badpre)
{
#pragma unroll
  for (int l = 0; l < HG_NPR; l++) dU[l] = 0.;
  int bad = 0;
  State q;
  if (PRE) q = qpre;
  if (G.mdim > 0) {
    bad = PRE ? badpre : get_state(ph, g, G.gam, q);
    double mhd[4][4];
    mhd_row(q, 0, mhd[0]);
    mhd_row(q, 1, mhd[1]);
    mhd_row(q, 2, mhd[2]);
    mhd_row(q, 3, mhd[3]);
    if (G.mdim == 3) {  // METRIC_DIM > 2: all four components (phys.c:143-154)
      const long cS = G.S, co = off3(G, i, j, k);
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
          dU[U1] += mhd[a][b] * G.conn3[(b * 10 + dyn_sym(1, a)) * cS + co];
          dU[U2] += mhd[a][b] * G.conn3[(b * 10 + dyn_sym(2, a)) * cS + co];
          dU[UU] += mhd[a][b] * G.conn3[(b * 10 + dyn_sym(0, a)) * cS + co];
          dU[U3] += mhd[a][b] * G.conn3[(b * 10 + dyn_sym(3, a)) * cS + co];
        }
    } else {
      const long cS = (long)G.T[0] * G.T[1];
      const long co = (long)(G.deg[1] ? 0 : j) * G.T[0] + (G.deg[0] ? 0 : i);
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) {
          dU[U1] += mhd[a][b] * __ldg(G.conn + ((b * 4 + 1) * 4 + a) * cS + co);
          dU[U2] += mhd[a][b] * __ldg(G.conn + ((b * 4 + 2) * 4 + a) * cS + co);
        }
    }
  }
  if (G.cooling == 1) {  // phys.c:162-172, source_cooling_func phys.c:541-582
    if (G.mdim == 0) bad = PRE ? badpre : get_state(ph, g, G.gam, q);
    const int bound = ((q.ucov[0] * (q.p + ph[UU] + ph[RHO] + q.bsq)) > (-ph[RHO])) ? 1 : 0;
    double f_cool = 0.;
    if (bound) {  // cooling_func_hr_disk, phys.c:779-783 (s_norm 1, q_exp 1/2)
      const double T_r = G.cool[G.T[0] + i], Omega_r = G.cool[i];
      const double E_ratio = (G.gam - 1.) * ph[UU] / (ph[RHO] * T_r);
      const double dE = E_ratio - 1.;
      // pow(x, 0.5) of the reference, as the correctly rounded square root
      f_cool = 1. * ph[UU] * Omega_r * sqrt(dE + fabs(dE));
    }
    dU[UU] -= f_cool * q.ucov[0];
    dU[U1] -= f_cool * q.ucov[1];
    dU[U2] -= f_cool * q.ucov[2];
    dU[U3] -= f_cool * q.ucov[3];
  }
  dU[UU] *= g.g;
  dU[U1] *= g.g;
  dU[U2] *= g.g;
  dU[U3] *= g.g;
  return bad;
}

// Conserved update of one zone (step_ch.c:320-370).
__device__ __forceinline__ void update_zone(const GridDev &G, int i, int j, int k, double Dt, const double *dU, double *U)
{
  const long S = G.S, o = off3(G, i, j, k);
  const long oi = o + G.st[0], oj = o + G.st[1], ok = o + G.st[2];
  const double *F0 = G.F[0], *F1 = G.F[1], *F2 = G.F[2];
#pragma unroll
  for (int l = 0; l < B1; l++) {
    const double a = F0[l * S + oi] - F0[l * S + o];
    const double b = F1[l * S + oj] - F1[l * S + o];
    const double c = F2[l * S + ok] - F2[l * S + o];
    U[l] += Dt * (-(a)*G.invdx[1] - (b)*G.invdx[2] - (c)*G.invdx[3] + dU[l]);
  }
  // induction fluxes after flux_ct: zeroed, then + fac * (sum of two EMFs)
  const double fac = G.ct_para ? 0.125 : 0.5;
  const double *E0 = G.emf[0], *E1 = G.emf[1], *E2 = G.emf[2];
  const long oij = o + G.st[0] + G.st[1], oik = o + G.st[0] + G.st[2], ojk = o + G.st[1] + G.st[2];
  // x1 faces
  const double f0b2_m = 0. + fac * (E2[o] + E2[oj]);
  const double f0b2_p = 0. + fac * (E2[oi] + E2[oij]);
  const double f0b3_m = 0. + (-fac) * (E1[o] + E1[ok]);
  const double f0b3_p = 0. + (-fac) * (E1[oi] + E1[oik]);
  // x2 faces
  const double f1b1_m = 0. + (-fac) * (E2[o] + E2[oi]);
  const double f1b1_p = 0. + (-fac) * (E2[oj] + E2[oij]);
  const double f1b3_m = 0. + fac * (E0[o] + E0[ok]);
  const double f1b3_p = 0. + fac * (E0[oj] + E0[ojk]);
  // x3 faces
  const double f2b1_m = 0. + fac * (E1[o] + E1[oi]);
  const double f2b1_p = 0. + fac * (E1[ok] + E1[oik]);
  const double f2b2_m = 0. + (-fac) * (E0[o] + E0[oj]);
  const double f2b2_p = 0. + (-fac) * (E0[ok] + E0[ojk]);
  const double zero = 0.;
  U[B1] += Dt * (-(zero - zero) * G.invdx[1] - (f1b1_p - f1b1_m) * G.invdx[2] - (f2b1_p - f2b1_m) * G.invdx[3] + dU[B1]);
  U[B2] += Dt * (-(f0b2_p - f0b2_m) * G.invdx[1] - (zero - zero) * G.invdx[2] - (f2b2_p - f2b2_m) * G.invdx[3] + dU[B2]);
  U[B3] += Dt * (-(f0b3_p - f0b3_m) * G.invdx[1] - (f1b3_p - f1b3_m) * G.invdx[2] - (zero - zero) * G.invdx[3] + dU[B3]);
}

// The update of advance() (step_ch.c:312-399) in two kernels over every
// physical zone, so that neither holds the geometry, the conserved-variable
// sources and the Newton solver's state at once:
//   k_update_cons  U(p_i), the geometric and cooling sources, the flux
//                  divergence with the CT-corrected induction fluxes -> U
//                  (the Uc planes) and the per-block M_tot partials;
//   k_update_c2p   the 2D Newton inversion of U, the queue for the rest of
//                  recover_primitives(), floors and gamma ceiling -> p_f.
// sub = 0 predictor (p_f = ph), 1 corrector (p_f = p).  The conserved update
// takes it as a template parameter: each substep's kernel holds only its own
// source path (fewer registers, no spill at the 3-block cap).
template <bool RS, int MDIM, int SUB>
__global__ void __launch_bounds__(HG_BLK, SUB == 0 ? HG_CONS0_MINB : HG_CONS_MINB) k_update_cons(const __grid_constant__ GridDev G,
                                                                    double dtfac, const double *__restrict__ p_h)
{
  constexpr int sub = SUB;
  const unsigned N0 = G.N[0], N1 = G.N[1];
  const unsigned total = (unsigned)G.capacity;  // < 2^31 (hg_init)
  const double Dt = dtfac * G.sc->dt;
  const long S = G.S;
  const double *p = G.p;
  double msum = 0.;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned tq = t / N0;
    const int i = HG_NGH + (int)(t - tq * N0);
    const int j = HG_NGH + (int)(tq % N1);
    const int k = HG_NGH + (int)(tq / N1);
    const long o = off3(G, i, j, k);
    Geom gl;
    if (MDIM != 0) load_geom(G, 3, i, j, gl, k, 0);
    const Geom &g = (MDIM == 0) ? G.g0 : gl;
    double pi[HG_NPR], U[HG_NPR], dU[HG_NPR];
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) {
      const double v = p[l * S + o];
      pi[l] = RS ? rs_roundtrip(G, v, l, i) : v;
    }
    State q;  // U(p_i) at the start of the step (U_gf[0])
    const int bad_i = get_state(pi, g, G.gam, q);
    if (bad_i && sub == 0) book(G, NF_GAMMA_CALC, i, j, k);
    primtoflux(pi, q, 0, g, U);
    if (sub == 0) {
      if (source_terms<true>(G, pi, g, i, j, k, dU, q, bad_i)) book(G, NF_GAMMA_CALC, i, j, k);
    } else {
      double phv[HG_NPR];
#pragma unroll
      for (int l = 0; l < HG_NPR; l++) {
        const double v = p_h[l * S + o];
        phv[l] = RS ? rs_roundtrip(G, v, l, i) : v;
      }
      if (MDIM == 3) {  // the corrector's sources take the geometry of n_mid
        Geom gh;
        load_geom(G, 3, i, j, gh, k, 1);
        if (source_terms<false>(G, phv, gh, i, j, k, dU, q, 0)) book(G, NF_GAMMA_CALC, i, j, k);
      } else {
        if (source_terms<false>(G, phv, g, i, j, k, dU, q, 0)) book(G, NF_GAMMA_CALC, i, j, k);
      }
    }
    update_zone(G, i, j, k, Dt, dU, U);
    msum += U[0];
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) G.Uc[l * S + o] = U[l];
  }
  const double bs = block_sum(msum);
  if (threadIdx.x == 0) G.blk[blockIdx.x] = bs;
}

template <bool RS, int MDIM>
__global__ void __launch_bounds__(HG_BLK, HG_C2P_MINB) k_update_c2p(const __grid_constant__ GridDev G, int sub,
                                                                   double *__restrict__ p_f)
{
  const unsigned N0 = G.N[0], N1 = G.N[1];
  const unsigned total = (unsigned)G.capacity;  // < 2^31 (hg_init)
  const long S = G.S;
  const double *p = G.p;
  unsigned int n_full = 0, n_floor = 0;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned tq = t / N0;
    const int i = HG_NGH + (int)(t - tq * N0);
    const int j = HG_NGH + (int)(tq % N1);
    const int k = HG_NGH + (int)(tq / N1);
    const long o = off3(G, i, j, k);
    Geom gl;
    if (MDIM != 0) load_geom(G, 3, i, j, gl, k, sub + 1);
    const Geom &g = (MDIM == 0) ? G.g0 : gl;
    double U[HG_NPR], pf[HG_NPR];
    // Newton guess: the predictor's p_f (= ph) holds the unscaled copy of p;
    // the corrector's p_f is p itself, rescaled in place by the predictor.
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) {
      U[l] = G.Uc[l * S + o];
      const double v = p[l * S + o];
      pf[l] = (RS && sub == 1) ? rs_roundtrip(G, v, l, i) : v;
    }
    double gamma = 0., bsq = 0.;
    const int ret = utoprim_2d(U, g, G.gam, pf, &gamma, &bsq);
    const bool ee = G.use_ee && ((pf[UU] < HG_BETA_MIN * bsq) || (pf[RHO] < HG_BETA_MIN * bsq));
    if (ret != 0 || check_gamma(gamma) == 2 || ee) {
      // rest of the recover_primitives() tree: queue the zone
      const int slot = atomicAdd(&G.sc->q_count, 1);
      if (slot < G.capacity) {
        G.q_idx[slot] = pack_ijk(i, j, k);
#pragma unroll
        for (int l = 0; l < HG_NPR; l++) G.q_U[(long)slot * HG_NPR + l] = U[l];
      } else {
        G.sc->err = 2;
      }
      continue;
    }
    // fast path of recover_primitives (step_ch.c:830-1018, FIXUP_TREE 3)
    n_full++;
    G.nfail[NF_USE_FULL_INV * S + o] += 1u;
    const double rf = G.floors[o], uf = G.floors[S + o];
    bool fl = false;
    if (pf[RHO] < rf) { pf[RHO] = rf; fl = true; }
    if (pf[UU] < uf) { pf[UU] = uf; fl = true; }
    if (fl) {
      n_floor++;
      G.nfail[NF_FLOOR * S + o] += 1u;
    }
    int pflag = PF_NONE;
    if (check_gamma(gamma)) {
      book(G, NF_GAMMA_MAX, i, j, k);
      pflag = PF_INTERP_V;
      flag_zone(G, PF_INTERP_V, i, j, k);
    }
    G.p_gamma[o] = gamma;
    if (pflag == PF_NONE) G.pflag[o] = PF_NONE;
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) put_state(G, p_f, l * S + o, pf[l]);
  }
  const unsigned int c_full = block_count(n_full);
  const unsigned int c_floor = block_count(n_floor);
  if (threadIdx.x == 0) {
    if (c_full) atomicAdd(&G.sc->nfailtot[NF_USE_FULL_INV], (unsigned long long)c_full);
    if (c_floor) atomicAdd(&G.sc->nfailtot[NF_FLOOR], (unsigned long long)c_floor);
  }
}

// ---------------------------------------------------------------------------
// fixup_entropy_eq(), fixup.c:335-454: entropy flux rebuilt from the face
// states of the six faces (recomputed here; the flux kernel does not store
// them) and the inversions Utoprim_1d_ee / Utoprim_1d_ee2.  pow() of the
// reference is the correctly rounded hg_cr_pow (hg_crpow.h).
template <bool RS>
__device__ __forceinline__ double ee_face_flux(const GridDev &G, const double *p_h, int d, int i, int j, int k, int slot)
{
  double pl[HG_NPR], pr[HG_NPR];
  face_prims<RS>(G, p_h, d, i, j, k, pl, pr);
  Geom g;
  load_geom(G, d, i, j, g, k, slot);
  State ql, qr;
  get_state(pl, g, G.gam, ql);
  get_state(pr, g, G.gam, qr);
  const int dim = d + 1;
  double cmaxl, cminl, cmaxr, cminr;
  vchar_fast(ql, g, dim, G.gam, &cmaxl, &cminl);
  vchar_fast(qr, g, dim, G.gam, &cmaxr, &cminr);
  const double a0 = 0. > cmaxl ? 0. : cmaxl;
  const double cmax = fabs(a0 > cmaxr ? a0 : cmaxr);
  const double a1 = 0. > -cminl ? 0. : -cminl;
  const double cmin = fabs(a1 > -cminr ? a1 : -cminr);
  const double ctop = cmin > cmax ? cmin : cmax;
  const double gam = G.gam;
  double s = (gam - 1.) * pl[UU] * hg_cr_pow(pl[RHO], 1. - gam);
  const double Ul = s * (g.g * ql.ucon[0]);
  const double Fl = s * (g.g * ql.ucon[dim]);
  s = (gam - 1.) * pr[UU] * hg_cr_pow(pr[RHO], 1. - gam);
  const double Ur = s * (g.g * qr.ucon[0]);
  const double Fr = s * (g.g * qr.ucon[dim]);
  if (G.flux == 1) return (cmax * Fl + cmin * Fr - cmax * cmin * (Ur - Ul)) / (cmax + cmin + HG_SMALL);
  return 0.5 * (Fl + Fr - ctop * (Ur - Ul));
}

// The six entropy face fluxes of every queued zone, one (zone, face) per
// thread, ahead of k_fallback: q_F[6 e + f], f = 0..2 the lower faces of
// x1..x3, 3..5 the upper ones.
template <bool RS>
__global__ void __launch_bounds__(HG_BLK, HG_EE_MINB) k_ee_faces(GridDev G, const double *__restrict__ p_h, int slot)
{
  const long n = 6L * min(G.sc->q_count, (int)G.capacity);
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const long e = t / 6;
    const int f = (int)(t % 6), d = f % 3, up = f / 3;
    int i, j, k;
    unpack_ijk(G.q_idx[e], i, j, k);
    G.q_F[t] = ee_face_flux<RS>(G, p_h, d, i + (up && d == 0), j + (up && d == 1), k + (up && d == 2), slot);
  }
}

template <bool RS>
__device__ __noinline__ int fixup_entropy_eq(const GridDev &G, long e, int i, int j, int k,
                                             const double *prim_old, double *prim, const Geom &geom,
                                             const Geom &geom_old, const double *Un, double Dt, double *gamma_out)
{
  double prim_backup[HG_NPR], gamma;
  for (int l = 0; l < HG_NPR; l++) prim_backup[l] = prim[l];
  const double gam = G.gam;
  gamma_calc(prim_old, geom_old, &gamma);
  const double S_old = geom_old.g * (gam - 1.) * prim_old[UU] * gamma /
                       (geom_old.alpha * hg_cr_pow(prim_old[RHO], (gam - 1.)));
  double Fm[3], Fp[3];
  for (int d = 0; d < 3; d++) {
    Fm[d] = G.q_F[6 * e + d];
    Fp[d] = G.q_F[6 * e + 3 + d];
  }
  const double Snew = S_old + Dt * (-(Fp[0] - Fm[0]) * G.invdx[1] - (Fp[1] - Fm[1]) * G.invdx[2] -
                                    (Fp[2] - Fm[2]) * G.invdx[3]);
  int ret = utoprim_1d_ee(Un, Snew, geom, gam, prim, &gamma);
  if ((!ret) && (check_gamma(gamma) == 2)) {
    for (int l = 0; l < HG_NPR; l++) prim[l] = prim_backup[l];
    ret = 1;
    gamma = 1.;
  }
  if (ret) {
    ret = utoprim_1d_ee2(Un, Snew, geom, gam, prim, &gamma);
    if ((!ret) && (check_gamma(gamma) == 2)) {
      for (int l = 0; l < HG_NPR; l++) prim[l] = prim_backup[l];
      ret = 1;
    }
    if (ret) gamma = 1.;
  }
  *gamma_out = gamma;
  if (!ret) book(G, NF_USE_EE, i, j, k);
  return ret;
}

// recover_primitives(), step_ch.c:801-1024 (FIXUP_TREE 3), full tree.
template <bool RS>
__global__ void __launch_bounds__(HG_BLK) k_fallback(GridDev G, int sub, double dtfac, const double *__restrict__ p_h,
                                                     double *__restrict__ p_f)
{
  const int n = min(G.sc->q_count, (int)G.capacity);
  const double Dt = dtfac * G.sc->dt;
  const long S = G.S;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    int i, j, k;
    unpack_ijk(G.q_idx[e], i, j, k);
    const long o = off3(G, i, j, k);
    double U[HG_NPR], pf[HG_NPR], pg[HG_NPR], pold[HG_NPR], pf2[HG_NPR];
    for (int l = 0; l < HG_NPR; l++) {
      U[l] = G.q_U[(long)e * HG_NPR + l];
      pold[l] = G.p[l * S + o];
      pf[l] = (sub == 0 || !RS) ? pold[l] : rs_roundtrip(G, pold[l], l, i);
      pg[l] = pf[l];
    }
    Geom g, g_old;
    load_geom(G, 3, i, j, g, k, sub + 1);
    if (G.mdim == 3) load_geom(G, 3, i, j, g_old, k, 0);  // geom_old of recover_primitives: n_beg
    else g_old = g;
    double gamma = 0., bsq = 0.;
    int ret = utoprim_2d(U, g, G.gam, pf, &gamma, &bsq);
    if ((!ret) && (check_gamma(gamma) == 2)) {
      for (int l = 0; l < B1; l++) pf[l] = pg[l];
      ret = 1;
      gamma = 1.;
    }
    if (ret) {
      ret = utoprim_1d(U, g, G.gam, pf, &gamma, &bsq);
      if ((!ret) && (check_gamma(gamma) == 2)) {
        for (int l = 0; l < B1; l++) pf[l] = pg[l];
        ret = 1;
      }
      if (ret) gamma = 1.;
    }
    double pgam = gamma;
    int use_ee = 0;
    if (G.use_ee && (ret || (pf[UU] < HG_BETA_MIN * bsq) || (pf[RHO] < HG_BETA_MIN * bsq))) use_ee = 1;
    int pflag = PF_NONE;
    bool done = false;
    if (!use_ee) {
      if (!ret) book(G, NF_USE_FULL_INV, i, j, k);
      else {
        book(G, NF_UTOPRIM, i, j, k);
        pflag = PF_INTERP_PRIM;
      }
    } else {
      if (!ret) {
        for (int l = 0; l < HG_NPR; l++) pf2[l] = pf[l];
      } else {
        book(G, NF_UTOPRIM, i, j, k);
      }
      for (int l = 0; l < B1; l++) pf[l] = pg[l];
      const int ret_ee = fixup_entropy_eq<RS>(G, e, i, j, k, pold, pf, g, g_old, U, Dt, &gamma);
      if (ret_ee) {
        if (ret) {
          book(G, NF_UTOPRIM_EE, i, j, k);
          pflag = PF_INTERP_PRIM;
          done = true;
        } else {
          book(G, NF_UTOPRIM_EE, i, j, k);
          for (int l = 0; l < HG_NPR; l++) pf[l] = pf2[l];
          gamma = pgam;
          book(G, NF_USE_FULL_INV, i, j, k);
        }
      }
    }
    if (!done) {
      pgam = gamma;
      const double rf = G.floors[o], uf = G.floors[S + o];
      bool fl = false;
      if (pf[RHO] < rf) { pf[RHO] = rf; fl = true; }
      if (pf[UU] < uf) { pf[UU] = uf; fl = true; }
      if (fl) book(G, NF_FLOOR, i, j, k);
      if (check_gamma(gamma)) {
        book(G, NF_GAMMA_MAX, i, j, k);
        pflag = PF_INTERP_V;
      }
    }
    G.p_gamma[o] = pgam;
    if (pflag != PF_NONE) flag_zone(G, pflag, i, j, k);
    else G.pflag[o] = PF_NONE;
    for (int l = 0; l < HG_NPR; l++) put_state(G, p_f, l * S + o, pf[l]);
  }
}

// ---------------------------------------------------------------------------
// Boundary conditions, bounds.c:58-211: every ghost zone copies the zone
// reached by applying the per-direction map (outflow: clamp to the physical
// range; periodic: wrap) in each direction.  The reference fills x1, then x2
// over all i, then x3 over all i,j, which composes to the same map.
__device__ __forceinline__ int bc_map(int x, int n, int periodic)
{
  const int s = HG_NGH, e = n + HG_NGH - 1;
  if (x < s) return periodic ? x + n : s;
  if (x > e) return periodic ? x - n : e;
  return x;
}

// x2 reflection of BC_SPHERICAL_OUTFLOW3 (bounds.c:522-546): ghost N2S-1-g
// copies N2S+g, ghost N2E+1+g copies N2E-g.
__device__ __forceinline__ int sph_reflect(int x, int n)
{
  const int s = HG_NGH, e = n + HG_NGH - 1;
  if (x < s) return 2 * s - 1 - x;
  if (x > e) return 2 * e + 1 - x;
  return x;
}

// inflow_check(), bounds.c:2304-2370 (dir = RR, USE_GAMMA_CEILING_X1DN_BC 0).
// Returns 1 if gamma_calc failed (ucon_calc's FAIL_GAMMA_CALC).
__device__ __forceinline__ int inflow_check(double *pr, const Geom &g, int type)
{
  double gamma;
  const int bad = gamma_calc(pr, g, &gamma);
  double ucon[4];
  ucon[0] = gamma * g.ncon[0];
  ucon[1] = pr[U1] - ucon[0] * g.beta[0];
  if (((ucon[1] > 0.) && (type == 0)) || ((ucon[1] < 0.) && (type == 1))) {
    gamma = g.alpha * ucon[0];
    pr[U1] /= gamma;
    pr[U2] /= gamma;
    pr[U3] /= gamma;
    pr[U1] = g.beta[0] * g.ncon[0];
    double vsq = 0.;
    for (int a = 1; a < 4; a++)
      for (int b = 1; b < 4; b++) vsq += g.gcov[a][b] * pr[U1 + a - 1] * pr[U1 + b - 1];
    if (fabs(vsq) < 1.e-13) vsq = fabs(vsq);
    if (vsq < 0.) vsq = 0.;
    if (vsq >= 1.) vsq = 1. - 1. / (HG_GAMMAMAX * HG_GAMMAMAX);
    gamma = 1. / sqrt(1. - vsq);
    pr[U1] *= gamma;
    pr[U2] *= gamma;
    pr[U3] *= gamma;
  }
  return bad;
}

// One ghost zone of BC_SPHERICAL_OUTFLOW3 (bounds.c:492-575).  The reference
// fills x1 ghosts (copy + inflow_check at the ghost's own geometry) over
// physical j,k, then x2 ghosts over all i (reflection, U2 and B2 flipped),
// then x3 ghosts over all i,j (periodic); composed per zone: take the zone
// the three maps reach, apply inflow_check at (ghost i, reflected j) if i is
// a ghost, then the flips if j is a ghost.  A gamma failure in inflow_check
// is booked only where the reference calls it (j and k physical).
__device__ __forceinline__ void bounds_spherical3(const GridDev &G, double *__restrict__ pa, int i, int j, int k,
                                                  long od, int slot)
{
  const int N0 = G.N[0], N1 = G.N[1], N2 = G.N[2];
  const int si = bc_map(i, N0, 0), sj = sph_reflect(j, N1), sk = bc_map(k, N2, 1);
  const long os = (long)si * G.st[0] + (long)sj * G.st[1] + (long)sk * G.st[2];
  double v[HG_NPR];
#pragma unroll
  for (int l = 0; l < HG_NPR; l++) v[l] = pa[l * G.S + os];
  if (i != si) {
    Geom g;
    load_geom(G, 3, i, sj, g, sk, slot);
    if (inflow_check(v, g, i > si ? 1 : 0) && j == sj && k == sk) book(G, NF_GAMMA_CALC, i, j, k);
  }
  if (j != sj) {
    v[U2] *= -1;
    v[B2] *= -1;
  }
#pragma unroll
  for (int l = 0; l < HG_NPR; l++) put_state(G, pa, l * G.S + od, v[l]);
}

// slot: the geometry level inflow_check reads (ncurr: n_mid after the
// predictor, n_end after the corrector; n_beg outside a step)
__global__ void __launch_bounds__(HG_BLK) k_bounds(GridDev G, double *__restrict__ pa, int conditional, int slot)
{
  if (conditional && !G.sc->bnd_phys) return;
  const int T0 = G.T[0], T1 = G.T[1], T2 = G.T[2];
  const int N0 = G.N[0], N1 = G.N[1], N2 = G.N[2];
  // ghost zones: x3 slabs, then x2 slabs, then x1 slabs (32-bit counts:
  // fewer than the 2^31 stored zones hg_init allows)
  const unsigned c1 = (unsigned)T0 * T1 * (T2 - (G.deg[2] ? 1 : N2));
  const unsigned c2 = (unsigned)T0 * (T1 - (G.deg[1] ? 1 : N1)) * (G.deg[2] ? 1 : N2);
  const unsigned c3 = (unsigned)(T0 - (G.deg[0] ? 1 : N0)) * (G.deg[1] ? 1 : N1) * (G.deg[2] ? 1 : N2);
  const unsigned total = c1 + c2 + c3;
  const int per = (G.bc == 1);
  const int fl = G.sc->failure_exists;
  const long S = G.S;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    int i, j, k;  // stored indices
    if (t < c1) {
      const unsigned q = t / (unsigned)T0;
      i = (int)(t - q * (unsigned)T0);
      j = (int)(q % (unsigned)T1);
      const int kg = (int)(q / (unsigned)T1);
      k = kg < HG_NGH ? kg : kg + N2;
    } else if (t < c1 + c2) {
      const unsigned u = t - c1, q = u / (unsigned)T0, w = (unsigned)(T1 - N1);
      i = (int)(u - q * (unsigned)T0);
      const int jg = (int)(q % w);
      j = jg < HG_NGH ? jg : jg + N1;
      k = HG_NGH + (int)(q / w);
    } else {
      const unsigned u = t - c1 - c2, w = (unsigned)(T0 - N0), q = u / w;
      const int ig = (int)(u - q * w);
      i = ig < HG_NGH ? ig : ig + N0;
      j = HG_NGH + (int)(q % (unsigned)N1);
      k = HG_NGH + (int)(q / (unsigned)N1);
    }
    // degenerate directions have no ghosts, so these are reference indices
    const long od = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
    if (G.bc == 10) {
      bounds_spherical3(G, pa, i, j, k, od, slot);
      G.pflag[od] = fl ? G.pflag[(long)bc_map(i, N0, 0) * G.st[0] + (long)sph_reflect(j, N1) * G.st[1] +
                                 (long)bc_map(k, N2, 1) * G.st[2]]
                       : 0;
      continue;
    }
    const int si = G.deg[0] ? i : bc_map(i, N0, per);
    const int sj = G.deg[1] ? j : bc_map(j, N1, per);
    const int sk = G.deg[2] ? k : bc_map(k, N2, per);
    const long os = (long)si * G.st[0] + (long)sj * G.st[1] + (long)sk * G.st[2];
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) put_state(G, pa, l * S + od, pa[l * S + os]);
    // pflag ghosts are copies while a failure exists in this substep; otherwise
    // every pflag of the reference is zero (step_ch.c:65-69, 123-127)
    G.pflag[od] = fl ? G.pflag[os] : 0;
  }
}

// ---------------------------------------------------------------------------
// fixup_interp_v / fixup_interp_prim (fixup.c:499-761) over the flagged list.
// A zone only reads unflagged neighbours, which no thread writes, so the
// zones are independent and the order of the reference's loop is immaterial.
__global__ void __launch_bounds__(HG_BLK) k_fixup(GridDev G, double *__restrict__ pv, int slot)
{
  const int n = min(G.sc->fl_count, (int)G.capacity);
  const long S = G.S;
  const int ngood_min_tab[4] = {13, 9, 6, 4};
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    int i, j, k;
    unpack_ijk(G.fl_idx[e], i, j, k);
    const long o = off3(G, i, j, k);
    const int which = G.pflag[o];
    if (which != PF_INTERP_V && which != PF_INTERP_PRIM) continue;
    const int lo = which == PF_INTERP_PRIM ? 0 : U1, hi = which == PF_INTERP_PRIM ? B1 - 1 : U3;
    unsigned int good = 0;  // bit (13 + ii + 3*(jj + 3*kk)) set if that neighbour is usable
    for (int kk = -1; kk <= 1; kk++)
      for (int jj = -1; jj <= 1; jj++)
        for (int ii = -1; ii <= 1; ii++)
          if (!G.pflag[off3(G, i + ii, j + jj, k + kk)]) good |= 1u << (13 + ii + 3 * (jj + 3 * kk));
    int ngood = 0;
    for (int m = 1; m <= 13; m++) {
      if (((good >> (13 + m)) & 1u) && ((good >> (13 - m)) & 1u)) ngood++;
      else good &= ~((1u << (13 + m)) | (1u << (13 - m)));
    }
    // icurr/jcurr/kcurr of the reference: the zone, or the last usable
    // neighbour visited by the gamma loop once that loop has run.
    int ci = i, cj = j, ck = k;
    double pc[HG_NPR], pold[HG_NPR];
    for (int l = 0; l < HG_NPR; l++) pc[l] = pv[l * S + o];
    for (int l = lo; l <= hi; l++) pold[l] = pc[l];
    Geom g;
    load_geom(G, 3, i, j, g, k, slot);
    double gamma, f, gamma_old;
    int i_ret;
    const int ngood_min = ngood_min_tab[G.nsd];
    if (which == PF_INTERP_PRIM && ngood < ngood_min) {
      gamma_calc(pc, g, &gamma);
      G.p_gamma[o] = gamma;
      book(G, NF_INTERP_PRIM, ci, cj, ck);
      continue;
    }
    if (which == PF_INTERP_V && ngood < ngood_min) {
      double pg = G.p_gamma[o];
      f = sqrt((HG_GAMMAMAX - 1.) * (HG_GAMMAMAX + 1.) / ((pg - 1.) * (pg + 1.)));
      pc[U1] *= f;
      pc[U2] *= f;
      pc[U3] *= f;
      G.p_gamma[o] = HG_GAMMAMAX;
      book(G, NF_GAMMA_MAX, ci, cj, ck);
      book(G, NF_INTERP_V, ci, cj, ck);
      for (int l = U1; l <= U3; l++) put_state(G, pv, l * S + o, pc[l]);
      continue;
    }
    for (int l = lo; l <= hi; l++) pc[l] = 0.;
    // the reference sums over ii (outer), jj, kk (inner)
    for (int ii = -1; ii <= 1; ii++)
      for (int jj = -1; jj <= 1; jj++)
        for (int kk = -1; kk <= 1; kk++)
          if ((good >> (13 + ii + 3 * (jj + 3 * kk))) & 1u) {
            const long on = off3(G, i + ii, j + jj, k + kk);
            for (int l = lo; l <= hi; l++) pc[l] += pv[l * S + on];
          }
    const int ng2 = ngood * 2;
    for (int l = lo; l <= hi; l++) pc[l] /= ng2;
    i_ret = gamma_calc(pc, g, &gamma);
    if (check_gamma(gamma)) {
      gamma_old = gamma;
      gamma = 0.;
      int ngood2 = 0;
      for (int ii = -1; ii <= 1; ii++)
        for (int jj = -1; jj <= 1; jj++)
          for (int kk = -1; kk <= 1; kk++)
            if ((good >> (13 + ii + 3 * (jj + 3 * kk))) & 1u) {
              Geom g2;
              load_geom(G, 3, i + ii, j + jj, g2, k + kk, slot);
              ci = i + ii;
              cj = j + jj;
              ck = k + kk;
              const long on = off3(G, i + ii, j + jj, k + kk);
              double pn[HG_NPR];
              for (int l = 0; l < HG_NPR; l++) pn[l] = pv[l * S + on];
              i_ret = gamma_calc(pn, g2, &f);
              if (!i_ret) {
                gamma += f;
                ngood2++;
              }
            }
      gamma /= ngood2;
      f = sqrt((gamma - 1.) * (gamma + 1.) / ((gamma_old - 1.) * (gamma_old + 1.)));
      pc[U1] *= f;
      pc[U2] *= f;
      pc[U3] *= f;
      i_ret = gamma_calc(pc, g, &gamma);
    }
    if (which == PF_INTERP_PRIM) {
      if (i_ret) {
        for (int l = U1; l <= U3; l++) pc[l] = pold[l];
        gamma_calc(pc, g, &gamma);
        book(G, NF_INTERP_PRIM, ci, cj, ck);
      }
      book(G, NF_USE_INTERP_PRIM, ci, cj, ck);
      if ((!i_ret) && check_gamma(gamma)) {
        f = sqrt((HG_GAMMAMAX - 1.) * (HG_GAMMAMAX + 1.) / ((gamma - 1.) * (gamma + 1.)));
        pc[U1] *= f;
        pc[U2] *= f;
        pc[U3] *= f;
        gamma = HG_GAMMAMAX;
        book(G, NF_GAMMA_MAX, ci, cj, ck);
      }
      G.p_gamma[o] = gamma;
    } else {
      if (i_ret || check_gamma(gamma)) {
        for (int l = U1; l <= U3; l++) pc[l] = pold[l];
        const double pg = G.p_gamma[o];
        f = sqrt((HG_GAMMAMAX - 1.) * (HG_GAMMAMAX + 1.) / ((pg - 1.) * (pg + 1.)));
        pc[U1] *= f;
        pc[U2] *= f;
        pc[U3] *= f;
        G.p_gamma[o] = HG_GAMMAMAX;
        book(G, NF_GAMMA_MAX, ci, cj, ck);
        book(G, NF_INTERP_V, ci, cj, ck);
      } else {
        book(G, NF_USE_INTERP_V, ci, cj, ck);
        G.p_gamma[o] = gamma;
      }
    }
    for (int l = lo; l <= hi; l++) put_state(G, pv, l * S + o, pc[l]);
  }
}

// ---------------------------------------------------------------------------
// fixup(), fixup.c:8-33 with fixup1zone (fixup.c:45-75): over the physical
// zones, gamma_calc (FAIL_GAMMA_CALC, gamma = 1 on failure), the rho/u floors
// (FAIL_FLOOR) and the gamma ceiling fixup_gamma (fixup.c:148-158,
// FAIL_GAMMA_MAX); all with state 0, so no zone is flagged.  This is the
// init-time pass the setups run before and after the magnetic field is set
// (init.torus.c:205-215).
__global__ void __launch_bounds__(HG_BLK) k_fixup_cells(GridDev G)
{
  const unsigned N0 = G.N[0], N1 = G.N[1];
  const unsigned total = (unsigned)G.capacity;  // < 2^31 (hg_init)
  const long S = G.S;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const unsigned tq = t / N0;
    const int i = HG_NGH + (int)(t - tq * N0);
    const int j = HG_NGH + (int)(tq % N1);
    const int k = HG_NGH + (int)(tq / N1);
    const long o = off3(G, i, j, k);
    Geom g;
    if (G.mdim != 0) load_geom(G, 3, i, j, g, k, 0);
    else g = G.g0;
    double pv[HG_NPR];
    for (int l = 0; l < HG_NPR; l++) pv[l] = G.p[l * S + o];
    double gamma;
    if (gamma_calc(pv, g, &gamma)) {
      book(G, NF_GAMMA_CALC, i, j, k);
      gamma = 1.;
    }
    bool fl = false;
    if (pv[RHO] < G.floors[o]) { pv[RHO] = G.floors[o]; fl = true; }
    if (pv[UU] < G.floors[S + o]) { pv[UU] = G.floors[S + o]; fl = true; }
    if (fl) book(G, NF_FLOOR, i, j, k);
    if (check_gamma(gamma)) {
      const double f = sqrt((HG_GAMMAMAX - 1.) * (HG_GAMMAMAX + 1.) / ((gamma - 1.) * (gamma + 1.)));
      pv[U1] *= f;
      pv[U2] *= f;
      pv[U3] *= f;
      book(G, NF_GAMMA_MAX, i, j, k);
    }
    for (int l = 0; l < HG_NPR; l++) G.p[l * S + o] = pv[l];
  }
}

// ---------------------------------------------------------------------------
__global__ void k_begin(DevScalars *sc)
{
  sc->maxs[0] = sc->maxs[1] = sc->maxs[2] = sc->maxs[3] = 0ull;
  sc->failure_exists = 0;
  sc->ftype[0] = sc->ftype[1] = sc->ftype[2] = 0;
  sc->bnd_phys = 0;
  sc->q_count = 0;
  sc->fl_count = 0;
}

// t += dx[0]; dx[0] = timestep() (step_ch.c:218-223, 546-623); M_tot.
__global__ void k_timestep(GridDev G, int nblk)
{
  __shared__ double red[1024];
  double s = 0.;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += G.blk[b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    DevScalars *sc = G.sc;
    sc->m_tot = red[0];
    const double c1 = __longlong_as_double((long long)sc->maxs[1]);
    const double c2 = __longlong_as_double((long long)sc->maxs[2]);
    const double c3 = __longlong_as_double((long long)sc->maxs[3]);
    sc->last_maxs[1] = c1;
    sc->last_maxs[2] = c2;
    sc->last_maxs[3] = c3;
    const double dt_old = sc->dt;
    const double t = sc->t + dt_old;
    const double dtsqij =
        sqrt((1. / 3.) / ((c1 * c1) / (G.dx[1] * G.dx[1]) + (c2 * c2) / (G.dx[2] * G.dx[2]) + (c3 * c3) / (G.dx[3] * G.dx[3])));
    double dtt = G.cour * dtsqij;
    if (dtt > HG_SAFE * dt_old) dtt = HG_SAFE * dt_old;
    if (t + dtt > (G.grid_length[0] + G.startx[0])) dtt = G.grid_length[0] + G.startx[0] - t;
    sc->t = t;
    sc->dt = dtt;
  }
}

// ---------------------------------------------------------------------------
// metric_dim 3: the time levels of the geometry and the connection.

__device__ __forceinline__ double *dyn_level(const GridDev &G, int slot)
{
  const int L = G.sc->lev[slot];
  return L == 0 ? G.geomL[0] : L == 1 ? G.geomL[1] : G.geomL[2];
}

// set_general_geometry (metric.c:3390-3499) for the time level `slot`, at
// t + tfac dx[0] (tfac 0, 0.5, 1 for n_beg, n_mid, n_end; metric.c:405-407,
// 3681-3683): the struct of_geom of the five positions of every stored zone.
__global__ void __launch_bounds__(HG_BLK) k_geom_level(GridDev G, int slot, double tfac)
{
  double *out = dyn_level(G, slot);
  const double t = G.sc->t + tfac * G.sc->dt;
  const bool pn = G.dyn.spacetime == HG_DYN_PN_BINARY;
  __shared__ PNBinary bin;  // the binary at the level's time, once per block
  if (pn) {
    if (threadIdx.x == 0) pn_binary(G.dyn, t, bin);
    __syncthreads();
  }
  const unsigned T0 = G.T[0], T1 = G.T[1];
  const unsigned total = (unsigned)HG_DYN_NPOS * (unsigned)G.S;  // < 2^31 (hg_init's bound on 5 planes)
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const unsigned pos = e / (unsigned)G.S, o = e - pos * (unsigned)G.S;
    const int i = (int)(o % T0), j = (int)((o / T0) % T1), k = (int)(o / (T0 * T1));
    Geom g;
    dyn_geom(G, (int)pos, i, j, k, t, g, pn ? &bin : nullptr);
    double *w = out + e;
    const long s = G.gS3;
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = a; b < 4; b++) {
        w[(HG_DP_GCON + dyn_sym(a, b)) * s] = g.gcon[a][b];
        w[(HG_DP_GCOV + dyn_sym(a, b)) * s] = g.gcov[a][b];
      }
    w[HG_DP_G * s] = g.g;
    w[HG_DP_GINV * s] = g.g_inv;
    w[HG_DP_ALPHA * s] = g.alpha;
    for (int a = 0; a < 3; a++) w[(HG_DP_BETA + a) * s] = g.beta[a];
    w[HG_DP_NCON0 * s] = g.ncon[0];
    if (G.geomF3[0] && pos < 3) {  // the mixed form's FP32 face geometry (hg_set_geometry's planes)
      const int L = G.sc->lev[slot];
      float *f = (L == 0 ? G.geomF3[0] : L == 1 ? G.geomF3[1] : G.geomF3[2]) + e;
      const long fs = 3 * (long)G.S;
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) f[(a * 4 + b) * fs] = (float)g.gcov[a][b];
      f[16 * fs] = (float)g.gcon[0][0];
      for (int jj = 1; jj <= 3; jj++) {
        f[(16 + jj) * fs] = (float)g.gcon[0][jj];
        f[(19 + jj) * fs] = (float)g.gcon[jj][jj];
      }
      f[23 * fs] = (float)g.ncon[0];
      for (int a = 0; a < 3; a++) f[(24 + a) * fs] = (float)g.beta[a];
      f[27 * fs] = (float)g.g;
    }
  }
}

// advance_geometry (metric.c:398-430), the rotation: the step's end becomes
// the next step's start; k_geom_level then fills n_mid and n_end.
__global__ void k_advance_geometry(DevScalars *sc)
{
  const int n = sc->lev[0];
  sc->lev[0] = sc->lev[2];
  sc->lev[2] = n;
}

// gcov of the level `slot` table at (pos, i, j, k), entry (a, b)
__device__ __forceinline__ double dyn_gcov_at(const GridDev &G, const double *lv, int pos, int i, int j, int k, int a,
                                              int b)
{
  return lv[(HG_DP_GCOV + dyn_sym(a, b)) * G.gS3 + (long)pos * G.S + off3(G, i, j, k)];
}

// set_general_conn (metric.c:3507-3648) at time t + tfac dx[0] from the
// level `slot` (ncurr): for every physical zone, conn_func_fd4
// (metric.c:212-247) -- the time derivative of gcov_func over +-dt_conn
// (conn.h:8-20), 4th-order differences of the stored gcov in x1, x2, x3
// (conn.h:44-86, weights invdx/6 and 4 invdx/3), on a physical x2 boundary
// the one-sided x2 stencils of conn_func_fd4_lo2 / _hi2 (metric.c:254-340,
// weights metric.c:3526-3540) -- and DGCOV_TO_CONN (conn.h:25-37) with the
// zone's gcon.  Written to conn3 as the 40 entries b <= c (HG_CONN3_PLANES).
#ifndef HG_CONN_MINB
#define HG_CONN_MINB 4
#endif
__global__ void __launch_bounds__(HG_BLK, HG_CONN_MINB) k_conn_dyn(GridDev G, int slot, double tfac)
{
  const double *lv = dyn_level(G, slot);
  const double t = G.sc->t + tfac * G.sc->dt;
  const double dtc = G.dyn.dt_conn, half_inv_dt_conn = 0.5 / dtc;
  const bool pn = G.dyn.spacetime == HG_DYN_PN_BINARY;
  __shared__ PNBinary bhl[2];  // the binary at t + dt_conn and t - dt_conn, once per block
  if (pn) {
    if (threadIdx.x < 2) pn_binary(G.dyn, threadIdx.x == 0 ? t + dtc : t - dtc, bhl[threadIdx.x]);
    __syncthreads();
  }
  const unsigned N0 = G.N[0], N1 = G.N[1];
  const unsigned total = (unsigned)G.capacity;
  const bool phys2 = (G.bc != 1);  // x2 boundaries physical (not periodic)
  const int N2S = HG_NGH, N2E = G.NE[1];
  double w1[4], w2[4];
  for (int d = 1; d < 4; d++) {
    w1[d] = G.invdx[d] / 6.;
    w2[d] = 4. * G.invdx[d] / 3.;
  }
  const double i2 = G.invdx[2];
  const double w_2lo[5] = {-0.5 * i2, -5. * i2 / 3., 3. * i2, -i2, i2 / 6.};
  const double w_2hi[5] = {-i2 / 6., i2, -3. * i2, 5. * i2 / 3., 0.5 * i2};
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const unsigned q = e / N0;
    const int i = HG_NGH + (int)(e - q * N0), j = HG_NGH + (int)(q % N1), k = HG_NGH + (int)(q / N1);
    // dg[sym(a, b)][c] = d_c gcov[a][b]: the stored gcov is symmetric, so the
    // 40 distinct derivatives stand for conn_func_fd4's 64 (the same values)
    constexpr int PA[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3}, PB[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
    double dg[10][4];
    {  // time component
      double gh[4][4], gl[4][4];
      dyn_gcov_func(G, 3, i, j, k, t + dtc, gh, pn ? &bhl[0] : nullptr);
      dyn_gcov_func(G, 3, i, j, k, t - dtc, gl, pn ? &bhl[1] : nullptr);
#pragma unroll
      for (int m = 0; m < 10; m++) dg[m][0] = (gh[PA[m]][PB[m]] - gl[PA[m]][PB[m]]) * half_inv_dt_conn;
    }
#pragma unroll
    for (int m = 0; m < 10; m++) {
      const int a = PA[m], b = PB[m];
      // x1: CENT i-1, FACE1 i, FACE1 i+1, CENT i+1
      dg[m][1] = w1[1] * (dyn_gcov_at(G, lv, 3, i - 1, j, k, a, b) - dyn_gcov_at(G, lv, 3, i + 1, j, k, a, b)) +
                 w2[1] * (dyn_gcov_at(G, lv, 0, i + 1, j, k, a, b) - dyn_gcov_at(G, lv, 0, i, j, k, a, b));
      if (phys2 && j == N2S) {
        dg[m][2] = w_2lo[0] * dyn_gcov_at(G, lv, 1, i, j, k, a, b) + w_2lo[1] * dyn_gcov_at(G, lv, 3, i, j, k, a, b) +
                   w_2lo[2] * dyn_gcov_at(G, lv, 1, i, j + 1, k, a, b) +
                   w_2lo[3] * dyn_gcov_at(G, lv, 3, i, j + 1, k, a, b) +
                   w_2lo[4] * dyn_gcov_at(G, lv, 1, i, j + 2, k, a, b);
      } else if (phys2 && j == N2E) {
        dg[m][2] = w_2hi[0] * dyn_gcov_at(G, lv, 1, i, j - 1, k, a, b) +
                   w_2hi[1] * dyn_gcov_at(G, lv, 3, i, j - 1, k, a, b) + w_2hi[2] * dyn_gcov_at(G, lv, 1, i, j, k, a, b) +
                   w_2hi[3] * dyn_gcov_at(G, lv, 3, i, j, k, a, b) + w_2hi[4] * dyn_gcov_at(G, lv, 1, i, j + 1, k, a, b);
      } else {
        dg[m][2] = w1[2] * (dyn_gcov_at(G, lv, 3, i, j - 1, k, a, b) - dyn_gcov_at(G, lv, 3, i, j + 1, k, a, b)) +
                   w2[2] * (dyn_gcov_at(G, lv, 1, i, j + 1, k, a, b) - dyn_gcov_at(G, lv, 1, i, j, k, a, b));
      }
      dg[m][3] = w1[3] * (dyn_gcov_at(G, lv, 3, i, j, k - 1, a, b) - dyn_gcov_at(G, lv, 3, i, j, k + 1, a, b)) +
                 w2[3] * (dyn_gcov_at(G, lv, 2, i, j, k + 1, a, b) - dyn_gcov_at(G, lv, 2, i, j, k, a, b));
    }
    // DGCOV_TO_CONN with tmp[l][b][cc] formed where it is used (the same
    // operations, without a second 64-entry array per thread)
    const long o = off3(G, i, j, k);
    const long oc = 3 * G.S + o;
    double gcon[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int l = 0; l < 4; l++) gcon[a][l] = lv[(HG_DP_GCON + dyn_sym(a, l)) * G.gS3 + oc];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int cc = b; cc < 4; cc++) {  // conn[a][cc][b] is the same double (HG_CONN3_PLANES)
          double v = 0.;
#pragma unroll
          for (int l = 0; l < 4; l++)
            v += gcon[a][l] * (0.5 * (dg[dyn_sym(b, l)][cc] + dg[dyn_sym(cc, l)][b] - dg[dyn_sym(cc, b)][l]));
          G.conn3[(a * 10 + dyn_sym(b, cc)) * G.S + o] = v;
        }
  }
}

// ---------------------------------------------------------------------------
// Host-side launch sequence of one step.
static void launch_geom_level(const GridDev &G, const LaunchCfg &L, cudaStream_t s, int slot, double tfac)
{
  k_geom_level<<<L.grid_upd, HG_BLK, 0, s>>>(G, slot, tfac);
}

static inline void mark(EventRec *r, int cls, cudaStream_t s)
{
  if (!r || r->n >= r->cap) return;
  r->cls[r->n] = cls;
  cudaEventRecord((cudaEvent_t)r->ev[r->n], s);
  r->n++;
}

// k_flux_strip keeps 16 * NF face states per thread in dynamic shared memory
// (16, 32 and 48 KiB per block for NF = 1, 2, 3; the limit is raised once
// per instantiation).  Longer strips save reconstruction work but their
// shared memory takes L1 capacity from the stencil loads: on the 192^3-class
// torus NF = 2 measured best, and hg_autotune chooses per grid.
template <bool RS, int MDIM, int d, int NF>
static void launch_strip_nf(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *ph, const int *lo,
                            const int *n, unsigned int mult, int slot)
{
  const size_t smem = sizeof(double) * 16 * NF * HG_BLK;
  k_flux_strip<RS, MDIM, d, NF>
      <<<L.grid_flux, HG_BLK, smem, s>>>(G, ph, lo[0], lo[1], lo[2], n[0], n[1], n[2], mult, slot);
}

template <bool RS, int MDIM, int d, int NF>
static cudaError_t strip_attr()
{
  return cudaFuncSetAttribute(k_flux_strip<RS, MDIM, d, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)(sizeof(double) * 16 * NF * HG_BLK));
}

template <bool RS, int MDIM>
static cudaError_t strip_attrs_rm()
{
  cudaError_t e = cudaSuccess;
  const cudaError_t r[9] = {strip_attr<RS, MDIM, 0, 1>(), strip_attr<RS, MDIM, 0, 2>(), strip_attr<RS, MDIM, 0, 3>(),
                            strip_attr<RS, MDIM, 1, 1>(), strip_attr<RS, MDIM, 1, 2>(), strip_attr<RS, MDIM, 1, 3>(),
                            strip_attr<RS, MDIM, 2, 1>(), strip_attr<RS, MDIM, 2, 2>(), strip_attr<RS, MDIM, 2, 3>()};
  for (cudaError_t x : r)
    if (x != cudaSuccess) e = x;
  return e;
}

// Blocks of k_fallback one SM holds at once.  Each queued zone is one long
// serial chain (nested Newton iterations), so the kernel is launched with
// every block the device holds: up to that many threads, each zone runs in a
// thread of its own instead of queueing behind another zone's chain.
int fallback_blocks_per_sm(bool rs)
{
  int n = 0;
  const cudaError_t e = rs ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fallback<true>, HG_BLK, 0)
                           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fallback<false>, HG_BLK, 0);
  if (e != cudaSuccess) cudaGetLastError();
  return (e == cudaSuccess && n > 0) ? n : 2;
}

// Kernel attributes that must be set before a launch (the strip kernels'
// shared memory above the default limit), once per device, outside any
// stream capture: called by hg_init.
cudaError_t prepare_kernels()
{
  const cudaError_t r[6] = {strip_attrs_rm<false, 0>(), strip_attrs_rm<true, 0>(), strip_attrs_rm<false, 2>(),
                            strip_attrs_rm<true, 2>(),  strip_attrs_rm<false, 3>(), strip_attrs_rm<true, 3>()};
  for (cudaError_t x : r)
    if (x != cudaSuccess) return x;
  return cudaSuccess;
}

// strips of L.strip_nf faces (1, 2 or 3: a launch-configuration choice)
template <bool RS, int MDIM, int d>
static void launch_strip(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *ph, const int *lo,
                         const int *n, unsigned int mult, int slot)
{
  if (L.strip_nf <= 1) launch_strip_nf<RS, MDIM, d, 1>(G, L, s, ph, lo, n, mult, slot);
  else if (L.strip_nf == 2) launch_strip_nf<RS, MDIM, d, 2>(G, L, s, ph, lo, n, mult, slot);
  else launch_strip_nf<RS, MDIM, d, 3>(G, L, s, ph, lo, n, mult, slot);
}

static void launch_flux_dir(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *ph, int d,
                            EventRec *R, int slot)
{
    int lo[3], n[3];
    unsigned int mult = 1;
    for (int a = 0; a < 3; a++) {
      if (G.deg[a]) {
        lo[a] = HG_NGH;
        n[a] = 1;
        mult *= (a == d) ? 2u : (G.ct_para ? 1u + 2u * HG_NGH : 3u);
      } else if (a == d) {
        lo[a] = HG_NGH;
        n[a] = G.N[a] + 1;
      } else if (G.ct_para) {
        lo[a] = 0;
        n[a] = G.N[a] + 2 * HG_NGH;
      } else {
        lo[a] = HG_NGH - 1;
        n[a] = G.N[a] + 2;
      }
    }
    mark(R, KC_FLUX, s);
    if (G.prec == HG_PREC_MIXED) {
      launch_flux_f32(G, L, s, d, lo, n, mult, slot);  // reads G.p32, filled from ph
      return;
    }
#define HG_FLUX(RSV, MD, DD) \
  k_flux<RSV, MD, DD><<<L.grid_flux, HG_BLK, 0, s>>>(G, ph, lo[0], lo[1], lo[2], n[0], n[1], n[2], mult, slot)
#define HG_STRIP(RSV, MD, DD) \
  launch_strip<RSV, MD, DD>(G, L, s, ph, lo, n, mult, slot)
#define HG_FLUX_D(RSV, MD) \
  if (d == 0) { if (G.deg[0] || !L.strip_x1) HG_FLUX(RSV, MD, 0); else HG_STRIP(RSV, MD, 0); } \
  else if (d == 1) { if (G.deg[1]) HG_FLUX(RSV, MD, 1); else HG_STRIP(RSV, MD, 1); } \
  else { if (G.deg[2]) HG_FLUX(RSV, MD, 2); else HG_STRIP(RSV, MD, 2); }
    if (G.mdim == 0) {
      if (G.rescale) { HG_FLUX_D(true, 0) }
      else { HG_FLUX_D(false, 0) }
    } else if (G.mdim == 3) {  // geometry of time level `slot`
      if (G.rescale) { HG_FLUX_D(true, 3) }
      else { HG_FLUX_D(false, 3) }
    } else {
      if (G.rescale) { HG_FLUX_D(true, 2) }
      else { HG_FLUX_D(false, 2) }
    }
#undef HG_FLUX_D
#undef HG_STRIP
#undef HG_FLUX
}

static void launch_substep(const GridDev &G, const LaunchCfg &L, cudaStream_t s, int sub, EventRec *R)
{
  const double *ph = sub == 0 ? G.p : G.ph;
  double *pf = sub == 0 ? G.ph : G.p;
  const double dtfac = sub == 0 ? 0.5 : 1.0;
  mark(R, KC_MISC, s);
  k_begin<<<1, 1, 0, s>>>(G.sc);
  // set_general_conn(t) before the predictor, set_general_conn(t + dx[0]/2)
  // before the corrector (step_ch.c:79-83, 128-133), from ncurr's level
  if (G.mdim == 3 && G.dyn.spacetime != HG_DYN_KS_SPHERICAL) {  // Kerr-Schild: static connection
    mark(R, KC_GEOM, s);
    k_conn_dyn<<<L.grid_upd, HG_BLK, 0, s>>>(G, sub, 0.5 * sub);
  }
  // (the mixed form's FP32 copy of ph is already current: put_state)
  for (int d = 0; d < 3; d++) launch_flux_dir(G, L, s, ph, d, R, sub);
  {
    int lo[3], n[3];
    for (int a = 0; a < 3; a++) {
      lo[a] = HG_NGH;
      n[a] = G.deg[a] ? 1 : G.N[a] + 1;
    }
    mark(R, KC_EMF, s);
    k_emf<<<L.grid_emf, HG_BLK, 0, s>>>(G, lo[0], lo[1], lo[2], n[0], n[1], n[2]);
  }
  mark(R, KC_UPDATE, s);
#define HG_UPD(RSV, MD)                                                                       \
  if (sub == 0) k_update_cons<RSV, MD, 0><<<L.grid_upd, HG_BLK, 0, s>>>(G, dtfac, ph);        \
  else k_update_cons<RSV, MD, 1><<<L.grid_upd, HG_BLK, 0, s>>>(G, dtfac, ph);                 \
  k_update_c2p<RSV, MD><<<L.grid_upd, HG_BLK, 0, s>>>(G, sub, pf)
  if (G.mdim == 0) {
    if (G.rescale) { HG_UPD(true, 0); }
    else { HG_UPD(false, 0); }
  } else if (G.mdim == 3) {
    if (G.rescale) { HG_UPD(true, 3); }
    else { HG_UPD(false, 3); }
  } else {
    if (G.rescale) { HG_UPD(true, 2); }
    else { HG_UPD(false, 2); }
  }
#undef HG_UPD
  mark(R, KC_FALLBACK, s);
  if (G.use_ee) {
    if (G.rescale) k_ee_faces<true><<<L.grid_fix * 6, HG_BLK, 0, s>>>(G, ph, sub);
    else k_ee_faces<false><<<L.grid_fix * 6, HG_BLK, 0, s>>>(G, ph, sub);
  }
  if (G.rescale) k_fallback<true><<<L.grid_fb, HG_BLK, 0, s>>>(G, sub, dtfac, ph, pf);
  else k_fallback<false><<<L.grid_fb, HG_BLK, 0, s>>>(G, sub, dtfac, ph, pf);
  mark(R, KC_BOUNDS, s);
  k_bounds<<<L.grid_bnd, HG_BLK, 0, s>>>(G, pf, 0, sub + 1);
  mark(R, KC_FIXUP, s);
  k_fixup<<<L.grid_fix, HG_BLK, 0, s>>>(G, pf, sub + 1);
  mark(R, KC_BOUNDS, s);
  k_bounds<<<L.grid_bnd, HG_BLK, 0, s>>>(G, pf, 1, sub + 1);
}

__global__ void k_reset_max(DevScalars *sc, int dim) { sc->maxs[dim] = 0ull; }

// ---------------------------------------------------------------------------
// Layout conversion between the reference's p[i][j][k][l] (NP innermost,
// every direction N+6 long) and the resident planes.  One thread per stored
// zone in the reference's order (k fastest), so the reference-side array is
// read/written in contiguous 64-byte runs.  A degenerate direction reads its
// one stored copy from the ghost-free reference index NG, and writes every
// reference copy of that direction.
__global__ void __launch_bounds__(HG_BLK) k_ref_to_planes(GridDev G, const double *__restrict__ ref, int NT1, int NT2,
                                                          double *__restrict__ out)
{
  const long total = G.S;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int k = (int)(t % G.T[2]);
    const int j = (int)((t / G.T[2]) % G.T[1]);
    const int i = (int)(t / ((long)G.T[2] * G.T[1]));
    const int ri = G.deg[0] ? HG_NGH : i, rj = G.deg[1] ? HG_NGH : j, rk = G.deg[2] ? HG_NGH : k;
    const double *src = ref + (((long)ri * NT1 + rj) * NT2 + rk) * HG_NPR;
    const long o = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) out[l * G.S + o] = src[l];
  }
}

__global__ void __launch_bounds__(HG_BLK) k_planes_to_ref(GridDev G, const double *__restrict__ in, int NT0, int NT1,
                                                          int NT2, double *__restrict__ ref)
{
  const long total = (long)NT0 * NT1 * NT2;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
    const int rk = (int)(t % NT2);
    const int rj = (int)((t / NT2) % NT1);
    const int ri = (int)(t / ((long)NT2 * NT1));
    const int i = G.deg[0] ? 0 : ri, j = G.deg[1] ? 0 : rj, k = G.deg[2] ? 0 : rk;
    const long o = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
    double *dst = ref + t * HG_NPR;
#pragma unroll
    for (int l = 0; l < HG_NPR; l++) dst[l] = in[l * G.S + o];
  }
}

// The same conversions when x1 and x3 both have ghosts (the usual 3D grid):
// the reference runs k fastest and the planes i fastest, so each block
// transposes a 32 (k) x 32 (i) tile of one x2 row through shared memory,
// four variables at a time; both sides are then read and written in
// contiguous runs.  grid (tiles of k, tiles of i, rows j), block (32, 8).
#define HG_TT 32
__global__ void __launch_bounds__(HG_TT * 8) k_ref_to_planes_tiled(GridDev G, const double *__restrict__ ref, int NT1,
                                                                 int NT2, double *__restrict__ out)
{
  __shared__ double tile[4][HG_TT][HG_TT + 1];
  const int k0 = blockIdx.x * HG_TT, i0 = blockIdx.y * HG_TT, j = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int T0 = G.T[0], T2 = G.T[2];
  const int rj = G.deg[1] ? HG_NGH : j;
  for (int lg = 0; lg < HG_NPR; lg += 4) {
    for (int ii = ty; ii < HG_TT; ii += 8) {
      const int i = i0 + ii, k = k0 + tx;
      if (i < T0 && k < T2) {
        const double *src = ref + (((long)i * NT1 + rj) * NT2 + k) * HG_NPR + lg;
#pragma unroll
        for (int v = 0; v < 4; v++) tile[v][tx][ii] = src[v];
      }
    }
    __syncthreads();
    for (int kk = ty; kk < HG_TT; kk += 8) {
      const int i = i0 + tx, k = k0 + kk;
      if (i < T0 && k < T2) {
        const long o = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
#pragma unroll
        for (int v = 0; v < 4; v++) out[(lg + v) * G.S + o] = tile[v][kk][tx];
      }
    }
    __syncthreads();
  }
}

// grid (tiles of k, tiles of i, reference rows rj over NT1), block (32, 8);
// a degenerate x2 reads its one stored row for every reference copy
__global__ void __launch_bounds__(HG_TT * 8) k_planes_to_ref_tiled(GridDev G, const double *__restrict__ in, int NT1,
                                                                 int NT2, double *__restrict__ ref)
{
  __shared__ double tile[4][HG_TT][HG_TT + 1];
  const int k0 = blockIdx.x * HG_TT, i0 = blockIdx.y * HG_TT, rj = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int T0 = G.T[0], T2 = G.T[2];
  const int j = G.deg[1] ? 0 : rj;
  for (int lg = 0; lg < HG_NPR; lg += 4) {
    for (int kk = ty; kk < HG_TT; kk += 8) {
      const int i = i0 + tx, k = k0 + kk;
      if (i < T0 && k < T2) {
        const long o = (long)i * G.st[0] + (long)j * G.st[1] + (long)k * G.st[2];
#pragma unroll
        for (int v = 0; v < 4; v++) tile[v][kk][tx] = in[(lg + v) * G.S + o];
      }
    }
    __syncthreads();
    for (int ii = ty; ii < HG_TT; ii += 8) {
      const int i = i0 + ii, k = k0 + tx;
      if (i < T0 && k < T2) {
        double *dst = ref + (((long)i * NT1 + rj) * NT2 + k) * HG_NPR + lg;
#pragma unroll
        for (int v = 0; v < 4; v++) dst[v] = tile[v][tx][ii];
      }
    }
    __syncthreads();
  }
}

void launch_ref_to_planes(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *ref, int NT1, int NT2,
                          double *out)
{
  if (!G.deg[0] && !G.deg[2] && G.T[1] <= 65535 && (G.T[0] + HG_TT - 1) / HG_TT <= 65535)
    k_ref_to_planes_tiled<<<dim3((G.T[2] + HG_TT - 1) / HG_TT, (G.T[0] + HG_TT - 1) / HG_TT, G.T[1]),
                            dim3(HG_TT, 8), 0, s>>>(G, ref, NT1, NT2, out);
  else
    k_ref_to_planes<<<L.grid_flux, HG_BLK, 0, s>>>(G, ref, NT1, NT2, out);
  if (G.p32 && out == G.p) launch_to_f32(G, L.grid_upd, s, G.p);  // the state set from the host
}

void launch_planes_to_ref(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *in, int NT0, int NT1,
                          int NT2, double *ref)
{
  if (!G.deg[0] && !G.deg[2] && NT1 <= 65535 && (G.T[0] + HG_TT - 1) / HG_TT <= 65535)
    k_planes_to_ref_tiled<<<dim3((G.T[2] + HG_TT - 1) / HG_TT, (G.T[0] + HG_TT - 1) / HG_TT, NT1), dim3(HG_TT, 8), 0,
                            s>>>(G, in, NT1, NT2, ref);
  else
    k_planes_to_ref<<<L.grid_flux, HG_BLK, 0, s>>>(G, in, NT0, NT1, NT2, ref);
}

// Fluxes of direction d from the resident primitives G.p (hg_face_flux).
void launch_face_flux(const GridDev &G, const LaunchCfg &L, cudaStream_t s, int d)
{
  k_reset_max<<<1, 1, 0, s>>>(G.sc, d + 1);
  if (G.prec == HG_PREC_MIXED) launch_to_f32(G, L.grid_upd, s, G.p);
  launch_flux_dir(G, L, s, G.p, d, nullptr, 0);
}

void launch_fixup_bounds(const GridDev &G, const LaunchCfg &L, cudaStream_t s)
{
  k_begin<<<1, 1, 0, s>>>(G.sc);
  k_fixup_cells<<<L.grid_upd, HG_BLK, 0, s>>>(G);
  k_bounds<<<L.grid_bnd, HG_BLK, 0, s>>>(G, G.p, 0, 0);
  if (G.p32) launch_to_f32(G, L.grid_upd, s, G.p);  // the FP32 copy of the state set from the host
}

// ---------------------------------------------------------------------------
// dump_ener()'s integrals (diag.c:704-815) of the last step and the largest
// divb_calc() (diag.c:503-612), per block; k_totals_final sums the blocks in
// order.  Layout of part / out: U[8], F[3][2][8] (direction, lower/upper
// boundary plane, variable; the induction components after flux-CT, from
// the EMFs as update_zone forms them), max |div B|.
#define HG_TOT 57
#define HG_TOT_BLOCKS 2048  // blocks of k_totals at most (its partials array)
__device__ __forceinline__ double ct_flux(const GridDev &G, int d, int l, long o)
{
  const double fac = G.ct_para ? 0.125 : 0.5;
  const double *E0 = G.emf[0], *E1 = G.emf[1], *E2 = G.emf[2];
  const long si = G.st[0], sj = G.st[1], sk = G.st[2];
  if (d == 0) {
    if (l == B2) return 0. + fac * (E2[o] + E2[o + sj]);
    if (l == B3) return 0. + (-fac) * (E1[o] + E1[o + sk]);
    return 0.;
  }
  if (d == 1) {
    if (l == B1) return 0. + (-fac) * (E2[o] + E2[o + si]);
    if (l == B3) return 0. + fac * (E0[o] + E0[o + sk]);
    return 0.;
  }
  if (l == B1) return 0. + fac * (E1[o] + E1[o + si]);
  if (l == B2) return 0. + (-fac) * (E0[o] + E0[o + sj]);
  return 0.;
}

__device__ __forceinline__ double divb_zone(const GridDev &G, int i, int j, int k)
{
  double f[3] = {0., 0., 0.};
#pragma unroll
  for (int di = -1; di <= 0; di++)
#pragma unroll
    for (int dj = -1; dj <= 0; dj++)
#pragma unroll
      for (int dk = -1; dk <= 0; dk++) {
        const long o = off3(G, i + di, j + dj, k + dk);
        double g;
        if (G.mdim == 0) g = G.g0.g;
        else if (G.mdim == 3) {
          const int L = G.sc->lev[0];
          g = (L == 0 ? G.geomL[0] : L == 1 ? G.geomL[1] : G.geomL[2])[HG_DP_G * G.gS3 + 3 * G.S + o];
        } else
          g = G.geomT[32 * G.gS + ((long)3 * G.T[1] + (G.deg[1] ? 0 : j + dj)) * G.T[0] + (G.deg[0] ? 0 : i + di)];
        const double b1 = G.p[B1 * G.S + o], b2 = G.p[B2 * G.S + o], b3 = G.p[B3 * G.S + o];
        f[0] += (di == 0 ? b1 : -b1) * g;
        f[1] += (dj == 0 ? b2 : -b2) * g;
        f[2] += (dk == 0 ? b3 : -b3) * g;
      }
  double divb = 0.;
  divb += f[0] * G.invdx[1];
  divb += f[1] * G.invdx[2];
  divb += f[2] * G.invdx[3];
  divb *= 0.25;
  return fabs(divb);
}

__global__ void __launch_bounds__(HG_BLK) k_totals(GridDev G, double *part)
{
  const int N0 = G.N[0], N1 = G.N[1], N2 = G.N[2];
  double u[HG_NPR], fs[48], dm = 0.;
  for (int l = 0; l < HG_NPR; l++) u[l] = 0.;
  for (int l = 0; l < 48; l++) fs[l] = 0.;
  const long zones = (long)N0 * N1 * N2;
  const long stride = (long)gridDim.x * blockDim.x;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < zones; t += stride) {
    const int i = HG_NGH + (int)(t % N0), j = HG_NGH + (int)((t / N0) % N1), k = HG_NGH + (int)(t / ((long)N0 * N1));
    const long o = off3(G, i, j, k);
    for (int l = 0; l < HG_NPR; l++) u[l] += G.Uc[l * G.S + o];
    const double v = divb_zone(G, i, j, k);
    dm = v > dm ? v : dm;
  }
  // boundary face planes: d = 0 (j,k), d = 1 (i,k), d = 2 (i,j)
  const long n_a[3] = {(long)N1 * N2, (long)N0 * N2, (long)N0 * N1};
  for (int d = 0; d < 3; d++)
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n_a[d]; t += stride) {
      int i, j, k;
      if (d == 0) { i = HG_NGH; j = HG_NGH + (int)(t % N1); k = HG_NGH + (int)(t / N1); }
      else if (d == 1) { i = HG_NGH + (int)(t % N0); j = HG_NGH; k = HG_NGH + (int)(t / N0); }
      else { i = HG_NGH + (int)(t % N0); j = HG_NGH + (int)(t / N0); k = HG_NGH; }
      for (int side = 0; side < 2; side++) {
        const int ii = (d == 0 && side) ? N0 + HG_NGH : i, jj = (d == 1 && side) ? N1 + HG_NGH : j;
        const int kk = (d == 2 && side) ? N2 + HG_NGH : k;
        const long o = off3(G, ii, jj, kk);
        for (int l = 0; l < HG_NPR; l++)
          fs[(d * 2 + side) * HG_NPR + l] += (l >= B1) ? ct_flux(G, d, l, o) : G.F[d][l * G.S + o];
      }
    }
  for (int l = 0; l < HG_NPR; l++) {
    const double b = block_sum(u[l]);
    if (threadIdx.x == 0) part[blockIdx.x * HG_TOT + l] = b;
  }
  for (int l = 0; l < 48; l++) {
    const double b = block_sum(fs[l]);
    if (threadIdx.x == 0) part[blockIdx.x * HG_TOT + 8 + l] = b;
  }
  __shared__ double red[HG_BLK / 32];
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const double w = __shfl_down_sync(0xffffffffu, dm, s);
    dm = w > dm ? w : dm;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dm;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
    for (int w = 1; w < HG_BLK / 32; w++) m = red[w] > m ? red[w] : m;
    part[blockIdx.x * HG_TOT + 56] = m;
  }
}

__global__ void k_totals_final(GridDev G, const double *part, int nblk, double *out)
{
  const int m = threadIdx.x;
  if (m >= HG_TOT) return;
  double s = 0.;
  for (int b = 0; b < nblk; b++) {
    const double v = part[b * HG_TOT + m];
    if (m == 56) s = v > s ? v : s;
    else s += v;
  }
  if (m < 8) s *= G.dx[1] * G.dx[2] * G.dx[3];
  else if (m < 56) {
    const int d = (m - 8) / 16;
    s *= d == 0 ? G.dx[2] * G.dx[3] : d == 1 ? G.dx[1] * G.dx[3] : G.dx[1] * G.dx[2];
  }
  out[m] = s;
}

void launch_totals(const GridDev &G, const LaunchCfg &L, cudaStream_t s, double *part, double *out)
{
  const int nb = L.grid_upd < HG_TOT_BLOCKS ? L.grid_upd : HG_TOT_BLOCKS;
  k_totals<<<nb, HG_BLK, 0, s>>>(G, part);
  k_totals_final<<<1, 64, 0, s>>>(G, part, nb, out);
}

// t, dx[0] and the error status of every member of a batch, for one copy
__global__ void k_gather_times(DevScalars *const *sc, int n, double *out)
{
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    out[3 * m] = sc[m]->t;
    out[3 * m + 1] = sc[m]->dt;
    out[3 * m + 2] = (double)sc[m]->err;
  }
}

void *gather_times_kernel() { return (void *)k_gather_times; }

void launch_bounds_only(const GridDev &G, const LaunchCfg &L, cudaStream_t s)
{
  k_begin<<<1, 1, 0, s>>>(G.sc);
  k_bounds<<<L.grid_bnd, HG_BLK, 0, s>>>(G, G.p, 0, 0);
  if (G.p32) launch_to_f32(G, L.grid_upd, s, G.p);
}

void launch_step(const GridDev &G, const LaunchCfg &L, cudaStream_t s, EventRec *R)
{
  launch_substep(G, L, s, 0, R);
  launch_substep(G, L, s, 1, R);
  mark(R, KC_MISC, s);
  k_timestep<<<1, 1024, 0, s>>>(G, L.grid_upd);
  if (G.mdim == 3) {  // advance_geometry() at the end of step_ch() (step_ch.c:225-227)
    mark(R, KC_GEOM, s);
    k_advance_geometry<<<1, 1, 0, s>>>(G.sc);
    launch_geom_level(G, L, s, 1, 0.5);
    launch_geom_level(G, L, s, 2, 1.0);
  }
  mark(R, KC_END, s);
}

// conn3 of the physical zones from rows (j + N1 i) of 64 that do not depend
// on k (a static axisymmetric connection)
__global__ void k_conn_broadcast(GridDev G, const double *rows)
{
  const unsigned N0 = G.N[0], N1 = G.N[1];
  for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < (unsigned)G.capacity; e += gridDim.x * blockDim.x) {
    const unsigned q = e / N0;
    const int ip = (int)(e - q * N0), jp = (int)(q % N1), kp = (int)(q / N1);
    const long o = off3(G, HG_NGH + ip, HG_NGH + jp, HG_NGH + kp);
    const double *r = rows + 64L * (jp + (long)N1 * ip);
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++)
        for (int c = b; c < 4; c++) G.conn3[(a * 10 + dyn_sym(b, c)) * G.S + o] = r[(a * 4 + b) * 4 + c];
  }
}

void launch_conn_broadcast(const GridDev &G, const LaunchCfg &L, cudaStream_t s, const double *rows)
{
  k_conn_broadcast<<<L.grid_upd, HG_BLK, 0, s>>>(G, rows);
}

// all three time levels at t (init_general_metric, metric.c:3664-3690)
void launch_geom_levels(const GridDev &G, const LaunchCfg &L, cudaStream_t s)
{
  launch_geom_level(G, L, s, 0, 0.0);
  launch_geom_level(G, L, s, 1, 0.5);
  launch_geom_level(G, L, s, 2, 1.0);
}

}  // namespace HG_KNS

#ifndef HG_FMA_BUILD

// ===========================================================================
// hg_face_flux_noalloc: hg_face_flux for callers that cannot allocate device
// memory.  Its only scratch -- the per-block maxima of the characteristic
// speed and a completion counter -- lives in the file-scope array below, so
// every GPU that loads the library holds it (256 KiB + 256 B) until exit.
// Host code never dereferences hg_na_scratch: it is a host-side stand-in for
// the symbol, and a kernel given its host address would fault or read the
// wrong memory.  Its device address comes from cudaGetSymbolAddress with the
// device current: looked up again on every call made outside stream capture
// (so a cudaDeviceReset, which reloads the module at a new address, is
// followed), and taken from the last lookup on that device during capture.
// ===========================================================================
namespace hg {

#define HG_NA_MAX_BLOCKS 32768  // one block per 128 faces: at most 4,194,304 faces per call
static __device__ __align__(256) unsigned long long hg_na_scratch[HG_NA_MAX_BLOCKS + 32];
static unsigned long long *hg_na_dev_ptr[64];  // last looked-up device address of hg_na_scratch, per device

// face_flux() without the failure bookkeeping (the caller gets fluxes only).
__device__ __forceinline__ double face_flux_na(const GridDev &G, const double *pl, const double *pr, const Geom &g,
                                               int d, double *__restrict__ Fd, long o)
{
  const int dim = d + 1;
  State ql, qr;
  get_state(pl, g, G.gam, ql);
  get_state(pr, g, G.gam, qr);
  double cmaxl, cminl, cmaxr, cminr;
  vchar_fast(ql, g, dim, G.gam, &cmaxl, &cminl);
  vchar_fast(qr, g, dim, G.gam, &cmaxr, &cminr);
  const double a0 = 0. > cmaxl ? 0. : cmaxl;
  const double cmax = fabs(a0 > cmaxr ? a0 : cmaxr);
  const double a1 = 0. > -cminl ? 0. : -cminl;
  const double cmin = fabs(a1 > -cminr ? a1 : -cminr);
  const double ctop = cmin > cmax ? cmin : cmax;
  const double gg = g.g;
#pragma unroll
  for (int l = 0; l < HG_NPR; l++) {
    const double Ul = flux_comp(pl, ql, 0, gg, l), Ur = flux_comp(pr, qr, 0, gg, l);
    const double Fl = flux_comp(pl, ql, dim, gg, l), Fr = flux_comp(pr, qr, dim, gg, l);
    Fd[l * G.S + o] = (G.flux == 1) ? (cmax * Fl + cmin * Fr - cmax * cmin * (Ur - Ul)) / (cmax + cmin + HG_SMALL)
                                    : 0.5 * (Fl + Fr - ctop * (Ur - Ul));
  }
  return ctop;
}

// One thread per face, one block per 128 faces; each block leaves its maximum
// in scratch[block], the last block to finish reduces them.
template <int d>
__global__ void __launch_bounds__(HG_BLK) k_flux_noalloc(const __grid_constant__ GridDev G,
                                                         const double *__restrict__ prims, int lo0, int lo1, int lo2,
                                                         int n0, int n1, int n2, double *max_out,
                                                         unsigned long long *scratch)
{
  // total <= HG_NA_MAX_BLOCKS * HG_BLK faces: the entry point rejects larger calls
  const unsigned total = (unsigned)n0 * n1 * n2;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  double vmax = 0.;
  if (t < total) {
    const int i = lo0 + (int)(t % n0);
    const int j = lo1 + (int)((t / n0) % n1);
    const int k = lo2 + (int)(t / ((long)n0 * n1));
    double pl[HG_NPR], pr[HG_NPR];
    face_prims<false>(G, prims, d, i, j, k, pl, pr);
    const double ctop = face_flux_na(G, pl, pr, G.g0, d, G.F[d], off3(G, i, j, k));
    if (i >= HG_NGH && i <= G.NE[0] && j >= HG_NGH && j <= G.NE[1] && k >= HG_NGH && k <= G.NE[2])
      if (ctop > vmax) vmax = ctop;
  }
  __shared__ double red[HG_BLK / 32];
  __shared__ bool last;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_down_sync(0xffffffffu, vmax, o);
    vmax = w > vmax ? w : vmax;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
  __syncthreads();
  unsigned long long *counter = scratch + HG_NA_MAX_BLOCKS;
  if (threadIdx.x == 0) {
    double m = red[0];
    for (int w = 1; w < HG_BLK / 32; w++) m = red[w] > m ? red[w] : m;
    scratch[blockIdx.x] = (unsigned long long)__double_as_longlong(m);
    __threadfence();
    last = (atomicAdd(counter, 1ull) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double m = 0.;
  for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    const double v = __longlong_as_double((long long)__ldcg(scratch + b));
    m = v > m ? v : m;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_down_sync(0xffffffffu, m, o);
    m = w > m ? w : m;
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < HG_BLK / 32; w++) m = red[w] > m ? red[w] : m;
    *max_out = m;
    *counter = 0ull;  // leave the counter at zero for the next call
  }
}

}  // namespace hg

#include <mutex>

#include "harmgpu.h"

extern "C" int hg_face_flux_noalloc(const hg_grid_desc *d, const double *geom, const double *prims, double *flux,
                                    double *max_char_speed, int32_t dir, void *stream)
{
  using namespace hg;
  if (!d || !geom || !prims || !flux || !max_char_speed || dir < 0 || dir > 2) return HG_ERR_BADARG;
  if (d->metric_dim != 0 || d->rescale_r != 0 || d->n1 < 2 || d->n2 < 2 || d->n3 < 2) return HG_ERR_BADARG;
  if (d->recon_type < 0 || d->recon_type > 5 || (d->flux_type != 0 && d->flux_type != 1)) return HG_ERR_BADARG;
  const int n[3] = {d->n1, d->n2, d->n3};
  int lo[3], cnt[3];
  for (int a = 0; a < 3; a++) {  // numerical_flux()'s face ranges (step_ch.c:668-675)
    if (a == dir) {
      lo[a] = HG_NGH;
      cnt[a] = n[a] + 1;
    } else if (d->use_flux_ct_para) {
      lo[a] = 0;
      cnt[a] = n[a] + 2 * HG_NGH;
    } else {
      lo[a] = HG_NGH - 1;
      cnt[a] = n[a] + 2;
    }
  }
  const long faces = (long)cnt[0] * cnt[1] * cnt[2];
  const long blocks = (faces + HG_BLK - 1) / HG_BLK;
  if (blocks > HG_NA_MAX_BLOCKS) {
    fprintf(stderr, "hg_face_flux_noalloc: %ld faces exceed the limit of %d faces per call\n", faces,
            HG_NA_MAX_BLOCKS * HG_BLK);
    return HG_ERR_BADARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HG_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return HG_ERR_CUDA;
  unsigned long long *scratch = nullptr;
  {
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (cap == cudaStreamCaptureStatusNone || !hg_na_dev_ptr[dev]) {
      // the address of the array on the current device (allocates nothing)
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, hg_na_scratch);
      if (e != cudaSuccess || !p) {
        fprintf(stderr, "hg_face_flux_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return HG_ERR_CUDA;
      }
      hg_na_dev_ptr[dev] = (unsigned long long *)p;
    }
    scratch = hg_na_dev_ptr[dev];
  }
  // the reference layout: variable innermost, k, j, i outermost
  GridDev G;
  memset(&G, 0, sizeof(G));
  const long st2 = HG_NPR, st1 = st2 * (n[2] + 2 * HG_NGH), st0 = st1 * (n[1] + 2 * HG_NGH);
  G.st[0] = st0;
  G.st[1] = st1;
  G.st[2] = st2;
  G.S = 1;
  for (int a = 0; a < 3; a++) {
    G.N[a] = n[a];
    G.T[a] = n[a] + 2 * HG_NGH;
    G.NE[a] = n[a] + HG_NGH - 1;
  }
  G.recon = d->recon_type;
  G.flux = d->flux_type;
  G.gam = d->gam;
  G.F[dir] = flux;
  Geom &g = G.g0;
  memcpy(g.gcon, geom, 16 * 8);
  memcpy(g.gcov, geom + 16, 16 * 8);
  g.g = geom[32];
  g.g_inv = geom[33];
  g.alpha = geom[34];
  for (int a = 0; a < 3; a++) g.beta[a] = geom[35 + a];
  for (int a = 0; a < 4; a++) g.ncon[a] = geom[38 + a];
  if (cudaMemsetAsync(scratch + HG_NA_MAX_BLOCKS, 0, sizeof(unsigned long long), s) != cudaSuccess)
    return HG_ERR_CUDA;
  if (dir == 0)
    k_flux_noalloc<0><<<(unsigned)blocks, HG_BLK, 0, s>>>(G, prims, lo[0], lo[1], lo[2], cnt[0], cnt[1], cnt[2],
                                                          max_char_speed, scratch);
  else if (dir == 1)
    k_flux_noalloc<1><<<(unsigned)blocks, HG_BLK, 0, s>>>(G, prims, lo[0], lo[1], lo[2], cnt[0], cnt[1], cnt[2],
                                                          max_char_speed, scratch);
  else
    k_flux_noalloc<2><<<(unsigned)blocks, HG_BLK, 0, s>>>(G, prims, lo[0], lo[1], lo[2], cnt[0], cnt[1], cnt[2],
                                                          max_char_speed, scratch);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "hg_face_flux_noalloc: launch failed: %s\n", cudaGetErrorString(e));
    return HG_ERR_CUDA;
  }
  return HG_OK;
}

#endif  // HG_FMA_BUILD
