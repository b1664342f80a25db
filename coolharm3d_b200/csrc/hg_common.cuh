// hg_common.cuh -- device helpers shared by the FP64 kernels (hg_kernels.cu)
// and the FP32 flux kernel of the mixed-precision form (hg_mixed.cu).
#pragma once
#include "hg_phys.cuh"

namespace hg {

#define HG_BLK 128

__device__ __forceinline__ int rs_type(int l) { return l == RHO ? 0 : (l == UU ? 2 : 1); }

// One value of the state written at plane offset `at` (l * S + o).  The
// mixed form keeps the FP32 copy its flux kernels read in step with every
// write, so no conversion pass runs before each substep: whichever array a
// step kernel writes (ph in the predictor, p in the corrector) is the next
// substep's flux input.
__device__ __forceinline__ void put_state(const GridDev &G, double *a, long at, double v)
{
  a[at] = v;
  if (G.p32) G.p32[at] = (float)v;
}

__device__ __forceinline__ void block_max_atomic(double v, unsigned long long *dst)
{
  __shared__ double red[HG_BLK / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double w = __shfl_down_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = red[0];
    for (int w = 1; w < HG_BLK / 32; w++) m = red[w] > m ? red[w] : m;
    // the maximum only grows: skip the atomic when it cannot raise it
    if (m > 0. && m > __longlong_as_double((long long)*(volatile unsigned long long *)dst))
      atomicMax(dst, (unsigned long long)__double_as_longlong(m));
  }
}

// FAIL_GAMMA_CALC at a face: the reference computes each face once per ghost
// copy of a degenerate direction (numerical_flux's ranges), booking it once
// per copy; mult is that number of copies.
__device__ __forceinline__ void book_face(const GridDev &G, int i, int j, int k, unsigned int mult)
{
  atomicAdd(&G.nfail[NF_GAMMA_CALC * G.S + off3(G, i, j, k)], mult);
  atomicAdd(&G.sc->nfailtot[NF_GAMMA_CALC], (unsigned long long)mult);
}

}  // namespace hg
