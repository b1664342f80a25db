// hg_peak.cu -- the device's FP64 peak, measured: the denominator of the
// step's FP64 roofline fraction (achieved FP64 operations per second over
// the rate a kernel that does nothing but FP64 fused multiply-adds reaches).
//
// k_fp64_peak: every thread runs HG_PK_CHAINS independent multiply-add chains
// (a = a*b + c) for `iters` iterations, so the FP64 pipe always has
// independent work; one fma counts as two FP64 operations.  The grid fills
// every SM with 4 blocks of 256 threads.  The chains' results are summed into
// `sink` so that no work can be dropped by the compiler.
#include <cuda_runtime.h>

#include <cstdio>

#include "harmgpu.h"

namespace hg {

#define HG_PK_CHAINS 8
#define HG_PK_BLOCK 256

__global__ void __launch_bounds__(HG_PK_BLOCK) k_fp64_peak(double b, double c, int iters, double *sink)
{
  double a[HG_PK_CHAINS];
#pragma unroll
  for (int q = 0; q < HG_PK_CHAINS; q++) a[q] = (double)(threadIdx.x + q) * 1e-3;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < HG_PK_CHAINS; q++) a[q] = fma(a[q], b, c);
  }
  double s = 0.;
#pragma unroll
  for (int q = 0; q < HG_PK_CHAINS; q++) s += a[q];
  if (s == 12345.678) *sink = s;  // never true for these inputs; keeps the chains live
}

}  // namespace hg

extern "C" int hg_fp64_peak(int32_t device, double *tflops, double *ms)
{
  if (!tflops) return HG_ERR_BADARG;
  if (cudaSetDevice(device) != cudaSuccess) return HG_ERR_CUDA;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return HG_ERR_CUDA;
  double *sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStream_t s = nullptr;
  int rc = HG_ERR_CUDA;
  const int blocks = 4 * sms, iters = 1 << 14;
  float best = 1e30f;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess || cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
    goto done;
  for (int rep = 0; rep < 6; rep++) {  // the first launch warms up; the best of the rest counts
    if (cudaEventRecord(e0, s) != cudaSuccess) goto done;
    hg::k_fp64_peak<<<blocks, HG_PK_BLOCK, 0, s>>>(1.0000001, 1e-9, iters, sink);
    if (cudaGetLastError() != cudaSuccess || cudaEventRecord(e1, s) != cudaSuccess ||
        cudaEventSynchronize(e1) != cudaSuccess)
      goto done;
    float t = 0.f;
    if (cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) goto done;
    if (rep > 0 && t < best) best = t;
  }
  *tflops = 2.0 * HG_PK_CHAINS * (double)iters * blocks * HG_PK_BLOCK / (best * 1e-3) / 1e12;
  if (ms) *ms = best;
  rc = HG_OK;
done:
  if (rc != HG_OK) {
    fprintf(stderr, "hg_fp64_peak: %s\n", cudaGetErrorString(cudaGetLastError()));
  }
  if (s) cudaStreamDestroy(s);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (sink) cudaFree(sink);
  return rc;
}
