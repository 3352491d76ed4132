// Measured arithmetic peaks used as roofline denominators for the CUDA-core kernels: long
// chains of independent fused multiply-adds (8 accumulators per thread, 4 resident blocks of
// 256 threads per SM), timed with CUDA events, best of several launches.

#include <cstdio>

#include "rds_internal.h"

namespace
{

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(T *out, T a, T b, int iters)
{
  T x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k)
    x[k] = T(threadIdx.x + k) * T(1e-7);
  for (int i = 0; i < iters; ++i)
  {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      x[k] = fma(x[k], a, b);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    s += x[k];
  if (s == T(-1234.5)) // never true; keeps the chains alive
    out[0] = s;
}

} // namespace

extern "C" RDS_API rds_status rds_measure_peak(int precision, double *tflops)
{
  if (!tflops)
    return RDS_ERR_INVALID;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return RDS_ERR_CUDA;
  void *out = nullptr;
  if (cudaMalloc(&out, 16) != cudaSuccess)
    return RDS_ERR_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int blocks = sms * 4, threads = 256, iters = 1 << 14;
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep)
  {
    cudaEventRecord(e0);
    if (precision == RDS_FP64)
      fma_chains<double><<<blocks, threads>>>((double *)out, 0.999999, 1e-9, iters);
    else
      fma_chains<float><<<blocks, threads>>>((float *)out, 0.999999f, 1e-9f, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best)
      best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess)
    return RDS_ERR_CUDA;
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  *tflops            = flops / (best * 1e-3) / 1e12;
  return RDS_OK;
}
