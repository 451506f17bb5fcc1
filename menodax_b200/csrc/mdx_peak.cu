// Measured CUDA-core FMA throughput, the roofline denominator for the ensemble
// kernels: they are bound by FP64 (and, for the LU, FP32) issue on the CUDA
// cores, not by HBM and not by the tensor cores.  Eight independent FMA chains
// per thread over a device-filling grid, timed with CUDA events.
#include <cuda_runtime.h>

#include "../../include/menodax.h"

namespace {

template <typename T>
__global__ void fma_chains(T* out, int iters, T b, T c) {
  T a0 = (T)threadIdx.x, a1 = a0 + (T)1, a2 = a0 + (T)2, a3 = a0 + (T)3;
  T a4 = a0 + (T)4, a5 = a0 + (T)5, a6 = a0 + (T)6, a7 = a0 + (T)7;
#pragma unroll 4
  for (int i = 0; i < iters; ++i) {
    a0 = a0 * b + c; a1 = a1 * b + c; a2 = a2 * b + c; a3 = a3 * b + c;
    a4 = a4 * b + c; a5 = a5 * b + c; a6 = a6 * b + c; a7 = a7 * b + c;
  }
  const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == (T)-1.2345) out[blockIdx.x] = s;  // keeps the chains live; never true
}

template <typename T>
int measure(double* flops_per_s) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MDX_E_CUDA;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MDX_E_CUDA;
  const int threads = 256, blocks = sms * 8, iters = 1 << 14;
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T) * blocks) != cudaSuccess) return MDX_E_CUDA;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_chains<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    fma_chains<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return MDX_E_CUDA;
  *flops_per_s = 2.0 * 8.0 * (double)iters * threads * blocks / (best * 1e-3);
  return MDX_OK;
}

}  // namespace

extern "C" int mdx_measure_fma_peak(int double_precision, double* flops_per_s) {
  if (!flops_per_s) return MDX_E_INVALID;
  return double_precision ? measure<double>(flops_per_s) : measure<float>(flops_per_s);
}
