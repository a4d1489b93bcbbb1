// FMA-throughput microbenchmark: the FP64 and FP32 CUDA-core peaks that the roofline of the
// step kernels is reported against (measured on the device the kernels run on).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <string>

#include "../../include/kerrray_cuda.h"

namespace {

constexpr int kChains = 8;

template <class T>
__global__ void k_fma_chains(T* __restrict__ sink, int iters, T b, T c) {
  T a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == (T)-1.2345) sink[threadIdx.x] = s;  // never true for these inputs; keeps the chains live
}

template <class T>
int measure(int device, double* tflops) {
  if (cudaSetDevice(device) != cudaSuccess) return KRR_ERR_NO_DEVICE;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  T* sink = nullptr;
  if (cudaMalloc(&sink, 1024 * sizeof(T)) != cudaSuccess) return KRR_ERR_CUDA;
  const int block = 256, grid = sms * 8, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const T b = (T)0.999999, c = (T)1e-7;
  k_fma_chains<T><<<grid, block>>>(sink, 256, b, c);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    k_fma_chains<T><<<grid, block>>>(sink, iters, b, c);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    best = std::min(best, ms);
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) return KRR_ERR_CUDA;
  const double flops = 2.0 * (double)grid * block * kChains * (double)iters;
  *tflops = flops / (best * 1e-3) / 1e12;
  return KRR_OK;
}

}  // namespace

extern "C" KRR_API int krr_fma_peak(int device, int fp64, double* tflops) {
  if (!tflops) return KRR_ERR_INVALID;
  return fp64 ? measure<double>(device, tflops) : measure<float>(device, tflops);
}
