// adrt_probe.cu -- FMA-throughput probe: the FP64 and FP32 CUDA-core peaks
// that bound the solver (its products and eliminations run on the FMA pipes).
#include <cuda_runtime.h>

#include "../../include/adrt_b200.h"

namespace {

template <typename T, int CHAINS>
__global__ void fma_probe_kernel(T* out, int iters, T a, T b) {
  T acc[CHAINS];
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) acc[c] = T(threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) acc[c] = fma(acc[c], a, b);
  }
  T s = T(0);
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) s += acc[c];
  if (s == T(12345.678)) out[0] = s;  // keeps the chains live
}

template <typename T>
double run_probe(int sms) {
  constexpr int kChains = 8, kThreads = 256;
  const int blocks = sms * 8, iters = 1 << 14;
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const T a = T(0.999999), b = T(1e-7);
  fma_probe_kernel<T, kChains><<<blocks, kThreads>>>(out, iters, a, b);  // warm-up
  cudaEventRecord(e0);
  fma_probe_kernel<T, kChains><<<blocks, kThreads>>>(out, iters, a, b);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
  const double flops = 2.0 * blocks * kThreads * (double)iters * kChains;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

extern "C" int adrt_probe_fma_tflops(double* fp64_tflops, double* fp32_tflops) {
  if (!fp64_tflops || !fp32_tflops) return ADRT_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ADRT_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  *fp64_tflops = run_probe<double>(sms);
  *fp32_tflops = run_probe<float>(sms);
  return (*fp64_tflops > 0 && *fp32_tflops > 0) ? ADRT_OK : ADRT_ERR_CUDA;
}
