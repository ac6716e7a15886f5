// adrt_probe.cu -- throughput probes: the FP64 and FP32 CUDA-core FMA peaks,
// and the warp-level tensor-core peaks (DMMA f64, TF32 and BF16 mma.sync) of
// the instructions the solver's products and right-solves issue.
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

// Warp-level tensor-core throughput: CHAINS independent accumulators per
// warp, every lane's operands fixed (the values do not matter for the rate).
template <int KIND, int CHAINS>
__global__ void mma_probe_kernel(float* out, int iters, unsigned seed) {
  const unsigned a0 = (seed ^ threadIdx.x) & 0x3f80ffffu, a1 = (a0 * 3u) & 0x3f80ffffu;
  const unsigned a2 = (a0 * 5u) & 0x3f80ffffu, a3 = (a0 * 7u) & 0x3f80ffffu;
  const unsigned b0 = (a0 * 11u) & 0x3f80ffffu, b1 = (a0 * 13u) & 0x3f80ffffu;
  float acc[CHAINS][4];
  double dacc[CHAINS][2];
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) {
    acc[c][0] = acc[c][1] = acc[c][2] = acc[c][3] = 0.f;
    dacc[c][0] = dacc[c][1] = 0.0;
  }
  const double da = 1.0 + 1e-9 * threadIdx.x, db = 0.5;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) {
      if constexpr (KIND == 0) {
        asm volatile(
            "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+f"(acc[c][0]), "+f"(acc[c][1]), "+f"(acc[c][2]), "+f"(acc[c][3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
      } else if constexpr (KIND == 1) {
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
            "{%8,%9}, {%0,%1,%2,%3};\n"
            : "+f"(acc[c][0]), "+f"(acc[c][1]), "+f"(acc[c][2]), "+f"(acc[c][3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
      } else {
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(dacc[c][0]), "+d"(dacc[c][1])
                     : "d"(da), "d"(db));
      }
    }
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < CHAINS; ++c)
    s += acc[c][0] + acc[c][1] + acc[c][2] + acc[c][3] + (float)(dacc[c][0] + dacc[c][1]);
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}

template <int KIND>
double run_mma_probe(int sms) {
  constexpr int kChains = 4, kThreads = 256;
  const int blocks = sms * 4, iters = (KIND == 2) ? (1 << 12) : (1 << 14);
  // flops per warp-level instruction
  const double per = KIND == 0 ? 2.0 * 16 * 8 * 8 : KIND == 1 ? 2.0 * 16 * 8 * 16 : 2.0 * 8 * 8 * 4;
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  mma_probe_kernel<KIND, kChains><<<blocks, kThreads>>>(out, iters, 12345u);  // warm-up
  cudaEventRecord(e0);
  mma_probe_kernel<KIND, kChains><<<blocks, kThreads>>>(out, iters, 12345u);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
  const double warps = (double)blocks * kThreads / 32.0;
  return warps * iters * kChains * per / (ms * 1e-3) / 1e12;
}

}  // namespace

extern "C" int adrt_probe_mma_tflops(double* fp64_dmma_tflops, double* tf32_tflops,
                                     double* bf16_tflops) {
  if (!fp64_dmma_tflops || !tf32_tflops || !bf16_tflops) return ADRT_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ADRT_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  *fp64_dmma_tflops = run_mma_probe<2>(sms);
  *tf32_tflops = run_mma_probe<0>(sms);
  *bf16_tflops = run_mma_probe<1>(sms);
  return (*fp64_dmma_tflops > 0 && *tf32_tflops > 0 && *bf16_tflops > 0) ? ADRT_OK : ADRT_ERR_CUDA;
}

extern "C" int adrt_probe_fma_tflops(double* fp64_tflops, double* fp32_tflops) {
  if (!fp64_tflops || !fp32_tflops) return ADRT_ERR_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return ADRT_ERR_CUDA;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  *fp64_tflops = run_probe<double>(sms);
  *fp32_tflops = run_probe<float>(sms);
  return (*fp64_tflops > 0 && *fp32_tflops > 0) ? ADRT_OK : ADRT_ERR_CUDA;
}
