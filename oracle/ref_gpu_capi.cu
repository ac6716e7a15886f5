// TEST INFRASTRUCTURE (the comparison bar, never linked into the product):
// C entry point around the reference's own GPU solver,
// adrt::cuda::solveBatch (src_cuda/cuda_solver.cu:858-1003, and for N > 8
// solveBatchedCublas, src_cuda/cuda_batched_solver.cu:753-997), compiled
// unmodified from the reference sources with the reference's own CUDA flags
// (--use_fast_math, CMakeLists.txt:88-93) by `make -C oracle ref-gpu`.
//
// ref_gpu_time_batch() takes a batch in this library's host layout (FP64,
// include/adrt_b200.h), converts it to the reference's DeviceData (FP32,
// src_cuda/cuda_solver.cuh:42-68), calls solveBatch `warmup` times untimed
// and `steps` times between CUDA events on one stream, and returns the mean
// time of a call and the reference's TOA outputs.  The reference API has one
// scalar surface albedo, solar angle and Planck band per call
// (cuda_solver.cuh:18-40): per-wavenumber arrays are refused, so the caller
// passes a batch of scalar options.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../include/adrt_b200.h"
#include "cuda_solver.cuh"

namespace {
std::string g_err;

template <typename T>
struct DevBuf {
  T* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  bool put(const std::vector<float>& h) {
    if (cudaMalloc(&p, h.size() * sizeof(T)) != cudaSuccess) return false;
    return cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
  }
  bool alloc(size_t n) { return cudaMalloc(&p, n * sizeof(T)) == cudaSuccess; }
};

int fail(const char* msg) {
  g_err = msg;
  return -1;
}
}  // namespace

extern "C" const char* ref_gpu_last_error(void) { return g_err.c_str(); }

extern "C" int ref_gpu_time_batch(const adrt_batch_desc* d, const adrt_inputs* in, int steps,
                                  int warmup, double* ms_per_call, double* toa_fu,
                                  double* toa_fd, double* boa_fdir) {
  if (!d || !in || !ms_per_call || steps < 1) return fail("bad arguments");
  if (in->surface_albedo || in->solar_mu || in->wavenumber_low || in->wavenumber_high ||
      in->surface_emission || in->top_emission || d->index_from_bottom)
    return fail("the reference API takes scalar albedo, solar angle, band and emissions only");
  const size_t W = d->num_wavenumbers, L = d->num_layers, M = d->num_moments, lev = L + 1;
  adrt::cuda::BatchConfig c;
  c.num_wavenumbers = (int)W;
  c.num_layers = (int)L;
  c.num_quadrature = d->num_quadrature;
  c.num_moments_max = (int)M;
  c.use_delta_m = d->use_delta_m != 0;
  c.use_thermal_emission = d->use_thermal_emission != 0;
  c.use_diffusion_lower_bc = d->use_diffusion_lower_bc != 0;
  c.surface_albedo = d->surface_albedo;
  c.surface_emission = d->surface_emission;
  c.surface_temperature = d->surface_temperature;
  c.top_emission = d->top_emission;
  c.top_temperature = d->top_temperature;
  c.solar_flux = d->solar_flux;
  c.solar_mu = d->solar_mu;
  c.wavenumber_low = d->wavenumber_low;
  c.wavenumber_high = d->wavenumber_high;
  c.spectrum_scaling = d->spectrum_scaling;

  std::vector<float> tau(W * L), ssa(W * L);
  for (size_t i = 0; i < W * L; ++i) {
    tau[i] = (float)in->delta_tau[i];
    ssa[i] = (float)in->single_scat_albedo[i];
  }
  const bool shared = d->moment_layout == ADRT_MOMENTS_SHARED;
  std::vector<float> mom(shared ? L * M : W * L * M);
  for (size_t w = 0; w < (shared ? 1 : W); ++w)
    for (size_t l = 0; l < L; ++l)
      for (size_t m = 0; m < M; ++m) {
        const size_t src = d->moment_layout == ADRT_MOMENTS_SHARED ? l * M + m
                           : d->moment_layout == ADRT_MOMENTS_PER_WAVENUMBER
                               ? w * M + m
                               : (w * L + l) * M + m;
        mom[(w * L + l) * M + m] = (float)in->phase_moments[src];
      }
  std::vector<float> temp, planck;
  if (d->use_thermal_emission) {
    if (!in->temperature) return fail("temperature missing");
    temp.resize(W * lev);
    for (size_t w = 0; w < W; ++w)
      for (size_t l = 0; l < lev; ++l)
        temp[w * lev + l] =
            (float)in->temperature[(d->temperature_per_wavenumber ? w * lev : 0) + l];
  } else if (in->planck_levels) {
    planck.resize(W * lev);
    for (size_t i = 0; i < W * lev; ++i) planck[i] = (float)in->planck_levels[i];
  }

  DevBuf<float> dtau, dssa, dmom, dtemp, dpl, dfu, dfd, dfdir;
  if (!dtau.put(tau) || !dssa.put(ssa) || !dmom.put(mom) ||
      (!temp.empty() && !dtemp.put(temp)) || (!planck.empty() && !dpl.put(planck)) ||
      !dfu.alloc(W) || !dfd.alloc(W) || !dfdir.alloc(W))
    return fail("device allocation or upload failed");
  adrt::cuda::DeviceData dd;
  dd.delta_tau = dtau.p;
  dd.single_scat_albedo = dssa.p;
  dd.phase_moments = dmom.p;
  dd.phase_moments_shared = shared;
  dd.temperature = dtemp.p;
  dd.planck_levels = dpl.p;
  dd.flux_up = dfu.p;
  dd.flux_down = dfd.p;
  dd.flux_direct = dfdir.p;

  cudaStream_t s;
  if (cudaStreamCreate(&s) != cudaSuccess) return fail("stream creation failed");
  for (int i = 0; i < warmup; ++i) adrt::cuda::solveBatch(c, dd, s);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaStreamSynchronize(s);
  cudaEventRecord(e0, s);
  for (int i = 0; i < steps; ++i) adrt::cuda::solveBatch(c, dd, s);
  cudaEventRecord(e1, s);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const cudaError_t err = cudaGetLastError();
  cudaStreamDestroy(s);
  if (err != cudaSuccess) return fail(cudaGetErrorString(err));
  *ms_per_call = ms / steps;
  std::vector<float> h(W);
  double* outs[3] = {toa_fu, toa_fd, boa_fdir};
  float* devs[3] = {dfu.p, dfd.p, dfdir.p};
  for (int k = 0; k < 3; ++k) {
    if (!outs[k]) continue;
    if (cudaMemcpy(h.data(), devs[k], W * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
      return fail("output copy failed");
    for (size_t w = 0; w < W; ++w) outs[k][w] = h[w];
  }
  return 0;
}
