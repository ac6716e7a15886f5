/// @file cuda_solver.hpp
/// @brief Source-compatible adrt::cuda batched API (BatchConfig, DeviceData,
///        solveBatch, solveBatchHost), served by the B200 engine.
///
/// Mirrors the reference's src_cuda/cuda_solver.cuh:18-98: the same structs,
/// field meanings and defaults, FP32 device arrays in the SoA layout
/// array[wav * stride + layer_or_level], TOA flux_up (times
/// spectrum_scaling), TOA flux_down and BOA flux_direct outputs.
///
/// Differences a caller may notice:
///   * solveBatch allocates nothing after the first call at a given size,
///     never synchronises the host, and is stream ordered;
///   * errors are reported (std::invalid_argument for invalid input,
///     std::runtime_error for CUDA failures) where the reference is silent;
///   * BatchConfig::precision selects the engine's precision form (the field
///     is new; its default keeps old callers compiling);
///   * the discrete scheme is the reference's CPU scheme (first-order start,
///     per-layer doubling counts, delta-M scaled beam), so results agree with
///     adrt::solve rather than with the reference GPU kernels.
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace adrt {
namespace cuda {

/// Precision form of the engine (adrt_precision in include/adrt_b200.h).
enum class Precision : int { FP64 = 0, Mixed = 1 };

/// Solver configuration (scalars shared across all wavenumbers).
struct BatchConfig {
  int num_wavenumbers = 0;
  int num_layers = 0;
  int num_quadrature = 8;   ///< N, 2..32
  int num_moments_max = 0;  ///< Legendre moments per set

  bool use_delta_m = false;
  bool use_thermal_emission = false;
  bool use_diffusion_lower_bc = false;

  double surface_albedo = 0.0;
  double surface_emission = 0.0;
  double surface_temperature = -1.0;
  double top_emission = 0.0;
  double top_temperature = -1.0;
  double solar_flux = 0.0;
  double solar_mu = 1.0;

  double wavenumber_low = 0.0;
  double wavenumber_high = 0.0;

  double spectrum_scaling = 1.0;  ///< applied to flux_up only

  Precision precision = Precision::FP64;
};

/// Device memory pointers (caller-owned), SoA layout.
struct DeviceData {
  const float* delta_tau;           ///< [nwav * nlay]
  const float* single_scat_albedo;  ///< [nwav * nlay]
  const float* phase_moments;       ///< [nwav * nlay * nmom] or [nlay * nmom]
  bool phase_moments_shared = false;

  const float* temperature = nullptr;    ///< [nwav * nlev] (thermal) or nullptr
  const float* planck_levels = nullptr;  ///< [nwav * nlev] or nullptr

  const float* surface_emission = nullptr;  ///< [nwav] or nullptr
  const float* top_emission = nullptr;      ///< [nwav] or nullptr

  float* flux_up = nullptr;      ///< [nwav] TOA upward flux (x spectrum_scaling)
  float* flux_down = nullptr;    ///< [nwav] TOA downward flux
  float* flux_direct = nullptr;  ///< [nwav] direct solar flux at the surface
};

/// Stream-ordered batched solve on the current device.  Uses a per-thread,
/// per-device engine that is created on the first call.
void solveBatch(const BatchConfig& config, const DeviceData& data, cudaStream_t stream = 0);

struct HostResult {
  std::vector<float> flux_up;
  std::vector<float> flux_down;
  std::vector<float> flux_direct;
};

/// Host-vector convenience wrapper (copies in, solves, copies out).
HostResult solveBatchHost(const BatchConfig& config, const std::vector<float>& delta_tau,
                          const std::vector<float>& single_scat_albedo,
                          const std::vector<float>& phase_moments, bool phase_moments_shared,
                          const std::vector<float>& planck_levels,
                          const std::vector<float>& temperature = {});

}  // namespace cuda
}  // namespace adrt
