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

// ---------------------------------------------------------------- raw inputs
/// Raw retrieval inputs (caller-owned device memory), as the reference's
/// RawDeviceData (src_cuda/cuda_solver.cuh:104-133): coefficient arrays are
/// level-major, array[level * nwav + wav], with the bottom of the atmosphere
/// at level 0; the phase moments keep the solver's top-first layer order.
struct RawDeviceData {
  const float* absorption_coeff;     ///< [nlev * nwav] absorption coefficient (cm^-1)
  const float* scattering_coeff;     ///< [nlev * nwav] scattering coefficient (cm^-1)
  const float* altitude;             ///< [nlev] altitude (cm), bottom first
  const float* temperature;          ///< [nlev] temperature (K), bottom first
  const double* wavenumber;          ///< [nwav] wavenumber (cm^-1)

  const float* phase_moments;        ///< [nlay * nmom] or [nwav * nlay * nmom]
  bool phase_moments_shared = false;

  const float* cloud_optical_depth = nullptr;  ///< [nlay * nwav] or nullptr

  float* flux_up = nullptr;      ///< [nwav] TOA upward flux (x spectrum_scaling)
  float* flux_down = nullptr;    ///< [nwav] TOA downward flux
  float* flux_direct = nullptr;  ///< [nwav] direct solar flux at the surface, or nullptr
};

/// Workspace of the reference's preprocessing path
/// (src_cuda/cuda_solver.cuh:137-156), kept for source compatibility.  The
/// engine forms optical depths, albedos and Planck levels inside its solve and
/// needs no intermediate arrays: allocate() only records the dimensions, and
/// the pointers stay null.
struct SolverWorkspaceGPU {
  float* delta_tau = nullptr;           ///< [nwav * nlay]
  float* single_scat_albedo = nullptr;  ///< [nwav * nlay]
  float* planck_levels = nullptr;       ///< [nwav * nlev]
  float* surface_emission = nullptr;    ///< [nwav]
  float* top_emission = nullptr;        ///< [nwav]
  int allocated_nwav = 0;
  int allocated_nlay = 0;

  void allocate(int nwav, int nlay);
  void free();
  ~SolverWorkspaceGPU() { free(); }
};

/// Solve from raw coefficients (src_cuda/cuda_solver.cuh:166-169): optical
/// depths by the trapezoid rule over altitude plus the cloud optical depth,
/// single-scattering albedos and single-wavenumber Planck levels are formed in
/// the solve.  Any N (the reference's overload without a workspace takes N <= 8).
void solveBatchFromCoefficients(const BatchConfig& config, const RawDeviceData& data,
                                cudaStream_t stream = 0);

/// The reference's workspace overload (src_cuda/cuda_solver.cuh:175-179): same
/// results as the overload without a workspace.
void solveBatchFromCoefficients(const BatchConfig& config, const RawDeviceData& data,
                                SolverWorkspaceGPU& workspace, cudaStream_t stream = 0);

}  // namespace cuda
}  // namespace adrt
