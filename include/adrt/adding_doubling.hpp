/// @file adding_doubling.hpp
/// @brief Source-compatible adrt::ADConfig / adrt::RTOutput / adrt::solve,
///        served by the B200 engine through the C ABI (include/adrt_b200.h).
///
/// Mirrors the reference's public CPU API (src/adding_doubling.hpp:32-298):
/// the same fields, defaults, validation messages and per-interface output
/// layout.  solve() runs one column on the GPU (a batch of one wavenumber).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

namespace adrt {

/// Results per interface: index 0 = top of atmosphere, index num_layers =
/// bottom (src/adding_doubling.hpp:32-50).
struct RTOutput {
  std::vector<double> flux_up;
  std::vector<double> flux_down;
  std::vector<double> mean_intensity;   ///< includes the direct beam
  std::vector<double> flux_divergence;  ///< 4 pi (1 - omega)(J - B), layer above
  std::vector<double> flux_direct;
  /// Temperature Jacobians [L+1][L+2] (levels 0..L, then the surface skin
  /// temperature) when ADConfig::compute_temperature_jacobian is set.
  std::vector<std::vector<double>> flux_up_temperature_jac;
  std::vector<std::vector<double>> flux_down_temperature_jac;
  std::vector<std::vector<double>> mean_intensity_temperature_jac;
  std::vector<std::vector<double>> flux_divergence_temperature_jac;
};

/// Column configuration (src/adding_doubling.hpp:63-247).
class ADConfig {
 public:
  int num_layers = 0;
  int num_quadrature = 8;

  bool use_thermal_emission = false;
  bool use_delta_m = false;
  bool use_diffusion_lower_bc = false;
  bool index_from_bottom = false;
  bool compute_temperature_jacobian = false;

  double surface_albedo = 0.0;
  double surface_emission = 0.0;
  double surface_temperature = -1.0;
  double top_emission = 0.0;
  double top_temperature = -1.0;
  double solar_flux = 0.0;
  double solar_mu = 1.0;

  double wavenumber_low = 0.0;
  double wavenumber_high = 0.0;

  std::vector<double> delta_tau;
  std::vector<double> single_scat_albedo;
  std::vector<double> temperature;
  std::vector<double> planck_levels;
  std::vector<std::vector<double>> phase_function_moments;

  ADConfig() = default;
  ADConfig(int nlyr, int nquad = 8) : num_layers(nlyr), num_quadrature(nquad) {}

  void allocate();
  /// @throws std::invalid_argument with the reference's messages.
  void validate() const;

  void setHenyeyGreenstein(double g, int lc = -1);
  void setDoubleHenyeyGreenstein(double f, double g1, double g2, int lc = -1);
  void setIsotropic(int lc = -1);
  void setRayleigh(int lc = -1);
};

/// Reusable per-thread workspace (src/workspace.hpp:17-48): here it owns a
/// GPU engine (device work buffers), created on first use.
class SolverWorkspace {
 public:
  SolverWorkspace();
  ~SolverWorkspace();
  SolverWorkspace(const SolverWorkspace&) = delete;
  SolverWorkspace& operator=(const SolverWorkspace&) = delete;
  void clear();
  void* engine();  ///< the adrt_engine* (C ABI handle)

 private:
  void* engine_ = nullptr;
};

RTOutput solve(const ADConfig& config);
RTOutput solve(const ADConfig& config, SolverWorkspace& workspace);

/// Gauss-Legendre nodes/weights on [0,1] (src/quadrature.cpp:11-51).
void gaussLegendre(int n, std::vector<double>& nodes, std::vector<double>& weights);

/// Band-integrated Planck function (src/planck.cpp:35-131), host evaluation.
double planckFunction(double wnumlo, double wnumhi, double temp);

/// Its temperature derivative (src/planck.cpp:135-175).
double planckFunctionDeriv(double wnumlo, double wnumhi, double temp);

}  // namespace adrt
