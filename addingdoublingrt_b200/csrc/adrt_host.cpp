// adrt_host.cpp -- the reference's C++ API (adrt::ADConfig / adrt::solve /
// adrt::cuda::solveBatch) implemented over the engine's C ABI.
//
// Built into libadrt_host.so, which links libadrt_b200.so; plain host C++,
// no CUDA code.  Validation messages, defaults and output layouts follow the
// reference (src/adding_doubling.hpp:32-298, src_cuda/cuda_solver.cuh:18-98).
#include <algorithm>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "adrt/adding_doubling.hpp"
#include "adrt/constants.hpp"
#include "adrt/cuda_solver.hpp"
#include "adrt_b200.h"

namespace adrt {
namespace {

[[noreturn]] void raise(int rc) {
  const std::string detail = adrt_last_status_detail();
  if (rc == ADRT_ERR_INVALID_ARGUMENT || rc == ADRT_ERR_UNSUPPORTED)
    throw std::invalid_argument(detail);
  throw std::runtime_error("adrt engine error " + std::to_string(rc) + ": " + detail);
}

void check(int rc) {
  if (rc != ADRT_OK) raise(rc);
}

template <class F>
void for_layers(int num_layers, int lc, F f) {
  const int start = (lc < 0) ? 0 : lc;
  const int end = (lc < 0) ? num_layers : lc + 1;
  for (int l = start; l < end; ++l) f(l);
}

}  // namespace

// ---------------------------------------------------------------- ADConfig
// allocate(), validate() and the phase helpers keep the reference's
// semantics and messages (src/adding_doubling.hpp:96-245).
void ADConfig::allocate() {
  delta_tau.assign(num_layers, 0.0);
  single_scat_albedo.assign(num_layers, 0.0);
  const int nmom = use_delta_m ? 2 * num_quadrature + 1 : 2 * num_quadrature;
  phase_function_moments.assign(num_layers, std::vector<double>(nmom, 0.0));
  for (auto& pm : phase_function_moments) pm[0] = 1.0;
  if (use_thermal_emission) temperature.assign(num_layers + 1, 0.0);
}

void ADConfig::validate() const {
  if (num_layers <= 0) throw std::invalid_argument("ADConfig: num_layers must be > 0");
  if (num_quadrature < 2) throw std::invalid_argument("ADConfig: num_quadrature must be >= 2");
  if (static_cast<int>(delta_tau.size()) != num_layers)
    throw std::invalid_argument("ADConfig: delta_tau size mismatch");
  if (static_cast<int>(single_scat_albedo.size()) != num_layers)
    throw std::invalid_argument("ADConfig: single_scat_albedo size mismatch");
  if (static_cast<int>(phase_function_moments.size()) != num_layers)
    throw std::invalid_argument("ADConfig: phase_function_moments size mismatch");
  for (int l = 0; l < num_layers; ++l) {
    if (delta_tau[l] < 0.0)
      throw std::invalid_argument("ADConfig: delta_tau[" + std::to_string(l) + "] < 0");
    if (single_scat_albedo[l] < 0.0 || single_scat_albedo[l] > 1.0)
      throw std::invalid_argument("ADConfig: single_scat_albedo[" + std::to_string(l) +
                                  "] out of [0,1]");
  }
  if (surface_albedo < 0.0 || surface_albedo > 1.0)
    throw std::invalid_argument("ADConfig: surface_albedo out of [0,1]");
  if (solar_flux > 0.0 && (solar_mu <= 0.0 || solar_mu > 1.0))
    throw std::invalid_argument("ADConfig: solar_mu must be in (0,1] when solar_flux > 0");
  if (use_thermal_emission) {
    if (static_cast<int>(temperature.size()) != num_layers + 1)
      throw std::invalid_argument("ADConfig: temperature size must be num_layers+1");
    for (int l = 0; l <= num_layers; ++l)
      if (temperature[l] < 0.0)
        throw std::invalid_argument("ADConfig: temperature[" + std::to_string(l) + "] < 0");
    if (wavenumber_low < 0.0 || wavenumber_high < wavenumber_low)
      throw std::invalid_argument("ADConfig: invalid wavenumber range");
  } else if (surface_temperature >= 0.0) {
    throw std::invalid_argument(
        "ADConfig: surface_temperature requires use_thermal_emission "
        "(use surface_emission for raw thermal sources)");
  } else if (top_temperature >= 0.0) {
    throw std::invalid_argument(
        "ADConfig: top_temperature requires use_thermal_emission "
        "(use top_emission for raw thermal sources)");
  }
  if (use_diffusion_lower_bc && !use_thermal_emission &&
      static_cast<int>(planck_levels.size()) != num_layers + 1)
    throw std::invalid_argument(
        "ADConfig: use_diffusion_lower_bc requires use_thermal_emission or planck_levels");
}

void ADConfig::setHenyeyGreenstein(double g, int lc) {
  for_layers(num_layers, lc, [&](int l) {
    double gk = 1.0;
    for (auto& m : phase_function_moments[l]) {
      m = gk;
      gk *= g;
    }
  });
}

void ADConfig::setDoubleHenyeyGreenstein(double f, double g1, double g2, int lc) {
  for_layers(num_layers, lc, [&](int l) {
    double g1k = 1.0, g2k = 1.0;
    for (auto& m : phase_function_moments[l]) {
      m = f * g1k + (1.0 - f) * g2k;
      g1k *= g1;
      g2k *= g2;
    }
  });
}

void ADConfig::setIsotropic(int lc) {
  for_layers(num_layers, lc, [&](int l) {
    auto& pm = phase_function_moments[l];
    std::fill(pm.begin(), pm.end(), 0.0);
    pm[0] = 1.0;
  });
}

void ADConfig::setRayleigh(int lc) {
  for_layers(num_layers, lc, [&](int l) {
    auto& pm = phase_function_moments[l];
    std::fill(pm.begin(), pm.end(), 0.0);
    pm[0] = 1.0;
    if (pm.size() > 2) pm[2] = 0.1;
  });
}

// ---------------------------------------------------------------- workspace
SolverWorkspace::SolverWorkspace() = default;
SolverWorkspace::~SolverWorkspace() { clear(); }

void SolverWorkspace::clear() {
  if (engine_) adrt_engine_destroy(static_cast<adrt_engine*>(engine_));
  engine_ = nullptr;
}

void* SolverWorkspace::engine() {
  if (!engine_) {
    adrt_engine_opts opts{-1, 0};
    adrt_engine* e = nullptr;
    check(adrt_engine_create(&opts, &e));
    engine_ = e;
  }
  return engine_;
}

// ---------------------------------------------------------------- solve
// One column = a batch of one wavenumber in FP64; per-layer moments of
// unequal length are zero-padded to the longest, which leaves the phase sums
// and the delta-M truncation fraction of every layer unchanged.
namespace {

// ADConfig::compute_temperature_jacobian (src/solver.cpp:117-341).  Row k of
// the Jacobian of F_up, F_down or J is the gradient of that output at
// interface k, so all 3 (L+1) rows come from one batched adjoint over copies
// of the column, each with a unit cotangent on its own output (temperatures,
// or Planck levels, per copy so the gradients stay apart).  Columns 0..L are
// the level temperatures (Planck levels without thermal emission), column
// L+1 the surface skin temperature when the surface radiates independently
// of the bottom level.  The flux-divergence rows follow from the J rows,
// divF_k = 4 pi (1 - omega) (J_k - B_k).
void temperature_jacobian(const ADConfig& c, adrt_batch_desc d, const std::vector<double>& moments,
                          adrt_engine* e, RTOutput& r) {
  const int L = c.num_layers, nint = L + 1, ndof = L + 2, K = 3 * nint;
  const bool thermal = c.use_thermal_emission;
  const bool planck_mode = !thermal && (int)c.planck_levels.size() == L + 1;
  double Bs = c.surface_emission;
  if (thermal) {
    const double Ts = c.surface_temperature >= 0.0 ? c.surface_temperature : c.temperature[
        c.index_from_bottom ? 0 : L];
    Bs = planckFunction(c.wavenumber_low, c.wavenumber_high, Ts);
  }
  const bool has_surface = !c.use_diffusion_lower_bc && (c.surface_albedo > 0.0 || Bs > 0.0);
  const bool surf_indep = has_surface && (thermal ? c.surface_temperature >= 0.0 : planck_mode);

  d.num_wavenumbers = K;
  d.moment_layout = ADRT_MOMENTS_SHARED;
  d.temperature_per_wavenumber = 1;
  auto rep = [&](const std::vector<double>& v) {
    std::vector<double> o((size_t)K * v.size());
    for (int k = 0; k < K; ++k) std::copy(v.begin(), v.end(), o.begin() + (size_t)k * v.size());
    return o;
  };
  const std::vector<double> dt = rep(c.delta_tau), om = rep(c.single_scat_albedo);
  const std::vector<double> src =
      rep(thermal ? c.temperature
                  : (planck_mode ? c.planck_levels : std::vector<double>(L + 1, 0.0)));
  adrt_inputs in{};
  in.delta_tau = dt.data();
  in.single_scat_albedo = om.data();
  in.phase_moments = moments.data();
  (thermal ? in.temperature : in.planck_levels) = src.data();
  std::vector<double> cot[3];
  for (int o = 0; o < 3; ++o) cot[o].assign((size_t)K * nint, 0.0);
  for (int row = 0; row < K; ++row) cot[row / nint][(size_t)row * nint + row % nint] = 1.0;
  adrt_cotangents ct{};
  ct.flux_up = cot[0].data();
  ct.flux_down = cot[1].data();
  ct.mean_intensity = cot[2].data();
  std::vector<double> g((size_t)K * nint, 0.0), gs(K, 0.0);
  adrt_gradients gr{};
  (thermal ? gr.temperature : gr.planck_levels) = g.data();
  gr.surface_emission = gs.data();
  check(adrt_adjoint_host(e, &d, &in, &ct, &gr));

  double ts_chain = 0.0;  // dB/dT at the skin temperature
  if (thermal && surf_indep) {
    check(adrt_planck_band_deriv(c.wavenumber_low, c.wavenumber_high, c.surface_temperature,
                                 &ts_chain));
  }
  std::vector<std::vector<double>>* J[3] = {&r.flux_up_temperature_jac,
                                            &r.flux_down_temperature_jac,
                                            &r.mean_intensity_temperature_jac};
  for (int o = 0; o < 3; ++o) J[o]->assign(nint, std::vector<double>(ndof, 0.0));
  const int bottom = c.index_from_bottom ? 0 : L;  // the bottom level's column
  for (int row = 0; row < K; ++row) {
    std::vector<double>& jr = (*J[row / nint])[row % nint];
    for (int m = 0; m <= L; ++m) jr[m] = g[(size_t)row * nint + m];
    if (surf_indep)
      jr[L + 1] = thermal ? gs[row] * ts_chain : gs[row];
    else if (has_surface && !thermal)
      jr[bottom] += gs[row];  // the surface source counts as the bottom level's
  }
  // divF_k = 4 pi (1 - omega_lyr) (J_k - B_k), lyr = the layer above interface k
  // (layer 0 at the top), in the caller's order
  auto& Jd = r.flux_divergence_temperature_jac;
  Jd.assign(nint, std::vector<double>(ndof, 0.0));
  for (int k = 0; k < nint; ++k) {
    const int ki = c.index_from_bottom ? L - k : k;  // top-first interface
    const int li = (ki == 0) ? 0 : ki - 1;
    const int lyr = c.index_from_bottom ? L - 1 - li : li;
    const double pref = 4.0 * PI * (1.0 - c.single_scat_albedo[lyr]);
    double chain_k = 1.0;  // dB_k / d(column k)
    if (thermal)
      check(adrt_planck_band_deriv(c.wavenumber_low, c.wavenumber_high, c.temperature[k],
                                   &chain_k));
    for (int m = 0; m < ndof; ++m)
      Jd[k][m] = pref * (r.mean_intensity_temperature_jac[k][m] - (m == k ? chain_k : 0.0));
  }
}

}  // namespace

RTOutput solve(const ADConfig& config, SolverWorkspace& workspace) {
  config.validate();
  const int L = config.num_layers;
  size_t M = 1;
  for (const auto& pm : config.phase_function_moments) M = std::max(M, pm.size());
  std::vector<double> moments((size_t)L * M, 0.0);
  for (int l = 0; l < L; ++l)
    std::copy(config.phase_function_moments[l].begin(), config.phase_function_moments[l].end(),
              moments.begin() + (size_t)l * M);

  adrt_batch_desc d{};
  d.num_wavenumbers = 1;
  d.num_layers = L;
  d.num_quadrature = config.num_quadrature;
  d.num_moments = (int)M;
  d.moment_layout = ADRT_MOMENTS_PER_LAYER;
  d.precision = ADRT_PRECISION_FP64;
  d.use_thermal_emission = config.use_thermal_emission;
  d.use_delta_m = config.use_delta_m;
  d.use_diffusion_lower_bc = config.use_diffusion_lower_bc;
  d.index_from_bottom = config.index_from_bottom;
  d.temperature_per_wavenumber = 0;
  d.surface_albedo = config.surface_albedo;
  d.surface_emission = config.surface_emission;
  d.surface_temperature = config.surface_temperature;
  d.top_emission = config.top_emission;
  d.top_temperature = config.top_temperature;
  d.solar_flux = config.solar_flux;
  d.solar_mu = config.solar_mu;
  d.wavenumber_low = config.wavenumber_low;
  d.wavenumber_high = config.wavenumber_high;
  d.spectrum_scaling = 1.0;

  adrt_inputs in{};
  in.delta_tau = config.delta_tau.data();
  in.single_scat_albedo = config.single_scat_albedo.data();
  in.phase_moments = moments.data();
  if (config.use_thermal_emission) in.temperature = config.temperature.data();
  if (!config.use_thermal_emission && (int)config.planck_levels.size() == L + 1)
    in.planck_levels = config.planck_levels.data();

  RTOutput r;
  r.flux_up.assign(L + 1, 0.0);
  r.flux_down.assign(L + 1, 0.0);
  r.mean_intensity.assign(L + 1, 0.0);
  r.flux_divergence.assign(L + 1, 0.0);
  r.flux_direct.assign(L + 1, 0.0);
  adrt_outputs out{};
  out.flux_up = r.flux_up.data();
  out.flux_down = r.flux_down.data();
  out.flux_direct = r.flux_direct.data();
  out.mean_intensity = r.mean_intensity.data();
  out.flux_divergence = r.flux_divergence.data();
  check(adrt_solve_batch_host(static_cast<adrt_engine*>(workspace.engine()), &d, &in, &out));
  if (config.compute_temperature_jacobian)
    temperature_jacobian(config, d, moments, static_cast<adrt_engine*>(workspace.engine()), r);
  return r;
}

RTOutput solve(const ADConfig& config) {
  thread_local SolverWorkspace ws;
  return solve(config, ws);
}

void gaussLegendre(int n, std::vector<double>& nodes, std::vector<double>& weights) {
  nodes.assign(n, 0.0);
  weights.assign(n, 0.0);
  check(adrt_gauss_legendre(n, nodes.data(), weights.data()));
}

double planckFunction(double wnumlo, double wnumhi, double temp) {
  double v = 0.0;
  check(adrt_planck_band(wnumlo, wnumhi, temp, &v));
  return v;
}

double planckFunctionDeriv(double wnumlo, double wnumhi, double temp) {
  double v = 0.0;
  check(adrt_planck_band_deriv(wnumlo, wnumhi, temp, &v));
  return v;
}

// ---------------------------------------------------------------- adrt::cuda
namespace cuda {
namespace {

adrt_engine* thread_engine() {
  thread_local std::unordered_map<int, SolverWorkspace> per_device;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cudaGetDevice failed");
  return static_cast<adrt_engine*>(per_device[dev].engine());
}

// The reference's temperature and planck_levels arrays are per wavenumber.
adrt_batch_desc to_desc(const BatchConfig& c, bool shared) {
  adrt_batch_desc d{};
  d.num_wavenumbers = c.num_wavenumbers;
  d.num_layers = c.num_layers;
  d.num_quadrature = c.num_quadrature;
  d.num_moments = c.num_moments_max;
  d.moment_layout = shared ? ADRT_MOMENTS_SHARED : ADRT_MOMENTS_PER_LAYER;
  d.precision = static_cast<int>(c.precision);
  d.use_thermal_emission = c.use_thermal_emission;
  d.use_delta_m = c.use_delta_m;
  d.use_diffusion_lower_bc = c.use_diffusion_lower_bc;
  d.index_from_bottom = 0;
  d.temperature_per_wavenumber = 1;
  d.surface_albedo = c.surface_albedo;
  d.surface_emission = c.surface_emission;
  d.surface_temperature = c.surface_temperature;
  d.top_emission = c.top_emission;
  d.top_temperature = c.top_temperature;
  d.solar_flux = c.solar_flux;
  d.solar_mu = c.solar_mu;
  d.wavenumber_low = c.wavenumber_low;
  d.wavenumber_high = c.wavenumber_high;
  d.spectrum_scaling = c.spectrum_scaling;
  return d;
}

}  // namespace

void solveBatch(const BatchConfig& config, const DeviceData& data, cudaStream_t stream) {
  const adrt_batch_desc d = to_desc(config, data.phase_moments_shared);
  adrt_inputs_f32 in{};
  in.delta_tau = data.delta_tau;
  in.single_scat_albedo = data.single_scat_albedo;
  in.phase_moments = data.phase_moments;
  in.temperature = config.use_thermal_emission ? data.temperature : nullptr;
  in.planck_levels = config.use_thermal_emission ? nullptr : data.planck_levels;
  in.surface_emission = data.surface_emission;
  in.top_emission = data.top_emission;
  adrt_outputs_f32 out{};
  out.toa_flux_up = data.flux_up;
  out.toa_flux_down = data.flux_down;
  out.boa_flux_direct = data.flux_direct;
  check(adrt_solve_batch_f32(thread_engine(), &d, &in, &out, stream));
}

void solveBatchFromCoefficients(const BatchConfig& config, const RawDeviceData& data,
                                cudaStream_t stream) {
  const adrt_batch_desc d = to_desc(config, data.phase_moments_shared);
  adrt_raw_inputs in{};
  in.absorption_coeff = data.absorption_coeff;
  in.scattering_coeff = data.scattering_coeff;
  in.altitude = data.altitude;
  in.temperature = data.temperature;
  in.wavenumber = data.wavenumber;
  in.cloud_optical_depth = data.cloud_optical_depth;
  in.phase_moments = data.phase_moments;
  adrt_outputs_f32 out{};
  out.toa_flux_up = data.flux_up;
  out.toa_flux_down = data.flux_down;
  out.boa_flux_direct = data.flux_direct;
  check(adrt_solve_batch_raw(thread_engine(), &d, &in, &out, stream));
}

void solveBatchFromCoefficients(const BatchConfig& config, const RawDeviceData& data,
                                SolverWorkspaceGPU& workspace, cudaStream_t stream) {
  workspace.allocate(config.num_wavenumbers, config.num_layers);
  solveBatchFromCoefficients(config, data, stream);
}

// The engine forms the intermediate quantities inside its solve, so the
// workspace only records the dimensions it was sized for.
void SolverWorkspaceGPU::allocate(int nwav, int nlay) {
  allocated_nwav = nwav;
  allocated_nlay = nlay;
}

void SolverWorkspaceGPU::free() {
  allocated_nwav = 0;
  allocated_nlay = 0;
}

HostResult solveBatchHost(const BatchConfig& config, const std::vector<float>& delta_tau,
                          const std::vector<float>& single_scat_albedo,
                          const std::vector<float>& phase_moments, bool phase_moments_shared,
                          const std::vector<float>& planck_levels,
                          const std::vector<float>& temperature) {
  const adrt_batch_desc d = to_desc(config, phase_moments_shared);
  auto widen = [](const std::vector<float>& v) { return std::vector<double>(v.begin(), v.end()); };
  const std::vector<double> dt = widen(delta_tau), om = widen(single_scat_albedo),
                            pm = widen(phase_moments), pl = widen(planck_levels),
                            tm = widen(temperature);
  adrt_inputs in{};
  in.delta_tau = dt.data();
  in.single_scat_albedo = om.data();
  in.phase_moments = pm.data();
  if (config.use_thermal_emission) {
    if (!tm.empty()) in.temperature = tm.data();
  } else if (!pl.empty()) {
    in.planck_levels = pl.data();
  }
  const size_t W = (size_t)config.num_wavenumbers;
  std::vector<double> fu(W), fd(W), fdir(W);
  adrt_outputs out{};
  out.toa_flux_up = fu.data();
  out.toa_flux_down = fd.data();
  out.boa_flux_direct = fdir.data();
  check(adrt_validate_batch(&d, &in));
  check(adrt_solve_batch_host(thread_engine(), &d, &in, &out));
  HostResult r;
  r.flux_up.assign(fu.begin(), fu.end());
  r.flux_down.assign(fd.begin(), fd.end());
  r.flux_direct.assign(fdir.begin(), fdir.end());
  return r;
}

}  // namespace cuda
}  // namespace adrt
