// ref_capi.cpp -- TEST INFRASTRUCTURE (oracle side), not part of the product.
//
// A C entry point around the reference's own CPU solver adrt::solve
// (src/solver.cpp:1704-1713), compiled unmodified from the reference
// sources together with the project-written Eigen subset in
// oracle/eigen_subset.  It maps the engine's batch description
// (include/adrt_b200.h) onto one adrt::ADConfig per wavenumber
// (src/adding_doubling.hpp:63-247) and runs the wavenumbers on
// std::thread workers, each owning one adrt::SolverWorkspace
// (src/workspace.hpp:17-22), so the same code serves as the golden-vector
// generator, the parity oracle and the timed CPU baseline.
//
// Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() load
// this library.
#include "adding_doubling.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../include/adrt_b200.h"

namespace {

std::mutex g_err_mu;
std::string g_err;

void set_err(const std::string& s) {
  std::lock_guard<std::mutex> lk(g_err_mu);
  g_err = s;
}

// Build the ADConfig of wavenumber w exactly as a caller of adrt::solve would.
adrt::ADConfig make_config(const adrt_batch_desc& d, const adrt_inputs& in, int w) {
  const int L = d.num_layers, M = d.num_moments;
  adrt::ADConfig c(L, d.num_quadrature);
  c.use_thermal_emission = d.use_thermal_emission != 0;
  c.use_delta_m = d.use_delta_m != 0;
  c.use_diffusion_lower_bc = d.use_diffusion_lower_bc != 0;
  c.index_from_bottom = d.index_from_bottom != 0;
  c.surface_albedo = in.surface_albedo ? in.surface_albedo[w] : d.surface_albedo;
  c.surface_emission = in.surface_emission ? in.surface_emission[w] : d.surface_emission;
  c.surface_temperature = d.surface_temperature;
  c.top_emission = in.top_emission ? in.top_emission[w] : d.top_emission;
  c.top_temperature = d.top_temperature;
  c.solar_flux = d.solar_flux;
  c.solar_mu = in.solar_mu ? in.solar_mu[w] : d.solar_mu;
  c.wavenumber_low = in.wavenumber_low ? in.wavenumber_low[w] : d.wavenumber_low;
  c.wavenumber_high = in.wavenumber_high ? in.wavenumber_high[w] : d.wavenumber_high;
  c.delta_tau.assign(in.delta_tau + (size_t)w * L, in.delta_tau + (size_t)(w + 1) * L);
  c.single_scat_albedo.assign(in.single_scat_albedo + (size_t)w * L,
                              in.single_scat_albedo + (size_t)(w + 1) * L);
  c.phase_function_moments.assign(L, std::vector<double>(M, 0.0));
  for (int l = 0; l < L; ++l) {
    const double* src = nullptr;
    if (d.moment_layout == ADRT_MOMENTS_SHARED)
      src = in.phase_moments + (size_t)l * M;
    else if (d.moment_layout == ADRT_MOMENTS_PER_WAVENUMBER)
      src = in.phase_moments + (size_t)w * M;
    else
      src = in.phase_moments + ((size_t)w * L + l) * M;
    std::copy(src, src + M, c.phase_function_moments[l].begin());
  }
  if (c.use_thermal_emission && in.temperature) {
    const double* t = d.temperature_per_wavenumber ? in.temperature + (size_t)w * (L + 1)
                                                   : in.temperature;
    c.temperature.assign(t, t + L + 1);
  }
  if (in.planck_levels)
    c.planck_levels.assign(in.planck_levels + (size_t)w * (L + 1),
                           in.planck_levels + (size_t)(w + 1) * (L + 1));
  return c;
}

void store(const adrt_batch_desc& d, const adrt_outputs& o, int w, const adrt::RTOutput& r) {
  const size_t n = (size_t)d.num_layers + 1;
  auto put = [&](double* dst, const std::vector<double>& v) {
    if (dst) std::copy(v.begin(), v.end(), dst + (size_t)w * n);
  };
  put(o.flux_up, r.flux_up);
  put(o.flux_down, r.flux_down);
  put(o.flux_direct, r.flux_direct);
  put(o.mean_intensity, r.mean_intensity);
  put(o.flux_divergence, r.flux_divergence);
  // RTOutput is in the caller's level order; TOA is level n-1 when the
  // arrays are indexed from the bottom (src/solver.cpp:711-719).
  const size_t toa = d.index_from_bottom ? n - 1 : 0, boa = d.index_from_bottom ? 0 : n - 1;
  if (o.toa_flux_up) o.toa_flux_up[w] = r.flux_up[toa] * d.spectrum_scaling;
  if (o.toa_flux_down) o.toa_flux_down[w] = r.flux_down[toa];
  if (o.boa_flux_direct) o.boa_flux_direct[w] = r.flux_direct[boa];
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

// Solve wavenumbers [w0, w1) of a batch with the reference CPU solver on
// `nthreads` threads.  Returns 0, or -1 with ref_last_error() set when the
// reference throws (validate() / planckFunction std::invalid_argument).
int ref_solve_batch_range(const adrt_batch_desc* desc, const adrt_inputs* in,
                          const adrt_outputs* out, int w0, int w1, int nthreads) {
  if (!desc || !in || !out) return -1;
  if (nthreads < 1) nthreads = 1;
  std::atomic<int> next(w0);
  std::atomic<int> failed(0);
  auto worker = [&]() {
    adrt::SolverWorkspace ws;
    for (;;) {
      int w = next.fetch_add(1);
      if (w >= w1 || failed.load()) break;
      try {
        adrt::ADConfig c = make_config(*desc, *in, w);
        adrt::RTOutput r = adrt::solve(c, ws);
        store(*desc, *out, w, r);
      } catch (const std::exception& e) {
        set_err(std::string("wavenumber ") + std::to_string(w) + ": " + e.what());
        failed.store(1);
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nthreads; ++t) pool.emplace_back(worker);
  worker();
  for (auto& t : pool) t.join();
  return failed.load() ? -1 : 0;
}

int ref_solve_batch(const adrt_batch_desc* desc, const adrt_inputs* in,
                    const adrt_outputs* out, int nthreads) {
  return ref_solve_batch_range(desc, in, out, 0, desc ? desc->num_wavenumbers : 0, nthreads);
}

// One wavenumber with the reference's analytic temperature Jacobian
// (src/solver.cpp:117-341).  jac_* are [(L+1) x (L+2)] row-major or NULL.
int ref_solve_column_jacobian(const adrt_batch_desc* desc, const adrt_inputs* in, int w,
                              const adrt_outputs* out, double* jac_flux_up,
                              double* jac_flux_down, double* jac_mean_intensity,
                              double* jac_flux_divergence) {
  try {
    adrt::ADConfig c = make_config(*desc, *in, w);
    c.compute_temperature_jacobian = true;
    adrt::RTOutput r = adrt::solve(c);
    adrt_batch_desc d1 = *desc;
    store(d1, *out, 0, r);
    auto put = [&](double* dst, const std::vector<std::vector<double>>& J) {
      if (!dst) return;
      size_t k = 0;
      for (const auto& row : J)
        for (double v : row) dst[k++] = v;
    };
    put(jac_flux_up, r.flux_up_temperature_jac);
    put(jac_flux_down, r.flux_down_temperature_jac);
    put(jac_mean_intensity, r.mean_intensity_temperature_jac);
    put(jac_flux_divergence, r.flux_divergence_temperature_jac);
    return 0;
  } catch (const std::exception& e) {
    set_err(e.what());
    return -1;
  }
}

// Reference utilities exposed for the oracle's own pinning tests.
int ref_gauss_legendre(int n, double* nodes, double* weights) {
  std::vector<double> x, w;
  adrt::gaussLegendre(n, x, w);
  std::copy(x.begin(), x.end(), nodes);
  std::copy(w.begin(), w.end(), weights);
  return 0;
}

double ref_planck(double wnumlo, double wnumhi, double temp) {
  try {
    return adrt::planckFunction(wnumlo, wnumhi, temp);
  } catch (const std::exception& e) {
    set_err(e.what());
    return -1.0;
  }
}

}  // extern "C"
