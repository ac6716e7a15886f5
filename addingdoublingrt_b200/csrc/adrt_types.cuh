// adrt_types.cuh -- device-side descriptors shared by the solver kernels and
// the host engine.
#pragma once

#include <cstddef>
#include <cstdint>

namespace adrt_dev {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxN = 32;         // largest quadrature order (reference: N in 2..32)
constexpr int kMaxMoments = 512;  // Legendre moments per set

// Quadrature constants for one N (device memory owned by the engine).
struct QuadDev {
  const double* mu;  // [N] Gauss-Legendre nodes on [0,1]
  const double* wt;  // [N] weights
  const double* pl;  // [mmax][N] Legendre polynomials P_l(mu_i)
  int mmax;          // rows of pl
  double xfac;       // 0.5 / sum(mu w)   (src/solver.cpp:378-383)
};

// One column of a batch: W wavenumbers sharing L, N and the scalar options.
struct ColumnDev {
  int W, L, N, NP, M, moment_layout;
  int thermal, delta_m, diffusion, from_bottom, temp_per_wav;
  int precision;
  double surface_albedo, surface_emission, surface_temperature;
  double top_emission, top_temperature, solar_flux, solar_mu;
  double wn_lo, wn_hi, spectrum_scaling;
  const double *dtau, *ssa, *moments, *temperature, *planck;
  const double *albedo_w, *mu0_w, *wlo_w, *whi_w, *semis_w, *temis_w;
  double *fu, *fd, *fdir, *J, *divF, *toa_fu, *toa_fd, *boa_fdir;
  // raw retrieval inputs (all null unless the batch is given as coefficients):
  // level-major [(L+1) x W] absorption / scattering coefficients, altitude
  // and temperature [L+1], cloud optical depth [L x W] (or null), level and
  // layer 0 at the bottom; wavenumber [W]
  const float *raw_abs, *raw_scat, *raw_alt, *raw_temp, *raw_cloud;
  const double* raw_wn;
  QuadDev quad;
  long long task_begin;  // first flattened task index of this column
  // normalised P++ / P+- of the moment sets shared by every wavenumber (one
  // per layer, [L][2][NP][NP]), formed once per call; null: built per layer
  const double* ptab;
};

// Kernel parameters (passed by value).
struct SolveParams {
  const ColumnDev* cols;
  int ncols;
  long long ntasks;
  unsigned long long* counter;  // work counter, zeroed before each launch
  unsigned int* status;         // device status word (adrt_device_flag bits)
  char* scratch;                // nslots * slot_bytes
  size_t slot_bytes;
  int nslots;
  int max_layers;               // L of the largest column (sizes the slot)
  // Wavenumbers whose pivot-free solve met a weak pivot, solved again by a
  // second launch of the same kernel (redo_pass = 1) with partial pivoting
  // in every solve: redo[0] entries, redo[1] that pass's work counter,
  // redo[2 ..] their task indices (room for redo_cap).  Null: no list.
  unsigned long long* redo;
  long long redo_cap;
  int redo_pass;
  int pivot_all;  // every solve with partial pivoting (ADRT_PIVOTING_PARTIAL)
};

}  // namespace adrt_dev
