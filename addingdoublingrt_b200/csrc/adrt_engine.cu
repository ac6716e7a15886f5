// adrt_engine.cu -- host engine behind the C ABI of include/adrt_b200.h.
//
// The engine owns every device buffer a solve needs (quadrature tables, the
// per-slot work buffer, the work counter and the status word), so a solve
// launch allocates nothing once adrt_engine_reserve() has sized it, and the
// only stream operations are one memset and one kernel launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/adrt_b200.h"
#include "adrt_adjoint.cuh"
#include "adrt_tpw.cuh"

using namespace adrt_dev;

namespace {

thread_local std::string g_detail;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_detail = buf;
  return code;
}

}  // namespace

// Lets other translation units of the library report through
// adrt_last_status_detail() (not exported).
__attribute__((visibility("hidden"))) void adrt_internal_set_detail(const char* msg) {
  g_detail = msg;
}

namespace {

#define CUDA_TRY(expr)                                                             \
  do {                                                                             \
    cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(ADRT_ERR_CUDA, "%s failed: %s", #expr, cudaGetErrorString(e_));  \
  } while (0)

// Gauss-Legendre nodes and weights on [0,1]: Newton iteration on P_n from the
// Chebyshev-like start cos(pi (i + 3/4) / (n + 1/2)), stopping at |dz| < 1e-15
// -- the construction of the reference's src/quadrature.cpp:11-51, which the
// engine must reproduce to the last bit so that its quadrature matches.
void gauss_legendre01(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
    double pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double pk = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      pp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = -p1 / pp;
      z += dz;
      if (std::fabs(dz) < 1e-15) break;
    }
    const double wi = 2.0 / ((1.0 - z * z) * pp * pp);
    x[i] = (1.0 - z) / 2.0;
    x[n - 1 - i] = (1.0 + z) / 2.0;
    w[i] = wi / 2.0;
    w[n - 1 - i] = wi / 2.0;
  }
}

// Kernel table: one instantiation per padded order and precision form.
using LaunchFn = int (*)(const SolveParams&, const ColumnDev&, int grid, cudaStream_t);

template <int NP, int KIND>
struct Kern {
  using GD = Geo<NP, double>;
  static constexpr int kThreads = 128;
  static constexpr int kGroups = kThreads / GD::G;
  static size_t smem() { return (size_t)kGroups * GroupLayout<NP, KIND>::bytes; }
  // records are sized for FP64 (the mixed form's class-D wavenumbers)
  static size_t slot_bytes(int lmax) { return SlotLayout<GD>::bytes(lmax); }
  static int max_blocks_per_sm() {
    static int cached = -1;
    if (cached < 0) {
      cudaFuncSetAttribute(solve_kernel<NP, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem());
      int nb = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, solve_kernel<NP, KIND>, kThreads, smem());
      cached = nb > 0 ? nb : 1;
    }
    return cached;
  }
  // Both passes: the solve, then the re-solve of the wavenumbers it listed
  // (a launch whose groups find an empty list and return at once when none
  // met a weak pivot).
  // (p.redo_pass already set: the re-solve pass alone, over the list as it is)
  static int launch(const SolveParams& p, const ColumnDev& c0, int grid, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    if (p.redo && !p.redo_pass) e = cudaMemsetAsync(p.redo, 0, 2 * sizeof(unsigned long long), s);
    if (e == cudaSuccess && !p.redo_pass) {
      solve_kernel<NP, KIND><<<grid, kThreads, smem(), s>>>(p, c0);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && p.redo) {
      SolveParams q = p;
      q.redo_pass = 1;
      solve_kernel<NP, KIND><<<grid, kThreads, smem(), s>>>(q, c0);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) return fail(ADRT_ERR_CUDA, "solve kernel launch: %s", cudaGetErrorString(e));
    return ADRT_OK;
  }
};

struct KernInfo {
  int np, groups;
  size_t (*slot_bytes)(int);
  int (*max_blocks)();
  LaunchFn launch;
};

template <int NP, int KIND>
KernInfo kinfo() {
  return KernInfo{NP, Kern<NP, KIND>::kGroups, &Kern<NP, KIND>::slot_bytes,
                  &Kern<NP, KIND>::max_blocks_per_sm, &Kern<NP, KIND>::launch};
}

int padded_order(int n) { return n <= 4 ? 4 : n <= 8 ? 8 : n <= 16 ? 16 : 32; }

KernInfo pick(int n, int precision) {
  const int np = padded_order(n);
  if (precision == ADRT_PRECISION_MIXED) {
    switch (np) {
      case 4: return kinfo<4, KIND_MIXED>();
      case 8: return kinfo<8, KIND_MIXED>();
      case 16: return kinfo<16, KIND_MIXED>();
      default: return kinfo<32, KIND_MIXED>();
    }
  }
  switch (np) {
    case 4: return kinfo<4, KIND_FP64>();
    case 8: return kinfo<8, KIND_FP64>();
    case 16: return kinfo<16, KIND_FP64>();
    default: return kinfo<32, KIND_FP64>();
  }
}

}  // namespace

// The host entry splits batches of at least 2 x kHostChunkMin wavenumbers into
// up to four chunks so that the copies overlap the solves; a chunk then keeps
// every resident thread group busy for several wavenumbers.
constexpr size_t kHostChunkMin = 8192;
// Room of the re-solve list: wavenumbers of one launch whose pivot-free solve
// met a weak pivot (none on physical inputs; beyond it ADRT_FLAG_PIVOT_UNRESOLVED).
constexpr long long kRedoCap = 65536;

struct adrt_engine {
  int device = 0;
  int num_sms = 0;
  size_t max_ws = 0;
  cudaStream_t last_stream = nullptr;
  char* scratch = nullptr;
  char* adj_scratch = nullptr;  // adjoint work buffer (larger slots)
  size_t adj_scratch_bytes = 0;
  size_t scratch_bytes = 0;
  unsigned long long* counter = nullptr;
  unsigned int* status = nullptr;
  unsigned long long* redo = nullptr;  // re-solve list (SolveParams::redo), kRedoCap entries
  ColumnDev* d_cols = nullptr;
  size_t d_cols_cap = 0;
  ColumnDev* h_cols = nullptr;       // pinned staging of the column table
  cudaEvent_t cols_copied = nullptr;  // the last table upload has been read
  struct Quad {
    double* buf = nullptr;
    int mmax = 0;
    QuadDev dev{};
  } quad[kMaxN + 1];
  // FP64 staging of the FP32 entry point (grows outside stream capture only)
  char* stage = nullptr;
  size_t stage_bytes = 0;
  // host entry: device staging (grows only), copy-in / solve / copy-out
  // streams and the events of two chunk buffers
  char* hstage = nullptr;
  size_t hstage_bytes = 0;
  cudaStream_t hs[3] = {nullptr, nullptr, nullptr};
  // shared-moment phase tables of a batch (layout ADRT_MOMENTS_SHARED)
  double* ptab = nullptr;
  size_t ptab_bytes = 0;
  cudaEvent_t hev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  std::mutex hmu;  // one host-entry call at a time per engine
  std::mutex mu;
  int adjoint_mode = ADRT_ADJOINT_RECORD;
  int pivoting = ADRT_PIVOTING_TENSOR_CORE;
  // uneven batches: warp mapping for every order, occupancy-limited grid,
  // longest columns first (adrt_engine_autotune_uneven replaces it)
  adrt_uneven_plan plan{{ADRT_MAPPING_WARP, ADRT_MAPPING_WARP, ADRT_MAPPING_WARP}, 0, 1,
                        {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}}};
};

namespace {

int set_device(adrt_engine* e) {
  CUDA_TRY(cudaSetDevice(e->device));
  return ADRT_OK;
}

}  // namespace

// Host copy of the quadrature table of order n: nodes [n], weights [n], then
// P_l(mu_i) for l < mmax ([mmax][n]); *xfac = 0.5 / sum(mu w).  Shared with
// the allocation-free entry point (not exported), so both upload the same bits.
__attribute__((visibility("hidden"))) void adrt_internal_quad_table(int n, int mmax,
                                                                    std::vector<double>& host,
                                                                    double* xfac) {
  std::vector<double> x, w;
  gauss_legendre01(n, x, w);
  host.assign((size_t)2 * n + (size_t)mmax * n, 0.0);
  for (int i = 0; i < n; ++i) {
    host[i] = x[i];
    host[n + i] = w[i];
  }
  double* pl = host.data() + 2 * n;
  for (int i = 0; i < n; ++i) pl[i] = 1.0;
  if (mmax > 1)
    for (int i = 0; i < n; ++i) pl[n + i] = x[i];
  for (int l = 2; l < mmax; ++l)
    for (int i = 0; i < n; ++i)
      pl[l * n + i] = ((2 * l - 1) * x[i] * pl[(l - 1) * n + i] - (l - 1) * pl[(l - 2) * n + i]) / l;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += x[i] * w[i];
  *xfac = 0.5 / s;
}

namespace {

// Quadrature table for order n with Legendre rows up to mmax.
int ensure_quad(adrt_engine* e, int n, int mmax) {
  auto& q = e->quad[n];
  if (q.buf && q.mmax >= mmax) return ADRT_OK;
  mmax = std::max(mmax, 2 * n);
  std::vector<double> host;
  double xfac = 0.0;
  adrt_internal_quad_table(n, mmax, host, &xfac);
  if (q.buf) {
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(q.buf);
    q.buf = nullptr;
  }
  if (cudaMalloc(&q.buf, host.size() * sizeof(double)) != cudaSuccess)
    return fail(ADRT_ERR_OUT_OF_MEMORY, "quadrature table allocation failed");
  CUDA_TRY(cudaMemcpy(q.buf, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice));
  q.mmax = mmax;
  q.dev.mu = q.buf;
  q.dev.wt = q.buf + n;
  q.dev.pl = q.buf + 2 * n;
  q.dev.mmax = mmax;
  q.dev.xfac = xfac;
  return ADRT_OK;
}

int check_desc(const adrt_batch_desc* d) {
  if (!d) return fail(ADRT_ERR_INVALID_ARGUMENT, "null batch description");
  if (d->num_wavenumbers < 1) return fail(ADRT_ERR_INVALID_ARGUMENT, "num_wavenumbers must be >= 1");
  if (d->num_layers <= 0) return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: num_layers must be > 0");
  if (d->num_quadrature < 2) return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: num_quadrature must be >= 2");
  if (d->num_quadrature > kMaxN)
    return fail(ADRT_ERR_UNSUPPORTED, "num_quadrature %d > 32 is not supported", d->num_quadrature);
  if (d->num_moments < 1 || d->num_moments > kMaxMoments)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "num_moments must be in 1..%d", kMaxMoments);
  if (d->moment_layout < 0 || d->moment_layout > 2)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "unknown moment_layout %d", d->moment_layout);
  if (d->precision != ADRT_PRECISION_FP64 && d->precision != ADRT_PRECISION_MIXED)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "unknown precision %d", d->precision);
  if (d->surface_albedo < 0.0 || d->surface_albedo > 1.0)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: surface_albedo out of [0,1]");
  if (d->solar_flux > 0.0 && (d->solar_mu <= 0.0 || d->solar_mu > 1.0))
    return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: solar_mu must be in (0,1] when solar_flux > 0");
  if (d->use_thermal_emission) {
    if (d->wavenumber_low < 0.0 || d->wavenumber_high < d->wavenumber_low)
      return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: invalid wavenumber range");
  } else if (d->surface_temperature >= 0.0) {
    return fail(ADRT_ERR_INVALID_ARGUMENT,
                "ADConfig: surface_temperature requires use_thermal_emission "
                "(use surface_emission for raw thermal sources)");
  } else if (d->top_temperature >= 0.0) {
    return fail(ADRT_ERR_INVALID_ARGUMENT,
                "ADConfig: top_temperature requires use_thermal_emission "
                "(use top_emission for raw thermal sources)");
  }
  return ADRT_OK;
}

int check_inputs(const adrt_batch_desc* d, const adrt_inputs* in) {
  if (!in) return fail(ADRT_ERR_INVALID_ARGUMENT, "null inputs");
  if (!in->delta_tau) return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: delta_tau size mismatch");
  if (!in->single_scat_albedo)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: single_scat_albedo size mismatch");
  if (!in->phase_moments)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: phase_function_moments size mismatch");
  if (d->use_thermal_emission && !in->temperature)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: temperature size must be num_layers+1");
  if (d->use_diffusion_lower_bc && !d->use_thermal_emission && !in->planck_levels)
    return fail(ADRT_ERR_INVALID_ARGUMENT,
                "ADConfig: use_diffusion_lower_bc requires use_thermal_emission or planck_levels");
  return ADRT_OK;
}

}  // namespace

// The argument checks of adrt_solve_batch (description, then inputs), for the
// library's other entry points (not exported).
__attribute__((visibility("hidden"))) int adrt_internal_check_batch(const adrt_batch_desc* d,
                                                                    const adrt_inputs* in) {
  int rc = check_desc(d);
  if (rc) return rc;
  return check_inputs(d, in);
}

namespace {

ColumnDev make_column(adrt_engine* e, const adrt_batch_desc* d, const adrt_inputs* in,
                      const adrt_outputs* out) {
  ColumnDev c{};
  c.W = d->num_wavenumbers;
  c.L = d->num_layers;
  c.N = d->num_quadrature;
  c.NP = padded_order(d->num_quadrature);
  c.M = d->num_moments;
  c.moment_layout = d->moment_layout;
  c.thermal = d->use_thermal_emission;
  c.delta_m = d->use_delta_m;
  c.diffusion = d->use_diffusion_lower_bc;
  c.from_bottom = d->index_from_bottom;
  c.temp_per_wav = d->temperature_per_wavenumber;
  c.precision = d->precision;
  c.surface_albedo = d->surface_albedo;
  c.surface_emission = d->surface_emission;
  c.surface_temperature = d->surface_temperature;
  c.top_emission = d->top_emission;
  c.top_temperature = d->top_temperature;
  c.solar_flux = d->solar_flux;
  c.solar_mu = d->solar_mu;
  c.wn_lo = d->wavenumber_low;
  c.wn_hi = d->wavenumber_high;
  c.spectrum_scaling = d->spectrum_scaling;
  c.dtau = in->delta_tau;
  c.ssa = in->single_scat_albedo;
  c.moments = in->phase_moments;
  c.temperature = in->temperature;
  c.planck = in->planck_levels;
  c.albedo_w = in->surface_albedo;
  c.mu0_w = in->solar_mu;
  c.wlo_w = in->wavenumber_low;
  c.whi_w = in->wavenumber_high;
  c.semis_w = in->surface_emission;
  c.temis_w = in->top_emission;
  if (out) {
    c.fu = out->flux_up;
    c.fd = out->flux_down;
    c.fdir = out->flux_direct;
    c.J = out->mean_intensity;
    c.divF = out->flux_divergence;
    c.toa_fu = out->toa_flux_up;
    c.toa_fd = out->toa_flux_down;
    c.boa_fdir = out->boa_flux_direct;
  }
  c.quad = e->quad[d->num_quadrature].dev;
  c.task_begin = 0;
  return c;
}

// Size the work buffer for (kernel, lmax); grows only outside stream capture.
int ensure_scratch(adrt_engine* e, const KernInfo& k, int lmax, int* grid, size_t* slot_bytes) {
  const int bps = k.max_blocks();
  *slot_bytes = (k.slot_bytes(lmax) + 255) & ~size_t(255);
  int blocks = bps * e->num_sms;
  size_t need = (size_t)blocks * k.groups * (*slot_bytes);
  if (e->max_ws && need > e->max_ws) {
    blocks = (int)(e->max_ws / ((size_t)k.groups * (*slot_bytes)));
    if (blocks < 1)
      return fail(ADRT_ERR_WORKSPACE, "workspace limit %zu B below one slot (%zu B)", e->max_ws,
                  *slot_bytes);
    need = (size_t)blocks * k.groups * (*slot_bytes);
  }
  if (need > e->scratch_bytes) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (e->last_stream) cudaStreamIsCapturing(e->last_stream, &cap);
    if (cap != cudaStreamCaptureStatusNone)
      return fail(ADRT_ERR_WORKSPACE,
                  "work buffer too small during stream capture; call adrt_engine_reserve first");
    if (e->scratch) {
      CUDA_TRY(cudaDeviceSynchronize());
      cudaFree(e->scratch);
      e->scratch = nullptr;
      e->scratch_bytes = 0;
    }
    if (cudaMalloc(&e->scratch, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(ADRT_ERR_OUT_OF_MEMORY, "work buffer allocation of %zu B failed", need);
    }
    e->scratch_bytes = need;
  }
  *grid = (int)(e->scratch_bytes / ((size_t)k.groups * (*slot_bytes)));
  *grid = std::min(*grid, bps * e->num_sms);
  return ADRT_OK;
}

// Element counts of the input (adrt_inputs field order) and output
// (adrt_outputs field order) arrays of a batch.
void input_counts(const adrt_batch_desc* d, size_t n[11]) {
  const size_t W = d->num_wavenumbers, L = d->num_layers, M = d->num_moments;
  n[0] = W * L;
  n[1] = W * L;
  n[2] = d->moment_layout == ADRT_MOMENTS_SHARED ? L * M
         : d->moment_layout == ADRT_MOMENTS_PER_WAVENUMBER ? W * M : W * L * M;
  n[3] = (d->temperature_per_wavenumber ? W : 1) * (L + 1);
  n[4] = W * (L + 1);
  for (int i = 5; i < 11; ++i) n[i] = W;
}
void output_counts(const adrt_batch_desc* d, size_t n[8]) {
  const size_t W = d->num_wavenumbers, L = d->num_layers;
  for (int i = 0; i < 5; ++i) n[i] = W * (L + 1);
  for (int i = 5; i < 8; ++i) n[i] = W;
}
size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

__global__ void widen_kernel(const float* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}
__global__ void narrow_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = static_cast<float>(in[i]);
}
int cast_grid(size_t n, int num_sms) {
  const size_t b = (n + 255) / 256;
  const size_t cap = (size_t)num_sms * 8;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

// Phase matrices of the moment sets every wavenumber shares (one per layer),
// once per call: phase_table_kernel forms set u's normalised P++ / P+- into
// table[u], which the solve reads instead of rebuilding them per wavenumber
// and layer.  The table grows outside stream capture only.
int ensure_ptab(adrt_engine* e, int np, int layers, cudaStreamCaptureStatus cap) {
  const size_t need = (size_t)layers * 2 * np * np * sizeof(double);
  if (need <= e->ptab_bytes) return ADRT_OK;
  if (cap != cudaStreamCaptureStatusNone)
    return fail(ADRT_ERR_WORKSPACE,
                "phase table too small during stream capture; call adrt_engine_reserve first");
  if (e->ptab) {
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(e->ptab);
    e->ptab = nullptr;
    e->ptab_bytes = 0;
  }
  if (cudaMalloc(&e->ptab, need) != cudaSuccess) {
    cudaGetLastError();
    return fail(ADRT_ERR_OUT_OF_MEMORY, "phase table allocation failed");
  }
  e->ptab_bytes = need;
  return ADRT_OK;
}

template <int NP>
int launch_ptab(const ColumnDev& c, double* tab, int sets, cudaStream_t s) {
  static bool ready = false;
  if (!ready) {
    CUDA_TRY(cudaFuncSetAttribute(phase_table_kernel<NP>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)AdjGroup<NP>::bytes));
    ready = true;
  }
  phase_table_kernel<NP><<<sets, AdjGeo<NP>::G, AdjGroup<NP>::bytes, s>>>(c, tab);
  CUDA_TRY(cudaGetLastError());
  return ADRT_OK;
}

int phase_table(adrt_engine* e, ColumnDev& c, cudaStream_t s) {
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  int rc = ensure_ptab(e, c.NP, c.L, cap);
  if (rc) return rc;
  switch (c.NP) {
    case 4: rc = launch_ptab<4>(c, e->ptab, c.L, s); break;
    case 8: rc = launch_ptab<8>(c, e->ptab, c.L, s); break;
    case 16: rc = launch_ptab<16>(c, e->ptab, c.L, s); break;
    default: rc = launch_ptab<32>(c, e->ptab, c.L, s); break;
  }
  if (rc) return rc;
  c.ptab = e->ptab;
  return ADRT_OK;
}

// adrt_solve_batch after argument checks, with e->mu held.  With `relist`,
// only the re-solve pass runs, over those wavenumbers.
int solve_locked(adrt_engine* e, const adrt_batch_desc* d, const adrt_inputs* in,
                 const adrt_outputs* out, cudaStream_t s, const adrt_raw_inputs* raw = nullptr,
                 const std::vector<unsigned long long>* relist = nullptr) {
  int rc;
  if ((rc = set_device(e))) return rc;
  e->last_stream = s;
  if ((rc = ensure_quad(e, d->num_quadrature, d->num_moments))) return rc;
  KernInfo k = pick(d->num_quadrature, d->precision);
  int grid;
  size_t sb;
  if ((rc = ensure_scratch(e, k, d->num_layers, &grid, &sb))) return rc;
  ColumnDev c0 = make_column(e, d, in, out);
  if (raw) {
    c0.raw_abs = raw->absorption_coeff;
    c0.raw_scat = raw->scattering_coeff;
    c0.raw_alt = raw->altitude;
    c0.raw_temp = raw->temperature;
    c0.raw_cloud = raw->cloud_optical_depth;
    c0.raw_wn = raw->wavenumber;
  }
  SolveParams p{};
  p.cols = nullptr;
  p.ncols = 1;
  p.ntasks = d->num_wavenumbers;
  p.counter = e->counter;
  p.status = e->status;
  p.scratch = e->scratch;
  p.slot_bytes = sb;
  p.nslots = grid * k.groups;
  p.max_layers = d->num_layers;
  p.redo = e->redo;
  p.redo_cap = kRedoCap;
  p.pivot_all = e->pivoting == ADRT_PIVOTING_PARTIAL;
  const int need_blocks = (d->num_wavenumbers + k.groups - 1) / k.groups;
  grid = std::min(grid, need_blocks);
  if (!raw && d->moment_layout == ADRT_MOMENTS_SHARED && (rc = phase_table(e, c0, s))) return rc;
  CUDA_TRY(cudaMemsetAsync(e->counter, 0, sizeof(unsigned long long), s));
  if (relist) {
    CUDA_TRY(cudaStreamSynchronize(s));
    CUDA_TRY(cudaMemcpy(e->redo, relist->data(), relist->size() * sizeof(unsigned long long),
                        cudaMemcpyHostToDevice));
    p.redo_pass = 1;
  }
  return k.launch(p, c0, grid, s);
}

// ------------------------------------------------------------- uneven batches
// One column of an uneven launch: its description and the wavenumbers to
// solve (all of them, or the autotuner's sample: the first W).
struct UnevenColumn {
  const adrt_column_desc* c;
  int W;
};

int warp_blocks_per_sm_max() {
  static int bps = -1;
  if (bps < 0) {
    const size_t smem = 4 * kMultiGroupBytes;
    cudaFuncSetAttribute(solve_kernel_multi<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, solve_kernel_multi<0>, 128, smem);
    if (bps < 1) bps = 1;
  }
  return bps;
}

template <int NP>
int tpw_blocks_per_sm() {
  static int bps = -1;
  if (bps < 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, tpw::solve_kernel_tpw<NP>, 128, 0);
    if (bps < 1) bps = 1;
  }
  return bps;
}

// Thread-per-wavenumber work memory: every thread of the launch holds its
// own records (about (L+1) x 3 NP^2 doubles, 0.97 MB at NP = 16, L = 150),
// so the launch is capped by this budget (or the engine's workspace limit).
constexpr size_t kThreadMappingBudget = size_t(16) << 30;

size_t tpw_slot_bytes(int np, int lmax) {
  const size_t d = np == 4 ? tpw::slot_doubles<4>(lmax)
                   : np == 8 ? tpw::slot_doubles<8>(lmax) : tpw::slot_doubles<16>(lmax);
  return d * sizeof(double);
}

long long tpw_slots(adrt_engine* e, int np, int lmax, long long ntasks) {
  const int bps = np == 4 ? tpw_blocks_per_sm<4>() : np == 8 ? tpw_blocks_per_sm<8>()
                                                             : tpw_blocks_per_sm<16>();
  long long n = (long long)bps * e->num_sms * 128;
  const size_t budget = e->max_ws ? e->max_ws : kThreadMappingBudget;
  n = std::min<long long>(n, (long long)(budget / tpw_slot_bytes(np, lmax)));
  return std::min<long long>(n, ntasks);
}

// Grow the engine's work buffer to `need` bytes (outside stream capture).
int grow_scratch(adrt_engine* e, size_t need, cudaStreamCaptureStatus cap) {
  if (need <= e->scratch_bytes) return ADRT_OK;
  if (cap != cudaStreamCaptureStatusNone)
    return fail(ADRT_ERR_WORKSPACE, "work buffer too small during stream capture");
  CUDA_TRY(cudaDeviceSynchronize());
  cudaFree(e->scratch);
  e->scratch = nullptr;
  e->scratch_bytes = 0;
  if (cudaMalloc(&e->scratch, need) != cudaSuccess) {
    cudaGetLastError();
    return fail(ADRT_ERR_OUT_OF_MEMORY, "work buffer allocation of %zu B failed", need);
  }
  e->scratch_bytes = need;
  return ADRT_OK;
}

// The uneven launch under `plan`, with e->mu held.  Columns are split into
// the warp launch (N <= 16: every mixed column, and FP64 columns whose order
// maps to warps), one thread-per-wavenumber launch per order (FP64 columns
// whose order maps to threads) and the N = 32 launch; all run back to back on
// the stream, each from its own work counter, over one column table.
int uneven_locked(adrt_engine* e, std::vector<UnevenColumn>& cv, cudaStream_t s,
                  const adrt_uneven_plan& plan) {
  int rc;
  if ((rc = set_device(e))) return rc;
  e->last_stream = s;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  const int ncols = (int)cv.size();
  for (auto& c : cv)
    if ((rc = ensure_quad(e, c.c->desc.num_quadrature, c.c->desc.num_moments))) return rc;
  // parts: 0 warp, 1..3 thread mapping at NP = 4, 8, 16, 4 the N = 32 kernel
  std::vector<int> part[5];
  int lmax[5] = {1, 1, 1, 1, 1};
  int any_mixed_l = 0;
  for (int i = 0; i < ncols; ++i) {
    const adrt_batch_desc& d = cv[i].c->desc;
    if (cv[i].W < 1) continue;
    const int np = padded_order(d.num_quadrature);
    const int oi = np == 4 ? 0 : np == 8 ? 1 : 2;
    int k;
    if (np == 32) {
      k = 4;
      any_mixed_l |= d.precision == ADRT_PRECISION_MIXED;
    } else if (d.precision == ADRT_PRECISION_FP64 && plan.mapping[oi] == ADRT_MAPPING_THREAD) {
      k = 1 + oi;
    } else {
      k = 0;
    }
    part[k].push_back(i);
    lmax[k] = std::max(lmax[k], d.num_layers);
  }
  // longest columns first (cost ~ L NP^3 per wavenumber), so the persistent
  // kernels' dynamic task queues end with short tasks
  auto cost = [&](int i) {
    const double np = padded_order(cv[i].c->desc.num_quadrature);
    return (double)cv[i].c->desc.num_layers * np * np * np;
  };
  if (plan.cost_order)
    for (auto& pv : part)
      std::stable_sort(pv.begin(), pv.end(), [&](int a, int b) { return cost(a) > cost(b); });
  int nused = 0;
  for (auto& pv : part) nused += (int)pv.size();
  if (nused == 0) return ADRT_OK;
  if (e->d_cols_cap < (size_t)nused) {
    if (cap != cudaStreamCaptureStatusNone)
      return fail(ADRT_ERR_WORKSPACE, "column table too small during capture");
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(e->d_cols);
    if (e->h_cols) cudaFreeHost(e->h_cols);
    e->d_cols = nullptr;
    e->h_cols = nullptr;
    e->d_cols_cap = 0;
    if (cudaMalloc(&e->d_cols, sizeof(ColumnDev) * nused) != cudaSuccess ||
        cudaMallocHost(&e->h_cols, sizeof(ColumnDev) * nused) != cudaSuccess)
      return fail(ADRT_ERR_OUT_OF_MEMORY, "column table allocation failed");
    e->d_cols_cap = nused;
    if (!e->cols_copied) CUDA_TRY(cudaEventCreateWithFlags(&e->cols_copied, cudaEventDisableTiming));
  }
  // the previous upload must have left the pinned staging before it is rewritten
  if (cap == cudaStreamCaptureStatusNone && e->cols_copied) CUDA_TRY(cudaEventSynchronize(e->cols_copied));
  long long totals[5] = {0, 0, 0, 0, 0};
  int first[5];
  int nt = 0;
  for (int k = 0; k < 5; ++k) {
    first[k] = nt;
    for (int i : part[k]) {
      const adrt_column_desc* c = cv[i].c;
      ColumnDev col = make_column(e, &c->desc, &c->in, &c->out);
      col.W = cv[i].W;
      col.task_begin = totals[k];
      totals[k] += cv[i].W;
      e->h_cols[nt++] = col;
    }
  }
  CUDA_TRY(cudaMemcpyAsync(e->d_cols, e->h_cols, sizeof(ColumnDev) * nused, cudaMemcpyHostToDevice, s));
  // (in a capture the copy runs at each replay, from the staging as it is
  // then; recording the event there would leave it a captured event)
  if (e->cols_copied && cap == cudaStreamCaptureStatusNone)
    CUDA_TRY(cudaEventRecord(e->cols_copied, s));
  // the warp launch: one wavenumber per warp, all orders <= 16, one launch
  if (!part[0].empty()) {
    const size_t smem = 4 * kMultiGroupBytes;
    const int bmax = warp_blocks_per_sm_max();
    const int bps = plan.warp_blocks_per_sm ? std::min(plan.warp_blocks_per_sm, bmax) : bmax;
    const size_t sb = (SlotLayout<Geo<16, double>>::bytes(lmax[0]) + 255) & ~size_t(255);
    long long blocks = (long long)bps * e->num_sms;
    if (e->max_ws) {
      blocks = std::min<long long>(blocks, (long long)(e->max_ws / (4 * sb)));
      if (blocks < 1) return fail(ADRT_ERR_WORKSPACE, "workspace limit below one slot (%zu B)", sb);
    }
    if ((rc = grow_scratch(e, (size_t)blocks * 4 * sb, cap))) return rc;
    blocks = std::min<long long>(blocks, (totals[0] + 3) / 4);
    SolveParams p{};
    p.cols = e->d_cols + first[0];
    p.ncols = (int)part[0].size();
    p.ntasks = totals[0];
    p.counter = e->counter;
    p.status = e->status;
    p.scratch = e->scratch;
    p.slot_bytes = sb;
    p.nslots = (int)blocks * 4;
    p.max_layers = lmax[0];
    p.redo = e->redo;
    p.redo_cap = kRedoCap;
    p.pivot_all = e->pivoting == ADRT_PIVOTING_PARTIAL;
    CUDA_TRY(cudaMemsetAsync(e->counter, 0, sizeof(unsigned long long), s));
    CUDA_TRY(cudaMemsetAsync(e->redo, 0, 2 * sizeof(unsigned long long), s));
    solve_kernel_multi<0><<<(int)blocks, 128, smem, s>>>(p);
    CUDA_TRY(cudaGetLastError());
    p.redo_pass = 1;  // the listed wavenumbers again, pivoted
    solve_kernel_multi<0><<<(int)blocks, 128, smem, s>>>(p);
    CUDA_TRY(cudaGetLastError());
  }
  // the thread-per-wavenumber launches, one per order
  for (int k = 1; k <= 3; ++k) {
    if (part[k].empty()) continue;
    const int np = k == 1 ? 4 : k == 2 ? 8 : 16;
    const long long nslots = tpw_slots(e, np, lmax[k], totals[k]);
    if (nslots < 1)
      return fail(ADRT_ERR_WORKSPACE, "workspace below one thread-mapping slot (%zu B)",
                  tpw_slot_bytes(np, lmax[k]));
    if ((rc = grow_scratch(e, (size_t)nslots * tpw_slot_bytes(np, lmax[k]), cap))) return rc;
    SolveParams p{};
    p.cols = e->d_cols + first[k];
    p.ncols = (int)part[k].size();
    p.ntasks = totals[k];
    p.counter = e->counter + 1 + k;
    p.status = e->status;
    p.scratch = e->scratch;
    p.slot_bytes = tpw_slot_bytes(np, lmax[k]);
    p.nslots = (int)nslots;
    p.max_layers = lmax[k];
    CUDA_TRY(cudaMemsetAsync(e->counter + 1 + k, 0, sizeof(unsigned long long), s));
    const int grid = (int)((nslots + 127) / 128);
    if (np == 4) tpw::solve_kernel_tpw<4><<<grid, 128, 0, s>>>(p);
    else if (np == 8) tpw::solve_kernel_tpw<8><<<grid, 128, 0, s>>>(p);
    else tpw::solve_kernel_tpw<16><<<grid, 128, 0, s>>>(p);
    CUDA_TRY(cudaGetLastError());
  }
  // columns of N > 16: one launch of the N = 32 kernel (per-column precision)
  if (!part[4].empty()) {
    KernInfo k = pick(32, any_mixed_l ? ADRT_PRECISION_MIXED : ADRT_PRECISION_FP64);
    int grid;
    size_t sb;
    if ((rc = ensure_scratch(e, k, lmax[4], &grid, &sb))) return rc;
    SolveParams p{};
    p.cols = e->d_cols + first[4];
    p.ncols = (int)part[4].size();  // 1: the kernel takes the column from c0
    p.ntasks = totals[4];
    p.counter = e->counter + 1;  // its own work counter
    p.status = e->status;
    p.scratch = e->scratch;
    p.slot_bytes = sb;
    p.nslots = grid * k.groups;
    p.max_layers = lmax[4];
    p.redo = e->redo;
    p.redo_cap = kRedoCap;
    p.pivot_all = e->pivoting == ADRT_PIVOTING_PARTIAL;
    grid = (int)std::min<long long>(grid, totals[4]);
    CUDA_TRY(cudaMemsetAsync(e->counter + 1, 0, sizeof(unsigned long long), s));
    ColumnDev c0 = e->h_cols[first[4]];
    if ((rc = k.launch(p, c0, grid, s))) return rc;
  }
  return ADRT_OK;
}

}  // namespace

// ====================================================================== C ABI
// Channel sums of a spectrum: one block per channel at a time (grid-stride
// over channels), each thread a strided partial sum in wavenumber order, then
// a fixed-shape block reduction.  HBM-bound: 8 or 16 bytes per wavenumber.
__global__ void __launch_bounds__(256) band_integrate_kernel(const double* __restrict__ spec,
                                                             const double* __restrict__ wgt,
                                                             long long W,
                                                             const long long* __restrict__ off,
                                                             int nch, double* __restrict__ out,
                                                             unsigned* status) {
  __shared__ double part[8];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int b = blockIdx.x; b < nch; b += gridDim.x) {
    const long long lo = off[b], hi = off[b + 1];
    const bool ok = lo >= 0 && lo <= hi && hi <= W;
    double acc = 0.0;
    if (ok) {
      for (long long w = lo + t; w < hi; w += blockDim.x)
        acc += (wgt ? wgt[w] : 1.0) * spec[w];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    if (t == 0) {
      double sum = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) sum += part[i];
      if (ok) {
        out[b] = sum;
      } else {
        out[b] = __longlong_as_double(0x7ff8000000000000ll);
        atomicOr(status, (unsigned)ADRT_FLAG_BAD_INPUT);
      }
    }
    __syncthreads();
  }
}

extern "C" {

const char* adrt_last_status_detail(void) { return g_detail.c_str(); }
const char* adrt_version(void) { return "adrt-b200 0.1.0 (sm_100a)"; }

int adrt_engine_create(const adrt_engine_opts* opts, adrt_engine** out) {
  if (!out) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine out-pointer");
  *out = nullptr;
  int dev = 0;
  if (opts && opts->device >= 0) {
    dev = opts->device;
  } else {
    CUDA_TRY(cudaGetDevice(&dev));
  }
  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (dev >= ndev) return fail(ADRT_ERR_INVALID_ARGUMENT, "device %d not present", dev);
  auto* e = new adrt_engine();
  e->device = dev;
  e->max_ws = opts ? opts->max_workspace_bytes : 0;
  int rc = set_device(e);
  if (rc) {
    delete e;
    return rc;
  }
  cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaMalloc(&e->counter, 64) != cudaSuccess || cudaMalloc(&e->status, 64) != cudaSuccess ||
      cudaMalloc(&e->redo, sizeof(unsigned long long) * (2 + kRedoCap)) != cudaSuccess) {
    delete e;
    return fail(ADRT_ERR_OUT_OF_MEMORY, "engine allocation failed");
  }
  cudaMemset(e->status, 0, 64);
  *out = e;
  return ADRT_OK;
}

int adrt_engine_destroy(adrt_engine* e) {
  if (!e) return ADRT_OK;
  cudaSetDevice(e->device);
  cudaDeviceSynchronize();
  cudaFree(e->scratch);
  cudaFree(e->counter);
  cudaFree(e->status);
  cudaFree(e->redo);
  cudaFree(e->d_cols);
  if (e->h_cols) cudaFreeHost(e->h_cols);
  if (e->cols_copied) cudaEventDestroy(e->cols_copied);
  for (auto& q : e->quad) cudaFree(q.buf);
  cudaFree(e->hstage);
  for (auto& st : e->hs)
    if (st) cudaStreamDestroy(st);
  for (auto& ev : e->hev)
    if (ev) cudaEventDestroy(ev);
  cudaFree(e->stage);
  cudaFree(e->adj_scratch);
  cudaFree(e->ptab);
  delete e;
  return ADRT_OK;
}

int adrt_engine_reserve(adrt_engine* e, const adrt_batch_desc* d) {
  if (!e) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine");
  int rc = check_desc(d);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(e->mu);
  if ((rc = set_device(e))) return rc;
  if ((rc = ensure_quad(e, d->num_quadrature, d->num_moments))) return rc;
  KernInfo k = pick(d->num_quadrature, d->precision);
  int grid;
  size_t sb;
  if (d->moment_layout == ADRT_MOMENTS_SHARED &&
      (rc = ensure_ptab(e, padded_order(d->num_quadrature), d->num_layers,
                        cudaStreamCaptureStatusNone)))
    return rc;
  return ensure_scratch(e, k, d->num_layers, &grid, &sb);
}

int adrt_engine_workspace_bytes(const adrt_engine* e, size_t* bytes) {
  if (!e || !bytes) return fail(ADRT_ERR_INVALID_ARGUMENT, "null argument");
  *bytes = e->scratch_bytes;
  return ADRT_OK;
}

int adrt_engine_device(const adrt_engine* e, int* device) {
  if (!e || !device) return fail(ADRT_ERR_INVALID_ARGUMENT, "null argument");
  *device = e->device;
  return ADRT_OK;
}

int adrt_engine_read_status(adrt_engine* e, int* flags) {
  if (!e || !flags) return fail(ADRT_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(e->mu);
  int rc = set_device(e);
  if (rc) return rc;
  CUDA_TRY(cudaDeviceSynchronize());
  unsigned int v = 0;
  CUDA_TRY(cudaMemcpy(&v, e->status, sizeof v, cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemset(e->status, 0, sizeof v));
  *flags = (int)v;
  return ADRT_OK;
}

int adrt_validate_batch(const adrt_batch_desc* d, const adrt_inputs* in) {
  int rc = check_desc(d);
  if (rc) return rc;
  if ((rc = check_inputs(d, in))) return rc;
  const int W = d->num_wavenumbers, L = d->num_layers;
  for (int w = 0; w < W; ++w) {
    for (int l = 0; l < L; ++l) {
      const double t = in->delta_tau[(size_t)w * L + l];
      const double o = in->single_scat_albedo[(size_t)w * L + l];
      if (!(t >= 0.0)) return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: delta_tau[%d] < 0 (wavenumber %d)", l, w);
      if (!(o >= 0.0 && o <= 1.0))
        return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: single_scat_albedo[%d] out of [0,1] (wavenumber %d)", l, w);
    }
    const double a = in->surface_albedo ? in->surface_albedo[w] : d->surface_albedo;
    if (!(a >= 0.0 && a <= 1.0)) return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: surface_albedo out of [0,1]");
    const double m0 = in->solar_mu ? in->solar_mu[w] : d->solar_mu;
    if (d->solar_flux > 0.0 && !(m0 > 0.0 && m0 <= 1.0))
      return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: solar_mu must be in (0,1] when solar_flux > 0");
    if (d->use_thermal_emission) {
      const double lo = in->wavenumber_low ? in->wavenumber_low[w] : d->wavenumber_low;
      const double hi = in->wavenumber_high ? in->wavenumber_high[w] : d->wavenumber_high;
      if (!(lo >= 0.0 && hi >= lo)) return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: invalid wavenumber range");
    }
  }
  if (d->use_thermal_emission) {
    const size_t nt = (size_t)(d->temperature_per_wavenumber ? W : 1) * (L + 1);
    for (size_t i = 0; i < nt; ++i)
      if (!(in->temperature[i] >= 0.0))
        return fail(ADRT_ERR_INVALID_ARGUMENT, "ADConfig: temperature[%zu] < 0", i % (L + 1));
  }
  return ADRT_OK;
}

int adrt_solve_batch(adrt_engine* e, const adrt_batch_desc* d, const adrt_inputs* in,
                     const adrt_outputs* out, void* stream_ptr) {
  if (!e) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine");
  int rc = check_desc(d);
  if (rc) return rc;
  if ((rc = check_inputs(d, in))) return rc;
  if (!out) return fail(ADRT_ERR_INVALID_ARGUMENT, "null outputs");
  std::lock_guard<std::mutex> lk(e->mu);
  return solve_locked(e, d, in, out, static_cast<cudaStream_t>(stream_ptr));
}

int adrt_solve_batch_f32(adrt_engine* e, const adrt_batch_desc* d, const adrt_inputs_f32* in,
                         const adrt_outputs_f32* out, void* stream_ptr) {
  if (!e) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine");
  if (!in || !out) return fail(ADRT_ERR_INVALID_ARGUMENT, "null inputs or outputs");
  int rc = check_desc(d);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(e->mu);
  if ((rc = set_device(e))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  size_t nin[11], nout[8];
  input_counts(d, nin);
  output_counts(d, nout);
  const float* const* fin = &in->delta_tau;
  float* const* fout = &out->flux_up;
  size_t need = 0;
  for (int i = 0; i < 11; ++i)
    if (fin[i]) need += align256(nin[i] * sizeof(double));
  for (int i = 0; i < 8; ++i)
    if (fout[i]) need += align256(nout[i] * sizeof(double));
  if (need > e->stage_bytes) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cap);
    if (cap != cudaStreamCaptureStatusNone)
      return fail(ADRT_ERR_WORKSPACE, "FP32 staging buffer too small during stream capture");
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(e->stage);
    e->stage = nullptr;
    e->stage_bytes = 0;
    if (cudaMalloc(&e->stage, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(ADRT_ERR_OUT_OF_MEMORY, "FP32 staging allocation of %zu B failed", need);
    }
    e->stage_bytes = need;
  }
  adrt_inputs din{};
  adrt_outputs dout{};
  const double** dinp = &din.delta_tau;
  double** doutp = &dout.flux_up;
  size_t off = 0;
  for (int i = 0; i < 11; ++i) {
    if (!fin[i]) continue;
    double* dp = reinterpret_cast<double*>(e->stage + off);
    off += align256(nin[i] * sizeof(double));
    widen_kernel<<<cast_grid(nin[i], e->num_sms), 256, 0, s>>>(fin[i], dp, nin[i]);
    dinp[i] = dp;
  }
  for (int i = 0; i < 8; ++i) {
    if (!fout[i]) continue;
    doutp[i] = reinterpret_cast<double*>(e->stage + off);
    off += align256(nout[i] * sizeof(double));
  }
  CUDA_TRY(cudaGetLastError());
  if ((rc = check_inputs(d, &din))) return rc;
  if ((rc = solve_locked(e, d, &din, &dout, s))) return rc;
  for (int i = 0; i < 8; ++i) {
    if (!fout[i]) continue;
    narrow_kernel<<<cast_grid(nout[i], e->num_sms), 256, 0, s>>>(doutp[i], fout[i], nout[i]);
  }
  CUDA_TRY(cudaGetLastError());
  return ADRT_OK;
}

int adrt_solve_batch_raw(adrt_engine* e, const adrt_batch_desc* d0, const adrt_raw_inputs* in,
                         const adrt_outputs_f32* out, void* stream_ptr) {
  if (!e) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine");
  if (!d0 || !in || !out) return fail(ADRT_ERR_INVALID_ARGUMENT, "null description, inputs or outputs");
  if (!in->absorption_coeff || !in->scattering_coeff || !in->altitude || !in->temperature ||
      !in->wavenumber || !in->phase_moments)
    return fail(ADRT_ERR_INVALID_ARGUMENT,
                "raw inputs need absorption and scattering coefficients, altitude, temperature, "
                "wavenumber and phase moments");
  // the coefficients carry the sources (single-wavenumber Planck levels) and
  // their own bottom-first ordering; the moments are ordered from the top
  adrt_batch_desc d = *d0;
  d.use_thermal_emission = 0;
  d.index_from_bottom = 0;
  d.temperature_per_wavenumber = 0;
  int rc;
  {
    // the skin and top temperatures set single-wavenumber Planck emissions
    // here; the rest of the description follows the usual rules
    adrt_batch_desc v = d;
    v.surface_temperature = -1.0;
    v.top_temperature = -1.0;
    if ((rc = check_desc(&v))) return rc;
  }
  std::lock_guard<std::mutex> lk(e->mu);
  if ((rc = set_device(e))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  size_t nin[11], nout[8];
  input_counts(&d, nin);
  output_counts(&d, nout);
  const size_t nmom = nin[2];  // phase moments of this layout
  float* const* fout = &out->flux_up;
  size_t need = align256(nmom * sizeof(double));
  for (int i = 0; i < 8; ++i)
    if (fout[i]) need += align256(nout[i] * sizeof(double));
  if (need > e->stage_bytes) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cap);
    if (cap != cudaStreamCaptureStatusNone)
      return fail(ADRT_ERR_WORKSPACE, "FP32 staging buffer too small during stream capture");
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(e->stage);
    e->stage = nullptr;
    e->stage_bytes = 0;
    if (cudaMalloc(&e->stage, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(ADRT_ERR_OUT_OF_MEMORY, "FP32 staging allocation of %zu B failed", need);
    }
    e->stage_bytes = need;
  }
  adrt_inputs din{};
  adrt_outputs dout{};
  double* mom = reinterpret_cast<double*>(e->stage);
  size_t off = align256(nmom * sizeof(double));
  widen_kernel<<<cast_grid(nmom, e->num_sms), 256, 0, s>>>(in->phase_moments, mom, nmom);
  din.phase_moments = mom;
  double** doutp = &dout.flux_up;
  for (int i = 0; i < 8; ++i) {
    if (!fout[i]) continue;
    doutp[i] = reinterpret_cast<double*>(e->stage + off);
    off += align256(nout[i] * sizeof(double));
  }
  CUDA_TRY(cudaGetLastError());
  if ((rc = solve_locked(e, &d, &din, &dout, s, in))) return rc;
  for (int i = 0; i < 8; ++i) {
    if (!fout[i]) continue;
    narrow_kernel<<<cast_grid(nout[i], e->num_sms), 256, 0, s>>>(doutp[i], fout[i], nout[i]);
  }
  CUDA_TRY(cudaGetLastError());
  return ADRT_OK;
}

int adrt_gauss_legendre(int n, double* nodes, double* weights) {
  if (n < 1 || !nodes || !weights) return fail(ADRT_ERR_INVALID_ARGUMENT, "bad quadrature arguments");
  std::vector<double> x, w;
  gauss_legendre01(n, x, w);
  std::copy(x.begin(), x.end(), nodes);
  std::copy(w.begin(), w.end(), weights);
  return ADRT_OK;
}

int adrt_planck_band(double lo, double hi, double temp, double* out) {
  if (!out) return fail(ADRT_ERR_INVALID_ARGUMENT, "null output");
  if (temp < 0.0 || hi < lo || lo < 0.0)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "planckFunction: invalid arguments");
  *out = planck_band(lo, hi, temp);
  return ADRT_OK;
}

int adrt_planck_band_deriv(double lo, double hi, double temp, double* out) {
  if (!out) return fail(ADRT_ERR_INVALID_ARGUMENT, "null output");
  if (temp < 0.0 || hi < lo || lo < 0.0)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "planckFunctionDeriv: invalid arguments");
  *out = planck_band_deriv(lo, hi, temp);
  return ADRT_OK;
}

int adrt_engine_set_adjoint_mode(adrt_engine* e, int mode) {
  if (!e) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine");
  if (mode != ADRT_ADJOINT_RECORD && mode != ADRT_ADJOINT_RECOMPUTE)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "unknown adjoint mode %d", mode);
  std::lock_guard<std::mutex> lk(e->mu);
  e->adjoint_mode = mode;
  return ADRT_OK;
}

int adrt_engine_set_pivoting(adrt_engine* e, int mode) {
  if (!e) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine");
  if (mode != ADRT_PIVOTING_TENSOR_CORE && mode != ADRT_PIVOTING_PARTIAL)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "unknown pivoting mode %d", mode);
  std::lock_guard<std::mutex> lk(e->mu);
  e->pivoting = mode;
  return ADRT_OK;
}

// Hidden helper (not in the public header): the re-solve pass alone over the
// wavenumbers `tasks` of a batch, as if the solve had listed them (the list
// mechanism is otherwise reached only by a weak pivot).  Synchronous.
extern "C" int adrt_internal_resolve_listed(adrt_engine* e, const adrt_batch_desc* d,
                                            const adrt_inputs* in, const adrt_outputs* out,
                                            const long long* tasks, int ntasks) {
  if (!e || !d || !in || !out || !tasks || ntasks < 1 || ntasks > kRedoCap)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "bad re-solve list");
  int rc;
  if ((rc = adrt_internal_check_batch(d, in))) return rc;
  std::vector<unsigned long long> list(2 + ntasks, 0ull);
  list[0] = (unsigned long long)ntasks;
  for (int i = 0; i < ntasks; ++i) {
    if (tasks[i] < 0 || tasks[i] >= d->num_wavenumbers)
      return fail(ADRT_ERR_INVALID_ARGUMENT, "task %lld outside the batch", tasks[i]);
    list[2 + i] = (unsigned long long)tasks[i];
  }
  std::lock_guard<std::mutex> lk(e->mu);
  if ((rc = solve_locked(e, d, in, out, nullptr, nullptr, &list))) return rc;
  CUDA_TRY(cudaStreamSynchronize(nullptr));
  return ADRT_OK;
}

int adrt_band_integrate(adrt_engine* e, const double* spectrum, const double* weight,
                        long long num_wavenumbers, const long long* offsets, int nchannels,
                        double* out, void* stream_ptr) {
  if (!e || !spectrum || !offsets || !out)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine, spectrum, offsets or output");
  if (nchannels < 0 || num_wavenumbers < 0)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "negative channel or wavenumber count");
  if (nchannels == 0) return ADRT_OK;
  std::lock_guard<std::mutex> lk(e->mu);
  int rc;
  if ((rc = set_device(e))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  e->last_stream = s;
  const int grid = std::min(nchannels, e->num_sms * 8);
  band_integrate_kernel<<<grid, 256, 0, s>>>(spectrum, weight, num_wavenumbers, offsets, nchannels,
                                             out, e->status);
  CUDA_TRY(cudaGetLastError());
  return ADRT_OK;
}

int adrt_adjoint(adrt_engine* e, const adrt_batch_desc* d, const adrt_inputs* in,
                 const adrt_outputs* out, const adrt_cotangents* cot, const adrt_gradients* gr,
                 void* stream_ptr) {
  if (!e || !cot || !gr) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine, cotangents or gradients");
  int rc = check_desc(d);
  if (rc) return rc;
  if ((rc = check_inputs(d, in))) return rc;
  std::lock_guard<std::mutex> lk(e->mu);
  if ((rc = set_device(e))) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  e->last_stream = s;
  if ((rc = ensure_quad(e, d->num_quadrature, d->num_moments))) return rc;
  const int np = padded_order(d->num_quadrature);
  // Per chunk of wavenumbers: tape_kernel (the forward kernel's geometry)
  // leaves each wavenumber's state and doubling records in HBM, then
  // adjoint_kernel runs the reverse on them.
  struct AK {
    int groups, threads, fgroups, fthreads, gthreads, np, tile;
    size_t smem, fsmem, gsmem, scr, state;
    long long step;  // doubles per recorded doubling step
    const void *fn, *ffn, *tfn, *pfn;
    void (*launch)(const SolveParams&, const ColumnDev&, const AdjDev&, int, size_t, cudaStream_t);
    void (*flaunch)(const SolveParams&, const ColumnDev&, const AdjDev&, int, size_t, cudaStream_t);
    // per shared moment set: phase table, and the moment gradients' finish
    void (*tlaunch)(const ColumnDev&, double*, int, size_t, cudaStream_t);
    void (*plaunch)(const ColumnDev&, const AdjDev&, int, size_t, cudaStream_t);
  } k{};
  const int L = d->num_layers;
  auto make = [&](auto tag) {
    constexpr int NP = decltype(tag)::value;
    using GD = AdjGeo<NP>;
    using GC = Geo<NP, double>;
    k.groups = AdjKern<NP>::kGroups;
    k.threads = AdjKern<NP>::kThreads;
    k.smem = (size_t)k.groups * AdjGroup<NP>::bytes;
    k.scr = align256(AdjScratch<GD>::bytes(L, d->num_moments));
    k.state = align256(WavState<GC>::bytes(L));
    k.step = TapeLayout<GC>::STEP;
    k.fthreads = Kern<NP, KIND_FP64>::kThreads;
    k.fgroups = Kern<NP, KIND_FP64>::kGroups;
    k.fsmem = Kern<NP, KIND_FP64>::smem();
    k.fn = reinterpret_cast<const void*>(adjoint_kernel<NP>);
    k.ffn = reinterpret_cast<const void*>(tape_kernel<NP>);
    k.launch = [](const SolveParams& p, const ColumnDev& c, const AdjDev& a, int grid, size_t smem,
                  cudaStream_t st) {
      adjoint_kernel<NP><<<grid, AdjKern<NP>::kThreads, smem, st>>>(p, c, a);
    };
    k.flaunch = [](const SolveParams& p, const ColumnDev& c, const AdjDev& a, int grid,
                   size_t smem, cudaStream_t st) {
      tape_kernel<NP><<<grid, Kern<NP, KIND_FP64>::kThreads, smem, st>>>(p, c, a);
    };
    k.np = NP;
    k.tile = GD::G * GD::TE;
    k.gthreads = GD::G;
    k.gsmem = AdjGroup<NP>::bytes;
    k.tfn = reinterpret_cast<const void*>(phase_table_kernel<NP>);
    k.pfn = reinterpret_cast<const void*>(phase_finish_kernel<NP>);
    k.tlaunch = [](const ColumnDev& c, double* tab, int sets, size_t smem, cudaStream_t st) {
      phase_table_kernel<NP><<<sets, GD::G, smem, st>>>(c, tab);
    };
    k.plaunch = [](const ColumnDev& c, const AdjDev& a, int sets, size_t smem, cudaStream_t st) {
      phase_finish_kernel<NP><<<sets, GD::G, smem, st>>>(c, a);
    };
  };
  switch (np) {
    case 4: make(std::integral_constant<int, 4>{}); break;
    case 8: make(std::integral_constant<int, 8>{}); break;
    case 16: make(std::integral_constant<int, 16>{}); break;
    default: make(std::integral_constant<int, 32>{}); break;
  }
  CUDA_TRY(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem));
  CUDA_TRY(cudaFuncSetAttribute(k.ffn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.fsmem));
  CUDA_TRY(cudaFuncSetAttribute(k.tfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.gsmem));
  CUDA_TRY(cudaFuncSetAttribute(k.pfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.gsmem));
  int bps = 0, fbps = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k.fn, k.threads, k.smem));
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fbps, k.ffn, k.fthreads, k.fsmem));
  if (bps < 1) bps = 1;
  if (fbps < 1) fbps = 1;
  const long long W = d->num_wavenumbers;
  // chunk: one wavenumber per resident forward group, within the memory budget
  const long long rgroups = (long long)bps * e->num_sms * k.groups;
  const size_t rev_bytes = (size_t)rgroups * k.scr;
  const bool recompute = e->adjoint_mode == ADRT_ADJOINT_RECOMPUTE;
  const size_t per_w =
      k.state + (recompute ? 0 : (size_t)L * kTapeStepsPerLayer * k.step * sizeof(double));
  const size_t budget = e->max_ws ? e->max_ws : kAdjointMemory;
  // moment sets shared by every wavenumber (one per layer): their phase
  // matrices once per call, and per-block sums of the phase-matrix cotangents
  // (within kPhaseSumMemory and the budget; else the sets' adjoint runs per
  // layer)
  const bool shared_sets = d->moment_layout == ADRT_MOMENTS_SHARED;
  const int sum_blocks = bps * e->num_sms;
  const size_t ptab_bytes = shared_sets ? align256((size_t)L * 2 * k.np * k.np * sizeof(double)) : 0;
  size_t psum_bytes = (shared_sets && gr->phase_moments)
                          ? align256((size_t)L * sum_blocks * 2 * k.tile * sizeof(double)) : 0;
  if (psum_bytes > kPhaseSumMemory || budget < rev_bytes + per_w + ptab_bytes + psum_bytes)
    psum_bytes = 0;
  const size_t fixed = rev_bytes + ptab_bytes + psum_bytes + 512;
  if (budget < fixed + per_w)
    return fail(ADRT_ERR_WORKSPACE, "workspace limit below one adjoint chunk (%zu B)",
                fixed + per_w);
  long long wc = std::min<long long>(W, (long long)fbps * e->num_sms * k.fgroups);
  wc = std::max<long long>(1, std::min<long long>(wc, (long long)((budget - fixed) / per_w)));
  // ADRT_ADJOINT_RECOMPUTE: no record pool, every chain recomputed in the reverse
  const long long pool_cap = recompute ? 0 : wc * L * kTapeStepsPerLayer * k.step;
  const size_t ext = align256(rev_bytes + (size_t)wc * k.state + (size_t)pool_cap * sizeof(double) +
                              sizeof(unsigned long long));
  const size_t need = ext + ptab_bytes + psum_bytes;
  if (need > e->adj_scratch_bytes) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cap);
    if (cap != cudaStreamCaptureStatusNone)
      return fail(ADRT_ERR_WORKSPACE, "adjoint work buffer too small during stream capture");
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(e->adj_scratch);
    e->adj_scratch = nullptr;
    e->adj_scratch_bytes = 0;
    if (cudaMalloc(&e->adj_scratch, need) != cudaSuccess) {
      cudaGetLastError();
      return fail(ADRT_ERR_OUT_OF_MEMORY, "adjoint work buffer allocation of %zu B failed", need);
    }
    e->adj_scratch_bytes = need;
  }
  ColumnDev c0 = make_column(e, d, in, out);
  SolveParams p{};
  p.cols = nullptr;
  p.ncols = 1;
  p.counter = e->counter;
  p.status = e->status;
  p.pivot_all = e->pivoting == ADRT_PIVOTING_PARTIAL;  // the taping forward's solves
  p.scratch = e->adj_scratch;
  p.slot_bytes = k.scr;
  p.max_layers = L;
  AdjDev a{};
  a.c_fu = cot->flux_up;
  a.c_fd = cot->flux_down;
  a.c_J = cot->mean_intensity;
  a.c_fdir = cot->flux_direct;
  a.g_tau = gr->delta_tau;
  a.g_ssa = gr->single_scat_albedo;
  a.g_mom = gr->phase_moments;
  a.g_temp = gr->temperature;
  a.g_planck = gr->planck_levels;
  a.g_semis = gr->surface_emission;
  a.state = e->adj_scratch + rev_bytes;
  a.state_bytes = k.state;
  a.pool = reinterpret_cast<double*>(a.state + (size_t)wc * k.state);
  a.pool_cap = pool_cap;
  a.pool_used = reinterpret_cast<unsigned long long*>(a.pool + pool_cap);
  a.ptab = ptab_bytes ? reinterpret_cast<double*>(e->adj_scratch + ext) : nullptr;
  a.pacc = psum_bytes ? reinterpret_cast<double*>(e->adj_scratch + ext + ptab_bytes) : nullptr;
  a.pacc_blocks = sum_blocks;
  if (ptab_bytes) {
    k.tlaunch(c0, const_cast<double*>(a.ptab), L, k.gsmem, s);
    CUDA_TRY(cudaGetLastError());
    c0.ptab = a.ptab;  // the taping forward reads the table too
  }
  if (psum_bytes) CUDA_TRY(cudaMemsetAsync(a.pacc, 0, psum_bytes, s));
  for (long long w0 = 0; w0 < W; w0 += wc) {
    const long long nw = std::min(wc, W - w0);
    a.w0 = w0;
    p.ntasks = nw;
    const int fgrid = (int)std::min<long long>((long long)fbps * e->num_sms,
                                               (nw + k.fgroups - 1) / k.fgroups);
    const int rgrid = (int)std::min<long long>((long long)bps * e->num_sms,
                                               (nw + k.groups - 1) / k.groups);
    p.nslots = rgrid * k.groups;
    CUDA_TRY(cudaMemsetAsync(e->counter, 0, sizeof(unsigned long long), s));
    CUDA_TRY(cudaMemsetAsync(a.pool_used, 0, sizeof(unsigned long long), s));
    k.flaunch(p, c0, a, fgrid, k.fsmem, s);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemsetAsync(e->counter, 0, sizeof(unsigned long long), s));
    k.launch(p, c0, a, rgrid, k.smem, s);
    CUDA_TRY(cudaGetLastError());
  }
  if (psum_bytes) {
    k.plaunch(c0, a, L, k.gsmem, s);
    CUDA_TRY(cudaGetLastError());
  }
  return ADRT_OK;
}

int adrt_solve_batch_uneven(adrt_engine* e, const adrt_column_desc* cols, int ncols,
                            void* stream_ptr) {
  if (!e || !cols || ncols < 1) return fail(ADRT_ERR_INVALID_ARGUMENT, "bad uneven-batch arguments");
  int rc;
  for (int i = 0; i < ncols; ++i) {
    if ((rc = check_desc(&cols[i].desc))) return rc;
    if ((rc = check_inputs(&cols[i].desc, &cols[i].in))) return rc;
  }
  std::lock_guard<std::mutex> lk(e->mu);
  std::vector<UnevenColumn> cv(ncols);
  for (int i = 0; i < ncols; ++i) cv[i] = UnevenColumn{&cols[i], cols[i].desc.num_wavenumbers};
  return uneven_locked(e, cv, static_cast<cudaStream_t>(stream_ptr), e->plan);
}

int adrt_engine_set_uneven_plan(adrt_engine* e, const adrt_uneven_plan* plan) {
  if (!e || !plan) return fail(ADRT_ERR_INVALID_ARGUMENT, "null argument");
  for (int m : plan->mapping)
    if (m != ADRT_MAPPING_WARP && m != ADRT_MAPPING_THREAD)
      return fail(ADRT_ERR_INVALID_ARGUMENT, "unknown mapping %d", m);
  if (plan->warp_blocks_per_sm < 0)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "warp_blocks_per_sm must be >= 0");
  std::lock_guard<std::mutex> lk(e->mu);
  e->plan = *plan;
  return ADRT_OK;
}

int adrt_engine_get_uneven_plan(const adrt_engine* e, adrt_uneven_plan* plan) {
  if (!e || !plan) return fail(ADRT_ERR_INVALID_ARGUMENT, "null argument");
  *plan = e->plan;
  return ADRT_OK;
}

int adrt_engine_autotune_uneven(adrt_engine* e, const adrt_column_desc* cols, int ncols,
                                void* stream_ptr, adrt_uneven_plan* out) {
  if (!e || !cols || ncols < 1) return fail(ADRT_ERR_INVALID_ARGUMENT, "bad uneven-batch arguments");
  int rc;
  for (int i = 0; i < ncols; ++i) {
    if ((rc = check_desc(&cols[i].desc))) return rc;
    if ((rc = check_inputs(&cols[i].desc, &cols[i].in))) return rc;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  std::lock_guard<std::mutex> lk(e->mu);
  if ((rc = set_device(e))) return rc;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cap);
  if (cap != cudaStreamCaptureStatusNone)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "the autotuner times launches: not during a capture");
  adrt_uneven_plan plan = e->plan;
  for (auto& r : plan.ns_per_wavenumber) r[0] = r[1] = 0.0;
  cudaEvent_t ev0, ev1;
  CUDA_TRY(cudaEventCreate(&ev0));
  CUDA_TRY(cudaEventCreate(&ev1));
  // ns per wavenumber of `cv` under `p` (one warm-up run, then one timed).
  // With give_up > 0 the warm-up run is timed too (allocation included), and
  // a mapping already slower than give_up ns per wavenumber there keeps that
  // figure without the second run.
  auto time_plan = [&](std::vector<UnevenColumn>& cv, const adrt_uneven_plan& p, double* ns,
                       double give_up = 0.0) -> int {
    long long n = 0;
    for (auto& c : cv) n += c.W;
    if (n == 0) return ADRT_OK;
    if (give_up > 0.0) CUDA_TRY(cudaEventRecord(ev0, s));
    int r = uneven_locked(e, cv, s, p);
    if (r) return r;
    if (give_up > 0.0) {
      CUDA_TRY(cudaEventRecord(ev1, s));
      CUDA_TRY(cudaEventSynchronize(ev1));
      float ms0 = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&ms0, ev0, ev1));
      if (ms0 * 1e6 / (double)n > give_up) {
        *ns = ms0 * 1e6 / (double)n;
        return ADRT_OK;
      }
    }
    CUDA_TRY(cudaEventRecord(ev0, s));
    if ((r = uneven_locked(e, cv, s, p))) return r;
    CUDA_TRY(cudaEventRecord(ev1, s));
    CUDA_TRY(cudaEventSynchronize(ev1));
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, ev0, ev1));
    *ns = ms * 1e6 / (double)n;
    return ADRT_OK;
  };
  // 1. per padded order: the two mappings on a sample of that order's FP64
  //    wavenumbers, large enough for several waves of either launch
  const int orders[3] = {4, 8, 16};
  for (int oi = 0; oi < 3 && !rc; ++oi) {
    std::vector<int> ids;
    int lmax = 1;
    for (int i = 0; i < ncols; ++i)
      if (padded_order(cols[i].desc.num_quadrature) == orders[oi] &&
          cols[i].desc.precision == ADRT_PRECISION_FP64) {
        ids.push_back(i);
        lmax = std::max(lmax, cols[i].desc.num_layers);
      }
    if (ids.empty()) continue;
    const long long warp_slots = (long long)warp_blocks_per_sm_max() * e->num_sms * 4;
    const long long thread_slots = tpw_slots(e, orders[oi], lmax, 1ll << 40);
    const long long want = 3 * std::max(warp_slots, thread_slots);
    std::vector<UnevenColumn> cv;
    long long taken = 0;
    // the same share of every column (columns differ in L and W)
    long long total = 0;
    for (int i : ids) total += cols[i].desc.num_wavenumbers;
    const double frac = std::min(1.0, (double)want / (double)total);
    for (int i : ids) {
      const int w = std::max(1, (int)std::ceil(frac * cols[i].desc.num_wavenumbers));
      cv.push_back(UnevenColumn{&cols[i], std::min(w, cols[i].desc.num_wavenumbers)});
      taken += cv.back().W;
    }
    (void)taken;
    adrt_uneven_plan p = plan;
    double ns[2] = {0.0, 0.0};
    p.mapping[oi] = ADRT_MAPPING_WARP;
    rc = time_plan(cv, p, &ns[0]);
    if (rc) break;
    // the thread mapping first on an eighth of the sample; one more than four
    // times slower there per wavenumber is not timed on the whole sample (at
    // N = 16 that takes seconds).  The pilot fills at most 3/8 of the thread
    // slots, which inflates its time per wavenumber by less than 4x, so a
    // mapping it drops is slower than the warp mapping on the whole sample.
    std::vector<UnevenColumn> pilot = cv;
    for (auto& c : pilot) c.W = std::max(1, c.W / 8);
    p.mapping[oi] = ADRT_MAPPING_THREAD;
    // (a warm-up pilot fifty times slower than the warp mapping -- the thread
    // mapping at N = 16, whose every launch lasts one whole wavenumber's
    // solve, seconds -- is not run a second time)
    rc = time_plan(pilot, p, &ns[1], 50.0 * ns[0]);
    if (!rc && !(ns[1] > 4.0 * ns[0])) rc = time_plan(cv, p, &ns[1]);
    if (rc) break;
    plan.ns_per_wavenumber[oi][0] = ns[0];
    plan.ns_per_wavenumber[oi][1] = ns[1];
    plan.mapping[oi] = (ns[1] > 0.0 && ns[1] < ns[0]) ? ADRT_MAPPING_THREAD : ADRT_MAPPING_WARP;
  }
  // 2. the warp launch's grid cap, on a sample of everything it runs
  if (!rc) {
    std::vector<UnevenColumn> cv;
    long long total = 0;
    for (int i = 0; i < ncols; ++i) {
      const int np = padded_order(cols[i].desc.num_quadrature);
      const bool warp = np <= 16 && (cols[i].desc.precision != ADRT_PRECISION_FP64 ||
                                     plan.mapping[np == 4 ? 0 : np == 8 ? 1 : 2] ==
                                         ADRT_MAPPING_WARP);
      if (warp) total += cols[i].desc.num_wavenumbers;
    }
    const long long want = 3ll * warp_blocks_per_sm_max() * e->num_sms * 4;
    const double frac = total ? std::min(1.0, (double)want / (double)total) : 0.0;
    for (int i = 0; i < ncols && total; ++i) {
      const int np = padded_order(cols[i].desc.num_quadrature);
      if (np > 16) continue;
      const int w = std::max(1, (int)std::ceil(frac * cols[i].desc.num_wavenumbers));
      cv.push_back(UnevenColumn{&cols[i], std::min(w, cols[i].desc.num_wavenumbers)});
    }
    double best = 0.0;
    int best_b = 0;
    for (int b = warp_blocks_per_sm_max(); b >= 1 && !rc && !cv.empty(); --b) {
      adrt_uneven_plan p = plan;
      p.warp_blocks_per_sm = b;
      double ns = 0.0;
      rc = time_plan(cv, p, &ns);
      if (!rc && (best_b == 0 || ns < best)) {
        best = ns;
        best_b = b;
      }
    }
    plan.warp_blocks_per_sm = (best_b == warp_blocks_per_sm_max()) ? 0 : best_b;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (rc) return rc;
  e->plan = plan;
  if (out) *out = plan;
  return ADRT_OK;
}

int adrt_solve_batch_host(adrt_engine* e, const adrt_batch_desc* d, const adrt_inputs* hin,
                          const adrt_outputs* hout) {
  if (!e) return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine");
  int rc = check_desc(d);
  if (rc) return rc;
  if ((rc = check_inputs(d, hin))) return rc;
  if (!hout) return fail(ADRT_ERR_INVALID_ARGUMENT, "null outputs");
  std::lock_guard<std::mutex> hl(e->hmu);
  {
    std::lock_guard<std::mutex> lk(e->mu);
    if ((rc = set_device(e))) return rc;
  }
  // Arrays split by wavenumber into chunks (per-wavenumber arrays) or copied
  // once (shared moments, a common temperature profile).  Chunk i is copied
  // in on hs[0], solved on hs[1] and copied out on hs[2], into one of two
  // buffer sets, so the copies of one chunk overlap the solves of its
  // neighbours; hev[b] / hev[2+b] / hev[4+b] mark buffer set b's copy-in,
  // solve and copy-out.
  const size_t W = d->num_wavenumbers, L = d->num_layers, M = d->num_moments;
  const bool mom_w = d->moment_layout != ADRT_MOMENTS_SHARED;
  const size_t mom_per = d->moment_layout == ADRT_MOMENTS_PER_WAVENUMBER ? M : L * M;
  struct Arr {
    const double* h;
    size_t per;   // elements per wavenumber, or total elements when shared
    bool per_w;
  };
  const Arr ins[11] = {{hin->delta_tau, L, true},
                       {hin->single_scat_albedo, L, true},
                       {hin->phase_moments, mom_w ? mom_per : L * M, mom_w},
                       {hin->temperature, L + 1, d->temperature_per_wavenumber != 0},
                       {hin->planck_levels, L + 1, true},
                       {hin->surface_albedo, 1, true},
                       {hin->solar_mu, 1, true},
                       {hin->wavenumber_low, 1, true},
                       {hin->wavenumber_high, 1, true},
                       {hin->surface_emission, 1, true},
                       {hin->top_emission, 1, true}};
  double* const* outs_h = &hout->flux_up;
  const size_t out_per[8] = {L + 1, L + 1, L + 1, L + 1, L + 1, 1, 1, 1};
  const int nchunks = (int)std::max<size_t>(1, std::min<size_t>(4, W / kHostChunkMin));
  const size_t wc = (W + nchunks - 1) / nchunks;
  auto a256 = [](size_t b) { return (b + 255) & ~size_t(255); };
  size_t shared_b = 0, set_b = 0;
  for (const auto& a : ins) {
    if (!a.h) continue;
    if (a.per_w)
      set_b += a256(wc * a.per * sizeof(double));
    else
      shared_b += a256(a.per * sizeof(double));
  }
  for (int i = 0; i < 8; ++i)
    if (outs_h[i]) set_b += a256(wc * out_per[i] * sizeof(double));
  const int nsets = nchunks > 1 ? 2 : 1;
  const size_t total = shared_b + nsets * set_b;
  if (!e->hs[0]) {
    for (auto& st : e->hs) CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& ev : e->hev) CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  }
  if (total > e->hstage_bytes) {
    CUDA_TRY(cudaDeviceSynchronize());
    cudaFree(e->hstage);
    e->hstage = nullptr;
    e->hstage_bytes = 0;
    if (cudaMalloc(&e->hstage, total) != cudaSuccess) {
      cudaGetLastError();
      return fail(ADRT_ERR_OUT_OF_MEMORY, "host-entry staging allocation of %zu B failed", total);
    }
    e->hstage_bytes = total;
  }
  cudaStream_t sin = e->hs[0], scmp = e->hs[1], sout = e->hs[2];
  const double* shared_d[11] = {};
  size_t off = 0;
  rc = ADRT_OK;
  for (int i = 0; i < 11 && rc == ADRT_OK; ++i) {
    if (!ins[i].h || ins[i].per_w) continue;
    double* dp = reinterpret_cast<double*>(e->hstage + off);
    off += a256(ins[i].per * sizeof(double));
    if (cudaMemcpyAsync(dp, ins[i].h, ins[i].per * sizeof(double), cudaMemcpyHostToDevice,
                        sin) != cudaSuccess)
      rc = fail(ADRT_ERR_CUDA, "host-to-device copy failed");
    shared_d[i] = dp;
  }
  const size_t set0 = off;
  for (int c = 0; c < nchunks && rc == ADRT_OK; ++c) {
    const size_t w0 = c * wc, n = std::min(wc, W - w0);
    if (n == 0) break;
    const int b = c % nsets;
    char* base = e->hstage + set0 + b * set_b;
    adrt_inputs din{};
    adrt_outputs dout{};
    const double** din_p = &din.delta_tau;
    double** dout_p = &dout.flux_up;
    size_t o = 0;
    // copy-in of this set waits for the solve that last read it
    if (c >= nsets) CUDA_TRY(cudaStreamWaitEvent(sin, e->hev[2 + b], 0));
    for (int i = 0; i < 11 && rc == ADRT_OK; ++i) {
      if (!ins[i].h) continue;
      if (!ins[i].per_w) {
        din_p[i] = shared_d[i];
        continue;
      }
      double* dp = reinterpret_cast<double*>(base + o);
      o += a256(wc * ins[i].per * sizeof(double));
      if (cudaMemcpyAsync(dp, ins[i].h + w0 * ins[i].per, n * ins[i].per * sizeof(double),
                          cudaMemcpyHostToDevice, sin) != cudaSuccess)
        rc = fail(ADRT_ERR_CUDA, "host-to-device copy failed");
      din_p[i] = dp;
    }
    for (int i = 0; i < 8; ++i) {
      if (!outs_h[i]) continue;
      dout_p[i] = reinterpret_cast<double*>(base + o);
      o += a256(wc * out_per[i] * sizeof(double));
    }
    if (rc != ADRT_OK) break;
    CUDA_TRY(cudaEventRecord(e->hev[b], sin));
    // the solve waits for its inputs and for the copy-out of this set's last chunk
    CUDA_TRY(cudaStreamWaitEvent(scmp, e->hev[b], 0));
    if (c >= nsets) CUDA_TRY(cudaStreamWaitEvent(scmp, e->hev[4 + b], 0));
    adrt_batch_desc dc = *d;
    dc.num_wavenumbers = (int)n;
    if ((rc = adrt_solve_batch(e, &dc, &din, &dout, scmp))) break;
    CUDA_TRY(cudaEventRecord(e->hev[2 + b], scmp));
    CUDA_TRY(cudaStreamWaitEvent(sout, e->hev[2 + b], 0));
    for (int i = 0; i < 8 && rc == ADRT_OK; ++i) {
      if (!outs_h[i]) continue;
      if (cudaMemcpyAsync(outs_h[i] + w0 * out_per[i], dout_p[i], n * out_per[i] * sizeof(double),
                          cudaMemcpyDeviceToHost, sout) != cudaSuccess)
        rc = fail(ADRT_ERR_CUDA, "device-to-host copy failed");
    }
    CUDA_TRY(cudaEventRecord(e->hev[4 + b], sout));
  }
  cudaError_t se = cudaStreamSynchronize(sout);
  if (se == cudaSuccess) se = cudaStreamSynchronize(scmp);
  if (se == cudaSuccess) se = cudaStreamSynchronize(sin);
  if (rc == ADRT_OK && se != cudaSuccess)
    rc = fail(ADRT_ERR_CUDA, "solve failed: %s", cudaGetErrorString(se));
  return rc;
}

int adrt_adjoint_host(adrt_engine* e, const adrt_batch_desc* d, const adrt_inputs* hin,
                      const adrt_cotangents* hcot, const adrt_gradients* hgr) {
  if (!e || !hin || !hcot || !hgr)
    return fail(ADRT_ERR_INVALID_ARGUMENT, "null engine, inputs, cotangents or gradients");
  int rc = check_desc(d);
  if (rc) return rc;
  if ((rc = check_inputs(d, hin))) return rc;
  {
    std::lock_guard<std::mutex> lk(e->mu);
    if ((rc = set_device(e))) return rc;
  }
  const size_t W = d->num_wavenumbers, L = d->num_layers, M = d->num_moments;
  const size_t nmom = d->moment_layout == ADRT_MOMENTS_SHARED ? L * M
                      : d->moment_layout == ADRT_MOMENTS_PER_WAVENUMBER ? W * M : W * L * M;
  const size_t ntemp = (d->temperature_per_wavenumber ? W : 1) * (L + 1);
  struct Arr {
    const double* h;
    size_t n;
  };
  const Arr ins[11] = {{hin->delta_tau, W * L}, {hin->single_scat_albedo, W * L},
                       {hin->phase_moments, nmom}, {hin->temperature, ntemp},
                       {hin->planck_levels, W * (L + 1)}, {hin->surface_albedo, W},
                       {hin->solar_mu, W}, {hin->wavenumber_low, W},
                       {hin->wavenumber_high, W}, {hin->surface_emission, W},
                       {hin->top_emission, W}};
  const Arr cots[4] = {{hcot->flux_up, W * (L + 1)}, {hcot->flux_down, W * (L + 1)},
                       {hcot->mean_intensity, W * (L + 1)}, {hcot->flux_direct, W * (L + 1)}};
  double* const grads_h[6] = {hgr->delta_tau, hgr->single_scat_albedo, hgr->phase_moments,
                              hgr->temperature, hgr->planck_levels, hgr->surface_emission};
  const size_t grad_n[6] = {W * L, W * L, nmom, ntemp, W * (L + 1), W};
  auto a256 = [](size_t b) { return (b + 255) & ~size_t(255); };
  size_t total = 0;
  for (const auto& a : ins)
    if (a.h) total += a256(a.n * sizeof(double));
  for (const auto& a : cots)
    if (a.h) total += a256(a.n * sizeof(double));
  for (int i = 0; i < 6; ++i)
    if (grads_h[i]) total += a256(grad_n[i] * sizeof(double));
  char* dbuf = nullptr;
  if (cudaMalloc(&dbuf, total) != cudaSuccess) {
    cudaGetLastError();
    return fail(ADRT_ERR_OUT_OF_MEMORY, "host-entry staging allocation of %zu B failed", total);
  }
  cudaStream_t s = nullptr;
  adrt_inputs din{};
  adrt_cotangents dcot{};
  adrt_gradients dgr{};
  const double** din_p = &din.delta_tau;
  const double** dcot_p = &dcot.flux_up;
  double** dgr_p = &dgr.delta_tau;
  size_t off = 0;
  rc = ADRT_OK;
  auto put = [&](const double* h, size_t n) -> double* {
    double* dp = reinterpret_cast<double*>(dbuf + off);
    off += a256(n * sizeof(double));
    if (cudaMemcpyAsync(dp, h, n * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
      rc = fail(ADRT_ERR_CUDA, "host-to-device copy failed");
    return dp;
  };
  for (int i = 0; i < 11 && rc == ADRT_OK; ++i)
    if (ins[i].h) din_p[i] = put(ins[i].h, ins[i].n);
  for (int i = 0; i < 4 && rc == ADRT_OK; ++i)
    if (cots[i].h) dcot_p[i] = put(cots[i].h, cots[i].n);
  // gradients that the adjoint adds to start from the caller's values
  for (int i = 0; i < 6 && rc == ADRT_OK; ++i)
    if (grads_h[i]) dgr_p[i] = put(grads_h[i], grad_n[i]);
  if (rc == ADRT_OK) rc = adrt_adjoint(e, d, &din, nullptr, &dcot, &dgr, s);
  for (int i = 0; i < 6 && rc == ADRT_OK; ++i)
    if (grads_h[i] && cudaMemcpyAsync(grads_h[i], dgr_p[i], grad_n[i] * sizeof(double),
                                      cudaMemcpyDeviceToHost, s) != cudaSuccess)
      rc = fail(ADRT_ERR_CUDA, "device-to-host copy failed");
  cudaError_t se = cudaStreamSynchronize(s);
  cudaFree(dbuf);
  if (rc == ADRT_OK && se != cudaSuccess)
    rc = fail(ADRT_ERR_CUDA, "adjoint failed: %s", cudaGetErrorString(se));
  return rc;
}

}  // extern "C"
