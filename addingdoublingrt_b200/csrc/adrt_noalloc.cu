// adrt_noalloc.cu -- adrt_solve_batch_noalloc: the batched solve for callers
// that must not allocate device memory.
//
// Some callers cannot call cudaMalloc: code that runs while a framework's
// caching allocator (PyTorch, JAX/XLA) has already reserved nearly all of
// the GPU's memory, so a raw allocation fails or fragments the pool; code on
// a real-time or retrieval path where an allocation's implicit device
// synchronisation is not acceptable; and plugin hosts that give a library
// only the buffers they pass in.  For them this entry point keeps all of the
// solver's work memory in one fixed array compiled into the library.
//
// The work memory is a file-scope __device__ array of kNoAllocScratchBytes
// (64 MiB) on every GPU that loads the library, held until the process
// exits.  It holds a 256-byte header (work counter, status word), the
// quadrature table of the call's N, and as many per-wavenumber work slots
// as fit; fewer slots than the engine uses means fewer wavenumbers in flight
// at once, not a different result.  Every call shares the array and it keeps
// the last call's contents: the counter, status word and quadrature table are
// rewritten by each call before its kernel runs, so calls that overlap on the
// GPU (on different streams, or from different host threads) race and must
// not be issued.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/adrt_b200.h"
#include "adrt_kernel.cuh"

using namespace adrt_dev;

void adrt_internal_set_detail(const char* msg);  // adrt_engine.cu

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr size_t kHeaderBytes = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) char g_noalloc_scratch[kNoAllocScratchBytes];

// The persistent solve loop of solve_kernel (adrt_kernel.cuh), with its
// slots, counter and status word in the static work memory.
template <int NP, int KIND>
__global__ void __launch_bounds__(128) solve_kernel_static(SolveParams P, ColumnDev col0) {
  using GD = Geo<NP, double>;
  using GF = Geo<NP, float>;
  using GL = GroupLayout<NP, KIND>;
  constexpr int G = GD::G;
  const int gib = threadIdx.x / G;
  const int t = threadIdx.x % G;
  const int bar = 1 + gib;
  const unsigned goff = (unsigned)(gib * GL::bytes);
  const unsigned tb = goff + (unsigned)CommonLayout<NP>::bytes;
  const int slot = blockIdx.x * (blockDim.x / G) + gib;
  if (slot >= P.nslots) return;  // the whole group leaves together
  char* sl = P.scratch + (size_t)slot * P.slot_bytes;
  for (unsigned i = (unsigned)t * 4u; i < (unsigned)GL::bytes; i += (unsigned)G * 4u)
    *sp<unsigned>(goff + i) = 0u;
  gsync<G>(bar);
  ColumnDev* colp = sp<ColumnDev>(goff + CommonLayout<NP>::col);
  if (t == 0) *colp = col0;
  long long* task_s = sp<long long>(goff + CommonLayout<NP>::misc + 32);
  for (;;) {
    long long task;
    if constexpr (G == 32) {
      unsigned long long v = 0;
      if (t == 0) v = atomicAdd(P.counter, 1ull);
      task = (long long)__shfl_sync(0xffffffffu, v, 0);
    } else {
      gsync<G>(bar);
      if (t == 0) *task_s = (long long)atomicAdd(P.counter, 1ull);
      gsync<G>(bar);
      task = *task_s;
    }
    if (task >= P.ntasks) break;
    const int w = (int)task;
    gsync<G>(bar);
    const int any =
        wav_prologue<NP>(goff, t, bar, w, sl, P.max_layers, P.status, KIND == KIND_MIXED);
    if constexpr (KIND == KIND_FP64) {
      wav_body<GD, MODE_FP64>(goff, tb, 0u, t, bar, w, sl, P.max_layers, P.status);
    } else if (!any) {
      wav_body<GF, MODE_MIX_S>(goff, tb, 0u, t, bar, w, sl, P.max_layers, P.status);
    } else {
      wav_body<GD, MODE_MIX_D>(goff, tb, tb + (unsigned)GL::lamF_in_D, t, bar, w, sl,
                               P.max_layers, P.status);
    }
  }
}

int na_fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  adrt_internal_set_detail(buf);
  return code;
}

// Device address of the static work memory, looked up once per device.
std::mutex g_na_mu;
char* g_na_addr[kMaxDevices] = {};

int na_setup(int dev, char** addr) {
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return na_fail(ADRT_ERR_CUDA, "cudaGetSymbolAddress of the static work memory: %s",
                     cudaGetErrorString(e));
    g_na_addr[dev] = static_cast<char*>(p);
  }
  *addr = g_na_addr[dev];
  return ADRT_OK;
}

struct NaKern {
  int groups;
  size_t smem;
  size_t (*slot_bytes)(int);
  cudaError_t (*prepare)(size_t);
  int (*blocks_per_sm)(size_t);
  void (*launch)(const SolveParams&, const ColumnDev&, int, size_t, cudaStream_t);
};

template <int NP, int KIND>
NaKern na_kern() {
  using GD = Geo<NP, double>;
  NaKern k;
  k.groups = 128 / GD::G;
  k.smem = (size_t)k.groups * GroupLayout<NP, KIND>::bytes;
  k.slot_bytes = [](int lmax) { return SlotLayout<GD>::bytes(lmax); };
  k.prepare = [](size_t smem) {
    return cudaFuncSetAttribute(solve_kernel_static<NP, KIND>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  };
  k.blocks_per_sm = [](size_t smem) {
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, solve_kernel_static<NP, KIND>, 128, smem);
    return nb > 0 ? nb : 1;
  };
  k.launch = [](const SolveParams& p, const ColumnDev& c, int grid, size_t smem,
                cudaStream_t s) { solve_kernel_static<NP, KIND><<<grid, 128, smem, s>>>(p, c); };
  return k;
}

NaKern na_pick(int n, int precision) {
  const int np = n <= 4 ? 4 : n <= 8 ? 8 : n <= 16 ? 16 : 32;
  if (precision == ADRT_PRECISION_MIXED) {
    switch (np) {
      case 4: return na_kern<4, KIND_MIXED>();
      case 8: return na_kern<8, KIND_MIXED>();
      case 16: return na_kern<16, KIND_MIXED>();
      default: return na_kern<32, KIND_MIXED>();
    }
  }
  switch (np) {
    case 4: return na_kern<4, KIND_FP64>();
    case 8: return na_kern<8, KIND_FP64>();
    case 16: return na_kern<16, KIND_FP64>();
    default: return na_kern<32, KIND_FP64>();
  }
}

}  // namespace

extern "C" int adrt_solve_batch_noalloc(const adrt_batch_desc* d, const adrt_inputs* in,
                                        const adrt_outputs* out, void* stream_ptr) {
  if (!d || !in || !out) return na_fail(ADRT_ERR_INVALID_ARGUMENT, "null argument");
  if (d->num_wavenumbers < 1 || d->num_layers < 1)
    return na_fail(ADRT_ERR_INVALID_ARGUMENT, "num_wavenumbers and num_layers must be >= 1");
  if (d->num_quadrature < 2 || d->num_quadrature > kMaxN)
    return na_fail(ADRT_ERR_UNSUPPORTED, "num_quadrature %d outside 2..%d", d->num_quadrature,
                   kMaxN);
  if (d->num_moments < 1 || d->num_moments > kMaxMoments)
    return na_fail(ADRT_ERR_INVALID_ARGUMENT, "num_moments must be in 1..%d", kMaxMoments);
  if (d->moment_layout < 0 || d->moment_layout > 2)
    return na_fail(ADRT_ERR_INVALID_ARGUMENT, "unknown moment_layout %d", d->moment_layout);
  if (d->precision != ADRT_PRECISION_FP64 && d->precision != ADRT_PRECISION_MIXED)
    return na_fail(ADRT_ERR_INVALID_ARGUMENT, "unknown precision %d", d->precision);
  if (!in->delta_tau || !in->single_scat_albedo || !in->phase_moments ||
      (d->use_thermal_emission && !in->temperature))
    return na_fail(ADRT_ERR_INVALID_ARGUMENT, "missing input array");
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return na_fail(ADRT_ERR_CUDA, "no usable current device");
  char* base = nullptr;
  int rc = na_setup(dev, &base);
  if (rc) return rc;

  // quadrature table of this N: nodes, weights, P_l(mu_i) for l < mmax
  const int n = d->num_quadrature;
  const int mmax = d->num_moments > 2 * n ? d->num_moments : 2 * n;
  std::vector<double> q((size_t)2 * n + (size_t)mmax * n);
  if ((rc = adrt_gauss_legendre(n, q.data(), q.data() + n)))
    return na_fail(rc, "quadrature set-up failed");
  double* pl = q.data() + 2 * n;
  double sum_mw = 0.0;
  for (int i = 0; i < n; ++i) {
    pl[i] = 1.0;
    if (mmax > 1) pl[n + i] = q[i];
    sum_mw += q[i] * q[n + i];
  }
  for (int l = 2; l < mmax; ++l)
    for (int i = 0; i < n; ++i)
      pl[l * n + i] = ((2 * l - 1) * q[i] * pl[(l - 1) * n + i] - (l - 1) * pl[(l - 2) * n + i]) / l;
  const size_t qbytes = (q.size() * sizeof(double) + 255) & ~size_t(255);

  NaKern k = na_pick(n, d->precision);
  const size_t slot = (k.slot_bytes(d->num_layers) + 255) & ~size_t(255);
  const size_t room = kNoAllocScratchBytes - kHeaderBytes - qbytes;
  if (slot > room)
    return na_fail(ADRT_ERR_WORKSPACE,
                   "one wavenumber needs %zu bytes of work memory at L=%d, N=%d; the static "
                   "work memory holds %zu (reduce num_layers)",
                   slot, d->num_layers, n, room);
  cudaError_t e = k.prepare(k.smem);
  if (e != cudaSuccess) return na_fail(ADRT_ERR_CUDA, "kernel set-up: %s", cudaGetErrorString(e));
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long resident = (long long)k.blocks_per_sm(k.smem) * sms * k.groups;
  long long nslots = (long long)(room / slot);
  if (nslots > resident) nslots = resident;
  if (nslots > d->num_wavenumbers) nslots = d->num_wavenumbers;
  const int grid = (int)((nslots + k.groups - 1) / k.groups);

  double* qdev = reinterpret_cast<double*>(base + kHeaderBytes);
  if ((e = cudaMemsetAsync(base, 0, kHeaderBytes, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(qdev, q.data(), q.size() * sizeof(double), cudaMemcpyHostToDevice,
                           s)) != cudaSuccess)
    return na_fail(ADRT_ERR_CUDA, "work memory set-up: %s", cudaGetErrorString(e));

  ColumnDev c{};
  c.W = d->num_wavenumbers;
  c.L = d->num_layers;
  c.N = n;
  c.NP = n <= 4 ? 4 : n <= 8 ? 8 : n <= 16 ? 16 : 32;
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
  c.fu = out->flux_up;
  c.fd = out->flux_down;
  c.fdir = out->flux_direct;
  c.J = out->mean_intensity;
  c.divF = out->flux_divergence;
  c.toa_fu = out->toa_flux_up;
  c.toa_fd = out->toa_flux_down;
  c.boa_fdir = out->boa_flux_direct;
  c.quad.mu = qdev;
  c.quad.wt = qdev + n;
  c.quad.pl = qdev + 2 * n;
  c.quad.mmax = mmax;
  c.quad.xfac = 0.5 / sum_mw;
  c.task_begin = 0;

  SolveParams p{};
  p.cols = nullptr;
  p.ncols = 1;
  p.ntasks = d->num_wavenumbers;
  p.counter = reinterpret_cast<unsigned long long*>(base);
  p.status = reinterpret_cast<unsigned int*>(base + 8);
  p.scratch = base + kHeaderBytes + qbytes;
  p.slot_bytes = slot;
  p.nslots = (int)nslots;
  p.max_layers = d->num_layers;
  k.launch(p, c, grid, k.smem, s);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return na_fail(ADRT_ERR_CUDA, "solve kernel launch: %s", cudaGetErrorString(e));
  return ADRT_OK;
}
