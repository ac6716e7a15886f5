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
// quadrature tables of every order N = 2..32 (uploaded once per device and
// order, by the first call that uses that order), and as many
// per-wavenumber work slots as fit; fewer slots than the engine uses means
// fewer wavenumbers in flight at once, not a different result.  Every call
// shares the array and it keeps the last call's contents: the counter is
// reset by each call before its kernel runs and the status word collects
// the flags of every call until adrt_noalloc_read_status clears it, so calls
// that overlap on the GPU (on different streams, or from different host
// threads) race and must not be issued.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/adrt_b200.h"
#include "adrt_kernel.cuh"

using namespace adrt_dev;

// adrt_engine.cu (hidden, not exported)
void adrt_internal_set_detail(const char* msg);
int adrt_internal_check_batch(const adrt_batch_desc* d, const adrt_inputs* in);
void adrt_internal_quad_table(int n, int mmax, std::vector<double>& host, double* xfac);

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
constexpr size_t kHeaderBytes = 256;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 128;

static __device__ __align__(256) char g_noalloc_scratch[kNoAllocScratchBytes];

// Quadrature tables: order n at quad_offset(n), Legendre rows up to
// kMaxMoments, so one table serves every moment count.
constexpr size_t quad_doubles(int n) { return (size_t)(2 + kMaxMoments) * n; }
constexpr size_t quad_offset(int n) {
  size_t off = kHeaderBytes;
  for (int m = 2; m < n; ++m) off += (quad_doubles(m) * sizeof(double) + 255) & ~size_t(255);
  return off;
}
// The re-solve list (SolveParams::redo): two counters and kRedoCap task
// indices after the quadrature tables, then the wavenumber slots.
constexpr long long kRedoCap = 4096;
constexpr size_t kRedoOffset = quad_offset(kMaxN + 1);
constexpr size_t kSlotsOffset =
    kRedoOffset + (((2 + kRedoCap) * sizeof(unsigned long long) + 255) & ~size_t(255));
static_assert(kSlotsOffset < kNoAllocScratchBytes / 8, "quadrature tables fit well inside");

int na_fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  adrt_internal_set_detail(buf);
  return code;
}

// Launch facts of one kernel instantiation, looked up once per device.
struct NaKernState {
  bool ready = false;
  int blocks_per_sm = 0;
};

// Per-device state: the array's device address, the SM count, which
// quadrature orders are uploaded (and their 0.5 / sum(mu w)), and the
// kernels' launch facts [padded order index][kind].
struct NaDevice {
  char* addr = nullptr;
  int sms = 0;
  bool quad_ready[kMaxN + 1] = {};
  double xfac[kMaxN + 1] = {};
  NaKernState kern[4][2];
};
std::mutex g_na_mu;
NaDevice g_na[kMaxDevices];

// Set-up on the current device `dev` (its first call): the device address of
// the static array (cudaGetSymbolAddress, checked) and the SM count.
int na_device(int dev, NaDevice** out) {
  NaDevice& d = g_na[dev];
  if (!d.addr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
      return na_fail(ADRT_ERR_CUDA, "cudaGetSymbolAddress of the static work memory: %s",
                     cudaGetErrorString(e));
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || sms < 1)
      return na_fail(ADRT_ERR_CUDA, "SM count of device %d: %s", dev, cudaGetErrorString(e));
    d.sms = sms;
    d.addr = static_cast<char*>(p);
  }
  *out = &d;
  return ADRT_OK;
}

// The quadrature table of order n in the static array, uploaded by the first
// call of this order on this device (a synchronous copy: that call must not be
// made during a stream capture).
int na_quad(NaDevice& d, int n, cudaStream_t s) {
  if (d.quad_ready[n]) return ADRT_OK;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
    return na_fail(ADRT_ERR_WORKSPACE,
                   "the first call with num_quadrature=%d on this device uploads its quadrature "
                   "table and cannot be captured: make one call with this order before capture",
                   n);
  std::vector<double> host;
  double xfac = 0.0;
  adrt_internal_quad_table(n, kMaxMoments, host, &xfac);
  const cudaError_t e = cudaMemcpy(d.addr + quad_offset(n), host.data(),
                                   host.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess)
    return na_fail(ADRT_ERR_CUDA, "quadrature table upload: %s", cudaGetErrorString(e));
  d.xfac[n] = xfac;
  d.quad_ready[n] = true;
  return ADRT_OK;
}

// A pointer the kernels may dereference on device `dev`: device memory of
// `dev`, managed memory, or pinned host memory mapped into the device's
// address space.  Plain (unregistered) host memory and other devices' memory
// are refused.
bool na_device_pointer(const void* p, int dev) {
  if (!p) return true;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  switch (a.type) {
    case cudaMemoryTypeDevice: return a.device == dev;
    case cudaMemoryTypeManaged: return true;
    case cudaMemoryTypeHost: return a.devicePointer != nullptr;
    default: return false;
  }
}

int na_check_pointers(const adrt_inputs* in, const adrt_outputs* out, int dev) {
  const void* ins[] = {in->delta_tau,     in->single_scat_albedo, in->phase_moments,
                       in->temperature,   in->planck_levels,      in->surface_albedo,
                       in->solar_mu,      in->wavenumber_low,     in->wavenumber_high,
                       in->surface_emission, in->top_emission};
  const char* inames[] = {"delta_tau",     "single_scat_albedo", "phase_moments",
                          "temperature",   "planck_levels",      "surface_albedo",
                          "solar_mu",      "wavenumber_low",     "wavenumber_high",
                          "surface_emission", "top_emission"};
  for (int i = 0; i < 11; ++i)
    if (!na_device_pointer(ins[i], dev))
      return na_fail(ADRT_ERR_INVALID_ARGUMENT,
                     "input %s is not device memory of device %d (host arrays go through "
                     "adrt_solve_batch_host)", inames[i], dev);
  const void* outs[] = {out->flux_up,          out->flux_down,     out->flux_direct,
                        out->mean_intensity,   out->flux_divergence, out->toa_flux_up,
                        out->toa_flux_down,    out->boa_flux_direct};
  for (int i = 0; i < 8; ++i)
    if (!na_device_pointer(outs[i], dev))
      return na_fail(ADRT_ERR_INVALID_ARGUMENT, "output %d is not device memory of device %d",
                     i, dev);
  return ADRT_OK;
}

// The engine's persistent solve kernel, instantiated in this file.
struct NaKern {
  int groups;
  size_t smem;
  size_t (*slot_bytes)(int);
  cudaError_t (*prepare)(size_t, int*);
  void (*launch)(const SolveParams&, const ColumnDev&, int, size_t, cudaStream_t);
};

template <int NP, int KIND>
NaKern na_kern() {
  using GD = Geo<NP, double>;
  NaKern k;
  k.groups = kThreads / GD::G;
  k.smem = (size_t)k.groups * GroupLayout<NP, KIND>::bytes;
  k.slot_bytes = [](int lmax) { return SlotLayout<GD>::bytes(lmax); };
  k.prepare = [](size_t smem, int* bps) {
    cudaError_t e = cudaFuncSetAttribute(solve_kernel<NP, KIND>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, solve_kernel<NP, KIND>, kThreads,
                                                         smem);
  };
  k.launch = [](const SolveParams& p, const ColumnDev& c, int grid, size_t smem,
                cudaStream_t s) { solve_kernel<NP, KIND><<<grid, kThreads, smem, s>>>(p, c); };
  return k;
}

int na_order_index(int np) { return np == 4 ? 0 : np == 8 ? 1 : np == 16 ? 2 : 3; }

NaKern na_pick(int np, int precision) {
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
  // the checks of adrt_solve_batch, so both refuse the same batches
  int rc = adrt_internal_check_batch(d, in);
  if (rc) return rc;
  if (!out) return na_fail(ADRT_ERR_INVALID_ARGUMENT, "null outputs");
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return na_fail(ADRT_ERR_CUDA, "no usable current device");
  if ((rc = na_check_pointers(in, out, dev))) return rc;

  std::lock_guard<std::mutex> lk(g_na_mu);
  NaDevice* nd = nullptr;
  if ((rc = na_device(dev, &nd))) return rc;
  const int n = d->num_quadrature;
  if ((rc = na_quad(*nd, n, s))) return rc;

  const int np = n <= 4 ? 4 : n <= 8 ? 8 : n <= 16 ? 16 : 32;
  const int kind = d->precision == ADRT_PRECISION_MIXED ? 1 : 0;
  NaKern k = na_pick(np, d->precision);
  NaKernState& ks = nd->kern[na_order_index(np)][kind];
  if (!ks.ready) {
    int bps = 0;
    const cudaError_t e = k.prepare(k.smem, &bps);
    if (e != cudaSuccess || bps < 1)
      return na_fail(ADRT_ERR_CUDA, "kernel set-up: %s", cudaGetErrorString(e));
    ks.blocks_per_sm = bps;
    ks.ready = true;
  }
  const size_t slot = (k.slot_bytes(d->num_layers) + 255) & ~size_t(255);
  const size_t room = kNoAllocScratchBytes - kSlotsOffset;
  // whole blocks of slots: every thread group of a launched block owns one
  long long blocks = (long long)(room / slot) / k.groups;
  if (blocks < 1)
    return na_fail(ADRT_ERR_WORKSPACE,
                   "one block of %d wavenumber slots needs %zu bytes of work memory at L=%d, "
                   "N=%d; the static work memory holds %zu (reduce num_layers)",
                   k.groups, slot * k.groups, d->num_layers, n, room);
  blocks = std::min<long long>(blocks, (long long)ks.blocks_per_sm * nd->sms);
  blocks = std::min<long long>(blocks, (d->num_wavenumbers + k.groups - 1) / k.groups);

  char* base = nd->addr;
  cudaError_t e0 = cudaMemsetAsync(base, 0, sizeof(unsigned long long), s);
  if (e0 == cudaSuccess)
    e0 = cudaMemsetAsync(base + kRedoOffset, 0, 2 * sizeof(unsigned long long), s);
  if (e0 != cudaSuccess)
    return na_fail(ADRT_ERR_CUDA, "work counter reset: %s", cudaGetErrorString(e0));

  ColumnDev c{};
  c.W = d->num_wavenumbers;
  c.L = d->num_layers;
  c.N = n;
  c.NP = np;
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
  const double* q = reinterpret_cast<const double*>(base + quad_offset(n));
  c.quad.mu = q;
  c.quad.wt = q + n;
  c.quad.pl = q + 2 * n;
  c.quad.mmax = kMaxMoments;
  c.quad.xfac = nd->xfac[n];
  c.task_begin = 0;

  SolveParams p{};
  p.cols = nullptr;
  p.ncols = 1;
  p.ntasks = d->num_wavenumbers;
  p.counter = reinterpret_cast<unsigned long long*>(base);
  p.status = reinterpret_cast<unsigned int*>(base + 8);
  p.scratch = base + kSlotsOffset;
  p.slot_bytes = slot;
  p.nslots = (int)(blocks * k.groups);
  p.max_layers = d->num_layers;
  p.redo = reinterpret_cast<unsigned long long*>(base + kRedoOffset);
  p.redo_cap = kRedoCap;
  k.launch(p, c, (int)blocks, k.smem, s);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {  // the re-solve pass over the listed wavenumbers
    SolveParams q = p;
    q.redo_pass = 1;
    k.launch(q, c, (int)blocks, k.smem, s);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess)
    return na_fail(ADRT_ERR_CUDA, "solve kernel launch: %s", cudaGetErrorString(e));
  return ADRT_OK;
}

extern "C" int adrt_noalloc_read_status(void* stream_ptr, int* flags) {
  if (!flags) return na_fail(ADRT_ERR_INVALID_ARGUMENT, "null flags");
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return na_fail(ADRT_ERR_CUDA, "no usable current device");
  std::lock_guard<std::mutex> lk(g_na_mu);
  NaDevice* nd = nullptr;
  int rc = na_device(dev, &nd);
  if (rc) return rc;
  unsigned int v = 0;
  unsigned int* st = reinterpret_cast<unsigned int*>(nd->addr + 8);
  cudaError_t e = cudaMemcpyAsync(&v, st, sizeof v, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemsetAsync(st, 0, sizeof v, s);
  if (e != cudaSuccess)
    return na_fail(ADRT_ERR_CUDA, "status read: %s", cudaGetErrorString(e));
  *flags = (int)v;
  return ADRT_OK;
}
