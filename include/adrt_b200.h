/*
 * adrt_b200.h -- C ABI of the B200 adding-doubling radiative-transfer engine.
 *
 * Plain C: pointers, sizes and status codes only.  Every entry point returns
 * an int status (ADRT_OK == 0, negative on error); a human-readable detail of
 * the last error on the calling thread is returned by adrt_last_status_detail().
 *
 * What each entry point replaces in the reference (NewStrangeWorlds/
 * AddingDoublingRT):
 *
 *   adrt_solve_batch         adrt::cuda::solveBatch(const BatchConfig&, const DeviceData&,
 *                            cudaStream_t)                         src_cuda/cuda_solver.cuh:77-80
 *                            (device buffers, stream ordered, no host sync).  Outputs are
 *                            per interface (src/adding_doubling.hpp:32-50), not TOA only.
 *   adrt_solve_batch_host    adrt::cuda::solveBatchHost(...)      src_cuda/cuda_solver.cuh:85-98
 *                            (host buffers; copies in, solves, copies out, synchronises).
 *   adrt_solve_batch_host    with W = 1 also serves adrt::solve(const ADConfig&)
 *                            (src/adding_doubling.hpp:258; RTOutput per-interface layout).
 *   adrt_validate_batch      ADConfig::validate()                  src/adding_doubling.hpp:123-174
 *   adrt_engine_create/...   SolverWorkspaceGPU                    src_cuda/cuda_solver.cuh:140-156
 *                            (the engine owns every device work buffer; nothing is
 *                            allocated inside a solve once adrt_engine_reserve succeeded).
 *
 * Array layouts (all row-major, wavenumber-major, TOA = layer/level 0 unless
 * index_from_bottom is set, exactly as the reference's DeviceData SoA layout
 * "array[wav * stride + layer_or_level]", src_cuda/cuda_solver.cuh:44):
 *   delta_tau, single_scat_albedo          [W * L]
 *   phase_moments                          see adrt_moment_layout
 *   temperature                            [L+1] shared, or [W * (L+1)]
 *   planck_levels                          [W * (L+1)]
 *   per-wavenumber scalars (optional)      [W]
 *   outputs flux_up/flux_down/flux_direct/
 *           mean_intensity/flux_divergence [W * (L+1)]   (NULL = not written)
 *   outputs toa_flux_up/toa_flux_down/
 *           boa_flux_direct                [W]           (reference DeviceData outputs)
 */
#ifndef ADRT_B200_H_
#define ADRT_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum adrt_status {
  ADRT_OK = 0,
  ADRT_ERR_INVALID_ARGUMENT = -1, /* ADConfig::validate() failure, bad sizes / pointers */
  ADRT_ERR_UNSUPPORTED = -2,      /* e.g. num_quadrature outside 2..32 on the GPU path */
  ADRT_ERR_CUDA = -3,             /* a CUDA runtime call failed */
  ADRT_ERR_OUT_OF_MEMORY = -4,    /* device work-buffer allocation failed */
  ADRT_ERR_WORKSPACE = -5,        /* the reserved work buffer is too small (capture mode) */
  ADRT_ERR_NUMERICAL = -6         /* device status word reported a numerical fault */
};

/* Device status word bits (adrt_engine_read_status). */
enum adrt_device_flag {
  ADRT_FLAG_SINGULAR_PIVOT = 1, /* an LU pivot was exactly zero (reference: silent inv=0) */
  ADRT_FLAG_NONFINITE = 2,      /* a non-finite flux was produced */
  ADRT_FLAG_BAD_INPUT = 4,      /* tau < 0, omega outside [0,1], T < 0 seen on the device, a
                                   layer so thick that the doubling rule asks for more than 64
                                   doublings (solved at 64), or a channel range outside the
                                   spectrum (band integration) */
  ADRT_FLAG_PIVOT_FALLBACK = 8, /* a pivot-free tensor-core right-solve met a pivot below 1e-10;
                                   its wavenumber was solved again with partial pivoting in
                                   every solve (results valid) */
  ADRT_FLAG_PIVOT_UNRESOLVED = 16 /* more such wavenumbers in one launch than the re-solve list
                                     holds (65536; 4096 for adrt_solve_batch_noalloc): the
                                     excess keep their pivot-free results */
};

/* ---------------------------------------------------------------- config */
enum adrt_precision {
  ADRT_PRECISION_FP64 = 0, /* every operation in FP64 (the plain GPU form) */
  ADRT_PRECISION_MIXED = 1 /* FP32 products, FP64 where conditioning needs it */
};

enum adrt_moment_layout {
  ADRT_MOMENTS_SHARED = 0,        /* [L * M]: same for every wavenumber (reference
                                     DeviceData::phase_moments_shared = true) */
  ADRT_MOMENTS_PER_WAVENUMBER = 1,/* [W * M]: one set per wavenumber, same for every layer */
  ADRT_MOMENTS_PER_LAYER = 2      /* [W * L * M]: per wavenumber and layer (reference
                                     phase_moments_shared = false) */
};

/* Scalars shared by every wavenumber of a batch.  Field meanings follow
 * adrt::ADConfig (src/adding_doubling.hpp:63-94) and adrt::cuda::BatchConfig
 * (src_cuda/cuda_solver.cuh:18-40). */
typedef struct adrt_batch_desc {
  int num_wavenumbers; /* W >= 1 */
  int num_layers;      /* L >= 1 */
  int num_quadrature;  /* N, 2..32 */
  int num_moments;     /* M >= 1 Legendre moments per set */
  int moment_layout;   /* enum adrt_moment_layout */
  int precision;       /* enum adrt_precision */

  int use_thermal_emission;   /* Planck levels from temperature (band-integrated) */
  int use_delta_m;            /* delta-M scaling (truncation fraction = chi[2N] when M > 2N) */
  int use_diffusion_lower_bc; /* diffusion-approximation lower boundary */
  int index_from_bottom;      /* user arrays indexed BOA (0) -> TOA */
  int temperature_per_wavenumber; /* temperature is [W*(L+1)] instead of shared [L+1] */

  double surface_albedo;      /* used when inputs.surface_albedo == NULL */
  double surface_emission;    /* raw, when !use_thermal_emission and inputs.surface_emission == NULL */
  double surface_temperature; /* >= 0 with thermal: surface emits B(T_s) */
  double top_emission;        /* raw, when !use_thermal_emission and inputs.top_emission == NULL */
  double top_temperature;     /* >= 0 with thermal: TOA downwelling B(T_top) */
  double solar_flux;          /* F0 */
  double solar_mu;            /* used when inputs.solar_mu == NULL */
  double wavenumber_low;      /* band, used when inputs.wavenumber_low == NULL */
  double wavenumber_high;
  double spectrum_scaling;    /* applied to toa_flux_up only (reference BatchConfig) */
} adrt_batch_desc;

/* Inputs (device pointers for adrt_solve_batch, host pointers for the
 * *_host entry points).  FP64 throughout so that near-conservative albedos
 * (1 - omega down to 1e-7) are represented exactly. */
typedef struct adrt_inputs {
  const double* delta_tau;          /* [W*L] */
  const double* single_scat_albedo; /* [W*L] */
  const double* phase_moments;      /* see moment_layout */
  const double* temperature;        /* [L+1] or [W*(L+1)]; thermal only */
  const double* planck_levels;      /* [W*(L+1)] or NULL; non-thermal sources */
  const double* surface_albedo;     /* [W] or NULL */
  const double* solar_mu;           /* [W] or NULL */
  const double* wavenumber_low;     /* [W] or NULL */
  const double* wavenumber_high;    /* [W] or NULL */
  const double* surface_emission;   /* [W] or NULL */
  const double* top_emission;       /* [W] or NULL */
} adrt_inputs;

typedef struct adrt_outputs {
  double* flux_up;         /* [W*(L+1)] diffuse upward flux per interface */
  double* flux_down;       /* [W*(L+1)] diffuse downward flux */
  double* flux_direct;     /* [W*(L+1)] attenuated direct beam */
  double* mean_intensity;  /* [W*(L+1)] J including the direct beam */
  double* flux_divergence; /* [W*(L+1)] 4 pi (1 - omega) (J - B) */
  double* toa_flux_up;     /* [W] flux_up[0] * spectrum_scaling */
  double* toa_flux_down;   /* [W] flux_down[0] */
  double* boa_flux_direct; /* [W] flux_direct[L] */
} adrt_outputs;

/* ---------------------------------------------------------------- engine */
typedef struct adrt_engine adrt_engine;

typedef struct adrt_engine_opts {
  int device;                  /* CUDA device ordinal; -1 = current device */
  size_t max_workspace_bytes;  /* 0 = no limit on the device work buffer */
} adrt_engine_opts;

int adrt_engine_create(const adrt_engine_opts* opts, adrt_engine** out);
int adrt_engine_destroy(adrt_engine* engine);

/* Pre-size the engine's device work buffer for batches up to this shape, so
 * that later adrt_solve_batch calls allocate nothing (and can be captured in
 * a CUDA graph). */
int adrt_engine_reserve(adrt_engine* engine, const adrt_batch_desc* desc);

/* Bytes of device work buffer the engine currently holds. */
int adrt_engine_workspace_bytes(const adrt_engine* engine, size_t* bytes);

/* The CUDA device ordinal the engine runs on; device pointers given to it
 * must be memory of that device. */
int adrt_engine_device(const adrt_engine* engine, int* device);

/* Synchronise the engine's last stream and read (and clear) the device status
 * word (enum adrt_device_flag bits). */
int adrt_engine_read_status(adrt_engine* engine, int* flags);

/* ---------------------------------------------------------------- solves */

/* Batched solve, device buffers, stream ordered; returns after enqueueing. */
int adrt_solve_batch(adrt_engine* engine, const adrt_batch_desc* desc,
                     const adrt_inputs* in, const adrt_outputs* out, void* cuda_stream);

/* Batched solve from host buffers: host->device copies, solve, device->host
 * copies, stream synchronised before return. */
int adrt_solve_batch_host(adrt_engine* engine, const adrt_batch_desc* desc,
                          const adrt_inputs* host_in, const adrt_outputs* host_out);

/* FP32 device arrays, the element type of the reference's DeviceData
 * (src_cuda/cuda_solver.cuh:45-68).  Same fields and layouts as adrt_inputs /
 * adrt_outputs. */
typedef struct adrt_inputs_f32 {
  const float* delta_tau;
  const float* single_scat_albedo;
  const float* phase_moments;
  const float* temperature;
  const float* planck_levels;
  const float* surface_albedo;
  const float* solar_mu;
  const float* wavenumber_low;
  const float* wavenumber_high;
  const float* surface_emission;
  const float* top_emission;
} adrt_inputs_f32;

typedef struct adrt_outputs_f32 {
  float* flux_up;
  float* flux_down;
  float* flux_direct;
  float* mean_intensity;
  float* flux_divergence;
  float* toa_flux_up;
  float* toa_flux_down;
  float* boa_flux_direct;
} adrt_outputs_f32;

/* Batched solve from FP32 device arrays, stream ordered: replaces
 * adrt::cuda::solveBatch(const BatchConfig&, const DeviceData&, cudaStream_t)
 * (src_cuda/cuda_solver.cuh:77-80) for callers holding FP32 data.  The inputs
 * are widened into an engine-owned FP64 staging buffer on the stream, solved,
 * and the requested outputs narrowed back.  Allocates only when the staging
 * buffer must grow (never during stream capture: size it with one call first). */
int adrt_solve_batch_f32(adrt_engine* engine, const adrt_batch_desc* desc,
                         const adrt_inputs_f32* in, const adrt_outputs_f32* out,
                         void* cuda_stream);

/* Raw retrieval inputs (device, FP32 as the reference's RawDeviceData,
 * src_cuda/cuda_solver.cuh:104-133).  Levels and layers of the coefficient
 * arrays are counted from the bottom of the atmosphere (level 0 = BOA); the
 * phase moments keep the solver's top-first layer order. */
typedef struct adrt_raw_inputs {
  const float* absorption_coeff;     /* [(L+1) * W] level-major, cm^-1 */
  const float* scattering_coeff;     /* [(L+1) * W] level-major, cm^-1 */
  const float* altitude;             /* [L+1] cm */
  const float* temperature;          /* [L+1] K */
  const double* wavenumber;          /* [W] cm^-1 */
  const float* cloud_optical_depth;  /* [L * W] layer-major, or NULL */
  const float* phase_moments;        /* per desc->moment_layout; layer 0 = top */
} adrt_raw_inputs;

/* Batched solve from raw absorption / scattering coefficients: replaces
 * adrt::cuda::solveBatchFromCoefficients (src_cuda/cuda_solver.cuh:166-179,
 * src_cuda/cuda_solver.cu:1193-1353).  Layer optical depths by the trapezoid
 * rule over altitude (plus the cloud optical depth), single-scattering albedo
 * = scattering depth / optical depth, and single-wavenumber Planck levels are
 * formed inside the solve's prologue (no intermediate arrays); the surface
 * emits B(T_BOA) (or B(surface_temperature) when >= 0) and the top sees
 * B(T_TOA) (or B(top_temperature) when >= 0).  desc's use_thermal_emission,
 * index_from_bottom and temperature_per_wavenumber are ignored.  Outputs as
 * adrt_solve_batch_f32 (the reference writes toa_flux_up, toa_flux_down and
 * boa_flux_direct).  Any N (the reference's workspace-free overload takes
 * N <= 8). */
int adrt_solve_batch_raw(adrt_engine* engine, const adrt_batch_desc* desc,
                         const adrt_raw_inputs* in, const adrt_outputs_f32* out,
                         void* cuda_stream);

/* Validate a batch description and (host) inputs with the rules of
 * ADConfig::validate() (src/adding_doubling.hpp:123-174) applied to every
 * wavenumber.  Returns ADRT_ERR_INVALID_ARGUMENT with a detail message. */
int adrt_validate_batch(const adrt_batch_desc* desc, const adrt_inputs* host_in);

/* Batched solve that allocates no device memory (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc -- inside a framework
 * whose caching allocator already holds the GPU's memory, on a latency-bound
 * path where an allocation's implicit synchronisation is not acceptable, or
 * in a plugin host that only hands over its own buffers.  Same arguments,
 * argument checks and results as adrt_solve_batch, without an engine: the
 * work memory is one fixed 64 MiB array compiled into the library (present
 * on every GPU that loads it, until the process exits).  Arrays must be
 * memory of the current device (or managed / mapped pinned memory); plain
 * host arrays are refused with ADRT_ERR_INVALID_ARGUMENT.  The first call on
 * a device looks up that array's device address, and the first call with
 * each num_quadrature uploads that order's quadrature table (synchronously);
 * make those calls before any stream capture (a capturing first call is
 * refused with ADRT_ERR_WORKSPACE).  A batch of which one block of
 * wavenumber slots (4 at N <= 16, 1 at N = 32; about (L+1) x 25 KB per
 * wavenumber at N = 32 in FP64) does not fit is rejected with
 * ADRT_ERR_WORKSPACE.  All calls share the array and it keeps the last
 * call's contents; each call resets its work counter, so calls that overlap
 * on the GPU race and must not be issued.  The device status word collects
 * the flags of every call until adrt_noalloc_read_status reads and clears
 * it. */
int adrt_solve_batch_noalloc(const adrt_batch_desc* desc, const adrt_inputs* in,
                             const adrt_outputs* out, void* cuda_stream);

/* Synchronise `cuda_stream` and read (and clear) the device status word of
 * adrt_solve_batch_noalloc calls on the current device (enum adrt_device_flag
 * bits), as adrt_engine_read_status does for an engine.  Allocates nothing
 * (no counterpart in the reference). */
int adrt_noalloc_read_status(void* cuda_stream, int* flags);

/* ------------------------------------------------------------- adjoint */

/* Cotangents of a scalar loss with respect to the per-interface outputs
 * ([W*(L+1)] device arrays in the output layout, NULL = zero). */
typedef struct adrt_cotangents {
  const double* flux_up;
  const double* flux_down;
  const double* mean_intensity;
  const double* flux_direct;
} adrt_cotangents;

/* Gradients (device arrays in the input layouts, NULL = not wanted).
 * delta_tau and single_scat_albedo [W*L] are overwritten; phase_moments,
 * temperature and planck_levels are ADDED to (shared layouts sum over the
 * wavenumbers), so zero them first. */
typedef struct adrt_gradients {
  double* delta_tau;
  double* single_scat_albedo;
  double* phase_moments;
  double* temperature;
  double* planck_levels;
  double* surface_emission; /* [W], overwritten: d/d(surface emission) -- the
                               surface_emission input without thermal emission, or
                               B(surface_temperature) with thermal emission and
                               surface_temperature >= 0 (times dB/dT gives d/dT_s) */
} adrt_gradients;

/* How adrt_adjoint's backward pass gets each layer's doubling chain. */
enum adrt_adjoint_mode {
  ADRT_ADJOINT_RECORD = 0,   /* default: the forward pass records the chains (up
                                to a record pool; chains beyond it are recomputed) */
  ADRT_ADJOINT_RECOMPUTE = 1 /* the forward pass keeps only the per-layer R, T and
                                sources for the adding; every chain is recomputed in
                                the backward pass */
};

/* Select the engine's adjoint mode (enum adrt_adjoint_mode); both give the
 * same gradients to round-off. */
int adrt_engine_set_adjoint_mode(adrt_engine* engine, int mode);

/* Pivoting of the FP64 right-solves (I - R R')^{-1} (no counterpart in the
 * reference, whose solves always pivot: src/matrix.hpp:120-124). */
enum adrt_pivoting {
  ADRT_PIVOTING_TENSOR_CORE = 0, /* default: pivot-free tensor-core elimination (the
                                    matrices are diagonally dominant), partial pivoting
                                    for unstable first-order starts, and a pivoted
                                    re-solve of any wavenumber that meets a weak pivot */
  ADRT_PIVOTING_PARTIAL = 1      /* every solve with the reference's partial pivoting */
};
int adrt_engine_set_pivoting(adrt_engine* engine, int mode);

/* Reverse-mode adjoint of the batched solve: given the loss cotangents,
 * the gradients with respect to delta_tau, single_scat_albedo, the phase
 * moments and the level temperatures (through dB/dT, the reference's
 * planckFunctionDeriv, src/planck.cpp:135-175) or the Planck levels.  The
 * derivative is that of the discrete scheme at fixed doubling counts; it
 * generalises the reference's analytic temperature Jacobian
 * (src/solver.cpp:117-341) to all inputs.  FP64; the forward pass records
 * every layer's doubling chain for the backward pass (in chunks of
 * wavenumbers; chains beyond the record pool are recomputed), or, in
 * ADRT_ADJOINT_RECOMPUTE mode, the backward pass recomputes them all.  `out` may be
 * NULL or receive the forward outputs.  With delta-M truncation in effect
 * (use_delta_m with num_moments > 2N) the gradients are those of the
 * unscaled inputs: tau' = (1 - omega f) tau, omega' = omega (1 - f) /
 * (1 - omega f) and chi*_l = (chi_l - f) / (1 - f), f = chi_2N, are
 * differentiated through (src/solver.cpp:441-501), f included. */
int adrt_adjoint(adrt_engine* engine, const adrt_batch_desc* desc, const adrt_inputs* in,
                 const adrt_outputs* out, const adrt_cotangents* cot,
                 const adrt_gradients* grads, void* cuda_stream);

/* adrt_adjoint from host buffers: copies in (the gradients too, since some
 * are added to), runs the adjoint, copies the gradients back and
 * synchronises.  Serves adrt::solve with ADConfig::compute_temperature_jacobian
 * (src/solver.cpp:117-341), whose Jacobian rows are gradients of single
 * outputs. */
int adrt_adjoint_host(adrt_engine* engine, const adrt_batch_desc* desc, const adrt_inputs* in,
                      const adrt_cotangents* cotangents, const adrt_gradients* gradients);

/* ------------------------------------------------------- uneven batches */

/* One column of an uneven batch (reference: several solveBatch calls).
 * Every pointer is a device pointer; arrays follow adrt_inputs / adrt_outputs
 * for this column's own W, L, N and M. */
typedef struct adrt_column_desc {
  adrt_batch_desc desc;
  adrt_inputs in;
  adrt_outputs out;
} adrt_column_desc;

/* Solve many columns of different W, L, N in ONE launch of the persistent
 * solver kernel per mapping (the engine's uneven plan, below; by default one
 * launch of the warp-per-wavenumber kernel for every N <= 16 and one of the
 * N = 32 kernel).  Replaces one adrt::cuda::solveBatch call per column
 * (src_cuda/cuda_solver.cuh:77-80).  The column table is copied to the device
 * by the engine; the call neither allocates nor synchronises the host once a
 * call of the same size has been made, so it can be captured in a graph. */
int adrt_solve_batch_uneven(adrt_engine* engine, const adrt_column_desc* cols, int ncols,
                            void* cuda_stream);

/* How an uneven batch is mapped onto the GPU (no counterpart in the
 * reference).  For padded orders 4, 8 and 16, the FP64 columns either run
 * one wavenumber per warp in the persistent multi-order kernel
 * (ADRT_MAPPING_WARP, the default) or one wavenumber per thread
 * (ADRT_MAPPING_THREAD: the reference's solveKernel mapping,
 * src_cuda/cuda_solver.cu:131-493, on this engine's scheme and outputs);
 * mixed-precision columns always take the warp mapping.  warp_blocks_per_sm
 * caps the warp launch's grid (0 = the occupancy limit); cost_order sorts the
 * columns longest first (L N^3 per wavenumber) so that the dynamic task
 * queue ends with short tasks.  ns_per_wavenumber holds what the autotuner
 * measured for [order 4, 8, 16][warp, thread] (0 = not measured; a thread
 * mapping more than 4x slower on an eighth of the sample keeps that
 * pilot's figure). */
enum adrt_mapping { ADRT_MAPPING_WARP = 0, ADRT_MAPPING_THREAD = 1 };
typedef struct adrt_uneven_plan {
  int mapping[3];
  int warp_blocks_per_sm;
  int cost_order;
  double ns_per_wavenumber[3][2];
} adrt_uneven_plan;

/* Autotune the uneven plan for this batch's shape: for every padded order
 * present with FP64 columns, both mappings solve a sample of that order's
 * wavenumbers (at least a few waves of the GPU's resident slots), and the
 * faster one per wavenumber is kept; then the warp launch's grid cap is
 * chosen the same way.  Results (including the measured times) go to `out`
 * (may be NULL) and become the engine's plan.  Synchronises the stream; do
 * not call it during a stream capture.  The sample solves write the sampled
 * wavenumbers' outputs, which the next solve of the batch overwrites. */
int adrt_engine_autotune_uneven(adrt_engine* engine, const adrt_column_desc* cols, int ncols,
                                void* cuda_stream, adrt_uneven_plan* out);

/* Set (e.g. a fixed mapping to compare against) or read the engine's plan. */
int adrt_engine_set_uneven_plan(adrt_engine* engine, const adrt_uneven_plan* plan);
int adrt_engine_get_uneven_plan(const adrt_engine* engine, adrt_uneven_plan* plan);

/* ---------------------------------------------------------- utilities */

/* Measured FP64 and FP32 FMA throughput (TFLOP/s) of the current device: the
 * roofline denominators of the solver kernels, whose products and
 * eliminations run on the CUDA-core FMA pipes.  Engine utility; the reference
 * has no counterpart. */
int adrt_probe_fma_tflops(double* fp64_tflops, double* fp32_tflops);

/* Measured warp-level tensor-core throughput (TFLOP/s) of the current device:
 * mma.sync m8n8k4 f64 (the FP64 products and right-solves), m16n8k8 tf32 (the
 * mixed form's FP32 products, three per product) and m16n8k16 bf16.  Engine
 * utility; the reference has no counterpart. */
int adrt_probe_mma_tflops(double* fp64_dmma_tflops, double* tf32_tflops, double* bf16_tflops);

/* Gauss-Legendre nodes and weights on [0,1], the engine's own quadrature
 * (replaces adrt::gaussLegendre, src/quadrature.cpp:11-51). */
int adrt_gauss_legendre(int n, double* nodes, double* weights);

/* Band-integrated Planck function on the host, the algorithm the engine runs
 * on the device (replaces adrt::planckFunction, src/planck.cpp:35-131).
 * ADRT_ERR_INVALID_ARGUMENT where the reference throws. */
int adrt_planck_band(double wavenumber_low, double wavenumber_high, double temperature,
                     double* out);

/* d/dT of the band-integrated Planck function: replaces
 * adrt::planckFunctionDeriv (src/planck.cpp:135-175, declared in
 * src/planck.hpp:27). */
int adrt_planck_band_deriv(double wnumlo, double wnumhi, double temp, double* out);

/* Band integration of a spectrum on the device, the reduction after a solve
 * (e.g. TOA flux_up into instrument channels): for each channel b,
 *   out[b] = sum over w in [offsets[b], offsets[b+1]) of weight[w] * spectrum[w]
 * (weight null: 1).  offsets holds nchannels + 1 non-decreasing indices into
 * [0, num_wavenumbers]; a channel whose range is not is written NaN and sets
 * ADRT_FLAG_BAD_INPUT.  Device pointers, stream-ordered, no allocation; each
 * channel is summed by one block in a fixed order, so the result does not
 * depend on the launch.  The reference's batched path scales flux_up by
 * spectrum_scaling (src_cuda/cuda_solver.cu:481, cuda_solver.cuh:39) and
 * leaves this reduction to its caller. */
int adrt_band_integrate(adrt_engine* engine, const double* spectrum, const double* weight,
                        long long num_wavenumbers, const long long* offsets, int nchannels,
                        double* out, void* stream);

/* --------------------------------------------------------------- errors */
const char* adrt_last_status_detail(void);
const char* adrt_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ADRT_B200_H_ */
