"""ctypes mirrors of the C ABI structs in include/adrt_b200.h.

Every Python entry point of the package (and the tests and bench harness)
passes arrays to the native library through these structs.  Field order and
types must match the header exactly.
"""
from __future__ import annotations

import ctypes as C

ADRT_OK = 0
ADRT_ERR_INVALID_ARGUMENT = -1
ADRT_ERR_UNSUPPORTED = -2
ADRT_ERR_CUDA = -3
ADRT_ERR_OUT_OF_MEMORY = -4
ADRT_ERR_WORKSPACE = -5
ADRT_ERR_NUMERICAL = -6

ADRT_FLAG_SINGULAR_PIVOT = 1
ADRT_FLAG_NONFINITE = 2
ADRT_FLAG_BAD_INPUT = 4
ADRT_FLAG_PIVOT_FALLBACK = 8
ADRT_FLAG_PIVOT_UNRESOLVED = 16
PIVOTING_TENSOR_CORE = 0
PIVOTING_PARTIAL = 1

PRECISION_FP64 = 0
PRECISION_MIXED = 1

MOMENTS_SHARED = 0
MOMENTS_PER_WAVENUMBER = 1
MOMENTS_PER_LAYER = 2

ADJOINT_RECORD = 0      # the forward pass records the doubling chains
ADJOINT_RECOMPUTE = 1   # the backward pass recomputes them

_dp = C.POINTER(C.c_double)


class BatchDesc(C.Structure):
    _fields_ = [
        ("num_wavenumbers", C.c_int),
        ("num_layers", C.c_int),
        ("num_quadrature", C.c_int),
        ("num_moments", C.c_int),
        ("moment_layout", C.c_int),
        ("precision", C.c_int),
        ("use_thermal_emission", C.c_int),
        ("use_delta_m", C.c_int),
        ("use_diffusion_lower_bc", C.c_int),
        ("index_from_bottom", C.c_int),
        ("temperature_per_wavenumber", C.c_int),
        ("surface_albedo", C.c_double),
        ("surface_emission", C.c_double),
        ("surface_temperature", C.c_double),
        ("top_emission", C.c_double),
        ("top_temperature", C.c_double),
        ("solar_flux", C.c_double),
        ("solar_mu", C.c_double),
        ("wavenumber_low", C.c_double),
        ("wavenumber_high", C.c_double),
        ("spectrum_scaling", C.c_double),
    ]


INPUT_FIELDS = (
    "delta_tau",
    "single_scat_albedo",
    "phase_moments",
    "temperature",
    "planck_levels",
    "surface_albedo",
    "solar_mu",
    "wavenumber_low",
    "wavenumber_high",
    "surface_emission",
    "top_emission",
)

OUTPUT_FIELDS = (
    "flux_up",
    "flux_down",
    "flux_direct",
    "mean_intensity",
    "flux_divergence",
    "toa_flux_up",
    "toa_flux_down",
    "boa_flux_direct",
)

INTERFACE_OUTPUTS = OUTPUT_FIELDS[:5]


class Inputs(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in INPUT_FIELDS]


class Outputs(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in OUTPUT_FIELDS]


OUTPUT_F32_FIELDS = OUTPUT_FIELDS  # same order, float pointers


class OutputsF32(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in OUTPUT_F32_FIELDS]


RAW_INPUT_FIELDS = ("absorption_coeff", "scattering_coeff", "altitude", "temperature",
                    "wavenumber", "cloud_optical_depth", "phase_moments")


class RawInputs(C.Structure):
    """adrt_raw_inputs: FP32 coefficient arrays (level 0 = bottom), FP64 wavenumbers."""
    _fields_ = [(f, C.c_void_p) for f in RAW_INPUT_FIELDS]


COTANGENT_FIELDS = ("flux_up", "flux_down", "mean_intensity", "flux_direct")
GRADIENT_FIELDS = ("delta_tau", "single_scat_albedo", "phase_moments", "temperature",
                   "planck_levels", "surface_emission")


class Cotangents(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in COTANGENT_FIELDS]


class Gradients(C.Structure):
    _fields_ = [(f, C.c_void_p) for f in GRADIENT_FIELDS]


class ColumnDesc(C.Structure):
    _fields_ = [("desc", BatchDesc), ("inp", Inputs), ("out", Outputs)]


MAPPING_WARP = 0
MAPPING_THREAD = 1


class UnevenPlan(C.Structure):
    """adrt_uneven_plan: mapping per padded order 4 / 8 / 16, the warp launch's
    blocks per SM (0 = occupancy limit), longest-first ordering, and the
    autotuner's measured ns per wavenumber [order][warp, thread]."""
    _fields_ = [("mapping", C.c_int * 3), ("warp_blocks_per_sm", C.c_int),
                ("cost_order", C.c_int), ("ns_per_wavenumber", (C.c_double * 2) * 3)]

    def as_dict(self) -> dict:
        return {"mapping": {o: ("thread" if self.mapping[i] else "warp")
                            for i, o in enumerate((4, 8, 16))},
                "warp_blocks_per_sm": self.warp_blocks_per_sm, "cost_order": self.cost_order,
                "ns_per_wavenumber": {o: {"warp": self.ns_per_wavenumber[i][0],
                                          "thread": self.ns_per_wavenumber[i][1]}
                                      for i, o in enumerate((4, 8, 16))}}


def array_counts(d: BatchDesc) -> dict:
    """Elements of every input, output, cotangent and gradient array of a batch
    (the sizes adrt_solve_batch and adrt_adjoint read and write)."""
    W, L, M = d.num_wavenumbers, d.num_layers, d.num_moments
    mom = {MOMENTS_SHARED: L * M, MOMENTS_PER_WAVENUMBER: W * M}.get(d.moment_layout, W * L * M)
    temp = (W if d.temperature_per_wavenumber else 1) * (L + 1)
    n = {"delta_tau": W * L, "single_scat_albedo": W * L, "phase_moments": mom,
         "temperature": temp, "planck_levels": W * (L + 1)}
    for f in INPUT_FIELDS[5:]:
        n[f] = W
    out = {f: W * (L + 1) for f in INTERFACE_OUTPUTS}
    out.update({f: W for f in OUTPUT_FIELDS[5:]})
    return {"in": n, "out": out, "cot": {f: W * (L + 1) for f in COTANGENT_FIELDS},
            "grad": {f: (n[f] if f != "surface_emission" else W) for f in GRADIENT_FIELDS}}


class EngineOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("max_workspace_bytes", C.c_size_t)]


DESC_INT_FIELDS = tuple(n for n, t in BatchDesc._fields_ if t is C.c_int)
DESC_FLOAT_FIELDS = tuple(n for n, t in BatchDesc._fields_ if t is C.c_double)


def make_desc(**kw) -> BatchDesc:
    """BatchDesc with the reference's defaults (ADConfig / BatchConfig)."""
    d = BatchDesc()
    d.num_quadrature = 8
    d.moment_layout = MOMENTS_SHARED
    d.surface_temperature = -1.0
    d.top_temperature = -1.0
    d.solar_mu = 1.0
    d.spectrum_scaling = 1.0
    for k, v in kw.items():
        if not hasattr(d, k):
            raise AttributeError(f"adrt_batch_desc has no field {k!r}")
        setattr(d, k, v)
    return d


def desc_to_dict(d: BatchDesc) -> dict:
    return {n: getattr(d, n) for n, _ in BatchDesc._fields_}
