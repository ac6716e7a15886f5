"""Host-side batch container and the seeded synthetic workloads.

`Batch` holds one batch description (adrt_batch_desc) and its host arrays in
the layouts of include/adrt_b200.h.  The generators build the five workloads
the engine is measured and checked on (numpy default_rng(seed), wavenumber-
major SoA, TOA = layer/level 0).  They stand in for the retrieval inputs the
reference's batched API was written for (src_cuda/cuda_solver.cuh:4-6) and
extend the synthetic atmosphere of the reference benchmark
(tests/benchmark_cuda.cu:37-91) to per-wavenumber bands, albedos, solar
angles and double Henyey-Greenstein moments.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi


@dataclass
class Batch:
    desc: _abi.BatchDesc
    arrays: dict = field(default_factory=dict)  # name -> float64 C-contiguous ndarray

    # ------------------------------------------------------------ shape helpers
    @property
    def W(self) -> int:
        return self.desc.num_wavenumbers

    @property
    def L(self) -> int:
        return self.desc.num_layers

    @property
    def N(self) -> int:
        return self.desc.num_quadrature

    def set(self, name: str, value) -> None:
        if name not in _abi.INPUT_FIELDS:
            raise KeyError(name)
        if value is None:
            self.arrays.pop(name, None)
        else:
            self.arrays[name] = np.ascontiguousarray(value, dtype=np.float64)

    def inputs_struct(self) -> _abi.Inputs:
        s = _abi.Inputs()
        for f in _abi.INPUT_FIELDS:
            a = self.arrays.get(f)
            setattr(s, f, a.ctypes.data if a is not None else None)
        return s

    def alloc_outputs(self, which=_abi.OUTPUT_FIELDS) -> dict:
        nint = self.L + 1
        out = {}
        for f in which:
            n = self.W * nint if f in _abi.INTERFACE_OUTPUTS else self.W
            out[f] = np.zeros(n, dtype=np.float64)
        return out

    @staticmethod
    def outputs_struct(out: dict) -> _abi.Outputs:
        s = _abi.Outputs()
        for f in _abi.OUTPUT_FIELDS:
            a = out.get(f)
            setattr(s, f, a.ctypes.data if a is not None else None)
        return s

    def subset(self, idx) -> "Batch":
        """A batch holding only wavenumbers `idx` (per-wavenumber arrays sliced)."""
        idx = np.asarray(idx, dtype=np.int64)
        d = _abi.BatchDesc.from_buffer_copy(self.desc)
        d.num_wavenumbers = int(idx.size)
        W, L = self.W, self.L
        b = Batch(d)
        for name, a in self.arrays.items():
            if name in ("delta_tau", "single_scat_albedo"):
                b.set(name, a.reshape(W, L)[idx])
            elif name == "phase_moments":
                if self.desc.moment_layout == _abi.MOMENTS_SHARED:
                    b.set(name, a)
                elif self.desc.moment_layout == _abi.MOMENTS_PER_WAVENUMBER:
                    b.set(name, a.reshape(W, -1)[idx])
                else:
                    b.set(name, a.reshape(W, L, -1)[idx])
            elif name == "temperature":
                if self.desc.temperature_per_wavenumber:
                    b.set(name, a.reshape(W, L + 1)[idx])
                else:
                    b.set(name, a)
            elif name == "planck_levels":
                b.set(name, a.reshape(W, L + 1)[idx])
            else:  # per-wavenumber scalars
                b.set(name, a[idx])
        return b

    def nbytes_inputs(self) -> int:
        return int(sum(a.nbytes for a in self.arrays.values()))


# ---------------------------------------------------------------- moments


def hg_moments(g, M):
    """Henyey-Greenstein Legendre moments chi_m = g^m (ADConfig::setHenyeyGreenstein,
    src/adding_doubling.hpp:181-193)."""
    g = np.asarray(g, dtype=np.float64)
    return g[..., None] ** np.arange(M)


def dhg_moments(f, g1, g2, M):
    """Double Henyey-Greenstein chi_m = f g1^m + (1-f) g2^m
    (ADConfig::setDoubleHenyeyGreenstein, src/adding_doubling.hpp:200-215)."""
    m = np.arange(M)
    f = np.asarray(f, dtype=np.float64)[..., None]
    return f * np.asarray(g1, dtype=np.float64)[..., None] ** m + (1.0 - f) * (
        np.asarray(g2, dtype=np.float64)[..., None] ** m
    )


def level_temperatures(rng, L):
    """Lapse profile 180 K (TOA) -> 300 K (BOA) plus N(0, 2 K) noise per level."""
    l = np.arange(L + 1, dtype=np.float64)
    return 180.0 + 120.0 * l / L + rng.normal(0.0, 2.0, size=L + 1)


# ---------------------------------------------------------------- workloads


def config1(W=1000, L=20, seed=1) -> Batch:
    """Solar only, N=8, shared HG(0.7) moments (16), albedo 0.3, delta-M on."""
    rng = np.random.default_rng(seed)
    N, M = 8, 16
    d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                       moment_layout=_abi.MOMENTS_SHARED, use_delta_m=1,
                       solar_flux=1.0, solar_mu=0.5, surface_albedo=0.3)
    b = Batch(d)
    b.set("delta_tau", rng.uniform(0.01, 0.5, size=(W, L)))
    b.set("single_scat_albedo", np.full((W, L), 0.9))
    b.set("phase_moments", np.tile(0.7 ** np.arange(M), (L, 1)))
    return b


def _band(W, w_index=None):
    w = np.arange(W, dtype=np.float64) if w_index is None else w_index
    lo = 500.0 + 2500.0 * w / W
    return lo, lo + 0.025


def config2(W=100_000, L=100, seed=2, precision=_abi.PRECISION_FP64) -> Batch:
    """Thermal + solar, N=16, per-wavenumber double-HG moments (32), 500-3000 cm^-1."""
    rng = np.random.default_rng(seed)
    N, M = 16, 32
    d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                       moment_layout=_abi.MOMENTS_PER_WAVENUMBER, precision=precision,
                       use_thermal_emission=1, use_delta_m=1, surface_temperature=300.0,
                       solar_flux=1.0)
    b = Batch(d)
    b.set("delta_tau", 10.0 ** rng.uniform(-4.0, 1.0, size=(W, L)))
    b.set("single_scat_albedo", rng.uniform(0.0, 0.99, size=(W, L)))
    g1 = rng.uniform(0.5, 0.9, size=W)
    g2 = rng.uniform(-0.5, 0.0, size=W)
    f = rng.uniform(0.7, 0.95, size=W)
    b.set("phase_moments", dhg_moments(f, g1, g2, M))
    b.set("temperature", level_temperatures(rng, L))
    b.set("surface_albedo", rng.uniform(0.0, 0.3, size=W))
    b.set("solar_mu", rng.uniform(0.1, 1.0, size=W))
    lo, hi = _band(W)
    b.set("wavenumber_low", lo)
    b.set("wavenumber_high", hi)
    return b


def config2_scalar(W=100_000, L=100, seed=2, precision=_abi.PRECISION_FP64) -> Batch:
    """Config 2's shape (W x 100 layers, N=16, 32 double-HG moments, thermal +
    solar, the same optical-depth, albedo and temperature distributions) within
    the reference GPU API's limits (src_cuda/cuda_solver.cuh:18-40, and the
    per-layer phase tables of src_cuda/cuda_batched_solver.cu:112-180): moment
    sets shared over wavenumbers (one per layer), one surface albedo (0.15),
    solar cosine (0.55) and Planck band (1000-1000.025 cm^-1) per batch.  The
    workload on which the engine and the reference's own GPU solver are timed
    side by side."""
    rng = np.random.default_rng(seed)
    N, M = 16, 32
    d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                       moment_layout=_abi.MOMENTS_SHARED, precision=precision,
                       use_thermal_emission=1, use_delta_m=1, surface_temperature=300.0,
                       solar_flux=1.0, solar_mu=0.55, surface_albedo=0.15,
                       wavenumber_low=1000.0, wavenumber_high=1000.025)
    b = Batch(d)
    b.set("delta_tau", 10.0 ** rng.uniform(-4.0, 1.0, size=(W, L)))
    b.set("single_scat_albedo", rng.uniform(0.0, 0.99, size=(W, L)))
    f = rng.uniform(0.7, 0.95, size=L)
    b.set("phase_moments", dhg_moments(f, rng.uniform(0.5, 0.9, size=L),
                                       rng.uniform(-0.5, 0.0, size=L), M))
    b.set("temperature", level_temperatures(rng, L))
    return b


def config3(W=20_000, L=60, seed=3, precision=_abi.PRECISION_FP64) -> Batch:
    """Precision stress: N=32, 1-omega = 10^U(-7,-1), tau = 10^U(-5,3), HG g~U(0,0.95),
    diffusion lower boundary, thermal + solar."""
    rng = np.random.default_rng(seed)
    N, M = 32, 64
    d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                       moment_layout=_abi.MOMENTS_PER_WAVENUMBER, precision=precision,
                       use_thermal_emission=1, use_delta_m=1, use_diffusion_lower_bc=1,
                       solar_flux=1.0, solar_mu=0.5)
    b = Batch(d)
    one_minus = 10.0 ** rng.uniform(-7.0, -1.0, size=(W, L))
    b.set("single_scat_albedo", 1.0 - one_minus)
    b.set("delta_tau", 10.0 ** rng.uniform(-5.0, 3.0, size=(W, L)))
    b.set("phase_moments", hg_moments(rng.uniform(0.0, 0.95, size=W), M))
    b.set("temperature", level_temperatures(rng, L))
    lo, hi = _band(W)
    b.set("wavenumber_low", lo)
    b.set("wavenumber_high", hi)
    return b


def config5(W=10_000, L=60, seed=5, precision=_abi.PRECISION_FP64) -> Batch:
    """Adjoint workload: as config 2 but single-HG moments g_l per layer (shared over
    wavenumbers), N=16, 60 layers."""
    rng = np.random.default_rng(seed)
    N, M = 16, 32
    d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                       moment_layout=_abi.MOMENTS_SHARED, precision=precision,
                       use_thermal_emission=1, use_delta_m=1, surface_temperature=300.0,
                       solar_flux=1.0)
    b = Batch(d)
    b.set("delta_tau", 10.0 ** rng.uniform(-4.0, 1.0, size=(W, L)))
    b.set("single_scat_albedo", rng.uniform(0.0, 0.99, size=(W, L)))
    b.set("phase_moments", hg_moments(rng.uniform(0.5, 0.9, size=L), M))
    b.set("temperature", level_temperatures(rng, L))
    b.set("surface_albedo", rng.uniform(0.0, 0.3, size=W))
    b.set("solar_mu", rng.uniform(0.1, 1.0, size=W))
    lo, hi = _band(W)
    b.set("wavenumber_low", lo)
    b.set("wavenumber_high", hi)
    return b


def config4_columns(ncols=4096, seed=4, max_total=None):
    """Uneven batch: per column L~U{20..150}, N in {4,8,16}, W=floor(exp U(ln 256, ln 8192)),
    optical properties as config 2, source type uniform over solar / thermal / both.
    Returns a list of Batch (one per column)."""
    rng = np.random.default_rng(seed)
    cols = []
    total = 0
    for c in range(ncols):
        L = int(rng.integers(20, 151))
        N = int(rng.choice([4, 8, 16]))
        W = int(np.floor(np.exp(rng.uniform(np.log(256.0), np.log(8192.0)))))
        src = int(rng.integers(0, 3))  # 0 solar, 1 thermal, 2 both
        M = 2 * N
        thermal = src in (1, 2)
        solar = src in (0, 2)
        d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                           moment_layout=_abi.MOMENTS_PER_WAVENUMBER,
                           precision=_abi.PRECISION_MIXED,
                           use_thermal_emission=int(thermal), use_delta_m=1,
                           surface_temperature=300.0 if thermal else -1.0,
                           solar_flux=1.0 if solar else 0.0)
        b = Batch(d)
        b.set("delta_tau", 10.0 ** rng.uniform(-4.0, 1.0, size=(W, L)))
        b.set("single_scat_albedo", rng.uniform(0.0, 0.99, size=(W, L)))
        b.set("phase_moments", dhg_moments(rng.uniform(0.7, 0.95, size=W),
                                           rng.uniform(0.5, 0.9, size=W),
                                           rng.uniform(-0.5, 0.0, size=W), M))
        if thermal:
            b.set("temperature", level_temperatures(rng, L))
            lo, hi = _band(W)
            b.set("wavenumber_low", lo)
            b.set("wavenumber_high", hi)
        b.set("surface_albedo", rng.uniform(0.0, 0.3, size=W))
        b.set("solar_mu", rng.uniform(0.1, 1.0, size=W))
        cols.append(b)
        total += W
        if max_total is not None and total >= max_total:
            break
    return cols


def config4_shapes(ncols=4096, seed=4):
    """The column shapes of config 4 (L, N, W, source type per column), drawn as
    config4_columns draws them."""
    rng = np.random.default_rng(seed)
    shapes = []
    for _ in range(ncols):
        L = int(rng.integers(20, 151))
        N = int(rng.choice([4, 8, 16]))
        W = int(np.floor(np.exp(rng.uniform(np.log(256.0), np.log(8192.0)))))
        src = int(rng.integers(0, 3))  # 0 solar, 1 thermal, 2 both
        shapes.append((L, N, W, src))
    return shapes


def config4_device(ncols=4096, seed=4, precision=_abi.PRECISION_MIXED, device="cuda",
                   fraction=1.0):
    """Config 4 generated on the device (the full batch, about 9.3e6
    wavenumber-columns and 40 GB of inputs and outputs, is too large to build
    on the host): the column shapes of config4_columns, per-wavenumber values
    from a seeded torch generator with config 4's distributions.  `fraction`
    keeps the first ceil(fraction W) wavenumbers of every column.  Returns
    [(desc, device inputs, device outputs)] for Engine.solve_uneven."""
    import torch
    g = torch.Generator(device=device).manual_seed(seed)
    f64 = dict(dtype=torch.float64, device=device)

    def U(lo, hi, *shape):
        return lo + (hi - lo) * torch.rand(*shape, generator=g, **f64)

    cols = []
    crng = np.random.default_rng(seed + 1000)
    for L, N, W, src in config4_shapes(ncols, seed):
        W = max(1, int(np.ceil(fraction * W)))
        M = 2 * N
        thermal, solar = src in (1, 2), src in (0, 2)
        d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                           moment_layout=_abi.MOMENTS_PER_WAVENUMBER, precision=precision,
                           use_thermal_emission=int(thermal), use_delta_m=1,
                           surface_temperature=300.0 if thermal else -1.0,
                           solar_flux=1.0 if solar else 0.0)
        m = torch.arange(M, **f64)
        f, g1, g2 = U(0.7, 0.95, W, 1), U(0.5, 0.9, W, 1), U(-0.5, 0.0, W, 1)
        ins = {"delta_tau": (10.0 ** U(-4.0, 1.0, W * L)).contiguous(),
               "single_scat_albedo": U(0.0, 0.99, W * L),
               "phase_moments": (f * g1 ** m + (1.0 - f) * g2 ** m).reshape(-1).contiguous(),
               "surface_albedo": U(0.0, 0.3, W), "solar_mu": U(0.1, 1.0, W)}
        if thermal:
            ins["temperature"] = torch.as_tensor(level_temperatures(crng, L), **f64)
            lo, hi = _band(W)
            ins["wavenumber_low"] = torch.as_tensor(lo, **f64)
            ins["wavenumber_high"] = torch.as_tensor(hi, **f64)
        outs = {k: torch.zeros(W * (L + 1), **f64) for k in _abi.INTERFACE_OUTPUTS}
        cols.append((d, ins, outs))
    return cols


def column_to_host(desc, ins, w) -> Batch:
    """Wavenumber w of a device column as a host batch of one (oracle checks)."""
    d = _abi.BatchDesc.from_buffer_copy(desc)
    d.num_wavenumbers = 1
    W, L, M = desc.num_wavenumbers, desc.num_layers, desc.num_moments
    b = Batch(d)
    for k, v in ins.items():
        if k in ("delta_tau", "single_scat_albedo"):
            b.set(k, v[w * L:(w + 1) * L].cpu().numpy().reshape(1, L))
        elif k == "phase_moments":
            b.set(k, v[w * M:(w + 1) * M].cpu().numpy().reshape(1, M))
        elif k == "temperature":
            b.set(k, v.cpu().numpy())
        else:
            b.set(k, v[w:w + 1].cpu().numpy())
    return b


def random_small(seed, N=None, L=None, W=None, **flags) -> Batch:
    """Small randomized batch exercising every option (parity tests)."""
    rng = np.random.default_rng(seed)
    N = N or int(rng.choice([2, 3, 4, 5, 8, 12, 16, 24, 32]))
    L = L or int(rng.integers(1, 9))
    W = W or int(rng.integers(1, 6))
    thermal = flags.pop("use_thermal_emission", int(rng.integers(0, 2)))
    delta_m = flags.pop("use_delta_m", int(rng.integers(0, 2)))
    diffusion = flags.pop("use_diffusion_lower_bc", int(rng.integers(0, 4) == 0))
    layout = flags.pop("moment_layout", int(rng.integers(0, 3)))
    M = flags.pop("num_moments", 2 * N + int(rng.integers(0, 3)))
    solar = flags.pop("solar_flux", float(rng.choice([0.0, 1.0, 2.5])))
    d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                       moment_layout=layout, use_thermal_emission=thermal, use_delta_m=delta_m,
                       use_diffusion_lower_bc=diffusion, solar_flux=solar,
                       solar_mu=float(rng.uniform(0.1, 1.0)))
    for k, v in flags.items():
        setattr(d, k, v)
    b = Batch(d)
    tau = 10.0 ** rng.uniform(-3.0, 1.5, size=(W, L))
    tau[rng.random(size=(W, L)) < 0.05] = 0.0
    b.set("delta_tau", tau)
    om = rng.uniform(0.0, 1.0, size=(W, L))
    om[rng.random(size=(W, L)) < 0.2] = 0.0
    om[rng.random(size=(W, L)) < 0.05] = 1.0
    b.set("single_scat_albedo", om)
    nsets = {0: L, 1: W, 2: W * L}[layout]
    g = rng.uniform(-0.3, 0.9, size=nsets)
    b.set("phase_moments", hg_moments(g, M))
    if thermal:
        b.set("temperature", 200.0 + 100.0 * rng.random(size=L + 1))
        lo = rng.uniform(100.0, 2000.0, size=W)
        b.set("wavenumber_low", lo)
        b.set("wavenumber_high", lo + rng.choice([0.01, 1.0, 300.0], size=W))
        if rng.random() < 0.5:
            d.surface_temperature = float(rng.uniform(250.0, 320.0))
        if rng.random() < 0.3:
            d.top_temperature = float(rng.choice([0.0, 150.0]))
    elif rng.random() < 0.5:
        b.set("planck_levels", rng.uniform(0.0, 2.0, size=(W, L + 1)))
        d.surface_emission = float(rng.uniform(0.0, 1.0))
        d.top_emission = float(rng.uniform(0.0, 0.5))
    if rng.random() < 0.7:
        b.set("surface_albedo", rng.uniform(0.0, 1.0, size=W) * (rng.random(size=W) < 0.8))
    else:
        d.surface_albedo = float(rng.uniform(0.0, 1.0))
    if rng.random() < 0.5:
        b.set("solar_mu", rng.uniform(0.05, 1.0, size=W))
    d.index_from_bottom = int(rng.random() < 0.25)
    return b
