"""PyTorch front end with the signature of the reference's JAX batch solver.

`solve_batch(config, delta_tau, ssa, phase_moments, planck_levels)` mirrors
src_jax/batch_solver.py:501-574 (BatchConfig :474-483): delta_tau and ssa
(nwav, nlay), phase_moments (nlay, nmom) shared by every wavenumber,
planck_levels (nwav, nlay+1); the surface emits planck_levels[:, -1] with
emissivity 1 - albedo and nothing comes down at the top, as in the JAX solver.
It returns (flux_up_toa, flux_down_boa), each (nwav,).

Differences from the JAX solver: the discrete scheme is the reference's CPU
scheme (first-order thin-layer start, per-layer doubling counts, delta-M
scaled beam), so results agree with adrt::solve; the solve runs on the B200
engine in FP64 (or the mixed form); and gradients come from the engine's
hand-written adjoint (adrt_adjoint) through a torch.autograd.Function, not
from automatic differentiation of the forward.  The adjoint is that of the
FP64 form, so a mixed-form solve whose inputs require gradients is refused.  Tensors are moved to the
current CUDA device and computed in float64; gradients are returned in the
inputs' dtypes.
"""
from __future__ import annotations

import torch

from . import _abi
from .engine import Engine

_engines: dict = {}


def _engine() -> Engine:
    dev = torch.cuda.current_device()
    if dev not in _engines:
        _engines[dev] = Engine(device=dev)
    return _engines[dev]


class BatchConfig:
    """Scalars of a batch (src_jax/batch_solver.py:474-483) plus the precision form."""

    def __init__(self):
        self.num_wavenumbers = 0
        self.num_layers = 0
        self.num_quadrature = 8
        self.num_moments_max = 16
        self.surface_albedo = 0.0
        self.solar_flux = 0.0
        self.solar_mu = 1.0
        self.precision = "fp64"  # or "mixed"


def _desc(config: BatchConfig, nwav: int, nlay: int, nmom: int) -> _abi.BatchDesc:
    return _abi.make_desc(
        num_wavenumbers=nwav, num_layers=nlay, num_quadrature=config.num_quadrature,
        num_moments=nmom, moment_layout=_abi.MOMENTS_SHARED,
        precision=_abi.PRECISION_MIXED if config.precision == "mixed" else _abi.PRECISION_FP64,
        use_thermal_emission=0, use_delta_m=0, surface_albedo=float(config.surface_albedo),
        solar_flux=float(config.solar_flux), solar_mu=float(config.solar_mu))


class _SolveBatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, config, delta_tau, ssa, phase_moments, planck_levels):
        dev = torch.device("cuda", torch.cuda.current_device())
        f64 = dict(dtype=torch.float64, device=dev)
        nwav, nlay = delta_tau.shape
        nmom = phase_moments.shape[1]
        ins = {
            "delta_tau": delta_tau.detach().to(**f64).contiguous(),
            "single_scat_albedo": ssa.detach().to(**f64).contiguous(),
            "phase_moments": phase_moments.detach().to(**f64).contiguous(),
            "planck_levels": planck_levels.detach().to(**f64).contiguous(),
        }
        ins["surface_emission"] = ins["planck_levels"][:, -1].contiguous()
        desc = _desc(config, nwav, nlay, nmom)
        n = nwav * (nlay + 1)
        outs = {"flux_up": torch.empty(n, **f64), "flux_down": torch.empty(n, **f64)}
        eng = _engine()
        eng.solve_device(desc, ins, outs, torch.cuda.current_stream())
        ctx.save_for_backward(delta_tau, ssa, phase_moments, planck_levels)
        ctx.desc, ctx.ins, ctx.nwav, ctx.nlay = desc, ins, nwav, nlay
        fu = outs["flux_up"].view(nwav, nlay + 1)[:, 0].clone()
        fd = outs["flux_down"].view(nwav, nlay + 1)[:, nlay].clone()
        return fu.to(delta_tau.dtype), fd.to(delta_tau.dtype)

    @staticmethod
    def backward(ctx, g_up, g_dn):
        delta_tau, ssa, phase_moments, planck_levels = ctx.saved_tensors
        nwav, nlay = ctx.nwav, ctx.nlay
        dev = ctx.ins["delta_tau"].device
        f64 = dict(dtype=torch.float64, device=dev)
        cot = {"flux_up": torch.zeros(nwav, nlay + 1, **f64),
               "flux_down": torch.zeros(nwav, nlay + 1, **f64)}
        if g_up is not None:
            cot["flux_up"][:, 0] = g_up.to(**f64)
        if g_dn is not None:
            cot["flux_down"][:, nlay] = g_dn.to(**f64)
        cot = {k: v.reshape(-1).contiguous() for k, v in cot.items()}
        gr = {
            "delta_tau": torch.zeros(nwav * nlay, **f64),
            "single_scat_albedo": torch.zeros(nwav * nlay, **f64),
            "phase_moments": torch.zeros_like(ctx.ins["phase_moments"]),
            "planck_levels": torch.zeros_like(ctx.ins["planck_levels"]),
            "surface_emission": torch.zeros(nwav, **f64),
        }
        _engine().adjoint(ctx.desc, ctx.ins, cot, gr, stream=torch.cuda.current_stream())
        gp = gr["planck_levels"].clone()
        gp[:, -1] += gr["surface_emission"]
        return (None,
                gr["delta_tau"].view(nwav, nlay).to(delta_tau.dtype),
                gr["single_scat_albedo"].view(nwav, nlay).to(ssa.dtype),
                gr["phase_moments"].to(phase_moments.dtype),
                gp.to(planck_levels.dtype))


def solve_batch(config: BatchConfig, delta_tau, ssa, phase_moments, planck_levels):
    """(flux_up_toa, flux_down_boa) of every wavenumber; differentiable in all four
    array arguments (src_jax/batch_solver.py:501-574)."""
    as_t = lambda x: x if torch.is_tensor(x) else torch.as_tensor(x, dtype=torch.float64)
    args = [as_t(delta_tau), as_t(ssa), as_t(phase_moments), as_t(planck_levels)]
    if config.precision == "mixed" and torch.is_grad_enabled() and any(
            a.requires_grad for a in args):
        # the adjoint differentiates the FP64 form; the mixed form's gradients
        # would belong to a different forward
        raise ValueError("gradients are available for precision='fp64' only; solve the mixed "
                         "form under torch.no_grad() or with inputs that do not require grad")
    return _SolveBatch.apply(config, *args)
