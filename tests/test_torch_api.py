"""torch front end with the JAX solver's signature (src_jax/batch_solver.py:501-574):
forward equals the engine / oracle, backward equals central finite differences
of the oracle (GPU)."""
import numpy as np
import pytest

from conftest import cuda_available
from addingdoublingrt_b200 import _abi, workloads
from oracle import oracle

pytestmark = pytest.mark.gpu


def inputs(seed=9, nwav=6, nlay=5, N=8):
    rng = np.random.default_rng(seed)
    tau = 10.0 ** rng.uniform(-2.0, 0.6, size=(nwav, nlay))
    ssa = rng.uniform(0.2, 0.95, size=(nwav, nlay))
    g = rng.uniform(0.3, 0.8, size=nlay)
    mom = workloads.hg_moments(g, 2 * N)
    planck = rng.uniform(0.2, 1.5, size=(nwav, nlay + 1))
    return tau, ssa, mom, planck


def oracle_batch(cfg, tau, ssa, mom, planck):
    nwav, nlay = tau.shape
    d = _abi.make_desc(num_wavenumbers=nwav, num_layers=nlay, num_quadrature=cfg.num_quadrature,
                       num_moments=mom.shape[1], moment_layout=_abi.MOMENTS_SHARED,
                       surface_albedo=cfg.surface_albedo, solar_flux=cfg.solar_flux,
                       solar_mu=cfg.solar_mu)
    b = workloads.Batch(d)
    b.set("delta_tau", tau)
    b.set("single_scat_albedo", ssa)
    b.set("phase_moments", mom)
    b.set("planck_levels", planck)
    b.set("surface_emission", planck[:, -1])
    return b


def oracle_toa_boa(cfg, tau, ssa, mom, planck):
    b = oracle_batch(cfg, tau, ssa, mom, planck)
    out = oracle.solve_oracle(b, 4, which=("flux_up", "flux_down"))
    L = tau.shape[1]
    return out["flux_up"].reshape(-1, L + 1)[:, 0], out["flux_down"].reshape(-1, L + 1)[:, L]


def test_solve_batch_forward_and_gradients():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    from addingdoublingrt_b200.torch_api import BatchConfig, solve_batch
    cfg = BatchConfig()
    cfg.num_quadrature = 8
    cfg.surface_albedo = 0.15
    cfg.solar_flux = 1.0
    cfg.solar_mu = 0.7
    tau, ssa, mom, planck = inputs()
    cfg.num_wavenumbers, cfg.num_layers = tau.shape
    cfg.num_moments_max = mom.shape[1]
    t = [torch.tensor(a, dtype=torch.float64, device="cuda", requires_grad=True)
         for a in (tau, ssa, mom, planck)]
    fu, fd = solve_batch(cfg, *t)
    rfu, rfd = oracle_toa_boa(cfg, tau, ssa, mom, planck)
    assert np.allclose(fu.detach().cpu().numpy(), rfu, rtol=1e-9, atol=1e-12)
    assert np.allclose(fd.detach().cpu().numpy(), rfd, rtol=1e-9, atol=1e-12)
    a = np.random.default_rng(1).normal(size=tau.shape[0])
    c = np.random.default_rng(2).normal(size=tau.shape[0])
    loss = (fu * torch.tensor(a, device="cuda")).sum() + (fd * torch.tensor(c, device="cuda")).sum()
    loss.backward()

    def L(tau_, ssa_, mom_, planck_):
        u, d = oracle_toa_boa(cfg, tau_, ssa_, mom_, planck_)
        return float(a @ u + c @ d)

    rng = np.random.default_rng(3)
    for k, arr in enumerate((tau, ssa, mom, planck)):
        grad = t[k].grad.detach().cpu().numpy()
        for _ in range(4):
            idx = tuple(int(rng.integers(0, s)) for s in arr.shape)
            # steps well above the scheme's own FP64 round-off (~1e-12 relative)
            h = 1e-4 * max(abs(arr[idx]), 0.05)
            ap, am = arr.copy(), arr.copy()
            ap[idx] += h
            am[idx] -= h
            args_p = [tau, ssa, mom, planck]
            args_m = [tau, ssa, mom, planck]
            args_p[k], args_m[k] = ap, am
            fdv = (L(*args_p) - L(*args_m)) / (2 * h)
            assert abs(grad[idx] - fdv) <= 2e-6 * max(1.0, abs(fdv)), (k, idx, grad[idx], fdv)

