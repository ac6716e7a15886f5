"""The adjoint (adrt_adjoint) against central finite differences of the oracle
and against the reference's own analytic temperature Jacobian (GPU).

The loss is L = sum over wavenumbers and interfaces of c . (F_up, F_down, J,
F_dir) with random cotangents c.  Finite differences perturb one input for all
wavenumbers at once (wavenumbers are independent) and use the oracle (the C
restatement, FP64).  The doubling count nn is piecewise constant in tau and
omega (src/doubling.hpp:20-26, 107-109); the adjoint differentiates the scheme
at fixed nn, so parameters whose perturbation would change nn are skipped.

The reference computes dF/dT analytically (src/solver.cpp:117-341); the
adjoint's temperature gradient contracted against the same cotangents must
match it.
"""
import os

import numpy as np
import pytest

from conftest import cuda_available
from addingdoublingrt_b200 import _abi, workloads
from oracle import oracle

pytestmark = pytest.mark.gpu

COT = ("flux_up", "flux_down", "mean_intensity", "flux_direct")


@pytest.fixture(scope="module")
def eng():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def small_batch(seed, N, W=5, L=7, layout=_abi.MOMENTS_SHARED, temp_per_wav=False):
    """Config-5-like: thermal + solar, single-HG moments, 2N moments (delta-M no-op)."""
    rng = np.random.default_rng(seed)
    M = 2 * N
    d = _abi.make_desc(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                       moment_layout=layout, use_thermal_emission=1, use_delta_m=1,
                       surface_temperature=300.0, solar_flux=1.0,
                       temperature_per_wavenumber=int(temp_per_wav))
    b = workloads.Batch(d)
    b.set("delta_tau", 10.0 ** rng.uniform(-2.5, 0.7, size=(W, L)))
    om = rng.uniform(0.1, 0.95, size=(W, L))
    om[:, 2] = 0.0  # one purely absorbing layer
    b.set("single_scat_albedo", om)
    nsets = {0: L, 1: W, 2: W * L}[layout]
    b.set("phase_moments", workloads.hg_moments(rng.uniform(0.4, 0.85, size=nsets), M))
    T = workloads.level_temperatures(rng, L)
    b.set("temperature", np.tile(T, (W, 1)) + rng.normal(0, 1, (W, L + 1)) if temp_per_wav else T)
    b.set("surface_albedo", rng.uniform(0.05, 0.3, size=W))
    b.set("solar_mu", rng.uniform(0.3, 1.0, size=W))
    lo = rng.uniform(600.0, 2000.0, size=W)
    b.set("wavenumber_low", lo)
    b.set("wavenumber_high", lo + 5.0)
    return b


def run_adjoint(eng, b, cot, which=("delta_tau", "single_scat_albedo", "phase_moments",
                                    "temperature")):
    import torch
    from addingdoublingrt_b200.engine import to_device
    di = to_device(b)
    dc = {k: torch.from_numpy(v).cuda() for k, v in cot.items()}
    dg = {k: torch.zeros_like(di[k]) for k in which}
    eng.adjoint(b.desc, di, dc, dg)
    torch.cuda.synchronize()
    assert eng.read_status() == 0
    return {k: v.cpu().numpy().reshape(b.arrays[k].shape) for k, v in dg.items()}


def loss_per_wav(b, cot):
    out = oracle.solve_oracle(b, 4, which=COT)
    return sum((cot[k] * out[k]).reshape(b.W, -1).sum(axis=1) for k in COT)


def nn_of(tau, om):
    lib = oracle.oracle_lib()
    return lib.oracle_num_doublings(float(tau), float(min(om, 1.0))) if tau > 0 and om > 0 else -1


def fd_layer_param(b, cot, name, rel=1e-5):
    """d loss / d name[w, l] by central differences (all wavenumbers at once);
    NaN where the perturbation changes the doubling count."""
    base = b.arrays[name].reshape(b.W, b.L)
    tau = b.arrays["delta_tau"].reshape(b.W, b.L)
    om = b.arrays["single_scat_albedo"].reshape(b.W, b.L)
    g = np.full((b.W, b.L), np.nan)
    for l in range(b.L):
        h = rel * np.maximum(np.abs(base[:, l]), 1e-3)
        # omega = 0 switches the layer to the pure-absorption branch: not differentiable
        ok = base[:, l] > h if name == "single_scat_albedo" else np.ones(b.W, bool)
        a_safe = base.copy()
        a_safe[~ok, l] = 0.5 if name == "single_scat_albedo" else a_safe[~ok, l]
        vals = []
        for sgn in (1.0, -1.0):
            a = a_safe.copy()
            a[:, l] += sgn * h
            for w in range(b.W):
                t2 = a[w, l] if name == "delta_tau" else tau[w, l]
                o2 = a[w, l] if name == "single_scat_albedo" else om[w, l]
                if ok[w] and nn_of(t2, o2) != nn_of(tau[w, l], om[w, l]):
                    ok[w] = False
            bb = workloads.Batch(_abi.BatchDesc.from_buffer_copy(b.desc), dict(b.arrays))
            bb.set(name, a)
            vals.append(loss_per_wav(bb, cot))
        g[:, l] = np.where(ok, (vals[0] - vals[1]) / (2 * h), np.nan)
    return g


def rel_err(ad, fd):
    m = ~np.isnan(fd)
    return float(np.max(np.abs(ad[m] - fd[m])) / np.max(np.abs(fd[m])))


@pytest.mark.parametrize("N", [4, 8, 16, 32])
def test_adjoint_tau_and_omega_match_finite_differences(eng, N):
    b = small_batch(11 + N, N)
    rng = np.random.default_rng(N)
    cot = {k: rng.normal(size=b.W * (b.L + 1)) for k in COT}
    ad = run_adjoint(eng, b, cot)
    for name in ("delta_tau", "single_scat_albedo"):
        fd = fd_layer_param(b, cot, name)
        e = rel_err(ad[name].reshape(b.W, b.L), fd)
        assert e < 2e-5, (name, N, e)


def test_adjoint_moments_and_temperatures_match_finite_differences(eng):
    b = small_batch(3, 8, W=4, L=6)
    rng = np.random.default_rng(3)
    cot = {k: rng.normal(size=b.W * (b.L + 1)) for k in COT}
    ad = run_adjoint(eng, b, cot)
    M = b.desc.num_moments
    chi = b.arrays["phase_moments"].reshape(b.L, M)
    fd = np.zeros_like(chi)
    h = 1e-5
    for l in range(b.L):
        for m in range(M):
            vals = []
            for sgn in (1.0, -1.0):
                c = chi.copy()
                c[l, m] += sgn * h
                bb = workloads.Batch(_abi.BatchDesc.from_buffer_copy(b.desc), dict(b.arrays))
                bb.set("phase_moments", c)
                vals.append(loss_per_wav(bb, cot).sum())
            fd[l, m] = (vals[0] - vals[1]) / (2 * h)
    e = rel_err(ad["phase_moments"].reshape(b.L, M), fd)
    assert e < 1e-4, ("phase_moments", e)
    T = b.arrays["temperature"]
    fdT = np.zeros_like(T)
    for l in range(b.L + 1):
        vals = []
        for sgn in (1.0, -1.0):
            a = T.copy()
            a[l] += sgn * 1e-3
            bb = workloads.Batch(_abi.BatchDesc.from_buffer_copy(b.desc), dict(b.arrays))
            bb.set("temperature", a)
            vals.append(loss_per_wav(bb, cot).sum())
        fdT[l] = (vals[0] - vals[1]) / 2e-3
    e = rel_err(ad["temperature"], fdT)
    assert e < 1e-4, ("temperature", e)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) absent")
def test_temperature_gradient_matches_reference_analytic_jacobian(eng):
    """Per wavenumber, dL/dT_l from the adjoint equals cot . J_T of the reference's
    analytic Jacobian (levels 0..L; the surface temperature column is not an input
    gradient here)."""
    import ctypes as C
    b = small_batch(21, 8, W=3, L=6, temp_per_wav=True)
    b.set("solar_mu", np.full(b.W, 0.6))
    rng = np.random.default_rng(21)
    cot = {k: rng.normal(size=b.W * (b.L + 1)) for k in COT}
    ad = run_adjoint(eng, b, cot)["temperature"].reshape(b.W, b.L + 1)
    lib = oracle.ref_lib()
    L = b.L
    for w in range(b.W):
        jac = {k: np.zeros((L + 1) * (L + 2)) for k in ("flux_up", "flux_down", "mean_intensity")}
        out = b.alloc_outputs()
        ins = b.inputs_struct()
        rc = lib.ref_solve_column_jacobian(C.byref(b.desc), C.byref(ins), w,
                                           C.byref(workloads.Batch.outputs_struct(out)),
                                           jac["flux_up"].ctypes.data, jac["flux_down"].ctypes.data,
                                           jac["mean_intensity"].ctypes.data, None)
        assert rc == 0, lib.ref_last_error()
        g = np.zeros(L + 1)
        for k in ("flux_up", "flux_down", "mean_intensity"):
            J = jac[k].reshape(L + 1, L + 2)[:, :L + 1]
            g += cot[k].reshape(b.W, L + 1)[w] @ J
        e = np.max(np.abs(ad[w] - g)) / np.max(np.abs(g))
        assert e < 1e-6, (w, e)


def fd_moments(b, cot, h=1e-5):
    """d loss / d chi by central differences over every moment set."""
    M = b.desc.num_moments
    chi = b.arrays["phase_moments"].reshape(-1, M)
    fd = np.zeros_like(chi)
    for s in range(chi.shape[0]):
        for m in range(M):
            vals = []
            for sgn in (1.0, -1.0):
                c = chi.copy()
                c[s, m] += sgn * h
                bb = workloads.Batch(_abi.BatchDesc.from_buffer_copy(b.desc), dict(b.arrays))
                bb.set("phase_moments", c)
                vals.append(loss_per_wav(bb, cot).sum())
            fd[s, m] = (vals[0] - vals[1]) / (2 * h)
    return fd


def fd_temperature(b, cot, h=1e-3):
    """d loss / d T_l by central differences: per wavenumber when the level
    temperatures are (wavenumbers are independent), else of the summed loss."""
    T = b.arrays["temperature"]
    per_w = bool(b.desc.temperature_per_wavenumber)
    Tm = T.reshape(b.W if per_w else 1, b.L + 1)
    fd = np.zeros(Tm.shape)
    for l in range(b.L + 1):
        vals = []
        for sgn in (1.0, -1.0):
            a = Tm.copy()
            a[:, l] += sgn * h
            bb = workloads.Batch(_abi.BatchDesc.from_buffer_copy(b.desc), dict(b.arrays))
            bb.set("temperature", a.reshape(T.shape))
            v = loss_per_wav(bb, cot)
            vals.append(v if per_w else v.sum())
        fd[:, l] = (vals[0] - vals[1]) / (2 * h)
    return fd.reshape(T.shape)


@pytest.mark.parametrize("layout", [_abi.MOMENTS_PER_WAVENUMBER, _abi.MOMENTS_PER_LAYER])
def test_adjoint_moment_layouts_match_finite_differences(eng, layout):
    """One moment set per wavenumber (its cotangent accumulated over the
    layers) and one per wavenumber and layer: tau, omega and moment gradients."""
    b = small_batch(31 + layout, 4, W=3, L=4, layout=layout)
    rng = np.random.default_rng(31 + layout)
    cot = {k: rng.normal(size=b.W * (b.L + 1)) for k in COT}
    ad = run_adjoint(eng, b, cot)
    for name in ("delta_tau", "single_scat_albedo"):
        fd = fd_layer_param(b, cot, name)
        e = rel_err(ad[name].reshape(b.W, b.L), fd)
        assert e < 2e-5, (name, layout, e)
    fd = fd_moments(b, cot)
    e = rel_err(ad["phase_moments"].reshape(fd.shape), fd)
    assert e < 1e-4, ("phase_moments", layout, e)


def thick_batch(seed, N, W=6, L=5, M=None, temp_per_wav=False):
    """Optically thick scattering layers (tau 300..1000, omega >= 0.3): about
    25 doublings per layer against the 12 per layer the record pool holds on
    average, so only part of the batch gets records and the reverse pass
    recomputes the other wavenumbers' doubling chains."""
    b = small_batch(seed, N, W=W, L=L, temp_per_wav=temp_per_wav)
    rng = np.random.default_rng(seed + 100)
    b.set("delta_tau", 10.0 ** rng.uniform(2.5, 3.0, size=(W, L)))
    b.set("single_scat_albedo", rng.uniform(0.3, 0.95, size=(W, L)))
    if M is not None:
        d = _abi.BatchDesc.from_buffer_copy(b.desc)
        d.num_moments = M
        arrays = dict(b.arrays)
        arrays["phase_moments"] = workloads.hg_moments(rng.uniform(0.4, 0.85, size=L), M)
        b = workloads.Batch(d, arrays)
    return b


PER_WAVENUMBER = ("delta_tau", "single_scat_albedo", "temperature", "surface_albedo",
                  "solar_mu", "wavenumber_low", "wavenumber_high")


def joined(a, b):
    """Batch of a's wavenumbers followed by b's (a's phase moments)."""
    d = _abi.BatchDesc.from_buffer_copy(a.desc)
    d.num_wavenumbers = a.W + b.W
    arrays = dict(a.arrays)
    for k in PER_WAVENUMBER:
        arrays[k] = np.concatenate([a.arrays[k].reshape(a.W, -1),
                                    b.arrays[k].reshape(b.W, -1)]).reshape(-1)
    return workloads.Batch(d, arrays)


def test_recomputed_doubling_chains_equal_recorded_ones(eng):
    """Chains that found no room in the record pool are recomputed in the
    reverse pass.  Six thick wavenumbers alone overflow the pool (most are
    recomputed); joined with sixty thin ones the pool holds every chain.  Their
    per-wavenumber gradients agree, and the temperature gradient of the
    recomputing batch matches finite differences."""
    N = 8
    thick = thick_batch(41, N, temp_per_wav=True)
    tau = thick.arrays["delta_tau"].reshape(thick.W, thick.L)
    om = thick.arrays["single_scat_albedo"].reshape(thick.W, thick.L)
    nn = np.array([[nn_of(tau[w, l], om[w, l]) for l in range(thick.L)]
                   for w in range(thick.W)])
    assert nn.mean() > 2 * 12, nn.mean()  # twice the pool's average allowance
    thin = small_batch(42, N, W=60, L=thick.L, temp_per_wav=True)
    thin.set("delta_tau", 10.0 ** np.random.default_rng(42).uniform(-4, -3, size=(60, thick.L)))
    both = joined(thick, thin)
    rng = np.random.default_rng(41)
    cot_both = {k: rng.normal(size=both.W * (both.L + 1)) for k in COT}
    cot = {k: v.reshape(both.W, -1)[:thick.W].reshape(-1).copy() for k, v in cot_both.items()}
    rec = run_adjoint(eng, both, cot_both)
    ad = run_adjoint(eng, thick, cot)
    for name in ("delta_tau", "single_scat_albedo", "temperature"):
        r = rec[name].reshape(both.W, -1)[:thick.W]
        g = ad[name].reshape(thick.W, -1)
        e = np.max(np.abs(g - r)) / np.max(np.abs(r))
        assert e < 1e-9, (name, e)
    fd = fd_temperature(thick, cot)
    e = rel_err(ad["temperature"].reshape(fd.shape), fd)
    assert e < 1e-4, ("temperature", e)


def test_delta_m_truncated_temperature_gradient_matches_finite_differences(eng):
    """delta-M with more than 2N moments scales tau, omega and the phase
    moments by the truncated fraction chi_2N; the temperature gradient of that
    scheme (here with recomputed chains as well) against finite differences."""
    N = 4
    b = thick_batch(43, N, M=3 * N)
    assert b.desc.use_delta_m and b.desc.num_moments > 2 * N
    rng = np.random.default_rng(43)
    cot = {k: rng.normal(size=b.W * (b.L + 1)) for k in COT}
    ad = run_adjoint(eng, b, cot, which=("temperature",))
    e = rel_err(ad["temperature"], fd_temperature(b, cot))
    assert e < 1e-4, ("temperature", e)


@pytest.mark.parametrize("layout", [_abi.MOMENTS_SHARED, _abi.MOMENTS_PER_WAVENUMBER,
                                    _abi.MOMENTS_PER_LAYER])
def test_delta_m_truncated_gradients_match_finite_differences(eng, layout):
    """With delta-M truncation (3N moments, f = chi_2N) the gradients in tau,
    omega and every moment -- through the scaled tau', omega' and chi* of
    src/solver.cpp:441-501, f included -- against central differences of the
    oracle, for the three moment layouts."""
    N = 8
    b = small_batch(61 + layout, N, W=3, L=5, layout=layout)
    M = 3 * N
    g = b.arrays["phase_moments"].reshape(-1, 2 * N)[:, 1]
    b.desc.num_moments = M
    b.set("phase_moments", workloads.hg_moments(g, M))
    assert np.all(g ** (2 * N) > 1e-12)  # truncation active in every set
    rng = np.random.default_rng(61)
    cot = {k: rng.normal(size=b.W * (b.L + 1)) for k in COT}
    ad = run_adjoint(eng, b, cot)
    for name in ("delta_tau", "single_scat_albedo"):
        fd = fd_layer_param(b, cot, name)
        e = rel_err(ad[name].reshape(b.W, b.L), fd)
        assert e < 2e-5, (name, layout, e)
    chi = b.arrays["phase_moments"].reshape(-1, M)
    fd = np.zeros_like(chi)
    h = 1e-6
    for s_ in range(chi.shape[0]):
        for m in range(M):
            vals = []
            for sgn in (1.0, -1.0):
                c = chi.copy()
                c[s_, m] += sgn * h
                bb = workloads.Batch(_abi.BatchDesc.from_buffer_copy(b.desc), dict(b.arrays))
                bb.set("phase_moments", c)
                vals.append(loss_per_wav(bb, cot).sum())
            fd[s_, m] = (vals[0] - vals[1]) / (2 * h)
    e = rel_err(ad["phase_moments"].reshape(-1, M), fd)
    assert e < 1e-4, ("phase_moments", layout, e)


def test_shared_moments_without_block_sums_match_per_layer_sets(eng):
    """Shared per-layer moments whose per-block cotangent sums would pass
    1 GB (here 1800 layers at N = 16) take the per-layer moment adjoint beside
    the phase-matrix table; the moment gradient equals that of the same
    moments given per wavenumber and layer, summed over the wavenumbers, and
    the other gradients are unchanged."""
    N, L, W = 16, 1800, 3
    b = small_batch(51, N, W=W, L=L)
    M = b.desc.num_moments
    rng = np.random.default_rng(51)
    cot = {k: rng.normal(size=W * (L + 1)) for k in COT}
    shared = run_adjoint(eng, b, cot)
    d = _abi.BatchDesc.from_buffer_copy(b.desc)
    d.moment_layout = _abi.MOMENTS_PER_LAYER
    arrays = dict(b.arrays)
    arrays["phase_moments"] = np.tile(b.arrays["phase_moments"].reshape(1, L, M),
                                      (W, 1, 1)).reshape(-1).copy()
    per = run_adjoint(eng, workloads.Batch(d, arrays), cot)
    g_per = per["phase_moments"].reshape(W, L, M).sum(axis=0)
    g_sh = shared["phase_moments"].reshape(L, M)
    assert np.max(np.abs(g_sh - g_per)) <= 1e-9 * np.max(np.abs(g_per))
    for k in ("delta_tau", "single_scat_albedo", "temperature"):
        assert np.max(np.abs(shared[k] - per[k])) <= 1e-9 * np.max(np.abs(per[k])), k


def test_recompute_mode_matches_record_mode(eng):
    """ADRT_ADJOINT_RECOMPUTE (every doubling chain recomputed in the backward
    pass, only the per-layer R, T and sources kept from the forward) gives the
    gradients of the default recording mode."""
    b = small_batch(61, 16, W=40, L=12)
    rng = np.random.default_rng(61)
    cot = {k: rng.normal(size=b.W * (b.L + 1)) for k in COT}
    rec = run_adjoint(eng, b, cot)
    eng.set_adjoint_mode(_abi.ADJOINT_RECOMPUTE)
    try:
        recomp = run_adjoint(eng, b, cot)
    finally:
        eng.set_adjoint_mode(_abi.ADJOINT_RECORD)
    for k in rec:
        assert np.max(np.abs(recomp[k] - rec[k])) <= 1e-9 * np.max(np.abs(rec[k])), k
