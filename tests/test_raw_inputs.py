"""Raw-coefficient entry point (adrt_solve_batch_raw; the reference's
adrt::cuda::solveBatchFromCoefficients, src_cuda/cuda_solver.cu:1193-1353).

The engine forms layer optical depths (trapezoid rule over altitude plus the
cloud optical depth), single-scattering albedos and single-wavenumber Planck
levels inside its solve.  As in the reference's own check
(tests/test_cuda_solver.cu:1587-1860), the fluxes must equal those of the
ordinary solve fed the preprocessed arrays, with per-wavenumber surface and
top emission; here the preprocessed arrays come from the oracle's FP64
restatement and the ordinary solve is the oracle itself and the engine's
FP64 entry point.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from addingdoublingrt_b200 import _abi, workloads
from oracle import oracle


def reference_case(cloud: bool):
    """The reference test's raw case: 4 wavenumbers, 5 layers, N = 4, 8
    isotropic moments, a non-uniform altitude grid and a cooling profile
    (tests/test_cuda_solver.cu:1602-1633), and its cloud variant (:1789-1793)."""
    W, L, M = 4, 5, 8
    wn = np.array([500.0, 1000.0, 1500.0, 2000.0])
    alt = np.array([0.0, 1e5, 3e5, 6e5, 1e6, 2e6], dtype=np.float32)
    temp = np.array([1500.0, 1300.0, 1100.0, 900.0, 700.0, 500.0], dtype=np.float32)
    lev = np.arange(L + 1)[:, None]
    w = np.arange(W)[None, :]
    ab = (np.float32(1e-6) * (1.0 + 0.5 * lev) * (1.0 + 0.3 * w)).astype(np.float32)
    sc = (np.float32(0.3) * ab).astype(np.float32)
    mom = np.zeros((L, M), dtype=np.float32)
    mom[:, 0] = 1.0
    cl = None
    if cloud:
        cl = np.repeat((0.01 * (np.arange(L) + 1))[:, None], W, axis=1).astype(np.float32)
    raw = dict(absorption_coeff=ab, scattering_coeff=sc, altitude=alt, temperature=temp,
               wavenumber=wn, cloud_optical_depth=cl, phase_moments=mom)
    desc = dict(num_wavenumbers=W, num_layers=L, num_quadrature=4, num_moments=M,
                moment_layout=_abi.MOMENTS_SHARED, surface_albedo=0.0)
    return desc, raw


def random_case(seed, W=300, L=40, N=16, M=40, shared=False):
    """Absorbing and scattering atmosphere with a cloud deck, solar beam,
    reflecting surface, skin and top temperatures and delta-M truncation."""
    rng = np.random.default_rng(seed)
    alt = np.cumsum(np.concatenate([[0.0], rng.uniform(2e4, 2e5, L)])).astype(np.float32)
    temp = np.linspace(320.0, 180.0, L + 1).astype(np.float32)
    wn = np.sort(rng.uniform(400.0, 3000.0, W))
    ab = (10.0 ** rng.uniform(-8, -4, (L + 1, W))).astype(np.float32)
    sc = (ab * rng.uniform(0.0, 3.0, (L + 1, W))).astype(np.float32)
    cl = np.zeros((L, W), dtype=np.float32)
    cl[3:8] = rng.uniform(0.0, 2.0, (5, W))
    g = rng.uniform(0.3, 0.85, L if shared else W * L)
    mom = workloads.hg_moments(g, M).astype(np.float32)
    raw = dict(absorption_coeff=ab, scattering_coeff=sc, altitude=alt, temperature=temp,
               wavenumber=wn, cloud_optical_depth=cl, phase_moments=mom)
    desc = dict(num_wavenumbers=W, num_layers=L, num_quadrature=N, num_moments=M,
                moment_layout=_abi.MOMENTS_SHARED if shared else _abi.MOMENTS_PER_LAYER,
                use_delta_m=1, surface_albedo=0.2, solar_flux=1.0, solar_mu=0.6,
                surface_temperature=330.0, top_temperature=2.7)
    return desc, raw


def oracle_fluxes(desc, raw):
    """TOA F_up, TOA F_down, BOA F_dir from the oracle on preprocessed arrays."""
    d = _abi.make_desc(**desc)
    pre = oracle.raw_preprocess(raw["absorption_coeff"], raw["scattering_coeff"],
                                raw["altitude"], raw["temperature"], raw["wavenumber"],
                                raw["cloud_optical_depth"], d.surface_temperature,
                                d.top_temperature)
    # the skin and top temperatures are now in the per-wavenumber emissions
    d.surface_temperature = -1.0
    d.top_temperature = -1.0
    b = workloads.Batch(d)
    for k in ("delta_tau", "single_scat_albedo", "planck_levels", "surface_emission",
              "top_emission"):
        b.set(k, pre[k])
    b.set("phase_moments", raw["phase_moments"].astype(np.float64))
    out = oracle.solve_oracle(b, 4, which=("toa_flux_up", "toa_flux_down", "boa_flux_direct"))
    return b, out


def engine_raw(eng, desc, raw):
    import torch
    d = _abi.make_desc(**desc)
    dev = {k: (torch.from_numpy(np.ascontiguousarray(v)).cuda() if v is not None else None)
           for k, v in raw.items()}
    ins = _abi.RawInputs(*[(dev[k].data_ptr() if dev[k] is not None else None)
                           for k in _abi.RAW_INPUT_FIELDS])
    W = d.num_wavenumbers
    outs = {k: torch.full((W,), np.nan, dtype=torch.float32, device="cuda")
            for k in ("toa_flux_up", "toa_flux_down", "boa_flux_direct")}
    o = _abi.OutputsF32(*[(outs[k].data_ptr() if k in outs else None)
                          for k in _abi.OUTPUT_F32_FIELDS])
    from addingdoublingrt_b200 import _lib
    _lib.check(eng.lib.adrt_solve_batch_raw(eng.handle, C.byref(d), C.byref(ins), C.byref(o),
                                            None))
    torch.cuda.synchronize()
    assert eng.read_status() == 0
    return {k: v.cpu().numpy().astype(np.float64) for k, v in outs.items()}


@pytest.fixture(scope="module")
def eng():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def close(a, b, rtol):
    scale = np.max(np.abs(b))
    return np.max(np.abs(a - b)) <= rtol * max(scale, 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("cloud", [False, True])
def test_reference_raw_case_matches_preprocessed_solve(eng, cloud):
    desc, raw = reference_case(cloud)
    got = engine_raw(eng, desc, raw)
    _, ref = oracle_fluxes(desc, raw)
    for k in ("toa_flux_up", "toa_flux_down"):
        # FP32 outputs of an FP64 solve
        assert close(got[k], ref[k], 2e-7), (k, got[k], ref[k])
    assert np.all(got["toa_flux_up"] > 0.0)


@pytest.mark.gpu
@pytest.mark.parametrize("shared", [True, False])
def test_random_raw_batch_matches_oracle(eng, shared):
    desc, raw = random_case(7 + shared, shared=shared)
    got = engine_raw(eng, desc, raw)
    b, ref = oracle_fluxes(desc, raw)
    for k in ("toa_flux_up", "toa_flux_down", "boa_flux_direct"):
        assert close(got[k], ref[k], 1e-6), (k, np.max(np.abs(got[k] - ref[k])))


@pytest.mark.gpu
def test_raw_matches_engine_fp64_path(eng):
    """The raw entry point and the ordinary FP64 entry point on the oracle's
    preprocessed arrays give the same fluxes (the reference's own pairing)."""
    import torch
    from addingdoublingrt_b200.engine import to_device, alloc_device_outputs
    desc, raw = random_case(3, W=200, L=30, N=8, M=24, shared=True)
    got = engine_raw(eng, desc, raw)
    b, _ = oracle_fluxes(desc, raw)
    di = to_device(b)
    do = alloc_device_outputs(b, which=("toa_flux_up", "toa_flux_down", "boa_flux_direct"))
    eng.solve_device(b.desc, di, do)
    torch.cuda.synchronize()
    for k in ("toa_flux_up", "toa_flux_down", "boa_flux_direct"):
        assert close(got[k], do[k].cpu().numpy(), 2e-7), k


def test_oracle_preprocessing_matches_fp32_procedure():
    """The oracle's FP64 preprocessing agrees with the reference test's FP32
    procedure (tests/test_cuda_solver.cu:1637-1677) to FP32 rounding."""
    desc, raw = reference_case(True)
    pre = oracle.raw_preprocess(raw["absorption_coeff"], raw["scattering_coeff"],
                                raw["altitude"], raw["temperature"], raw["wavenumber"],
                                raw["cloud_optical_depth"])
    f = np.float32
    W, L = desc["num_wavenumbers"], desc["num_layers"]
    ab, sc, alt, tmp = (raw[k] for k in ("absorption_coeff", "scattering_coeff", "altitude",
                                         "temperature"))
    for w in range(W):
        nu = f(raw["wavenumber"][w])
        for l in range(L):
            b = L - 1 - l
            dz = f(alt[b + 1] - alt[b])
            tau = f(dz * (f(ab[b + 1, w] + sc[b + 1, w]) + f(ab[b, w] + sc[b, w])) * f(0.5))
            sdep = f(dz * f(sc[b + 1, w] + sc[b, w]) * f(0.5))
            tau = f(tau + raw["cloud_optical_depth"][b, w])
            ssa = f(sdep / tau)
            assert abs(pre["delta_tau"][w, l] - tau) <= 1e-6 * tau
            assert abs(pre["single_scat_albedo"][w, l] - ssa) <= 1e-6 * ssa
        for lev in range(L + 1):
            t = f(tmp[L - lev])
            bb = f(1.19105e-08) * nu * nu * nu / f(np.exp(f(1.43879) * nu / t) - f(1.0))
            assert abs(pre["planck_levels"][w, lev] - bb) <= 1e-5 * bb
        assert pre["surface_emission"][w] == pre["planck_levels"][w, L]
        assert pre["top_emission"][w] == pre["planck_levels"][w, 0]
