"""The oracle is pinned before it is trusted (CPU only).

* The C restatement (oracle/adrt_oracle.c) reproduces the golden vectors --
  outputs of the reference's own solver compiled from its sources without FMA
  contraction -- to the last bit.
* Its pieces match the reference's utilities (quadrature, Planck, nn rule).
* The reference's own C++ suites (tests/test_ad_solver.cpp,
  tests/test_temperature_jacobian.cpp) are run against the reference build when
  the reference checkout is present (`make -C oracle check-ref`).
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from conftest import ROOT, golden_paths, load_golden
from addingdoublingrt_b200 import _abi, workloads
from oracle import oracle

GOLDEN = golden_paths()


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 60


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_restatement_reproduces_reference_bitwise(path):
    name, b, ref = load_golden(path)
    out = oracle.solve_oracle(b, 2)
    for k, v in ref.items():
        assert np.array_equal(out[k], v), (name, k, np.max(np.abs(out[k] - v)))


def test_gauss_legendre_weights_and_nodes():
    lib = oracle.oracle_lib()
    for n in (2, 3, 4, 8, 16, 32):
        x = np.zeros(n)
        w = np.zeros(n)
        lib.oracle_gauss_legendre(n, x.ctypes.data, w.ctypes.data)
        assert abs(w.sum() - 1.0) < 1e-14  # reference GaussLegendreWeightSum
        assert np.all((x > 0) & (x < 1))
        xr, wr = np.polynomial.legendre.leggauss(n)
        assert np.allclose(np.sort(x), (xr + 1) / 2, atol=1e-14)
        assert np.allclose(w[np.argsort(x)], wr / 2, atol=1e-14)


def test_planck_positive_and_stefan_boltzmann():
    lib = oracle.oracle_lib()
    assert lib.oracle_planck(500.0, 600.0, 300.0) > 0.0
    sigma = 5.67032e-8
    total = lib.oracle_planck(0.0, 1e5, 300.0)
    assert abs(total - sigma * 300.0 ** 4 / math.pi) / total < 1e-3
    assert lib.oracle_planck(500.0, 600.0, 0.0) == 0.0
    assert lib.oracle_planck(600.0, 500.0, 300.0) == -1.0  # invalid -> reference throws


def test_planck_derivative_matches_finite_difference():
    lib = oracle.oracle_lib()
    for lo, hi, T in ((500.0, 500.025, 250.0), (500.0, 1500.0, 280.0), (2000.0, 2000.0, 300.0)):
        h = 1e-3
        fd = (lib.oracle_planck(lo, hi, T + h) - lib.oracle_planck(lo, hi, T - h)) / (2 * h)
        an = lib.oracle_planck_deriv(lo, hi, T)
        assert abs(an - fd) <= 1e-5 * abs(fd) + 1e-30


def test_num_doublings_rule():
    lib = oracle.oracle_lib()
    assert lib.oracle_ipow0(0.005) == 4 and lib.oracle_ipow0(0.05) == 10
    assert lib.oracle_ipow0(0.1) == 16 and lib.oracle_ipow0(0.01) == 10
    for k in range(-20, 21):  # exact powers of two: ln(tau)/ln(2) is integral
        assert lib.oracle_num_doublings(2.0 ** k, 0.5) == max(1, k + 16)
    assert lib.oracle_num_doublings(3.0, 0.5) == 17
    assert lib.oracle_num_doublings(0.3, 0.5) == 15  # trunc toward zero of -1.74
    assert lib.oracle_num_doublings(1e-9, 0.001) == 1


@pytest.mark.skipif(not oracle.ref_available(strict=True), reason="reference build absent")
def test_reference_utilities_agree_with_restatement():
    ref = oracle.ref_lib(strict=True)
    lib = oracle.oracle_lib()
    for lo, hi, T in ((500.0, 500.025, 250.0), (500.0, 1500.0, 280.0), (10.0, 3000.0, 180.0)):
        assert ref.ref_planck(lo, hi, T) == lib.oracle_planck(lo, hi, T)
    for n in (2, 5, 16, 32):
        a, b = np.zeros(n), np.zeros(n)
        c, d = np.zeros(n), np.zeros(n)
        ref.ref_gauss_legendre(n, a.ctypes.data, b.ctypes.data)
        lib.oracle_gauss_legendre(n, c.ctypes.data, d.ctypes.data)
        assert np.array_equal(a, c) and np.array_equal(b, d)


@pytest.mark.skipif(not oracle.ref_available(strict=True), reason="reference build absent")
def test_restatement_matches_reference_on_fresh_random_batches():
    for seed in range(200, 230):
        b = workloads.random_small(seed)
        try:
            ref = oracle.solve_reference(b, 2, strict=True)
        except oracle.OracleError:
            with pytest.raises(oracle.OracleError):
                oracle.solve_oracle(b, 2)
            continue
        out = oracle.solve_oracle(b, 2)
        for k in ref:
            assert np.array_equal(out[k], ref[k]), (seed, k)


def test_validation_mirrors_reference():
    b = workloads.random_small(7, use_thermal_emission=0)
    b.arrays["delta_tau"][0] = -1.0
    with pytest.raises(oracle.OracleError, match="delta_tau"):
        oracle.solve_oracle(b, 1)
    b = workloads.random_small(7, use_thermal_emission=0)
    b.desc.surface_temperature = 300.0
    with pytest.raises(oracle.OracleError, match="surface_temperature requires"):
        oracle.solve_oracle(b, 1)


@pytest.mark.skipif(not os.path.isdir(os.path.join(oracle.reference_dir(), "tests")),
                    reason="reference checkout absent")
def test_reference_own_suites_pass_against_reference_build():
    r = oracle.make("check-ref", quiet=False, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "tests passed" in r.stdout


def test_flop_model_matches_expected_means():
    """Mean algorithmic flops per wavenumber-solve of the workloads, from the
    flop model of the branches the scheme takes (GEMM 2N^3, LU (2/3)N^3,
    triangular solve 2N^2 per right-hand side), within 15 % of the estimates
    2.4e6 (config 1), 7.6e7 (config 2) and 4.5e7 (config 5 forward)."""
    cases = {
        "cfg1": (workloads.config1(W=200), 2.4e6),
        "cfg2": (workloads.config2().subset(np.arange(0, 100_000, 500)), 7.6e7),
        "cfg5": (workloads.config5(W=200), 4.5e7),
    }
    for name, (b, expect) in cases.items():
        f = oracle.flops(b) / b.W
        assert 0.85 * expect < f < 1.15 * expect, (name, f)
