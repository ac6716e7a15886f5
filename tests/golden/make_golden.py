"""Generate the golden vectors in tests/golden/*.npz.

Each fixture holds one batch (description + inputs) and the outputs of the
reference's own CPU solver, adrt::solve (src/solver.cpp), compiled unmodified
from the reference sources against the project-written Eigen subset without
FMA contraction (oracle/_ref/libadrt_ref_strict.so; `make -C oracle ref`).

    python tests/golden/make_golden.py

Requires the reference checkout (only to build oracle/_ref); the fixtures are
committed so the tests need neither.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from addingdoublingrt_b200 import _abi, workloads  # noqa: E402
from oracle import oracle  # noqa: E402


def save(name: str, b: workloads.Batch, out: dict) -> None:
    payload = {"desc_" + k: np.asarray(v) for k, v in _abi.desc_to_dict(b.desc).items()}
    for k, v in b.arrays.items():
        payload["in_" + k] = v
    for k, v in out.items():
        payload["out_" + k] = v
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **payload)


def edge_cases():
    """Hand-built batches for the branches the reference tests exercise."""
    cases = []
    # single thin layer, isotropic, conservative, N=2 (smallest order)
    b = workloads.Batch(_abi.make_desc(num_wavenumbers=1, num_layers=1, num_quadrature=2,
                                       num_moments=4, solar_flux=1.0, solar_mu=0.5))
    b.set("delta_tau", [[0.03125]])  # 2^-5: exact power of two (nn truncation)
    b.set("single_scat_albedo", [[1.0]])
    b.set("phase_moments", [[1.0, 0.0, 0.0, 0.0]])
    cases.append(("edge_n2_pow2", b))
    # thick power-of-two layer, Rayleigh-like moments, N=16, surface albedo
    b = workloads.Batch(_abi.make_desc(num_wavenumbers=2, num_layers=2, num_quadrature=16,
                                       num_moments=32, solar_flux=1.0, solar_mu=0.6,
                                       surface_albedo=0.25))
    b.set("delta_tau", [[32.0, 0.5], [1.0, 2.0]])
    b.set("single_scat_albedo", [[0.99, 0.5], [1.0, 0.0]])
    m = np.zeros(32); m[0] = 1.0; m[2] = 0.1
    b.set("phase_moments", np.tile(m, (2, 1)))
    cases.append(("edge_rayleigh_thick", b))
    # pure absorption everywhere with thermal emission and a skin temperature
    b = workloads.Batch(_abi.make_desc(num_wavenumbers=3, num_layers=5, num_quadrature=8,
                                       num_moments=16, use_thermal_emission=1,
                                       wavenumber_low=500.0, wavenumber_high=1500.0,
                                       surface_temperature=310.0, surface_albedo=0.1))
    b.set("delta_tau", np.full((3, 5), 0.4))
    b.set("single_scat_albedo", np.zeros((3, 5)))
    b.set("phase_moments", workloads.hg_moments(np.full(5, 0.5), 16))
    b.set("temperature", np.linspace(200.0, 300.0, 6))
    cases.append(("edge_pure_absorption_thermal", b))
    # active delta-M truncation (M = 2N + 1), cold-space top, diffusion lower boundary
    b = workloads.Batch(_abi.make_desc(num_wavenumbers=2, num_layers=4, num_quadrature=8,
                                       num_moments=17, use_thermal_emission=1, use_delta_m=1,
                                       use_diffusion_lower_bc=1, top_temperature=0.0,
                                       wavenumber_low=600.0, wavenumber_high=700.0,
                                       solar_flux=1.0, solar_mu=0.7))
    b.set("delta_tau", [[0.5, 1.0, 2.0, 4.0], [0.1, 0.0, 3.0, 0.2]])
    b.set("single_scat_albedo", [[0.9, 0.8, 0.95, 0.5], [0.3, 0.6, 0.99, 0.0]])
    b.set("phase_moments", workloads.hg_moments(np.full(4, 0.85), 17))
    b.set("temperature", np.linspace(220.0, 290.0, 5))
    cases.append(("edge_deltam_diffusion_coldtop", b))
    # planck_levels mode, index_from_bottom, per-layer moments, fewer moments than 2N
    b = workloads.Batch(_abi.make_desc(num_wavenumbers=2, num_layers=3, num_quadrature=4,
                                       num_moments=5, moment_layout=_abi.MOMENTS_PER_LAYER,
                                       index_from_bottom=1, surface_emission=0.7,
                                       top_emission=0.2, surface_albedo=0.4))
    b.set("delta_tau", [[0.2, 0.7, 1.3], [2.0, 0.05, 0.6]])
    b.set("single_scat_albedo", [[0.5, 0.0, 0.9], [1.0, 0.2, 0.7]])
    b.set("phase_moments", workloads.hg_moments(np.array([[0.1, 0.5, 0.7], [0.0, 0.3, 0.9]]), 5))
    b.set("planck_levels", [[0.1, 0.2, 0.3, 0.4], [1.0, 0.9, 0.8, 0.7]])
    cases.append(("edge_planck_levels_from_bottom", b))
    # N=32 and N=3 / N=12 (orders outside the reference's fixed-size list)
    for n, seed in ((32, 101), (3, 102), (12, 103)):
        b = workloads.random_small(seed, N=n, L=4, W=2, use_thermal_emission=1,
                                   use_diffusion_lower_bc=0)
        cases.append((f"edge_n{n}", b))
    return cases


def main() -> None:
    if not oracle.ref_available(strict=True):
        raise SystemExit("oracle/_ref/libadrt_ref_strict.so missing: run `make -C oracle ref`")
    n = 0
    for seed in range(60):
        b = workloads.random_small(seed)
        try:
            out = oracle.solve_reference(b, 8, strict=True)
        except oracle.OracleError:
            continue  # the reference rejects this configuration (validate())
        save(f"random_{seed:03d}", b, out)
        n += 1
    for name, b in edge_cases():
        save(name, b, oracle.solve_reference(b, 8, strict=True))
        n += 1
    subsets = [
        ("config1", workloads.config1(W=1000).subset(np.arange(0, 1000, 100))),
        ("config2", workloads.config2().subset(np.arange(0, 100_000, 10_000))),
        ("config3", workloads.config3().subset(np.arange(0, 20_000, 4_000))),
        ("config5", workloads.config5().subset(np.arange(0, 10_000, 2_000))),
    ]
    for name, b in subsets:
        save(name, b, oracle.solve_reference(b, 8, strict=True))
        n += 1
    print(f"wrote {n} fixtures to {HERE}")


if __name__ == "__main__":
    main()
