"""The reference's own test suites run against this library's drop-in API.

oracle/Makefile (`engine-tests`) compiles the reference's
tests/test_ad_solver.cpp (the column solver: known answers from published
tables, energy conservation, validation errors, workspace reuse),
tests/test_temperature_jacobian.cpp (the analytic temperature Jacobians of
ADConfig::compute_temperature_jacobian against central differences) and
tests/test_cuda_solver.cu (the batched GPU API: solveBatch, solveBatchHost and
the raw-coefficient solveBatchFromCoefficients) unmodified, against
include/adrt/*.hpp and libadrt_host.so, so every adrt::solve / adrt::cuda::*
call they make runs on the B200 engine.  A suite passes when its process
exits 0 (the reference harnesses return their failure counts).
"""
import os
import subprocess

import pytest

from conftest import cuda_available

REF_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                       "_ref")


@pytest.mark.gpu
@pytest.mark.parametrize("suite", ["engine_ad_solver_tests", "engine_cuda_solver_tests"])
def test_reference_suite_passes_on_the_engine(suite):
    if not cuda_available():
        pytest.skip("no CUDA device")
    exe = os.path.join(REF_DIR, suite)
    if not os.path.exists(exe):
        pytest.skip(f"{suite} not built (needs the reference checkout at build time)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    tail = "\n".join((r.stdout + r.stderr).splitlines()[-25:])
    assert r.returncode == 0, tail
