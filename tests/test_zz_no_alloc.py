"""The allocation-free entry point adrt_solve_batch_noalloc (GPU).

Callers that cannot allocate device memory -- code running under a
framework's caching allocator that already holds the GPU, latency-bound
retrieval loops, plugin hosts that only lend their own buffers -- solve
through adrt_solve_batch_noalloc, whose work memory is a fixed array inside
the library.  This file checks, through the C ABI, that two calls in a row
give the same fluxes as the engine's adrt_solve_batch on the same inputs,
within the FP64 parity tolerance of the other GPU tests, and that a batch
too large for the fixed work memory is refused with a clear error.  It is
named to be collected last, and works alone in a fresh process or after the
other tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from addingdoublingrt_b200 import _abi, _lib, workloads

pytestmark = pytest.mark.gpu


def _call_noalloc(lib, desc, di, do):
    from addingdoublingrt_b200.engine import _ptr
    ins = _abi.Inputs()
    for f in _abi.INPUT_FIELDS:
        setattr(ins, f, _ptr(di.get(f)))
    outs = _abi.Outputs()
    for f in _abi.OUTPUT_FIELDS:
        setattr(outs, f, _ptr(do.get(f)))
    return lib.adrt_solve_batch_noalloc(C.byref(desc), C.byref(ins), C.byref(outs), None)


def _norm_err(x, ref, per):
    x = np.asarray(x).reshape(-1, per)
    ref = np.asarray(ref).reshape(-1, per)
    s = np.max(np.abs(ref), axis=1)
    s[s == 0] = 1.0
    return float(np.max(np.max(np.abs(x - ref), axis=1) / s))


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_noalloc_matches_engine_on_two_calls(precision):
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    from addingdoublingrt_b200.engine import Engine, alloc_device_outputs, to_device
    lib = _lib.load()
    b = workloads.config2(W=2048, precision=precision)
    di = to_device(b)
    eng = Engine()
    ref = alloc_device_outputs(b, _abi.OUTPUT_FIELDS)
    eng.solve_device(b.desc, di, ref)
    torch.cuda.synchronize()
    ref = {k: v.cpu().numpy() for k, v in ref.items()}
    eng.close()
    for call in range(2):
        do = alloc_device_outputs(b, _abi.OUTPUT_FIELDS)
        rc = _call_noalloc(lib, b.desc, di, do)
        assert rc == 0, lib.adrt_last_status_detail().decode()
        torch.cuda.synchronize()
        for k in _abi.INTERFACE_OUTPUTS:
            e = _norm_err(do[k].cpu().numpy(), ref[k], b.L + 1)
            assert e <= 1e-9, (call, k, e)
        for k in ("toa_flux_up", "toa_flux_down", "boa_flux_direct"):
            got = do[k].cpu().numpy()
            assert np.allclose(got, ref[k], rtol=1e-9, atol=1e-12 * np.max(np.abs(ref[k]))), (call, k)


def test_noalloc_rejects_a_batch_beyond_its_work_memory():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    lib = _lib.load()
    b = workloads.random_small(7, N=32, L=4, W=1)
    b.desc.num_layers = 4000  # one wavenumber would need ~100 MB of work memory
    b.set("delta_tau", np.full(4000, 0.1))
    b.set("single_scat_albedo", np.full(4000, 0.5))
    b.desc.moment_layout = _abi.MOMENTS_SHARED
    b.set("phase_moments", np.tile(b.arrays["phase_moments"].reshape(-1)[:b.desc.num_moments],
                                   4000))
    b.desc.use_thermal_emission = 0
    b.arrays.pop("temperature", None)
    b.arrays.pop("planck_levels", None)
    b.desc.use_diffusion_lower_bc = 0
    di = to_device(b)
    do = alloc_device_outputs(b, ("flux_up",))
    rc = _call_noalloc(lib, b.desc, di, do)
    assert rc == _abi.ADRT_ERR_WORKSPACE
    assert "work memory" in lib.adrt_last_status_detail().decode()
