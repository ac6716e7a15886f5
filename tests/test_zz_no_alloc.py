"""The allocation-free entry point adrt_solve_batch_noalloc.

Callers that cannot allocate device memory -- code running under a
framework's caching allocator that already holds the GPU, latency-bound
retrieval loops, plugin hosts that only lend their own buffers -- solve
through adrt_solve_batch_noalloc, whose work memory is a fixed array inside
the library.  This file checks, through the C ABI, that two calls in a row
give the same fluxes as the engine's adrt_solve_batch on the same inputs,
within the FP64 parity tolerance of the other GPU tests, and against the
oracle; that a batch too large for the fixed work memory, plain host arrays
and the batches adrt_solve_batch refuses are refused with a clear error; and
that its device status word is read and cleared by adrt_noalloc_read_status.
It is named to be collected last, and works alone in a fresh process or
after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from addingdoublingrt_b200 import _abi, _lib, workloads


def _call_noalloc(lib, desc, di, do, raw_ptrs=False):
    from addingdoublingrt_b200.engine import _ptr
    ptr = (lambda a: None if a is None else a.ctypes.data) if raw_ptrs else _ptr
    ins = _abi.Inputs()
    for f in _abi.INPUT_FIELDS:
        setattr(ins, f, ptr(di.get(f)))
    outs = _abi.Outputs()
    for f in _abi.OUTPUT_FIELDS:
        setattr(outs, f, ptr(do.get(f)))
    return lib.adrt_solve_batch_noalloc(C.byref(desc), C.byref(ins), C.byref(outs), None)


def _read_status(lib):
    v = C.c_int(-1)
    assert lib.adrt_noalloc_read_status(None, C.byref(v)) == 0, \
        lib.adrt_last_status_detail().decode()
    return v.value


def _norm_err(x, ref, per):
    x = np.asarray(x).reshape(-1, per)
    ref = np.asarray(ref).reshape(-1, per)
    s = np.max(np.abs(ref), axis=1)
    s[s == 0] = 1.0
    return float(np.max(np.max(np.abs(x - ref), axis=1) / s))


def test_noalloc_refuses_what_the_engine_refuses():
    """The entry point runs adrt_solve_batch's own argument checks first (no
    GPU is touched before they pass): a solar beam with solar_mu = 0, an
    albedo outside [0, 1], a surface temperature without thermal emission."""
    lib = _lib.load()
    cases = []
    b = workloads.config1(W=4)
    b.desc.solar_mu = 0.0
    cases.append((b, "solar_mu"))
    b = workloads.config1(W=4)
    b.desc.surface_albedo = 1.5
    cases.append((b, "surface_albedo"))
    b = workloads.config1(W=4)
    b.desc.surface_temperature = 300.0
    cases.append((b, "surface_temperature"))
    for b, word in cases:
        rc = _call_noalloc(lib, b.desc, b.arrays, b.alloc_outputs(("flux_up",)), raw_ptrs=True)
        assert rc == _abi.ADRT_ERR_INVALID_ARGUMENT
        assert word in lib.adrt_last_status_detail().decode()


@pytest.mark.gpu
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
    assert _read_status(lib) == 0


@pytest.mark.gpu
@pytest.mark.parametrize("N,L", [(16, 2000), (32, 1000)])
def test_noalloc_few_slots_against_the_oracle(N, L):
    """Batches so deep that the fixed work memory holds fewer wavenumber slots
    than the GPU has resident thread groups (one or two blocks of slots, the
    last wavenumbers taken by a partly idle grid), compared with the oracle."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    from oracle import oracle
    lib = _lib.load()
    b = workloads.random_small(11, N=N, L=L, W=9, use_thermal_emission=1)
    di = to_device(b)
    do = alloc_device_outputs(b, _abi.INTERFACE_OUTPUTS)
    rc = _call_noalloc(lib, b.desc, di, do)
    assert rc == 0, lib.adrt_last_status_detail().decode()
    torch.cuda.synchronize()
    ref = oracle.solve_oracle(b, which=_abi.INTERFACE_OUTPUTS)
    reff = oracle.solve_oracle(b, which=_abi.INTERFACE_OUTPUTS, fma=True)
    for k in _abi.INTERFACE_OUTPUTS:
        sens = _norm_err(reff[k], ref[k], b.L + 1)
        e = _norm_err(do[k].cpu().numpy(), ref[k], b.L + 1)
        assert e <= 1e-6 + 1000 * sens, (k, e, sens)
    assert _read_status(lib) & _abi.ADRT_FLAG_NONFINITE == 0


@pytest.mark.gpu
def test_noalloc_status_word_is_read_and_cleared():
    """A negative optical depth in the device arrays is flagged on the device
    (as by the engine); adrt_noalloc_read_status reports it once, then 0."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    lib = _lib.load()
    _read_status(lib)
    b = workloads.config1(W=4)
    b.arrays["delta_tau"].reshape(-1)[5] = -1.0
    di = to_device(b)
    do = alloc_device_outputs(b, ("flux_up",))
    assert _call_noalloc(lib, b.desc, di, do) == 0, lib.adrt_last_status_detail().decode()
    assert _read_status(lib) & _abi.ADRT_FLAG_BAD_INPUT
    assert _read_status(lib) == 0


@pytest.mark.gpu
def test_noalloc_refuses_host_arrays():
    """Plain host (numpy) arrays handed straight to the C entry point are
    refused before any kernel sees a host address."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    lib = _lib.load()
    b = workloads.config1(W=4)
    rc = _call_noalloc(lib, b.desc, b.arrays, b.alloc_outputs(("flux_up",)), raw_ptrs=True)
    assert rc == _abi.ADRT_ERR_INVALID_ARGUMENT
    assert "not device memory" in lib.adrt_last_status_detail().decode()


@pytest.mark.gpu
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
    b.desc.surface_temperature = -1.0
    b.desc.top_temperature = -1.0
    b.arrays.pop("temperature", None)
    b.arrays.pop("planck_levels", None)
    b.desc.use_diffusion_lower_bc = 0
    di = to_device(b)
    do = alloc_device_outputs(b, ("flux_up",))
    rc = _call_noalloc(lib, b.desc, di, do)
    assert rc == _abi.ADRT_ERR_WORKSPACE, lib.adrt_last_status_detail().decode()
    assert "work memory" in lib.adrt_last_status_detail().decode()


@pytest.mark.gpu
def test_noalloc_calls_take_no_device_memory():
    """After a first call (which loads the module and uploads the order's
    quadrature table), further calls leave the device's free memory exactly
    as it was: nothing is allocated, not even by the driver."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    lib = _lib.load()
    b = workloads.config2(W=4096, L=30)
    di = to_device(b)
    do = alloc_device_outputs(b, _abi.INTERFACE_OUTPUTS)
    assert _call_noalloc(lib, b.desc, di, do) == 0, lib.adrt_last_status_detail().decode()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    torch_bytes = torch.cuda.memory_allocated()
    for _ in range(3):
        assert _call_noalloc(lib, b.desc, di, do) == 0, lib.adrt_last_status_detail().decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert torch.cuda.memory_allocated() == torch_bytes
    assert _read_status(lib) & ~_abi.ADRT_FLAG_PIVOT_FALLBACK == 0


@pytest.mark.gpu
def test_noalloc_replays_from_a_cuda_graph():
    """After one eager call of the order (the quadrature table upload), a call
    can be captured in a CUDA graph: its counter resets and both passes (the
    solve and the re-solve pass) replay on new inputs written into the same
    buffers, equal to an eager call on those inputs."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    from addingdoublingrt_b200.engine import _ptr, alloc_device_outputs, to_device
    lib = _lib.load()
    b = workloads.config2(W=2048, L=40)
    di = to_device(b)
    do = alloc_device_outputs(b, _abi.INTERFACE_OUTPUTS)

    def call(stream):
        ins = _abi.Inputs()
        for f in _abi.INPUT_FIELDS:
            setattr(ins, f, _ptr(di.get(f)))
        outs = _abi.Outputs()
        for f in _abi.OUTPUT_FIELDS:
            setattr(outs, f, _ptr(do.get(f)))
        return lib.adrt_solve_batch_noalloc(C.byref(b.desc), C.byref(ins), C.byref(outs),
                                            C.c_void_p(stream.cuda_stream))

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        assert call(s) == 0, lib.adrt_last_status_detail().decode()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = call(s)
    assert rc == 0, lib.adrt_last_status_detail().decode()
    b2 = workloads.config2(W=2048, L=40, seed=78)
    for k, v in di.items():
        v.copy_(torch.from_numpy(b2.arrays[k]))
    for v in do.values():
        v.zero_()
    g.replay()
    torch.cuda.synchronize()
    got = {k: v.clone() for k, v in do.items()}
    assert call(torch.cuda.current_stream()) == 0
    torch.cuda.synchronize()
    for k in _abi.INTERFACE_OUTPUTS:
        assert torch.equal(got[k], do[k]), k
    assert not torch.equal(got["flux_up"], torch.zeros_like(got["flux_up"]))
    assert _read_status(lib) == 0
    del g
