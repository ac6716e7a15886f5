"""The C-ABI library loads and exports every entry point the header declares,
and its host-side validation mirrors ADConfig::validate()
(src/adding_doubling.hpp:123-174).  No GPU needed: nothing here launches."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from addingdoublingrt_b200 import _abi, _lib, workloads

HEADER = os.path.join(ROOT, "include", "adrt_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(adrt_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    for s in ("adrt_engine_create", "adrt_solve_batch", "adrt_solve_batch_host",
              "adrt_solve_batch_uneven", "adrt_last_status_detail"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(_lib.EXPORTS) <= set(declared_symbols())


def test_struct_layouts_match_header():
    # 11 ints + pad, then 10 doubles
    assert C.sizeof(_abi.BatchDesc) == 11 * 4 + 4 + 10 * 8
    assert C.sizeof(_abi.Inputs) == 11 * 8
    assert C.sizeof(_abi.Outputs) == 8 * 8


def _validate(b):
    lib = _lib.load()
    rc = lib.adrt_validate_batch(C.byref(b.desc), C.byref(b.inputs_struct()))
    return rc, lib.adrt_last_status_detail().decode()


def test_validate_accepts_workloads():
    for b in (workloads.config1(W=10), workloads.config2(W=10), workloads.config3(W=10),
              workloads.config5(W=10)):
        rc, msg = _validate(b)
        assert rc == 0, msg


@pytest.mark.parametrize("mutate,match", [
    (lambda b: b.arrays["delta_tau"].__setitem__(3, -0.1), "delta_tau"),
    (lambda b: b.arrays["single_scat_albedo"].__setitem__(0, 1.5), "single_scat_albedo"),
    (lambda b: setattr(b.desc, "num_layers", 0), "num_layers"),
    (lambda b: setattr(b.desc, "num_quadrature", 1), "num_quadrature"),
    (lambda b: b.set("surface_albedo", np.full(b.W, 1.2)), "surface_albedo"),
    (lambda b: b.set("solar_mu", np.zeros(b.W)), "solar_mu"),
    (lambda b: b.arrays["temperature"].__setitem__(0, -5.0), "temperature"),
    (lambda b: b.set("wavenumber_high", np.zeros(b.W)), "wavenumber"),
])
def test_validate_rejects_like_the_reference(mutate, match):
    b = workloads.config2(W=4)
    mutate(b)
    rc, msg = _validate(b)
    assert rc == _abi.ADRT_ERR_INVALID_ARGUMENT
    assert match in msg


def test_orders_above_32_are_unsupported():
    b = workloads.config2(W=2)
    b.desc.num_quadrature = 33
    rc, msg = _validate(b)
    assert rc == _abi.ADRT_ERR_UNSUPPORTED and "not supported" in msg


def test_validate_requires_thermal_for_surface_temperature():
    b = workloads.config1(W=2)
    b.desc.surface_temperature = 300.0
    rc, msg = _validate(b)
    assert rc == _abi.ADRT_ERR_INVALID_ARGUMENT and "requires use_thermal_emission" in msg
    b = workloads.config1(W=2)
    b.desc.top_temperature = 0.0
    rc, msg = _validate(b)
    assert rc == _abi.ADRT_ERR_INVALID_ARGUMENT and "top_temperature" in msg


def test_validate_diffusion_needs_sources():
    b = workloads.config1(W=2)
    b.desc.use_diffusion_lower_bc = 1
    rc, msg = _validate(b)
    assert rc == _abi.ADRT_ERR_INVALID_ARGUMENT and "diffusion" in msg


def test_version_string():
    assert b"sm_100a" in _lib.load().adrt_version()


def test_device_entry_points_refuse_host_arrays():
    """The device entry points' pointer helper refuses numpy arrays and CPU
    tensors (their addresses are host memory) before anything reaches a kernel."""
    import numpy as np
    import pytest
    import torch
    from addingdoublingrt_b200.engine import _ptr
    assert _ptr(None) is None
    for host in (np.zeros(4), torch.zeros(4, dtype=torch.float64)):
        with pytest.raises(TypeError):
            _ptr(host)


@pytest.mark.gpu
def test_device_methods_check_the_engine_device():
    """The engine reports its device (adrt_engine_device), and the Python device
    methods refuse tensors of another device before launching anything."""
    import torch
    from conftest import cuda_available
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import Engine, alloc_device_outputs, to_device
    eng = Engine()
    try:
        assert eng.device == torch.cuda.current_device()
        b = workloads.config5(W=8, L=4)
        di = to_device(b)
        do = alloc_device_outputs(b, ("toa_flux_up",))
        eng.solve_device(b.desc, di, do)
        torch.cuda.synchronize()
        real = eng.device
        eng.device = real + 1  # as if the tensors belonged to another GPU
        with pytest.raises(ValueError):
            eng.solve_device(b.desc, di, do)
        eng.device = real
        assert eng.read_status() == 0
    finally:
        eng.close()


@pytest.mark.parametrize("make", [workloads.config1, workloads.config2, workloads.config5])
def test_array_counts_match_the_batch_arrays(make):
    """The element counts the Python engine checks device arrays against are
    those of every input and output array of a batch."""
    b = make(W=40)
    n = _abi.array_counts(b.desc)
    for k, v in b.arrays.items():
        assert v.size == n["in"][k], k
    for k, v in b.alloc_outputs().items():
        assert v.size == n["out"][k], k


@pytest.mark.gpu
def test_short_device_arrays_are_refused_before_the_launch():
    import torch
    from conftest import cuda_available
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import Engine, alloc_device_outputs, to_device
    eng = Engine()
    try:
        b = workloads.config5(W=16, L=6)
        di = to_device(b)
        do = alloc_device_outputs(b, ("flux_up", "toa_flux_up"))
        short = dict(do)
        short["flux_up"] = do["flux_up"][:-1].contiguous()
        with pytest.raises(ValueError):
            eng.solve_device(b.desc, di, short)
        bad = dict(di)
        bad["delta_tau"] = di["delta_tau"].reshape(-1)[:-3].contiguous()
        with pytest.raises(ValueError):
            eng.solve_device(b.desc, bad, do)
        eng.solve_device(b.desc, di, do)
        torch.cuda.synchronize()
        assert eng.read_status() == 0
    finally:
        eng.close()


def test_mixed_form_refuses_gradients():
    """The adjoint differentiates the FP64 form, so a mixed-form solve whose
    inputs require gradients is refused before anything runs (no GPU needed)."""
    import torch
    from addingdoublingrt_b200 import torch_api
    cfg = torch_api.BatchConfig()
    cfg.precision = "mixed"
    rng = np.random.default_rng(3)
    tau, ssa, mom, planck = (torch.as_tensor(rng.uniform(0.1, 0.9, size=sh))
                             for sh in ((3, 2), (3, 2), (2, 16), (3, 3)))
    tau.requires_grad_(True)
    with pytest.raises(ValueError, match="fp64"):
        torch_api.solve_batch(cfg, tau, ssa, mom, planck)
