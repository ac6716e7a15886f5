"""Loader for the in-tree native library libadrt_b200.so (the C ABI of
include/adrt_b200.h).  There is no fallback: if the library is missing or
does not load, every solve raises."""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import _abi

_PKG = os.path.dirname(os.path.abspath(__file__))
# ADRT_LIBRARY may point at another build of the same library (tuning variants).
LIB_PATH = os.environ.get("ADRT_LIBRARY") or os.path.join(_PKG, "libadrt_b200.so")

_lock = threading.Lock()
_lib = None

EXPORTS = (
    "adrt_engine_create",
    "adrt_engine_destroy",
    "adrt_engine_reserve",
    "adrt_engine_workspace_bytes",
    "adrt_engine_read_status",
    "adrt_solve_batch",
    "adrt_solve_batch_host",
    "adrt_validate_batch",
    "adrt_solve_batch_uneven",
    "adrt_last_status_detail",
    "adrt_version",
    "adrt_probe_fma_tflops",
    "adrt_probe_mma_tflops",
    "adrt_solve_batch_f32",
    "adrt_gauss_legendre",
    "adrt_planck_band",
    "adrt_solve_batch_noalloc",
    "adrt_noalloc_read_status",
    "adrt_adjoint",
    "adrt_solve_batch_raw",
    "adrt_adjoint_host",
    "adrt_planck_band_deriv",
    "adrt_band_integrate",
    "adrt_engine_set_adjoint_mode",
    "adrt_engine_set_pivoting",
    "adrt_engine_device",
    "adrt_engine_autotune_uneven",
    "adrt_engine_set_uneven_plan",
    "adrt_engine_get_uneven_plan",
)


class NativeLibraryMissing(RuntimeError):
    pass


def load(build_if_missing: bool = False) -> C.CDLL:
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            if not build_if_missing:
                raise NativeLibraryMissing(
                    f"{LIB_PATH} not found; build it with `python -m addingdoublingrt_b200.build`")
            from . import build as _build
            _build.build()
        lib = C.CDLL(LIB_PATH)
        P = C.POINTER
        lib.adrt_engine_create.argtypes = [P(_abi.EngineOpts), P(C.c_void_p)]
        lib.adrt_engine_destroy.argtypes = [C.c_void_p]
        lib.adrt_engine_reserve.argtypes = [C.c_void_p, P(_abi.BatchDesc)]
        lib.adrt_engine_workspace_bytes.argtypes = [C.c_void_p, P(C.c_size_t)]
        lib.adrt_engine_read_status.argtypes = [C.c_void_p, P(C.c_int)]
        lib.adrt_solve_batch.argtypes = [C.c_void_p, P(_abi.BatchDesc), P(_abi.Inputs),
                                         P(_abi.Outputs), C.c_void_p]
        lib.adrt_solve_batch_host.argtypes = [C.c_void_p, P(_abi.BatchDesc), P(_abi.Inputs),
                                              P(_abi.Outputs)]
        lib.adrt_validate_batch.argtypes = [P(_abi.BatchDesc), P(_abi.Inputs)]
        lib.adrt_solve_batch_uneven.argtypes = [C.c_void_p, P(_abi.ColumnDesc), C.c_int,
                                                C.c_void_p]
        lib.adrt_last_status_detail.restype = C.c_char_p
        lib.adrt_version.restype = C.c_char_p
        lib.adrt_probe_fma_tflops.argtypes = [P(C.c_double), P(C.c_double)]
        lib.adrt_probe_mma_tflops.argtypes = [P(C.c_double), P(C.c_double), P(C.c_double)]
        lib.adrt_gauss_legendre.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        lib.adrt_planck_band.argtypes = [C.c_double, C.c_double, C.c_double, P(C.c_double)]
        lib.adrt_planck_band_deriv.argtypes = [C.c_double, C.c_double, C.c_double,
                                               P(C.c_double)]
        lib.adrt_solve_batch_f32.argtypes = [C.c_void_p, P(_abi.BatchDesc), C.c_void_p,
                                             C.c_void_p, C.c_void_p]
        lib.adrt_solve_batch_noalloc.argtypes = [P(_abi.BatchDesc), P(_abi.Inputs),
                                                 P(_abi.Outputs), C.c_void_p]
        lib.adrt_noalloc_read_status.argtypes = [C.c_void_p, P(C.c_int)]
        lib.adrt_adjoint_host.argtypes = [C.c_void_p, P(_abi.BatchDesc), P(_abi.Inputs),
                                          P(_abi.Cotangents), P(_abi.Gradients)]
        lib.adrt_solve_batch_raw.argtypes = [C.c_void_p, P(_abi.BatchDesc),
                                             P(_abi.RawInputs), P(_abi.OutputsF32), C.c_void_p]
        lib.adrt_engine_set_adjoint_mode.argtypes = [C.c_void_p, C.c_int]
        lib.adrt_engine_set_pivoting.argtypes = [C.c_void_p, C.c_int]
        lib.adrt_engine_device.argtypes = [C.c_void_p, P(C.c_int)]
        lib.adrt_engine_autotune_uneven.argtypes = [C.c_void_p, P(_abi.ColumnDesc), C.c_int,
                                                    C.c_void_p, P(_abi.UnevenPlan)]
        lib.adrt_engine_set_uneven_plan.argtypes = [C.c_void_p, P(_abi.UnevenPlan)]
        lib.adrt_engine_get_uneven_plan.argtypes = [C.c_void_p, P(_abi.UnevenPlan)]
        lib.adrt_band_integrate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_longlong,
                                            C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        lib.adrt_adjoint.argtypes = [C.c_void_p, P(_abi.BatchDesc), P(_abi.Inputs),
                                     C.c_void_p, P(_abi.Cotangents), P(_abi.Gradients),
                                     C.c_void_p]
        _lib = lib
        return lib


class ADRTError(RuntimeError):
    def __init__(self, code: int, detail: str):
        super().__init__(f"adrt error {code}: {detail}")
        self.code = code
        self.detail = detail


class InvalidArgument(ADRTError, ValueError):
    """Mirrors the reference's std::invalid_argument from ADConfig::validate()."""


def check(rc: int) -> None:
    if rc == _abi.ADRT_OK:
        return
    detail = load().adrt_last_status_detail().decode()
    if rc == _abi.ADRT_ERR_INVALID_ARGUMENT:
        raise InvalidArgument(rc, detail)
    raise ADRTError(rc, detail)
