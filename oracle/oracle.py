"""TEST INFRASTRUCTURE: Python access to the two CPU oracles.

* `liboracle.so`  -- the C restatement in adrt_oracle.c (the parity checker).
* `_ref/libadrt_ref.so` -- the reference's own CPU solver (src/solver.cpp and
  friends, compiled unmodified against the project-written Eigen subset);
  used to generate the golden vectors and as the timed CPU baseline.

Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() import
this module.  Nothing in the engine does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

from addingdoublingrt_b200 import _abi
from addingdoublingrt_b200.workloads import Batch

HERE = os.path.dirname(os.path.abspath(__file__))
_lock = threading.Lock()
_libs = {}


def reference_dir() -> str:
    """The reference checkout the recipe builds from: $ADRT_REFERENCE, else the
    conventional read-only checkout location.  May not exist (the GPU machine
    has only the prebuilt _ref/ files)."""
    return os.environ.get("ADRT_REFERENCE", "/root/reference")


def reference_present() -> bool:
    return os.path.isdir(os.path.join(reference_dir(), "src"))


def make(target: str, quiet: bool = True, jobs: int = 1, **kw) -> subprocess.CompletedProcess:
    """`make -C oracle <target> REF=<reference_dir()>`."""
    cmd = ["make", "-s", f"-j{jobs}", "-C", HERE, target, f"REF={reference_dir()}"]
    if quiet:
        kw.setdefault("stdout", subprocess.DEVNULL)
    return subprocess.run(cmd, **kw)


def _make(target: str) -> None:
    make(target, check=True)


def oracle_lib(fma: bool = False) -> C.CDLL:
    """The C restatement, built on first use if absent (gcc only).  `fma=True`
    gives the same code compiled with FMA contraction (sensitivity probe)."""
    key = "oracle_fma" if fma else "oracle"
    name = "liboracle_fma.so" if fma else "liboracle.so"
    with _lock:
        if key not in _libs:
            path = os.path.join(HERE, name)
            if not os.path.exists(path):
                _make(name)
            lib = C.CDLL(path)
            sig = [C.POINTER(_abi.BatchDesc), C.POINTER(_abi.Inputs), C.POINTER(_abi.Outputs)]
            lib.oracle_solve_batch.argtypes = sig + [C.c_int]
            lib.oracle_solve_batch_range.argtypes = sig + [C.c_int, C.c_int, C.c_int]
            lib.oracle_last_error.restype = C.c_char_p
            lib.oracle_planck.restype = C.c_double
            lib.oracle_planck.argtypes = [C.c_double] * 3
            lib.oracle_planck_deriv.restype = C.c_double
            lib.oracle_planck_deriv.argtypes = [C.c_double] * 3
            lib.oracle_gauss_legendre.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
            lib.oracle_num_doublings.argtypes = [C.c_double, C.c_double]
            lib.oracle_ipow0.argtypes = [C.c_double]
            lib.oracle_flops_batch.restype = C.c_double
            lib.oracle_flops_batch.argtypes = [C.POINTER(_abi.BatchDesc),
                                               C.POINTER(_abi.Inputs), C.c_int, C.c_int]
            _libs[key] = lib
        return _libs[key]


def ref_available(strict: bool = False) -> bool:
    name = "libadrt_ref_strict.so" if strict else "libadrt_ref.so"
    return os.path.exists(os.path.join(HERE, "_ref", name))


def ref_lib(strict: bool = False) -> C.CDLL:
    """The reference's own solver (oracle/_ref); raises if it was not built.
    `strict=True`: the build without FMA contraction (golden vectors)."""
    key = "ref_strict" if strict else "ref"
    name = "libadrt_ref_strict.so" if strict else "libadrt_ref.so"
    with _lock:
        if key not in _libs:
            path = os.path.join(HERE, "_ref", name)
            if not os.path.exists(path):
                raise FileNotFoundError(
                    f"{path} missing: build it with `make -C oracle ref REF=<checkout>` where the "
                    "reference sources are present")
            lib = C.CDLL(path)
            sig = [C.POINTER(_abi.BatchDesc), C.POINTER(_abi.Inputs), C.POINTER(_abi.Outputs)]
            lib.ref_solve_batch.argtypes = sig + [C.c_int]
            lib.ref_solve_batch_range.argtypes = sig + [C.c_int, C.c_int, C.c_int]
            lib.ref_last_error.restype = C.c_char_p
            lib.ref_planck.restype = C.c_double
            lib.ref_planck.argtypes = [C.c_double] * 3
            lib.ref_gauss_legendre.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
            lib.ref_solve_column_jacobian.argtypes = [
                C.POINTER(_abi.BatchDesc), C.POINTER(_abi.Inputs), C.c_int,
                C.POINTER(_abi.Outputs)] + [C.c_void_p] * 4
            _libs[key] = lib
        return _libs[key]


class OracleError(RuntimeError):
    pass


def _run(fn, errfn, batch: Batch, nthreads: int, which, w0=None, w1=None) -> dict:
    out = batch.alloc_outputs(which)
    d = batch.desc
    ins = batch.inputs_struct()
    outs = Batch.outputs_struct(out)
    if w0 is None:
        rc = fn(C.byref(d), C.byref(ins), C.byref(outs), int(nthreads))
    else:
        rc = fn(C.byref(d), C.byref(ins), C.byref(outs), int(w0), int(w1), int(nthreads))
    if rc != 0:
        raise OracleError(errfn().decode())
    return out


def solve_oracle(batch: Batch, nthreads: int = 0, which=_abi.OUTPUT_FIELDS,
                 fma: bool = False) -> dict:
    """All outputs of `batch` from the C restatement."""
    lib = oracle_lib(fma)
    return _run(lib.oracle_solve_batch, lib.oracle_last_error, batch,
                nthreads or os.cpu_count() or 1, which)


def solve_reference(batch: Batch, nthreads: int = 0, which=_abi.OUTPUT_FIELDS,
                    strict: bool = False) -> dict:
    """All outputs of `batch` from the reference's own solver (oracle/_ref)."""
    lib = ref_lib(strict)
    return _run(lib.ref_solve_batch, lib.ref_last_error, batch,
                nthreads or os.cpu_count() or 1, which)


def flops(batch: Batch, w0: int = 0, w1: int | None = None) -> float:
    """Algorithmic flops of wavenumbers [w0, w1) (reference branch counting)."""
    lib = oracle_lib()
    ins = batch.inputs_struct()
    return lib.oracle_flops_batch(C.byref(batch.desc), C.byref(ins), int(w0),
                                  int(batch.W if w1 is None else w1))


def rel_error(x: np.ndarray, ref: np.ndarray) -> float:
    """max |x - ref| / max(|ref|, 1e-12 max|ref|) over all elements."""
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = np.max(np.abs(ref)) if ref.size else 0.0
    if scale == 0.0:
        return float(np.max(np.abs(x - ref))) if x.size else 0.0
    den = np.maximum(np.abs(ref), 1e-12 * scale)
    return float(np.max(np.abs(x - ref) / den))


def norm_error(x: np.ndarray, ref: np.ndarray, per: int) -> float:
    """max |x - ref| normalised by each wavenumber's largest |ref| (rows of `per`)."""
    x = np.asarray(x, dtype=np.float64).reshape(-1, per)
    ref = np.asarray(ref, dtype=np.float64).reshape(-1, per)
    scale = np.max(np.abs(ref), axis=1, keepdims=True)
    scale[scale == 0.0] = 1.0
    return float(np.max(np.abs(x - ref) / scale))


def planck_single(temp, nu):
    """Single-wavenumber Planck function of the raw entry point,
    c1 nu^3 / (exp(c2 nu / T) - 1), c1 = 1.19105e-8, c2 = 1.43879, zero below
    1e-5 K (src_cuda/cuda_planck_single.cuh:19-35), in FP64."""
    temp = np.asarray(temp, dtype=np.float64)
    nu = np.asarray(nu, dtype=np.float64)
    with np.errstate(over="ignore", divide="ignore"):
        b = 1.19105e-08 * nu ** 3 / np.expm1(1.43879 * nu / np.where(temp < 1e-5, 1.0, temp))
    return np.where(temp < 1e-5, 0.0, b)


def raw_preprocess(absorption, scattering, altitude, temperature, wavenumber, cloud=None,
                   surface_temperature=-1.0, top_temperature=-1.0) -> dict:
    """FP64 restatement of the reference's raw-coefficient preprocessing
    (src_cuda/cuda_solver.cu:1131-1186, and the inline path :175-249, :428-440):
    coefficient arrays [(L+1), W] with level 0 at the bottom, altitude and
    temperature [L+1] bottom first, cloud optical depth [L, W] bottom first.
    Returns the solver's top-first arrays: delta_tau and single_scat_albedo
    [W, L], planck_levels [W, L+1], surface_emission and top_emission [W]."""
    ab = np.asarray(absorption, dtype=np.float64)
    sc = np.asarray(scattering, dtype=np.float64)
    alt = np.asarray(altitude, dtype=np.float64)
    tmp = np.asarray(temperature, dtype=np.float64)
    nu = np.asarray(wavenumber, dtype=np.float64)
    L = alt.size - 1
    dz = (alt[1:] - alt[:-1])[:, None]                      # [L, 1] bottom first
    ext = ab + sc
    tau = dz * (ext[1:] + ext[:-1]) * 0.5                    # [L, W]
    sdep = dz * (sc[1:] + sc[:-1]) * 0.5
    if cloud is not None:
        tau = tau + np.asarray(cloud, dtype=np.float64)
    tau = np.maximum(tau, 0.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        ssa = np.where(tau > 0.0, sdep / np.where(tau > 0.0, tau, 1.0), 0.0)
    B = planck_single(tmp[::-1][None, :], nu[:, None])      # [W, L+1] top first
    surf = planck_single(surface_temperature, nu) if surface_temperature >= 0.0 else B[:, L]
    top = planck_single(top_temperature, nu) if top_temperature >= 0.0 else B[:, 0]
    return {"delta_tau": tau[::-1].T.copy(), "single_scat_albedo": ssa[::-1].T.copy(),
            "planck_levels": B, "surface_emission": np.asarray(surf, dtype=np.float64),
            "top_emission": np.asarray(top, dtype=np.float64)}
