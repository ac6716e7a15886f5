"""Build the native engine in-tree: addingdoublingrt_b200/libadrt_b200.so.

    python -m addingdoublingrt_b200.build [--verbose]

nvcc cross-compiles for sm_100a only (no GPU needed at build time).  No
fast-math: the parity bar against the FP64 oracle depends on IEEE division,
square root and exp/log.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libadrt_b200.so")
HOST_LIB = os.path.join(PKG, "libadrt_host.so")
HOST_SOURCES = ["adrt_host.cpp"]
# The plain FP64 GPU form: the same engine with every product, right-solve and
# phase build on the CUDA cores (DFMA, the pivoted scalar Gauss-Jordan) and no
# tensor-core instruction -- the denominator of the mixed form's speed-up.
CUDA_CORE_LIB = os.path.join(PKG, "libadrt_b200_cudacore.so")
CUDA_CORE_FLAGS = ["-DADRT_GEMM_MMA=0", "-DADRT_GJ_MMA=0", "-DADRT_PHASE_MMA=0"]

SOURCES = ["adrt_engine.cu", "adrt_probe.cu", "adrt_noalloc.cu"]
HEADERS = ["adrt_types.cuh", "adrt_solver.cuh", "adrt_kernel.cuh", "adrt_adjoint.cuh",
           "adrt_tpw.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(HOST_LIB):
        return True
    t = min(os.path.getmtime(LIB), os.path.getmtime(HOST_LIB))
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + HOST_SOURCES]
    deps.append(os.path.join(ROOT, "include", "adrt_b200.h"))
    deps += [os.path.join(ROOT, "include", "adrt", f)
             for f in ("adding_doubling.hpp", "cuda_solver.hpp", "constants.hpp")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_host() -> str:
    """The reference-compatible C++ API (adrt::solve, adrt::cuda::solveBatch)
    over the C ABI: plain g++, linked against libadrt_b200.so."""
    cuda_inc = os.path.join(os.path.dirname(os.path.dirname(nvcc())), "include")
    tmp = HOST_LIB + ".tmp"
    subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall",
                    "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                    *[os.path.join(CSRC, f) for f in HOST_SOURCES],
                    "-L", PKG, "-ladrt_b200", "-Wl,-rpath,$ORIGIN", "-o", tmp], check=True)
    os.replace(tmp, HOST_LIB)
    return HOST_LIB


def build(verbose: bool = False, force: bool = False, extra=(), out: str | None = None) -> str:
    """Compile and link the engine.  `extra` adds nvcc flags (e.g. -D
    tuning macros) and `out` redirects the library (variant builds)."""
    target = out or LIB
    if not force and out is None and not _stale():
        return LIB
    objs = []
    tag = "" if out is None else "_" + os.path.basename(out).replace(".so", "")
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", tag + ".o"))
        cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = target + ".tmp"
    subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp,
                    *objs, "-lcudart"], check=True)
    os.replace(tmp, target)
    if out is None:
        build_host()
    return target


def build_all(verbose: bool = False) -> None:
    """The engine (and its C++ drop-in library) and the CUDA-core FP64 form,
    compiled in parallel."""
    import concurrent.futures as cf
    with cf.ThreadPoolExecutor(2) as ex:
        jobs = [ex.submit(build, verbose, True),
                ex.submit(build, verbose, True, CUDA_CORE_FLAGS, CUDA_CORE_LIB)]
        for j in jobs:
            j.result()


if __name__ == "__main__":
    build_all(verbose="--verbose" in sys.argv)
    print(LIB)
    print(CUDA_CORE_LIB)
