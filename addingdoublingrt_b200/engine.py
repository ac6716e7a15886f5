"""Python handle on the native engine.

`Engine` owns one adrt_engine (device work buffers) and solves batches held
either in host numpy arrays (`solve_host`, the adrt_solve_batch_host entry)
or in CUDA tensors (`solve_device`, the stream-ordered adrt_solve_batch
entry).  PyTorch is used only to hold device memory and streams.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi, _lib
from .workloads import Batch


class Engine:
    def __init__(self, device: int = -1, max_workspace_bytes: int = 0):
        self.lib = _lib.load()
        opts = _abi.EngineOpts(device=device, max_workspace_bytes=max_workspace_bytes)
        h = C.c_void_p()
        _lib.check(self.lib.adrt_engine_create(C.byref(opts), C.byref(h)))
        self.handle = h
        d = C.c_int()
        _lib.check(self.lib.adrt_engine_device(h, C.byref(d)))
        self.device = int(d.value)  # the CUDA ordinal the engine's kernels run on

    @staticmethod
    def _sizes(desc, groups):
        """Refuse arrays shorter than the batch needs (the kernels would read or
        write past their ends): groups = [(kind, {name: tensor}), ...]."""
        n = _abi.array_counts(desc)
        for kind, arrays in groups:
            for name, t in (arrays or {}).items():
                if t is not None and name in n[kind] and t.numel() < n[kind][name]:
                    raise ValueError(f"{name}: {t.numel()} elements, the batch needs "
                                     f"{n[kind][name]}")

    def _dev(self, t):
        """_ptr of a tensor that must live on the engine's device (another
        GPU's address would be dereferenced as a peer address)."""
        if t is not None and getattr(t, "is_cuda", False) and t.device.index != self.device:
            raise ValueError(f"tensor on cuda:{t.device.index}, engine on cuda:{self.device}")
        return _ptr(t)

    def close(self) -> None:
        if self.handle:
            self.lib.adrt_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, desc: _abi.BatchDesc) -> None:
        _lib.check(self.lib.adrt_engine_reserve(self.handle, C.byref(desc)))

    def workspace_bytes(self) -> int:
        v = C.c_size_t()
        _lib.check(self.lib.adrt_engine_workspace_bytes(self.handle, C.byref(v)))
        return int(v.value)

    def set_adjoint_mode(self, mode: int) -> None:
        """adrt_engine_set_adjoint_mode: _abi.ADJOINT_RECORD (default) or
        _abi.ADJOINT_RECOMPUTE (every doubling chain recomputed in the backward pass)."""
        _lib.check(self.lib.adrt_engine_set_adjoint_mode(self.handle, int(mode)))

    def set_pivoting(self, mode: int) -> None:
        """adrt_engine_set_pivoting: _abi.PIVOTING_TENSOR_CORE (default: pivot-free
        tensor-core solves with a pivoted re-solve on weak pivots) or
        _abi.PIVOTING_PARTIAL (every solve with the reference's partial pivoting)."""
        _lib.check(self.lib.adrt_engine_set_pivoting(self.handle, int(mode)))

    def read_status(self) -> int:
        v = C.c_int()
        _lib.check(self.lib.adrt_engine_read_status(self.handle, C.byref(v)))
        return int(v.value)

    # ------------------------------------------------------------------ host entry
    def solve_host(self, batch: Batch, which=_abi.OUTPUT_FIELDS, out: dict | None = None) -> dict:
        """adrt_solve_batch_host: host arrays in, host arrays out (synchronous)."""
        out = batch.alloc_outputs(which) if out is None else out
        ins = batch.inputs_struct()
        outs = Batch.outputs_struct(out)
        _lib.check(self.lib.adrt_solve_batch_host(self.handle, C.byref(batch.desc),
                                                  C.byref(ins), C.byref(outs)))
        return out

    # ------------------------------------------------------------------ device entry
    def solve_device(self, desc: _abi.BatchDesc, dev_inputs: dict, dev_outputs: dict,
                     stream=None) -> None:
        """adrt_solve_batch on CUDA tensors (float64, contiguous); stream ordered."""
        self._sizes(desc, [("in", dev_inputs), ("out", dev_outputs)])
        ins = _abi.Inputs()
        for f in _abi.INPUT_FIELDS:
            t = dev_inputs.get(f)
            setattr(ins, f, self._dev(t))
        outs = _abi.Outputs()
        for f in _abi.OUTPUT_FIELDS:
            setattr(outs, f, self._dev(dev_outputs.get(f)))
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        _lib.check(self.lib.adrt_solve_batch(self.handle, C.byref(desc), C.byref(ins),
                                             C.byref(outs), s))

    def adjoint(self, desc: _abi.BatchDesc, dev_inputs: dict, cotangents: dict, gradients: dict,
                dev_outputs: dict | None = None, stream=None) -> None:
        """adrt_adjoint on CUDA tensors: gradients of sum(cotangent * output) with respect to
        the inputs named in `gradients` (delta_tau and single_scat_albedo are overwritten,
        phase_moments / temperature / planck_levels are added to)."""
        self._sizes(desc, [("in", dev_inputs), ("cot", cotangents), ("grad", gradients),
                           ("out", dev_outputs)])
        ins = _abi.Inputs()
        for f in _abi.INPUT_FIELDS:
            setattr(ins, f, self._dev(dev_inputs.get(f)))
        cot = _abi.Cotangents()
        for f in _abi.COTANGENT_FIELDS:
            setattr(cot, f, self._dev(cotangents.get(f)))
        gr = _abi.Gradients()
        for f in _abi.GRADIENT_FIELDS:
            setattr(gr, f, self._dev(gradients.get(f)))
        outp = None
        if dev_outputs is not None:
            outs = _abi.Outputs()
            for f in _abi.OUTPUT_FIELDS:
                setattr(outs, f, self._dev(dev_outputs.get(f)))
            outp = C.byref(outs)
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        _lib.check(self.lib.adrt_adjoint(self.handle, C.byref(desc), C.byref(ins), outp,
                                         C.byref(cot), C.byref(gr), s))

    def band_integrate(self, spectrum, offsets, weight=None, out=None, stream=None):
        """adrt_band_integrate on CUDA tensors: out[b] = sum of weight * spectrum over
        wavenumbers offsets[b] .. offsets[b + 1] - 1 (float64 spectrum / weight, int64
        offsets of nchannels + 1 entries); returns out (float64, nchannels)."""
        import torch
        if offsets.dtype != torch.int64 or not offsets.is_contiguous() or not offsets.is_cuda:
            raise TypeError("offsets must be a contiguous int64 CUDA tensor")
        if offsets.device.index != self.device:
            raise ValueError(f"offsets on cuda:{offsets.device.index}, engine on cuda:{self.device}")
        nch = int(offsets.numel()) - 1
        if weight is not None and weight.numel() != spectrum.numel():
            raise ValueError("weight must have one entry per wavenumber of the spectrum")
        if out is None:
            out = torch.empty(max(nch, 0), dtype=torch.float64, device=spectrum.device)
        elif out.numel() < nch:
            raise ValueError(f"out holds {out.numel()} values for {nch} channels")
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        _lib.check(self.lib.adrt_band_integrate(self.handle, self._dev(spectrum), self._dev(weight),
                                                int(spectrum.numel()), offsets.data_ptr(), nch,
                                                self._dev(out), s))
        return out

    def _columns(self, columns: list):
        arr = (_abi.ColumnDesc * len(columns))()
        for i, (desc, di, do) in enumerate(columns):
            self._sizes(desc, [("in", di), ("out", do)])
            arr[i].desc = desc
            for f in _abi.INPUT_FIELDS:
                setattr(arr[i].inp, f, self._dev(di.get(f)))
            for f in _abi.OUTPUT_FIELDS:
                setattr(arr[i].out, f, self._dev(do.get(f)))
        return arr

    def autotune_uneven(self, columns: list, stream=None) -> _abi.UnevenPlan:
        """adrt_engine_autotune_uneven: time both mappings per order on samples of
        `columns` and keep the faster (the engine's plan from then on)."""
        arr = self._columns(columns)
        plan = _abi.UnevenPlan()
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        _lib.check(self.lib.adrt_engine_autotune_uneven(self.handle, arr, len(columns), s,
                                                        C.byref(plan)))
        return plan

    def uneven_plan(self) -> _abi.UnevenPlan:
        plan = _abi.UnevenPlan()
        _lib.check(self.lib.adrt_engine_get_uneven_plan(self.handle, C.byref(plan)))
        return plan

    def set_uneven_plan(self, plan: _abi.UnevenPlan) -> None:
        _lib.check(self.lib.adrt_engine_set_uneven_plan(self.handle, C.byref(plan)))

    def solve_uneven(self, columns: list, stream=None) -> None:
        """adrt_solve_batch_uneven: columns = [(desc, dev_inputs, dev_outputs), ...]."""
        arr = self._columns(columns)
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        _lib.check(self.lib.adrt_solve_batch_uneven(self.handle, arr, len(columns), s))


def _ptr(t):
    """Device address of a float64 CUDA tensor for the device entry points (a
    host array here would hand the kernels a host address)."""
    if t is None:
        return None
    if isinstance(t, np.ndarray) or not getattr(t, "is_cuda", False):
        raise TypeError("device entry points take CUDA tensors; host arrays go through "
                        "the host entry (solve_host)")
    if not t.is_contiguous():
        raise ValueError("device arrays must be contiguous")
    import torch
    if t.dtype != torch.float64:
        raise TypeError("device arrays must be float64")
    return t.data_ptr()


def to_device(batch: Batch, device="cuda") -> dict:
    import torch
    return {k: torch.from_numpy(v).to(device) for k, v in batch.arrays.items()}


def alloc_device_outputs(batch: Batch, which=_abi.OUTPUT_FIELDS, device="cuda") -> dict:
    import torch
    nint = batch.L + 1
    out = {}
    for f in which:
        n = batch.W * nint if f in _abi.INTERFACE_OUTPUTS else batch.W
        out[f] = torch.zeros(n, dtype=torch.float64, device=device)
    return out
