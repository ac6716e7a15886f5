"""Benchmark: wavenumber-solves/s of the batched adding-doubling solve.

Workload: 100,000 wavenumbers x 100 layers, N=16, thermal + solar, per-
wavenumber double Henyey-Greenstein moments (32), band-integrated Planck
levels over 500-3000 cm^-1 (seeded synthetic inputs, `workloads.config2`).

    python bench.py [--gpus N --steps K --warmup W] [--precision fp64|mixed]
    python bench.py --impl reference      # the reference's CPU solver on the host cores

One step = one solve of the whole batch with inputs resident in HBM (inputs
of 190 MB exceed the 126 MB L2, so no flush is needed between steps).  `e2e`
times the host entry point adrt_solve_batch_host (pinned host arrays in,
host arrays out, host<->device copies inside the timed region).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from addingdoublingrt_b200 import _abi, workloads  # noqa: E402

METRIC = "wavenumber-solves/s N=16 L=100: FP64 vs mixed @1e-6 rel err; adjoint/fwd time"
WORKLOAD = "config2: W=100000 wavenumbers x L=100 layers, N=16, M=32 per-wavenumber dHG moments, thermal+solar"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"])
    p.add_argument("--wavenumbers", type=int, default=100_000)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-check", action="store_true")
    p.add_argument("--only", default=None, choices=["fp64", "mixed"],
                   help="time one precision form only (profiling runs)")
    p.add_argument("--adjoint-wavenumbers", type=int, default=10_000,
                   help="wavenumbers of the config-5 adjoint timing")
    p.add_argument("--workload", default="config2",
                   choices=["config2", "config4", "adjoint", "band", "table"],
                   help="config2: the headline line; config4: uneven batch; adjoint: config 5; "
                        "band: band integration of a spectrum (--wavenumbers x 1000)")
    p.add_argument("--no-adjoint", action="store_true",
                   help="skip the adjoint/forward timing of the headline line")
    p.add_argument("--no-e2e", action="store_true", help="skip the host-entry (e2e) timing")
    p.add_argument("--no-config4", action="store_true",
                   help="skip the full config-4 uneven batch of the headline line")
    p.add_argument("--config4-fraction", type=float, default=1.0,
                   help="config 4 with the first ceil(f W) wavenumbers of every column "
                        "(profiling runs; the measured workload is f = 1)")
    p.add_argument("--no-cuda-core", action="store_true",
                   help="skip the CUDA-core FP64 form (the mixed form's denominator)")
    p.add_argument("--no-reference-gpu", action="store_true",
                   help="reference arm: skip the reference's own GPU solver "
                        "(oracle/_ref/libadrt_ref_gpu.so)")
    return p.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU baseline
def cpu_baseline(batch, seconds=12.0, threads=None):
    """The reference's own CPU solver (oracle/_ref, compiled from the reference
    sources) on the host cores, on a bounded sample of the same workload."""
    from oracle import oracle
    threads = threads or os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    rng = np.random.default_rng(0)
    n = max(threads * 2, 64)
    rate = None
    while True:
        idx = np.sort(rng.choice(batch.W, size=min(n, batch.W), replace=False))
        sub = batch.subset(idx)
        t0 = time.perf_counter()
        if kind == "reference":
            oracle.solve_reference(sub, threads)
        else:
            oracle.solve_oracle(sub, threads)
        dt = time.perf_counter() - t0
        rate = sub.W / dt
        if dt >= seconds or n >= batch.W:
            break
        n = int(min(batch.W, max(n * 2, rate * seconds * 1.1)))
    return {"value": rate, "unit": "wavenumber-solves/s", "cores": threads, "kind": kind,
            "sample": f"{sub.W} random wavenumbers of the same workload ({dt:.1f} s on "
                      f"{threads} threads)"}


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle
    batch = workloads.config2(W=args.wavenumbers)
    threads = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    rng = np.random.default_rng(1)
    sample = max(4 * threads, 256)
    solve = (lambda b: oracle.solve_reference(b, threads)) if kind == "reference" else \
        (lambda b: oracle.solve_oracle(b, threads))
    subs = [batch.subset(np.sort(rng.choice(batch.W, sample, replace=False)))
            for _ in range(args.warmup + args.steps)]
    for i in range(args.warmup):
        solve(subs[i])
    t0 = time.perf_counter()
    for i in range(args.steps):
        solve(subs[args.warmup + i])
    dt = time.perf_counter() - t0
    rate = sample * args.steps / dt
    line = {
        "metric": METRIC, "value": rate, "unit": "wavenumber-solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD, "sample_per_step": sample},
        "cpu_baseline": {"value": rate, "unit": "wavenumber-solves/s", "cores": threads,
                         "kind": kind,
                         "sample": f"{sample} random wavenumbers per step, {threads} threads"},
        "e2e": {"value": rate, "unit": "wavenumber-solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_gpu and args.gpus == 1:
        try:
            line["reference_gpu"] = reference_gpu(workloads.config2_scalar(W=args.wavenumbers))
            c1 = reference_gpu(workloads.config1(), steps=10, warmup=2)
            c1["workload"] = "config1 (W=1000 x 20 layers, N=8: the reference's solveKernel<8>)"
            line["reference_gpu_config1"] = c1
        except Exception as ex:  # the CPU line stands on its own
            line["reference_gpu"] = {"unavailable": str(ex)[:200]}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- adjoint and uneven
def time_adjoint(eng, W=10_000, reps=3, mode=_abi.ADJOINT_RECORD):
    """Forward and adjoint times of config 5 (10 000 x 60, N=16, thermal + solar,
    per-layer HG moments): gradients of TOA F_up and BOA F_down with respect to
    delta_tau, omega, the moments and the 61 level temperatures.  Returns
    (forward ms, adjoint ms) on the device, median of `reps`; `mode` is the
    engine's adjoint mode (doubling chains recorded, or recomputed in the
    backward pass)."""
    import torch
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    eng.set_adjoint_mode(mode)
    b = workloads.config5(W=W)
    di = to_device(b)
    do = alloc_device_outputs(b, _abi.INTERFACE_OUTPUTS)
    n = b.W * (b.L + 1)
    cot = {"flux_up": torch.zeros(n, dtype=torch.float64, device="cuda"),
           "flux_down": torch.zeros(n, dtype=torch.float64, device="cuda")}
    cot["flux_up"].view(b.W, -1)[:, 0] = 1.0
    cot["flux_down"].view(b.W, -1)[:, b.L] = 1.0
    gr = {k: torch.zeros_like(di[k])
          for k in ("delta_tau", "single_scat_albedo", "phase_moments", "temperature")}
    eng.solve_device(b.desc, di, do)
    eng.adjoint(b.desc, di, cot, gr)
    torch.cuda.synchronize()
    fw, ad = [], []
    for _ in range(reps):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        eng.solve_device(b.desc, di, do)
        e1.record()
        eng.adjoint(b.desc, di, cot, gr)
        e2.record()
        torch.cuda.synchronize()
        fw.append(e0.elapsed_time(e1))
        ad.append(e1.elapsed_time(e2))
    eng.set_adjoint_mode(_abi.ADJOINT_RECORD)
    return statistics.median(fw), statistics.median(ad)


def _time_uneven(eng, cols, reps=1, warmup=1):
    import torch
    for _ in range(warmup):
        eng.solve_uneven(cols)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        eng.solve_uneven(cols)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _prefix(cols, fraction):
    """Every column's first ceil(fraction W) wavenumbers (views of the same tensors)."""
    out = []
    for d, ins, outs in cols:
        W, L, M = d.num_wavenumbers, d.num_layers, d.num_moments
        w = max(1, int(np.ceil(fraction * W)))
        dd = _abi.BatchDesc.from_buffer_copy(d)
        dd.num_wavenumbers = w
        per = {"delta_tau": L, "single_scat_albedo": L, "phase_moments": M}
        ii = {k: (v if k == "temperature" else v[:w * per.get(k, 1)]) for k, v in ins.items()}
        oo = {k: v[:w * (L + 1)] for k, v in outs.items()}
        out.append((dd, ii, oo))
    return out


def run_config4(args, eng, line=True):
    """Config 4 in full: 4096 columns, L ~ U{20..150}, N in {4, 8, 16}, W log-uniform
    256..8192 (9.37e6 wavenumber-columns, generated on the device), solar /
    thermal / both.  The uneven plan is autotuned on the FP64 batch (mapping per
    order, warp-launch grid), the whole batch is solved in FP64 under it, and on
    a 5 % prefix of every column the autotuned plan is compared with the fixed
    thread-per-wavenumber mapping (the reference's solveKernel mapping) and with
    the warp mapping alone; the mixed form runs on the same prefix.  One
    wavenumber per column is checked against the oracle."""
    import torch
    from oracle import oracle
    t0 = time.perf_counter()
    cols = workloads.config4_device(ncols=4096, seed=4, precision=_abi.PRECISION_FP64,
                                    fraction=args.config4_fraction)
    gen_s = time.perf_counter() - t0
    total = sum(d.num_wavenumbers for d, _, _ in cols)
    saved = _abi.UnevenPlan.from_buffer_copy(eng.uneven_plan())
    t0 = time.perf_counter()
    plan = eng.autotune_uneven(cols)
    tune_s = time.perf_counter() - t0
    full_ms = _time_uneven(eng, cols, reps=1, warmup=1)
    status = eng.read_status()
    # one wavenumber per column against the oracle (FP64, autotuned plan)
    import concurrent.futures as cf
    checks = []
    for d, ins, outs in cols:
        w = d.num_wavenumbers // 2
        L = d.num_layers
        got = {k: outs[k][w * (L + 1):(w + 1) * (L + 1)].cpu().numpy()
               for k in ("flux_up", "flux_down", "mean_intensity")}
        checks.append((workloads.column_to_host(d, ins, w), got))

    def check(item):
        b, got = item
        ref = oracle.solve_oracle(b, 1, which=_abi.INTERFACE_OUTPUTS)
        sens = oracle.solve_oracle(b, 1, which=_abi.INTERFACE_OUTPUTS, fma=True)
        return (max(oracle.norm_error(got[k], ref[k], b.L + 1) for k in got),
                max(oracle.norm_error(sens[k], ref[k], b.L + 1) for k in got))

    with cf.ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        checked = list(ex.map(check, checks))
    err = max(e for e, _ in checked)
    sens_max = max(s_ for _, s_ in checked)
    # beyond the FP64 parity tests' tolerance (1e-9 + 1000 x the FMA sensitivity)
    beyond = sum(1 for e, s_ in checked if e > 1e-9 + 1000.0 * s_)
    sub = _prefix(cols, 0.05)
    nsub = sum(d.num_wavenumbers for d, _, _ in sub)
    tuned_ms = _time_uneven(eng, sub)
    fixed = _abi.UnevenPlan.from_buffer_copy(plan)
    for i in range(3):
        fixed.mapping[i] = _abi.MAPPING_THREAD
    fixed.warp_blocks_per_sm = 0
    eng.set_uneven_plan(fixed)
    thread_ms = _time_uneven(eng, sub)
    warp = _abi.UnevenPlan.from_buffer_copy(plan)
    for i in range(3):
        warp.mapping[i] = _abi.MAPPING_WARP
    warp.warp_blocks_per_sm = 0
    eng.set_uneven_plan(warp)
    warp_ms = _time_uneven(eng, sub)
    eng.set_uneven_plan(plan)
    for d, _, _ in sub:
        d.precision = _abi.PRECISION_MIXED
    mixed_ms = _time_uneven(eng, sub)
    eng.set_uneven_plan(saved)
    res = {
        "metric": "wavenumber-solves/s, uneven batch (config 4)", "value": total / (full_ms * 1e-3),
        "unit": "wavenumber-solves/s", "ms_per_step": full_ms, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic (generated on the device)",
        "config": {"workload": f"config4: 4096 columns, {total} wavenumber-columns, N in "
                               "{4,8,16}, L 20..150, FP64, autotuned plan"},
        "plan": plan.as_dict(), "autotune_s": tune_s, "generate_s": gen_s,
        "prefix_5pct": {"wavenumbers": nsub,
                        "autotuned_solves_per_s": nsub / (tuned_ms * 1e-3),
                        "thread_per_wavenumber_solves_per_s": nsub / (thread_ms * 1e-3),
                        "warp_per_wavenumber_solves_per_s": nsub / (warp_ms * 1e-3),
                        "autotuned_over_thread_per_wavenumber": thread_ms / tuned_ms,
                        "mixed_solves_per_s": nsub / (mixed_ms * 1e-3)},
        "oracle_check_one_wavenumber_per_column": {
            "max_normalized_error": err, "max_fp64_fma_sensitivity": sens_max,
            "beyond_1e-9_plus_1000x_sensitivity": beyond, "checked": len(checked)},
        "status": status}
    if line:
        print(json.dumps(res), flush=True)
    return res


def run_table(args, eng):
    """One line per configuration (1, 2, 3, 5) with the figures of the results
    table: FP64 and mixed solves/s of the whole batch (device arrays, CUDA
    events), their normalised error against the FP64 oracle on a sample (per
    output), the FP64 form's roofline fraction, and the reference's own CPU
    solver (oracle/_ref, else the C restatement) on one core and on all host
    cores, each a bounded sample."""
    import torch
    from oracle import oracle
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    from addingdoublingrt_b200 import _lib
    peaks = measured_peaks(_lib.load())
    kind = "reference" if oracle.ref_available() else "port"
    cpu_solve = (lambda b, n: oracle.solve_reference(b, n)) if kind == "reference" else \
        (lambda b, n: oracle.solve_oracle(b, n))
    cases = [("config1", lambda p: workloads.config1(), 1000),
             ("config2", lambda p: workloads.config2(precision=p), 2000),
             ("config3", lambda p: workloads.config3(precision=p), 500),
             ("config5", lambda p: workloads.config5(precision=p), 1000)]
    for name, make, nsample in cases:
        row = {"metric": f"table row: {name}", "unit": "wavenumber-solves/s"}
        outs = {}
        for pname, prec in (("fp64", _abi.PRECISION_FP64), ("mixed", _abi.PRECISION_MIXED)):
            b = make(prec)
            b.desc.precision = prec
            di = to_device(b)
            do = alloc_device_outputs(b, _abi.INTERFACE_OUTPUTS)
            eng.reserve(b.desc)
            for _ in range(2):
                eng.solve_device(b.desc, di, do)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(3):
                eng.solve_device(b.desc, di, do)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 3
            row[f"{pname}_solves_per_s"] = b.W / (ms * 1e-3)
            row[f"{pname}_ms"] = ms
            outs[pname] = (b, do)
            if pname == "fp64":
                fl = oracle.flops(b)
                row["fp64_roofline_frac"] = fl / (ms * 1e-3) / 1e12 / peaks["fp64_tflops"]
                row["W"], row["L"], row["N"] = b.W, b.L, b.N
        b = outs["fp64"][0]
        idx = np.linspace(0, b.W - 1, min(b.W, nsample)).astype(np.int64)
        sub = b.subset(idx)
        ref = oracle.solve_oracle(sub, os.cpu_count() or 1, which=_abi.INTERFACE_OUTPUTS)
        t = torch.as_tensor(idx, device="cuda")
        for pname, (bb, do) in outs.items():
            row[f"{pname}_normalized_error"] = {
                k: oracle.norm_error(do[k].view(-1, b.L + 1)[t].cpu().numpy().ravel(), ref[k],
                                     b.L + 1)
                for k in ("flux_up", "flux_down", "flux_direct", "mean_intensity")}
        # the reference's CPU solver: one core, and every host core
        for cores in (1, os.cpu_count() or 1):
            n = 8 * cores
            while True:
                sb = b.subset(np.arange(min(n, b.W)))
                t0 = time.perf_counter()
                cpu_solve(sb, cores)
                dt = time.perf_counter() - t0
                if dt > 3.0 or n >= b.W:
                    break
                n = int(min(b.W, n * max(2.0, 4.0 / max(dt, 1e-3))))
            row[f"cpu_{cores}_cores_solves_per_s"] = sb.W / dt
        row["cpu_kind"] = kind
        print(json.dumps(row), flush=True)


def run_band(args, eng):
    """Band integration of a spectrum into channels (adrt_band_integrate):
    --wavenumbers x 1000 wavenumbers of float64 spectrum and weights (inputs
    resident in HBM, larger than L2) into channels of 1000 wavenumbers.  HBM-
    bound: 16 bytes per wavenumber read."""
    import torch
    W = args.wavenumbers * 1000
    per = 1000
    g = torch.Generator(device="cuda").manual_seed(11)
    spec = torch.rand(W, dtype=torch.float64, device="cuda", generator=g)
    wgt = torch.rand(W, dtype=torch.float64, device="cuda", generator=g)
    off = torch.arange(0, W + 1, per, dtype=torch.int64, device="cuda")
    out = torch.empty(off.numel() - 1, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        eng.band_integrate(spec, off, wgt, out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        eng.band_integrate(spec, off, wgt, out)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    gbs = 16.0 * W / (ms * 1e-3) / 1e9
    peak, src = None, "measured (MEASURED_PEAKS.json)"
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    if not peak:  # the pool's earlier copy-bandwidth measurement
        peak, src = 6650.0, "fallback 6.65 TB/s copy bandwidth"
    ref = float((spec * wgt).sum())
    line = {"metric": "band integration GB/s", "value": gbs, "unit": "GB/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"band integration: {W} wavenumbers into {out.numel()} "
                                   f"channels of {per}, spectrum and weights in HBM"},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "frac": gbs / peak,
                         "unit": "GB/s", "peak_source": src},
            "sum_check": abs(float(out.sum()) - ref) / ref}
    print(json.dumps(line), flush=True)


def cuda_core_rate(args):
    """Solves/s of the plain FP64 GPU form -- the same engine built with every
    product, right-solve and phase build on the CUDA cores and no tensor-core
    instruction (addingdoublingrt_b200/libadrt_b200_cudacore.so) -- on the same
    workload, timed the same way in a child process (the library is chosen
    when the package loads)."""
    from addingdoublingrt_b200 import build as _build
    if not os.path.exists(_build.CUDA_CORE_LIB):
        return None
    env = dict(os.environ, ADRT_LIBRARY=_build.CUDA_CORE_LIB)
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        env.pop(k, None)
    cmd = [sys.executable, os.path.abspath(__file__), "--only", "fp64", "--no-check",
           "--no-adjoint", "--no-cpu-baseline", "--no-cuda-core", "--no-e2e",
           "--wavenumbers", str(args.wavenumbers), "--steps", str(max(1, min(args.steps, 3))),
           "--warmup", str(max(1, min(args.warmup, 2)))]
    r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=900)
    for line in reversed(r.stdout.strip().splitlines()):
        try:
            d = json.loads(line)
        except ValueError:
            continue
        return {"value": d["value"], "ms_per_step": d["ms_per_step"],
                "library": os.path.basename(_build.CUDA_CORE_LIB)}
    return {"value": None, "error": (r.stderr or r.stdout)[-300:]}


def reference_gpu(batch, steps=3, warmup=1):
    """The reference's own GPU solver (adrt::cuda::solveBatch, src_cuda,
    compiled unmodified with --use_fast_math into oracle/_ref/libadrt_ref_gpu.so)
    timed on `batch` between CUDA events (part of the reference arm).  The
    reference computes TOA F_up / F_down and BOA F_dir in FP32 with its own
    second-order layer start; its TOA F_up error is measured against the FP64
    oracle on a sample of 256 wavenumbers."""
    import ctypes as C
    from oracle import oracle
    path = os.path.join(ROOT, "oracle", "_ref", "libadrt_ref_gpu.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libadrt_ref_gpu.so not built"}
    lib = C.CDLL(path)
    lib.ref_gpu_time_batch.argtypes = [C.POINTER(_abi.BatchDesc), C.POINTER(_abi.Inputs),
                                       C.c_int, C.c_int, C.POINTER(C.c_double)] + [C.c_void_p] * 3
    lib.ref_gpu_last_error.restype = C.c_char_p
    W = batch.W
    ms = C.c_double()
    fu = np.zeros(W)
    rc = lib.ref_gpu_time_batch(C.byref(batch.desc), C.byref(batch.inputs_struct()), steps,
                                warmup, C.byref(ms), fu.ctypes.data, None, None)
    if rc != 0:
        return {"unavailable": lib.ref_gpu_last_error().decode()}
    idx = np.linspace(0, W - 1, min(W, 256)).astype(np.int64)
    ref = oracle.solve_oracle(batch.subset(idx), os.cpu_count() or 1,
                              which=("toa_flux_up",))["toa_flux_up"]
    scale = float(np.max(np.abs(ref))) or 1.0
    return {"solves_per_s": W / (ms.value * 1e-3), "ms_per_call": ms.value,
            "toa_flux_up_max_rel_err_vs_oracle": oracle_rel(fu[idx], ref),
            "toa_flux_up_median_rel_err_vs_oracle":
                float(np.median(np.abs(fu[idx] - ref) / np.maximum(np.abs(ref), 1e-12 * scale))),
            "library": "oracle/_ref/libadrt_ref_gpu.so (src_cuda, --use_fast_math, sm_100a)",
            "workload": REF_GPU_WORKLOAD}


REF_GPU_WORKLOAD = ("config2 shape within the reference GPU API (workloads.config2_scalar): "
                    "W x 100 layers, N=16, 32 moments shared per layer, scalar albedo / mu0 / band")


def engine_rate(eng, batch, steps=3, warmup=1):
    """The engine's FP64 solves/s on `batch` (device arrays, CUDA events)."""
    import torch
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    di = to_device(batch)
    do = alloc_device_outputs(batch, _abi.INTERFACE_OUTPUTS)
    eng.reserve(batch.desc)
    for _ in range(warmup):
        eng.solve_device(batch.desc, di, do)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        eng.solve_device(batch.desc, di, do)
    e1.record()
    torch.cuda.synchronize()
    return batch.W / (e0.elapsed_time(e1) / steps * 1e-3)


def oracle_rel(x, ref):
    scale = float(np.max(np.abs(ref))) or 1.0
    return float(np.max(np.abs(x - ref)) / scale)


# ---------------------------------------------------------------- ranks
def max_over_ranks(x: float, dist, device) -> float:
    """The slowest rank's value (every rank calls this in the same order)."""
    if not dist:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: int, world: int, seconds: float) -> float:
    """Whole-job throughput of a weak-scaling run: every rank processes its own
    units_per_rank, and the job takes as long as its slowest rank."""
    return units_per_rank * world / seconds


def rank_batch(W: int, rank: int, world: int, precision):
    """This rank's config-2 wavenumbers: with one rank the W-wavenumber batch;
    with several, a cost-balanced contiguous range of one W x world batch
    (weak scaling: about W wavenumbers of work per rank, no exchange)."""
    if world == 1:
        return workloads.config2(W=W, precision=precision)
    from addingdoublingrt_b200 import shard
    whole = workloads.config2(W=W * world, precision=precision)
    return shard.shard(whole, rank, world)[2]


# ---------------------------------------------------------------- engine arm
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from addingdoublingrt_b200.engine import Engine, alloc_device_outputs, to_device
    from addingdoublingrt_b200 import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    eng = Engine(device=local)
    if args.workload == "config4":
        return run_config4(args, eng)
    if args.workload == "band":
        return run_band(args, eng)
    if args.workload == "table":
        return run_table(args, eng)
    if args.workload == "adjoint":
        W = args.adjoint_wavenumbers
        fw, ad = time_adjoint(eng, W=W)
        fw2, ad2 = time_adjoint(eng, W=W, mode=_abi.ADJOINT_RECOMPUTE)
        print(json.dumps({"metric": "adjoint time / forward time, config 5", "value": ad / fw,
                          "unit": "ratio", "higher_is_better": False, "forward_ms": fw,
                          "adjoint_ms": ad, "adjoint_recompute_ms": ad2,
                          "adjoint_recompute_over_forward": ad2 / fw2,
                          "config": {"workload": f"config5: W={W} x L=60, "
                                                 "N=16, thermal + solar, FP64"}}))
        return
    results = {}
    precisions = [args.only] if args.only else ["fp64", "mixed"]
    for pname in precisions:
        prec = _abi.PRECISION_FP64 if pname == "fp64" else _abi.PRECISION_MIXED
        b = rank_batch(args.wavenumbers, rank, world, prec)
        di = to_device(b)
        do = alloc_device_outputs(b, which=_abi.INTERFACE_OUTPUTS)
        eng.reserve(b.desc)
        stream = torch.cuda.current_stream()
        for _ in range(args.warmup):
            eng.solve_device(b.desc, di, do, stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clk:
            ev0.record(stream)
            for _ in range(args.steps):
                eng.solve_device(b.desc, di, do, stream)
            ev1.record(stream)
            torch.cuda.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, "cuda")
        status = eng.read_status()
        results[pname] = {"ms": ms, "clocks": clk.summary(), "status": status,
                          "batch": b, "out": do}

    # accuracy against the oracle on a sample (rank 0)
    acc = {}
    if rank == 0 and not args.no_check:
        from oracle import oracle
        b0 = results[precisions[0]]["batch"]
        idx = np.arange(0, b0.W, max(1, b0.W // 200))
        ref = oracle.solve_oracle(b0.subset(idx), os.cpu_count() or 1,
                                  which=_abi.INTERFACE_OUTPUTS)
        L = b0.L
        for pname in precisions:
            out = {k: v.view(-1, L + 1)[torch.as_tensor(idx, device="cuda")].cpu().numpy().ravel()
                   for k, v in results[pname]["out"].items()}
            acc[pname] = {k: {"elementwise": oracle.rel_error(out[k], ref[k]),
                              "normalized": oracle.norm_error(out[k], ref[k], L + 1)}
                          for k in ("flux_up", "flux_down", "flux_direct", "mean_intensity")}

    # e2e through the host entry point (pinned host buffers, copies timed)
    pname = args.precision
    if args.only:
        pname = args.only
    elif pname == "auto":
        # the faster of the forms whose sampled normalised error is <= 1e-6
        ok = [p for p in precisions
              if p == "fp64" or (acc and max(v["normalized"] for v in acc[p].values()) <= 1e-6)]
        pname = min(ok, key=lambda p: results[p]["ms"])
    b = results[pname]["batch"]
    e2e_s, h2d, d2h = None, 0, 0
    if not args.no_e2e:
        hb = workloads.Batch(_abi.BatchDesc.from_buffer_copy(b.desc))
        pinned = {}
        for k, v in b.arrays.items():
            t = torch.from_numpy(v).pin_memory()
            pinned[k] = t
            hb.arrays[k] = t.numpy()
        hout = {k: torch.zeros(b.W * (b.L + 1), dtype=torch.float64).pin_memory().numpy()
                for k in _abi.INTERFACE_OUTPUTS}
        eng.solve_host(hb, out=hout)
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            eng.solve_host(hb, out=hout)
        e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps, dist, "cuda")
        h2d = int(sum(v.nbytes for v in hb.arrays.values()))
        d2h = int(sum(v.nbytes for v in hout.values()))
    cc = None
    if world == 1 and not args.no_cuda_core and not args.only:
        cc = cuda_core_rate(args)
    scalar_rate = None
    if world == 1 and not args.only:
        # the workload the reference arm times the reference's GPU solver on
        scalar_rate = engine_rate(eng, workloads.config2_scalar(W=args.wavenumbers))

    adj = {}
    if not args.no_adjoint:
        fw, ad = time_adjoint(eng)
        fw2, ad2 = time_adjoint(eng, mode=_abi.ADJOINT_RECOMPUTE)
        adj = {"adjoint_over_forward": ad / fw, "adjoint_config5_ms": ad, "forward_config5_ms": fw,
               "adjoint_recompute_over_forward": ad2 / fw2, "adjoint_recompute_config5_ms": ad2}
    c4 = None
    if world == 1 and not args.only and not args.no_config4:
        # free the headline batches first (config 4 holds 40 GB on the device)
        for r in results.values():
            r["out"] = {k: v.cpu() for k, v in r["out"].items()} if rank == 0 else None
        torch.cuda.empty_cache()
        try:
            c4 = run_config4(args, eng, line=False)
        except Exception as ex:
            c4 = {"error": str(ex)[:300]}
        torch.cuda.empty_cache()
    if rank == 0:
        from oracle import oracle
        fl = oracle.flops(b)  # algorithmic flops of the whole batch
        ms = results[pname]["ms"]
        peaks = measured_peaks(_lib.load())
        pk = peaks["fp64_tflops"] if pname == "fp64" else peaks["fp32_tflops"]
        tpk = tensor_peaks(_lib.load())
        achieved = fl / (ms * 1e-3) / 1e12
        traffic = None
        try:
            tj = json.load(open(os.path.join(ROOT, "profiles", "solve_kernel_traffic.json")))
            traffic = tj[f"{pname}_bytes_per_wavenumber"] * args.wavenumbers
        except Exception:
            pass
        roof = {"bound": "fp64" if pname == "fp64" else "fp32", "achieved": achieved,
                "peak": pk, "unit": "TFLOP/s", "frac": achieved / pk if pk else None,
                "traffic": traffic, "traffic_note": "ncu, scaled per wavenumber from a "
                "4000-wavenumber capture (profiles/solve_kernel_traffic.json)",
                "peak_source": peaks["source"] + " (of measured)",
                "flops_per_launch": fl}
        if pname == "fp64" and tpk and tpk.get("fp64_dmma_tflops"):
            # the FP64 products run on the FP64 tensor cores: their measured
            # DMMA rate (above the FMA rate) is the roof; the FMA fraction stays
            dm = tpk["fp64_dmma_tflops"]
            roof.update({"bound": "tensor", "peak": dm, "frac": achieved / dm,
                         "peak_source": "measured live: FP64 DMMA (mma.sync m8n8k4.f64) "
                                        "throughput probe on this GPU (of measured)",
                         "frac_of_fp64_fma_peak": achieved / pk if pk else None,
                         "fp64_fma_peak": pk})
        line = {
            "metric": METRIC,
            "value": job_rate(args.wavenumbers, world, ms * 1e-3),
            "unit": "wavenumber-solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if pname == "fp64" else "f32+f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": pname,
                       "wavenumbers_per_gpu": args.wavenumbers,
                       "l2": "inputs 190 MB > 126 MB L2, no flush",
                       "parallelism": (f"wavenumber shards x{world}: cost-balanced contiguous "
                                       "ranges of one batch, no exchange") if world > 1
                                      else "one GPU"},
            **{f"{p}_solves_per_s": job_rate(args.wavenumbers, world, results[p]["ms"] * 1e-3)
               for p in precisions},
            "mixed_over_fp64": (results["fp64"]["ms"] / results["mixed"]["ms"]
                                if len(precisions) == 2 else None),
            "fp64_cuda_core_solves_per_s": cc["value"] if cc else None,
            "fp64_solves_per_s_reference_gpu_workload": scalar_rate,
            "mixed_over_fp64_cuda_core": (job_rate(args.wavenumbers, world, results["mixed"]["ms"] * 1e-3)
                                          / cc["value"] if cc and cc.get("value") and
                                          "mixed" in results else None),
            "accuracy_vs_oracle": acc,
            "roofline": roof,
            "peaks": {"fp64_fma_tflops": peaks["fp64_tflops"],
                      "fp32_fma_tflops": peaks["fp32_tflops"], **(tpk or {}),
                      "source": "probe kernels on this GPU (csrc/adrt_probe.cu)"},
            "e2e": ({"value": job_rate(args.wavenumbers, world, e2e_s),
                     "unit": "wavenumber-solves/s",
                     "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h} if e2e_s else None),
            # per step: the solve kernel and its re-solve pass (empty unless a
            # wavenumber met a weak pivot)
            "gpu_launches": 2 * args.steps,
            **adj,
            "config4": c4,
            "clocks": results[pname]["clocks"],
            "device_status": {p: results[p]["status"] for p in precisions},
        }
        if "mixed" in results and pname != "mixed":
            # the mixed form's own roofline: its algorithmic flops against the
            # FP32 FMA peak (its FP32 products run as TF32 x3 tensor-core
            # tiles, the rest in FP64)
            am = fl / (results["mixed"]["ms"] * 1e-3) / 1e12
            line["roofline_mixed"] = {"bound": "fp32", "achieved": am,
                                      "peak": peaks["fp32_tflops"], "unit": "TFLOP/s",
                                      "frac": am / peaks["fp32_tflops"]
                                      if peaks["fp32_tflops"] else None}
            if tpk and tpk.get("tf32_mma_tflops"):
                line["roofline_mixed"]["frac_of_tf32_mma_peak"] = am / tpk["tf32_mma_tflops"]
        if not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(b)
            one = cpu_baseline(b, seconds=4.0, threads=1)
            line["cpu_baseline"]["value_1_thread"] = one["value"]
            line["cpu_baseline"]["sample_1_thread"] = one["sample"]
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def tensor_peaks(lib):
    """Warp-level tensor-core throughput of this GPU (adrt_probe_mma_tflops)."""
    import ctypes as C
    v = [C.c_double() for _ in range(3)]
    if hasattr(lib, "adrt_probe_mma_tflops") and \
            lib.adrt_probe_mma_tflops(*(C.byref(x) for x in v)) == 0:
        return {"fp64_dmma_tflops": v[0].value, "tf32_mma_tflops": v[1].value,
                "bf16_mma_tflops": v[2].value}
    return None


def measured_peaks(lib):
    """FP64 / FP32 FMA peaks: MEASURED_PEAKS.json when it holds them, else the
    engine's FMA-throughput probe run now on this GPU."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        mp = json.load(open(path))
    except Exception:
        mp = {}
    if "fp64_tflops" in mp and "fp32_tflops" in mp:
        return {"fp64_tflops": mp["fp64_tflops"], "fp32_tflops": mp["fp32_tflops"],
                "source": "MEASURED_PEAKS.json"}
    import ctypes as C
    f64 = C.c_double()
    f32 = C.c_double()
    if hasattr(lib, "adrt_probe_fma_tflops") and \
            lib.adrt_probe_fma_tflops(C.byref(f64), C.byref(f32)) == 0:
        return {"fp64_tflops": f64.value, "fp32_tflops": f32.value,
                "source": "measured live: FMA-throughput probe kernel"}
    return {"fp64_tflops": None, "fp32_tflops": None, "source": "unavailable"}


if __name__ == "__main__":
    main()
