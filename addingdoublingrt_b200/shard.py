"""One batch of wavenumbers split over ranks (one process per GPU).

Wavenumbers are independent and the phase moments and quadrature are
read-only, so a batch splits into contiguous wavenumber ranges with no
exchange between the ranks: each rank solves its range on its own GPU and
keeps its outputs.  The ranges are balanced by an estimate of each
wavenumber's work, not by count: every scattering layer costs its number of
doubling steps (the rule of src/doubling.hpp:20-26 and 107-109, as the
device's num_doublings applies it) plus a fixed share for its adding step;
a transparent or purely absorbing layer costs a small fixed share.  Columns
of an uneven batch are packed onto ranks by the engine's per-column cost
model (wavenumbers x layers x padded order cubed, csrc/adrt_engine.cu's
cost order), largest first.
"""
from __future__ import annotations

import numpy as np

#: work of one layer's adding step, in doubling steps
ADDING_SHARE = 2.0
#: work of a layer without scattering (its adding shortcut), in doubling steps
CLEAR_SHARE = 0.5
#: the device's bound on doubling steps per layer
MAX_DOUBLINGS = 64


def num_doublings(tau, omega) -> np.ndarray:
    """Doubling steps per layer: max(1, trunc(ln tau / ln 2) + ipow0(omega)),
    ipow0 = 4 / 10 / 16 below omega 0.01 / 0.1 / above, an exact power of two
    taking its exponent, bounded by 64 (src/doubling.hpp:20-26, 107-109)."""
    tau = np.asarray(tau, dtype=np.float64)
    om = np.minimum(np.asarray(omega, dtype=np.float64), 1.0)
    ip = np.where(om < 0.01, 4, np.where(om < 0.1, 10, 16))
    with np.errstate(divide="ignore", invalid="ignore"):
        m, e = np.frexp(tau)
        lg = np.where(m == 0.5, e - 1, np.trunc(np.log(tau) / np.log(2.0)))
    lg = np.where(np.isfinite(lg), lg, 0.0)
    nn = np.clip(lg + ip, 1, MAX_DOUBLINGS)
    return np.where(tau < 1e300, nn, MAX_DOUBLINGS).astype(np.int64)


def wavenumber_costs(batch) -> np.ndarray:
    """Estimated work of every wavenumber of a host batch, in doubling steps."""
    W, L = batch.W, batch.L
    tau = batch.arrays["delta_tau"].reshape(W, L)
    om = batch.arrays["single_scat_albedo"].reshape(W, L)
    scat = (tau > 0.0) & (om > 0.0)
    per_layer = np.where(scat, num_doublings(np.where(scat, tau, 1.0), om) + ADDING_SHARE,
                         CLEAR_SHARE)
    return per_layer.sum(axis=1)


def balanced_ranges(costs, world: int) -> list[tuple[int, int]]:
    """Contiguous [lo, hi) wavenumber ranges, one per rank, covering every
    wavenumber once, each cut where the running cost first reaches its share
    of the total: no range exceeds total / world by more than one
    wavenumber's cost.  With fewer wavenumbers than ranks the last ranks get
    empty ranges."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(costs, dtype=np.float64)
    if c.ndim != 1 or np.any(c < 0) or not np.all(np.isfinite(c)):
        raise ValueError("costs must be a finite non-negative vector")
    W = c.size
    csum = np.cumsum(c)
    total = float(csum[-1]) if W else 0.0
    cuts = [0]
    for k in range(1, world):
        if total > 0.0:
            j = int(np.searchsorted(csum, total * k / world, side="left")) + 1
        else:
            j = (W * k) // world
        cuts.append(min(max(j, cuts[-1]), W))
    cuts.append(W)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def shard(batch, rank: int, world: int):
    """This rank's range of a host batch: (lo, hi, sub-batch of wavenumbers
    lo..hi-1, per-wavenumber arrays sliced and shared ones kept)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    lo, hi = balanced_ranges(wavenumber_costs(batch), world)[rank]
    return lo, hi, batch.subset(np.arange(lo, hi))


def column_costs(descs) -> np.ndarray:
    """The engine's per-column cost model of an uneven batch: W x L x NP^3,
    NP the padded order (4, 8, 16 or 32)."""
    out = []
    for d in descs:
        n = d.num_quadrature
        NP = 4 if n <= 4 else 8 if n <= 8 else 16 if n <= 16 else 32
        out.append(float(d.num_wavenumbers) * d.num_layers * NP ** 3)
    return np.asarray(out, dtype=np.float64)


def pack_columns(costs, world: int) -> list[list[int]]:
    """Columns onto ranks, largest first, each onto the least-loaded rank
    (ties to the lowest rank); every rank's list in the columns' order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(costs, dtype=np.float64)
    load = np.zeros(world)
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(c.size), key=lambda i: (-c[i], i)):
        r = int(np.argmin(load))
        parts[r].append(i)
        load[r] += c[i]
    return [sorted(p) for p in parts]


__all__ = ["num_doublings", "wavenumber_costs", "balanced_ranges", "shard", "column_costs",
           "pack_columns", "ADDING_SHARE", "CLEAR_SHARE"]
