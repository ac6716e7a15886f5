"""Sharding one batch over ranks (addingdoublingrt_b200.shard): the doubling
count of the cost estimate against the oracle's rule, the cost-balanced
contiguous ranges and the column packing on their invariants, and on a GPU
the shards solved one after another against the whole batch's solve."""
import ctypes as C

import numpy as np
import pytest

from conftest import cuda_available
from addingdoublingrt_b200 import _abi, shard, workloads


def test_doubling_count_follows_the_oracle_rule():
    from oracle import oracle
    lib = oracle.oracle_lib()
    lib.oracle_num_doublings.restype = C.c_int
    rng = np.random.default_rng(0)
    tau = 10.0 ** rng.uniform(-6.0, 4.0, 4000)
    om = np.concatenate([rng.uniform(0.0, 1.0, 3000), [0.0, 0.00999, 0.01, 0.0999, 0.1, 1.0] * 166,
                         [0.5] * 4])[:4000]
    got = shard.num_doublings(tau, om)
    want = [lib.oracle_num_doublings(float(t), float(o)) for t, o in zip(tau, om)]
    assert np.array_equal(got, want)
    # exact powers of two take their exponent; non-finite depths the device bound
    assert list(shard.num_doublings([0.5, 1.0, 8.0], [0.5] * 3)) == [15, 16, 19]
    assert list(shard.num_doublings([np.inf, np.nan, 1e301], [0.5] * 3)) == [64] * 3


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_ranges_cover_the_batch_and_balance_the_cost(world):
    b = workloads.config2(W=257, L=20)
    c = shard.wavenumber_costs(b)
    assert c.shape == (257,) and np.all(c > 0)
    r = shard.balanced_ranges(c, world)
    assert len(r) == world and r[0][0] == 0 and r[-1][1] == 257
    assert all(r[i][1] == r[i + 1][0] and r[i][0] <= r[i][1] for i in range(world - 1))
    loads = [c[lo:hi].sum() for lo, hi in r]
    assert max(loads) <= c.sum() / world + c.max() + 1e-9
    # by cost, not by count: a batch whose second half is four times as
    # expensive puts more wavenumbers on the first rank
    if world == 2:
        skew = np.r_[np.ones(100), 4.0 * np.ones(100)]
        (lo0, hi0), _ = shard.balanced_ranges(skew, 2)
        assert hi0 - lo0 > 100


def test_ranges_edge_cases():
    assert shard.balanced_ranges([], 3) == [(0, 0)] * 3
    assert shard.balanced_ranges([1.0, 1.0], 4)[-1] == (2, 2)
    assert shard.balanced_ranges(np.zeros(10), 2) == [(0, 5), (5, 10)]
    for bad in ([-1.0, 1.0], [np.nan], [[1.0]]):
        with pytest.raises(ValueError):
            shard.balanced_ranges(bad, 2)
    with pytest.raises(ValueError):
        shard.balanced_ranges([1.0], 0)
    with pytest.raises(ValueError):
        shard.shard(workloads.config1(W=4), 2, 2)


def test_shards_keep_shared_arrays_and_slice_per_wavenumber_ones():
    b = workloads.config5(W=40)
    lo, hi, s = shard.shard(b, 1, 3)
    assert s.W == hi - lo and s.desc.num_wavenumbers == hi - lo
    assert np.array_equal(s.arrays["delta_tau"].reshape(-1, b.L),
                          b.arrays["delta_tau"].reshape(b.W, b.L)[lo:hi])
    assert np.array_equal(s.arrays["phase_moments"], b.arrays["phase_moments"])  # shared set


def test_column_packing():
    descs = [_abi.make_desc(num_wavenumbers=w, num_layers=l, num_quadrature=n)
             for w, l, n in [(8192, 150, 16), (256, 20, 4), (4000, 80, 8), (300, 150, 16),
                             (8000, 30, 4), (1000, 100, 16), (5000, 60, 8)]]
    c = shard.column_costs(descs)
    assert c[0] == 8192 * 150 * 16 ** 3 and c[1] == 256 * 20 * 4 ** 3
    for world in (1, 2, 3, 10):
        parts = shard.pack_columns(c, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(descs)))
        loads = [c[p].sum() if p else 0.0 for p in parts]
        assert max(loads) <= c.sum() / world + c.max()
        assert all(p == sorted(p) for p in parts)


@pytest.mark.gpu
def test_shards_solved_apart_match_the_whole_batch():
    """Every wavenumber's solve is independent of the others in the launch,
    so the shards' outputs, solved one after another, are the whole batch's
    bit for bit."""
    if not cuda_available():
        pytest.skip("no CUDA device")
    import torch
    from addingdoublingrt_b200.engine import Engine, alloc_device_outputs, to_device
    b = workloads.config2(W=3000, L=40)
    eng = Engine()
    whole = alloc_device_outputs(b, _abi.INTERFACE_OUTPUTS)
    eng.solve_device(b.desc, to_device(b), whole)
    parts = []
    for rank in range(3):
        lo, hi, s = shard.shard(b, rank, 3)
        out = alloc_device_outputs(s, _abi.INTERFACE_OUTPUTS)
        eng.solve_device(s.desc, to_device(s), out)
        parts.append((lo, hi, out))
    torch.cuda.synchronize()
    assert eng.read_status() == 0
    for k in _abi.INTERFACE_OUTPUTS:
        w = whole[k].view(b.W, b.L + 1)
        for lo, hi, out in parts:
            assert torch.equal(out[k].view(hi - lo, b.L + 1), w[lo:hi]), k
    eng.close()
