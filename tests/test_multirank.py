"""The multi-GPU path of bench.py on CPU: two gloo ranks.  The path splits
one batch into cost-balanced contiguous wavenumber ranges with no data-path
collective; only the timing reduction crosses ranks.  Every rank takes the
max-over-ranks step in the same order, the job rate is the units of all
ranks over the slowest rank's time, the ranks' ranges cover the batch once,
and each rank's shard solved on its own (by the oracle, standing in for the
GPU here) gives the whole batch's outputs for its range."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    import bench
    from addingdoublingrt_b200 import workloads
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle
        from addingdoublingrt_b200 import _abi
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        b = bench.rank_batch(6, rank, world, _abi.PRECISION_FP64)
        out = oracle.solve_oracle(b, 1, which=("flux_up",))["flux_up"]
        q.put((rank, slowest, b.arrays["delta_tau"].copy(), out))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_the_step_time_and_shard_the_work():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]  # both ranks see the slowest rank's time
    from oracle import oracle
    from addingdoublingrt_b200 import workloads
    whole = workloads.config2(W=12)
    # the ranges cover the batch once, in rank order
    assert np.array_equal(np.concatenate([r[2] for r in res]), whole.arrays["delta_tau"])
    assert all(r[2].size > 0 for r in res)
    ref = oracle.solve_oracle(whole, 1, which=("flux_up",))["flux_up"]
    assert np.array_equal(np.concatenate([r[3] for r in res]), ref)
    import bench
    assert bench.job_rate(1000, world, 0.5) == 4000.0
    assert np.isclose(bench.job_rate(100_000, 1, 0.537), 186219.7, rtol=1e-4)
