"""The multi-GPU path of bench.py on CPU: two gloo ranks (the path shards
wavenumbers across replicas with no data-path collective; only the timing
reduction crosses ranks).  Every rank takes the max-over-ranks step in the
same order, the job rate is the units of all ranks over the slowest rank's
time, and the ranks' synthetic shards differ."""
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
        slowest = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        b = workloads.config2(W=8, seed=bench.rank_seed(rank))
        q.put((rank, slowest, float(b.arrays["delta_tau"].sum())))
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
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]  # both ranks see the slowest rank's time
    assert res[0][2] != res[1][2]                # different wavenumber shards
    import bench
    assert bench.job_rate(1000, world, 0.5) == 4000.0
    assert np.isclose(bench.job_rate(100_000, 1, 0.537), 186219.7, rtol=1e-4)
