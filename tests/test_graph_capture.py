"""The batched solve inside a CUDA graph.  After adrt_engine_reserve the
device entry point allocates and synchronises nothing, so a caller can
capture it (here in a torch.cuda.CUDAGraph) and replay it on new inputs
written into the same device buffers; the replay equals a direct solve."""
import numpy as np
import pytest

from conftest import cuda_available
from addingdoublingrt_b200 import workloads

pytestmark = pytest.mark.gpu

WHICH = ("toa_flux_up", "toa_flux_down", "boa_flux_direct", "flux_up", "mean_intensity")


@pytest.fixture(scope="module")
def eng():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


@pytest.mark.parametrize("make", [workloads.config2, workloads.config5])
def test_solve_replays_from_a_cuda_graph(eng, make):
    import torch
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    b = make(W=3000)
    eng.reserve(b.desc)
    di = to_device(b)
    do = alloc_device_outputs(b, WHICH)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        eng.solve_device(b.desc, di, do, stream=s)  # warm: quadrature tables cached
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        eng.solve_device(b.desc, di, do, stream=s)
    # new inputs of the same shape in the captured buffers
    b2 = make(W=3000, seed=77)
    for k, v in di.items():
        v.copy_(torch.from_numpy(b2.arrays[k]))
    g.replay()
    torch.cuda.synchronize()
    got = {k: v.clone() for k, v in do.items()}
    ref = alloc_device_outputs(b2, WHICH)
    eng.solve_device(b2.desc, di, ref)
    torch.cuda.synchronize()
    for k in WHICH:
        assert torch.equal(got[k], ref[k]), k
    assert not torch.equal(got["toa_flux_up"], torch.zeros_like(got["toa_flux_up"]))
    assert eng.read_status() == 0
    del g


def test_uneven_batch_replays_from_a_cuda_graph(eng):
    """Columns of different N, L, W and precision in one captured launch; the
    replay (new inputs in the captured buffers) equals a direct uneven solve,
    and eager uneven solves work after the capture."""
    import torch
    from addingdoublingrt_b200.engine import alloc_device_outputs, to_device
    cols = workloads.config4_columns(ncols=12, seed=14)
    dev = [(c.desc, to_device(c), alloc_device_outputs(c, ("toa_flux_up", "toa_flux_down")))
           for c in cols]
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        eng.solve_uneven(dev, stream=s)  # warm: column table and work buffer sized
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        eng.solve_uneven(dev, stream=s)
    cols2 = workloads.config4_columns(ncols=12, seed=14)  # same shapes
    rng = np.random.default_rng(3)
    for (d, di, do), c in zip(dev, cols2):
        tau = c.arrays["delta_tau"] * rng.uniform(0.5, 2.0, size=c.arrays["delta_tau"].shape)
        di["delta_tau"].copy_(torch.from_numpy(tau))
    g.replay()
    torch.cuda.synchronize()
    got = [{k: v.clone() for k, v in do.items()} for _, _, do in dev]
    ref = [(d, di, {k: torch.zeros_like(v) for k, v in do.items()}) for d, di, do in dev]
    eng.solve_uneven(ref)  # eager, after the capture
    torch.cuda.synchronize()
    for g_out, (_, _, r_out) in zip(got, ref):
        for k in g_out:
            assert torch.equal(g_out[k], r_out[k]), k
    assert eng.read_status() == 0
    del g
