"""Band integration of a spectrum into channels (adrt_band_integrate), the
reduction after a solve that the reference leaves to its caller (its batched
path only scales flux_up by spectrum_scaling, src_cuda/cuda_solver.cu:481).
Checked against numpy on ragged channels, empty channels, unit weights and
out-of-range offsets."""
import numpy as np
import pytest

from conftest import cuda_available


@pytest.fixture(scope="module")
def eng():
    if not cuda_available():
        pytest.skip("no CUDA device")
    from addingdoublingrt_b200.engine import Engine
    e = Engine()
    yield e
    e.close()


def reference(spec, weight, offsets):
    w = np.ones_like(spec) if weight is None else weight
    return np.array([np.sum(w[a:b] * spec[a:b]) for a, b in zip(offsets[:-1], offsets[1:])])


def ragged_offsets(rng, W, nch):
    cuts = np.sort(rng.integers(0, W + 1, size=nch - 1))
    return np.concatenate([[0], cuts, [W]]).astype(np.int64)


@pytest.mark.gpu
@pytest.mark.parametrize("weighted", [False, True])
def test_channels_match_numpy(eng, weighted):
    import torch
    rng = np.random.default_rng(5 + weighted)
    W, nch = 200_003, 1537
    spec = rng.uniform(0.0, 2.0, W)
    weight = rng.uniform(0.01, 0.05, W) if weighted else None
    off = ragged_offsets(rng, W, nch)
    off[10:13] = off[10]  # empty channels
    off = np.maximum.accumulate(off)
    got = eng.band_integrate(torch.from_numpy(spec).cuda(), torch.from_numpy(off).cuda(),
                             None if weight is None else torch.from_numpy(weight).cuda())
    torch.cuda.synchronize()
    ref = reference(spec, weight, off)
    assert np.allclose(got.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    assert np.all(got.cpu().numpy()[10:12] == 0.0)
    assert eng.read_status() == 0


@pytest.mark.gpu
def test_one_channel_over_a_full_spectrum(eng):
    """The whole config-2 spectrum (100 000 wavenumbers) into one channel."""
    import torch
    rng = np.random.default_rng(9)
    spec = rng.uniform(0.0, 1.0, 100_000)
    off = np.array([0, spec.size], dtype=np.int64)
    got = eng.band_integrate(torch.from_numpy(spec).cuda(), torch.from_numpy(off).cuda())
    torch.cuda.synchronize()
    assert abs(got.item() - spec.sum()) <= 1e-12 * spec.sum()


@pytest.mark.gpu
def test_bad_offsets_flag_the_channel(eng):
    """A channel whose range leaves [0, W] or runs backwards is NaN and raises
    ADRT_FLAG_BAD_INPUT; the other channels are summed."""
    import torch
    spec = np.arange(10, dtype=np.float64)
    off = np.array([0, 4, 3, 10, 12], dtype=np.int64)
    got = eng.band_integrate(torch.from_numpy(spec).cuda(), torch.from_numpy(off).cuda())
    torch.cuda.synchronize()
    g = got.cpu().numpy()
    assert g[0] == spec[:4].sum() and np.isnan(g[1]) and g[2] == spec[3:].sum() and np.isnan(g[3])
    assert eng.read_status() & 4


@pytest.mark.gpu
def test_short_buffers_are_refused_before_the_launch(eng):
    """An output buffer with fewer entries than channels, or weights of another
    length than the spectrum, raise before anything is written."""
    import torch
    spec = torch.ones(100, dtype=torch.float64, device="cuda")
    off = torch.tensor([0, 50, 100], dtype=torch.int64, device="cuda")
    with pytest.raises(ValueError):
        eng.band_integrate(spec, off, out=torch.zeros(1, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        eng.band_integrate(spec, off, torch.ones(99, dtype=torch.float64, device="cuda"))
    got = eng.band_integrate(spec, off)
    torch.cuda.synchronize()
    assert got.cpu().tolist() == [50.0, 50.0]
