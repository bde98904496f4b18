"""GPU spectrum entry point (aem_dft) against numpy.

The post-processor takes numpy's FFT of the zero-padded series
(utility_scripts/post_processor.py:160-215); aem_dft evaluates the same sum
directly at chosen frequencies.  Checked: the padded-FFT bins (relative L2
<= 1e-10, FP64 accumulation on both sides), arbitrary off-grid frequencies
against a float64 direct sum, and bit-identical results on a repeat call.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _direct(x, dt, freqs):
    m = np.arange(len(x))
    return np.array([np.sum(x.astype(np.float64) * np.exp(-2j * np.pi * f * m * dt)) for f in freqs])


@pytest.mark.parametrize("n,padding", [(300, 10), (4000, 10), (17, 3)])
def test_dft_matches_padded_fft(n, padding, gpu_lib):
    import torch
    import alpineem_b200 as ab

    rng = np.random.default_rng(n)
    x = rng.standard_normal(n).astype(np.float32)
    dt = 1.9e-12
    N = (padding + 1) * n
    ref = np.fft.fft(np.concatenate((x.astype(np.float64), np.zeros(n * padding))))
    k = np.arange(0, N // 2, max(1, N // 700))
    freqs = k / (N * dt)
    got = ab.dft(torch.from_numpy(x).cuda(), dt, torch.from_numpy(freqs).cuda()).cpu().numpy()
    err = np.linalg.norm(got - ref[k]) / np.linalg.norm(ref[k])
    assert err <= TOL, err


def test_dft_off_grid_and_repeat(gpu_lib):
    import torch
    import alpineem_b200 as ab

    rng = np.random.default_rng(7)
    x = rng.standard_normal(5000).astype(np.float32)
    dt = 1.0e-12
    freqs = rng.uniform(1e9, 3e10, 512)
    xd, fd = torch.from_numpy(x).cuda(), torch.from_numpy(freqs).cuda()
    a = ab.dft(xd, dt, fd).cpu().numpy()
    b = ab.dft(xd, dt, fd).cpu().numpy()
    ref = _direct(x, dt, freqs)
    assert np.linalg.norm(a - ref) / np.linalg.norm(ref) <= TOL
    assert np.array_equal(a, b)
