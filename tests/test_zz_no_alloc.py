"""aem_dft_static, the spectrum entry point for callers that cannot allocate
device memory (hosts that keep all GPU memory in their own arena, plugin
callbacks that must not allocate), checked through the C ABI against the
allocating aem_dft on the same inputs.

Two calls in a row with different sizes, each compared with aem_dft, show
that the static scratch shared by all calls carries nothing from one call
to the next.  Oversized requests must fail cleanly.  This file sorts last
so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-10  # the tolerance of the aem_dft tests; the two paths agree bit for bit in practice


def _bind(lib):
    for name in ("aem_dft", "aem_dft_static"):
        f = getattr(lib, name)
        f.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                      ctypes.c_void_p, ctypes.c_void_p]
        f.restype = ctypes.c_int
    lib.aem_last_error.argtypes = [ctypes.c_void_p]
    lib.aem_last_error.restype = ctypes.c_char_p


def _spectrum(lib, fn, x, dt, freqs):
    import torch
    out = torch.empty(2 * freqs.numel(), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = getattr(lib, fn)(x.data_ptr(), x.numel(), dt, freqs.data_ptr(), freqs.numel(), out.data_ptr(), stream)
    assert rc == 0, lib.aem_last_error(None)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.complex128)


def test_static_matches_allocating_on_two_calls(gpu_lib):
    import torch
    _bind(gpu_lib)
    rng = np.random.default_rng(11)
    cases = [(6000, 512, 1.0e-12), (1500, 2048, 2.5e-12)]
    for n, nf, dt in cases:
        x = torch.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda()
        freqs = torch.from_numpy(rng.uniform(1e8, 0.5 / dt, nf)).cuda()
        ref = _spectrum(gpu_lib, "aem_dft", x, dt, freqs)
        got = _spectrum(gpu_lib, "aem_dft_static", x, dt, freqs)
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= TOL, (n, nf, err)


def test_static_rejects_oversize(gpu_lib):
    import torch
    _bind(gpu_lib)
    x = torch.zeros(64, dtype=torch.float32, device="cuda")
    freqs = torch.ones(65537, dtype=torch.float64, device="cuda")
    out = torch.empty(2 * 65537, dtype=torch.float64, device="cuda")
    rc = gpu_lib.aem_dft_static(x.data_ptr(), 64, 1e-12, freqs.data_ptr(), 65537, out.data_ptr(), None)
    assert rc == -3
    assert b"exceed the static scratch" in gpu_lib.aem_last_error(None)
