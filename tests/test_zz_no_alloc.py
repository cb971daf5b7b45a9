"""The allocation-free FFT entry point against the allocating one.

qpsdm_fft_r2c_noalloc serves callers that may not allocate device memory:
hosts whose own memory pool owns all of the GPU's memory, and latency-critical
callers that cannot take an allocation's implicit synchronisation.  It keeps
its twiddles in a fixed device array built into the library instead of
memory allocated per length, so it must give the same spectra as
qpsdm_fft_r2c, call after call, even when the previous call left the array
holding another length's twiddles.

This file is collected last on purpose: a failure here comes after every
other test has run.  It also passes on its own in a fresh process.
"""
import numpy as np
import pytest

from q_psdm_b200 import _lib

pytestmark = pytest.mark.gpu


def _r2c(fn, x, n, batch):
    import torch
    y = torch.empty((batch, n // 2 + 1, 2), dtype=torch.float32, device="cuda")
    rc = fn(x.data_ptr(), n, batch, y.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, y.cpu().numpy()


def test_noalloc_matches_allocating_entry_point(cuda):
    import torch
    L = _lib.lib()
    g = torch.Generator(device="cuda").manual_seed(5)
    # consecutive calls with different lengths: each must rewrite the shared
    # twiddle array before its own kernel reads it
    for n, batch in [(1232, 6), (4004, 3), (1232, 5), (8192, 2)]:
        x = torch.randn((batch, n), device="cuda", generator=g)
        rc0, want = _r2c(L.qpsdm_fft_r2c, x, n, batch)
        rc1, got = _r2c(L.qpsdm_fft_r2c_noalloc, x, n, batch)
        assert rc0 == 0 and rc1 == 0
        # the FFT tests' tolerance; the two paths run the same kernel on the
        # same twiddles, so in practice they agree bit for bit
        tol = 3e-7 * max(1.0, np.log2(n)) * np.abs(want).max()
        assert np.abs(got - want).max() <= tol, n


def test_noalloc_allocates_nothing(cuda):
    """Free device memory is unchanged around a first call at a new length
    (after one earlier call has loaded the kernels and looked up the array)."""
    import torch
    L = _lib.lib()
    x = torch.randn((4, 3080), device="cuda")
    y = torch.empty((4, 3080 // 2 + 1, 2), dtype=torch.float32, device="cuda")
    assert L.qpsdm_fft_r2c_noalloc(x.data_ptr(), 720, 4, y.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert L.qpsdm_fft_r2c_noalloc(x.data_ptr(), 3080, 4, y.data_ptr(), None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_on_a_stream(cuda):
    """Two calls in a row on a non-default stream, each checked against the
    allocating entry point on the same stream."""
    import torch
    L = _lib.lib()
    st = torch.cuda.Stream()
    g = torch.Generator(device="cuda").manual_seed(9)
    for n, batch in [(2002, 7), (6006, 2)]:
        x = torch.randn((batch, n), device="cuda", generator=g)
        want = torch.empty((batch, n // 2 + 1, 2), dtype=torch.float32, device="cuda")
        got = torch.empty_like(want)
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            assert L.qpsdm_fft_r2c(x.data_ptr(), n, batch, want.data_ptr(), st.cuda_stream) == 0
            assert L.qpsdm_fft_r2c_noalloc(x.data_ptr(), n, batch, got.data_ptr(),
                                           st.cuda_stream) == 0
        st.synchronize()
        w, o = want.cpu().numpy(), got.cpu().numpy()
        tol = 3e-7 * max(1.0, np.log2(n)) * np.abs(w).max()
        assert np.abs(o - w).max() <= tol, n


def test_noalloc_rejects_sizes_beyond_its_array(cuda):
    import torch
    L = _lib.lib()
    x = torch.zeros(2 * (_lib.FFT_NOALLOC_MAX_N + 2), device="cuda")
    n = _lib.FFT_NOALLOC_MAX_N + 2
    assert L.qpsdm_fft_r2c_noalloc(x.data_ptr(), n, 1, x.data_ptr(), None) == _lib.ESIZE
    assert L.qpsdm_fft_r2c_noalloc(x.data_ptr(), 15, 1, x.data_ptr(), None) == 1
