"""Batched real FFTs through the C ABI against the reference's pfarc golden
vectors and a float64 numpy transform."""
import os

import numpy as np
import pytest

from q_psdm_b200 import _lib

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_cpu_vectors.npz")
LENGTHS = [2, 16, 720, 728, 1008, 1232, 1260, 1540, 1716, 2002, 2520, 3080, 4004,
           5040, 6006]


@pytest.mark.parametrize("n", LENGTHS)
def test_r2c_matches_pfarc_and_numpy(cuda, n):
    import torch
    g = np.load(GOLD)
    rng = np.random.default_rng(n)
    batch = 7
    x = rng.standard_normal((batch, n)).astype(np.float32)
    x[0] = g[f"pfarc_in_{n}"]
    dx = torch.from_numpy(x).cuda()
    dy = torch.empty((batch, n // 2 + 1, 2), dtype=torch.float32, device="cuda")
    rc = _lib.lib().qpsdm_fft_r2c(dx.data_ptr(), n, batch, dy.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    y = dy.cpu().numpy()
    yc = y[..., 0].astype(np.float64) + 1j * y[..., 1]
    ref = np.fft.rfft(x.astype(np.float64), axis=1)
    tol = 3e-7 * max(1.0, np.log2(n))
    assert np.abs(yc - ref).max() <= tol * np.abs(ref).max()
    pf = g[f"pfarc_out_{n}"]
    pfc = pf[0::2].astype(np.float64) + 1j * pf[1::2]
    assert np.abs(yc[0] - pfc).max() <= 2 * tol * np.abs(pfc).max()


@pytest.mark.parametrize("n", LENGTHS)
def test_c2r_inverts(cuda, n):
    import torch
    rng = np.random.default_rng(100 + n)
    x = rng.standard_normal((5, n)).astype(np.float32)
    X = np.fft.rfft(x.astype(np.float64), axis=1)
    dX = torch.from_numpy(np.stack([X.real, X.imag], -1).astype(np.float32)).cuda()
    dy = torch.empty((5, n), dtype=torch.float32, device="cuda")
    assert _lib.lib().qpsdm_fft_c2r(dX.data_ptr(), n, 5, dy.data_ptr(), None) == 0
    torch.cuda.synchronize()
    y = dy.cpu().numpy() / n
    assert np.abs(y - x).max() <= 3e-7 * max(1.0, np.log2(n)) * np.abs(x).max() * 4


def test_bad_lengths_rejected(cuda):
    import torch
    d = torch.zeros(64, device="cuda")
    assert _lib.lib().qpsdm_fft_r2c(d.data_ptr(), 17 * 2, 1, d.data_ptr(), None) == 1
    assert _lib.lib().qpsdm_fft_r2c(d.data_ptr(), 15, 1, d.data_ptr(), None) == 1
