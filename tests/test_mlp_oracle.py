"""The surrogate network's CPU oracle, pinned on the CPU.

The reference has no learned component, so the oracle's gradient is pinned
by central finite differences of its own FP64 loss; its BF16 rounding by
known bit patterns.  The product's parameter layout and initialiser must
agree with the oracle's."""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from q_psdm_b200 import surrogate as S


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, (n, 5)).astype(np.float32)
    t = np.stack([np.sin(2 * x[:, 0]) + x[:, 4] ** 2, x[:, 1] * x[:, 2]], 1).astype(np.float32)
    return x, t


def test_layout_and_init_agree_with_product():
    assert M.NPARAM == S.NPARAM
    assert np.array_equal(M.init_params(5).astype(np.float32), S.init_params(5))


def test_bf16_rounding_known_values():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -3.0e-5, 0.0], np.float32)
    r = M.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                                # tie: to even
    assert r[2] == 1.0 + 2 ** -7                      # above the half-way point
    assert r[3] == 1.0                                # below it
    assert abs(r[4] - (-3.0e-5)) <= 2 ** -8 * 3.0e-5
    assert r[5] == 0.0


@pytest.mark.parametrize("w_out", [(1.0, 1.0), (0.3, 2.0)])
def test_oracle_gradient_matches_finite_differences(w_out):
    x, t = _data(37, 1)
    p = M.init_params(2, out_scale=1.0)
    rng = np.random.default_rng(3)
    P = M.unpack(p)
    for l in range(1, 5):
        P[f"b{l}"] = rng.standard_normal(M.H) * 0.1
    P["b5"][:2] = rng.standard_normal(2) * 0.1
    p = M.pack(P)
    shift, scale = np.zeros(5, np.float32), np.full(5, 0.7, np.float32)
    _, g = M.loss_and_grad(p, x, t, shift, scale, w_out)
    trainable = np.ones(M.NPARAM, bool)
    o = 0
    for name, shp in M.SHAPES:
        n = int(np.prod(shp))
        if name == "W1":
            trainable[o:o + n] = (np.arange(n) % M.NIN) < 5
        if name == "W5":
            trainable[o:o + n] = np.arange(n) < 2 * M.H
        if name == "b5":
            trainable[o:o + n] = np.arange(n) < 2
        o += n
    assert np.all(g[~trainable] == 0.0)
    idx = rng.choice(np.flatnonzero(trainable), 60, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        lp, _ = M.loss_and_grad(pp, x, t, shift, scale, w_out)
        lm, _ = M.loss_and_grad(pm, x, t, shift, scale, w_out)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_emulation_is_close_to_fp64():
    x, t = _data(300, 4)
    p = M.init_params(1, out_scale=1.0)
    shift, scale = np.zeros(5, np.float32), np.ones(5, np.float32)
    l64, g64 = M.loss_and_grad(p, x, t, shift, scale)
    l16, g16 = M.loss_and_grad(p, x, t, shift, scale, bf16_ops=True)
    assert abs(l16 - l64) < 2e-2 * l64
    assert np.linalg.norm(g16 - g64) < 3e-2 * np.linalg.norm(g64)
