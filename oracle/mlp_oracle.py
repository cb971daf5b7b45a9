"""CPU oracle of the traveltime / t* surrogate network (test infrastructure).

Only the tests and the benchmark's checker import this file; the product
path never does.  The reference has no learned component (it reads
precomputed tables, src/q-psdm.cu:2382-2627), so there is nothing of the
reference to pin against: this oracle is pinned instead by central finite
differences of its own FP64 loss (tests/test_mlp_oracle.py).

Network: 5 inputs (zero-padded to 16) -> 4 x 128 SiLU -> 2 outputs (padded
to 16).  Parameter vector, in order: W1 [128][16], b1 [128], W2 [128][128],
b2, W3, b3, W4, b4, W5 [16][128], b5 [16] (W[out][in]).  Loss:
    L = sum_s sum_j w_j (y_sj - t_sj)^2 / n.

``bf16=True`` rounds to bfloat16 (round to nearest even) at the points where
the tensor-core kernels store an operand in BF16: the weights, the
normalised inputs, every hidden activation, and the output-side gradients
dZ that feed a GEMM.  Sums are FP64 either way.
"""
from __future__ import annotations

import numpy as np

H, NIN, NOUT = 128, 16, 16
SHAPES = [("W1", (H, NIN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
          ("b3", (H,)), ("W4", (H, H)), ("b4", (H,)), ("W5", (NOUT, H)), ("b5", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, o = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], np.float64).reshape(shp)
        o += n
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in SHAPES])


def bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def features(x, shift, scale):
    """[n][5] raw inputs -> [n][16] normalised, zero-padded (FP32 as on the
    device)."""
    x = np.asarray(x, np.float32)
    f = np.zeros((x.shape[0], NIN), np.float32)
    f[:, :5] = (x - np.asarray(shift, np.float32)) * np.asarray(scale, np.float32)
    return f.astype(np.float64)


def forward(p, x, shift, scale, bf16_ops=False):
    """Outputs y [n][2] and the per-layer (Z, H) for backward."""
    P = unpack(p)
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    h = r(features(x, shift, scale))
    acts = [h]
    zs = []
    for l in range(1, 5):
        z = h @ r(P[f"W{l}"]).T
        zs.append(z)
        h = r(_silu(z + P[f"b{l}"]))
        acts.append(h)
    y = h @ r(P["W5"]).T + P["b5"]
    return y[:, :2], zs, acts


def loss_and_grad(p, x, t, shift, scale, w_out=(1.0, 1.0), bf16_ops=False):
    """FP64 loss and its gradient with respect to the parameter vector."""
    P = unpack(p)
    r = bf16 if bf16_ops else (lambda a: np.asarray(a, np.float64))
    n = x.shape[0]
    y, zs, acts = forward(p, x, shift, scale, bf16_ops)
    w = np.asarray(w_out, np.float64)
    e = y - np.asarray(t, np.float64)
    loss = float(np.sum(w * e * e) / n)
    d = np.zeros((n, NOUT))
    d[:, :2] = 2.0 * w * e / n
    G = {"b5": d.sum(0)}
    db = r(d)
    G["W5"] = db.T @ acts[4]
    dh = db @ r(P["W5"])
    for l in range(4, 0, -1):
        d = dh * _silu_grad(zs[l - 1] + P[f"b{l}"])
        G[f"b{l}"] = d.sum(0)
        db = r(d)
        G[f"W{l}"] = db.T @ acts[l - 1]
        dh = db @ r(P[f"W{l}"])
    # padding columns / rows are not parameters
    G["W1"][:, 5:] = 0.0
    G["W5"][2:, :] = 0.0
    G["b5"][2:] = 0.0
    return loss, pack(G)


def init_params(seed=0, out_scale=0.1):
    """He-normal hidden weights, small output layer, zero biases and pads."""
    rng = np.random.default_rng(seed)
    d = {}
    d["W1"] = np.zeros((H, NIN))
    d["W1"][:, :5] = rng.standard_normal((H, 5)) * np.sqrt(2.0 / 5)
    for l in (2, 3, 4):
        d[f"W{l}"] = rng.standard_normal((H, H)) * np.sqrt(2.0 / H)
    d["W5"] = np.zeros((NOUT, H))
    d["W5"][:2] = rng.standard_normal((2, H)) * np.sqrt(1.0 / H) * out_scale
    for l in range(1, 5):
        d[f"b{l}"] = np.zeros(H)
    d["b5"] = np.zeros(NOUT)
    return pack(d)
