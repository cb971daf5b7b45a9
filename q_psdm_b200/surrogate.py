"""Learned traveltime / t* surrogate on the tcgen05 tensor cores.

The network (5 -> 128 x 4 SiLU -> 2, ``csrc/mlp.cu``) maps a surface
position and an image point, (px, py, x, y, z), to corrections of the
linear-gradient background:

    T  = T_bg(r, z)          + y0 * 1e-3      (s)
    t* = T_bg(r, z) / q_ref  + y1 * 1e-3      (s)

with r the horizontal source-point distance and T_bg the exact v0 + kz z
traveltime.  The background carries the steep curvature of T in the source
position; the network learns only the smooth part that the velocity
anomalies and the Q layers add.

It is trained (on the GPU, by the library's own forward and backward
kernels) on the tables the eikonal generator writes at a coarse surface
spacing, and is then evaluated at the table nodes of a finer surface grid to
densify them.  The tables keep the last word on its error: every coarse surface
patch of every table cell whose corner nodes the network misses by more than
``gate_ms`` (2 ms) keeps plain bilinear interpolation of the coarse tables.
The reference has no counterpart; it reads precomputed tables only
(src/q-psdm.cu:2382-2627).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .tables import DESC_DTYPE, LineTables, cell_surface_nodes

NPARAM = 53776


def init_params(seed: int = 0, out_scale: float = 0.1) -> np.ndarray:
    """He-normal hidden weights, small output layer, zero biases and pads
    (parameter order of qpsdm_mlp_set_params)."""
    rng = np.random.default_rng(seed)
    H = 128
    parts = []
    w1 = np.zeros((H, 16))
    w1[:, :5] = rng.standard_normal((H, 5)) * np.sqrt(2.0 / 5)
    parts += [w1, np.zeros(H)]
    for _ in range(3):
        parts += [rng.standard_normal((H, H)) * np.sqrt(2.0 / H), np.zeros(H)]
    w5 = np.zeros((16, H))
    w5[:2] = rng.standard_normal((2, H)) * np.sqrt(1.0 / H) * out_scale
    parts += [w5, np.zeros(16)]
    p = np.concatenate([a.ravel() for a in parts]).astype(np.float32)
    assert p.size == NPARAM
    return p


class Mlp:
    """One network on one GPU (qpsdm_mlp_* handle).  Device buffers are
    torch tensors; every compute call goes to the library's kernels."""

    def __init__(self, device: int = 0, seed: int = 0, params: np.ndarray | None = None):
        import torch
        self.torch = torch
        self.L = _lib.lib()
        self.device = device
        self.dev = torch.device("cuda", device)
        h = C.c_void_p()
        _lib.check(self.L.qpsdm_mlp_create(device, C.byref(h)), what="mlp_create")
        self.h = h
        assert self.L.qpsdm_mlp_param_count() == NPARAM
        self.set_params(init_params(seed) if params is None else params)
        self.set_scaling(np.zeros(5), np.ones(5), (1.0, 1.0))

    def close(self):
        if self.h:
            self.L.qpsdm_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p) -> None:
        a = np.ascontiguousarray(p, np.float32)
        assert a.size == NPARAM
        _lib.check(self.L.qpsdm_mlp_set_params(self.h, a.ctypes.data), what="mlp_set_params")

    def params(self) -> np.ndarray:
        a = np.empty(NPARAM, np.float32)
        _lib.check(self.L.qpsdm_mlp_get_params(self.h, a.ctypes.data), what="mlp_get_params")
        return a

    def set_scaling(self, shift, scale, out_weight=(1.0, 1.0)) -> None:
        self.shift = np.ascontiguousarray(shift, np.float32)
        self.scale = np.ascontiguousarray(scale, np.float32)
        w = np.ascontiguousarray(out_weight, np.float32)
        _lib.check(self.L.qpsdm_mlp_set_scaling(self.h, self.shift.ctypes.data,
                                                self.scale.ctypes.data, w.ctypes.data),
                   what="mlp_set_scaling")

    def _dev(self, a, cols):
        t = self.torch
        if isinstance(a, t.Tensor):
            assert a.is_cuda and a.dtype == t.float32 and a.is_contiguous()
            assert a.shape[-1] == cols
            return a
        return t.from_numpy(np.ascontiguousarray(a, np.float32).reshape(-1, cols)).to(self.dev)

    def gradients(self, x, t):
        """(loss, gradient vector) over all samples, no update."""
        dx, dt = self._dev(x, 5), self._dev(t, 2)
        g = np.empty(NPARAM, np.float32)
        loss = C.c_float()
        _lib.check(self.L.qpsdm_mlp_gradients(self.h, dx.data_ptr(), dt.data_ptr(), dx.shape[0],
                                              g.ctypes.data, C.byref(loss), None),
                   what="mlp_gradients")
        return float(loss.value), g

    def train_step(self, x, t, lr: float, want_loss: bool = False):
        dx, dt = self._dev(x, 5), self._dev(t, 2)
        loss = C.c_float()
        _lib.check(self.L.qpsdm_mlp_train_step(self.h, dx.data_ptr(), dt.data_ptr(), dx.shape[0],
                                               float(lr), C.byref(loss) if want_loss else None,
                                               None),
                   what="mlp_train_step")
        return float(loss.value) if want_loss else None

    def forward(self, x, out=None):
        """y [n][2] (torch, on the device) for x [n][5]."""
        dx = self._dev(x, 5)
        n = dx.shape[0]
        y = out if out is not None else self.torch.empty((n, 2), dtype=self.torch.float32,
                                                         device=self.dev)
        _lib.check(self.L.qpsdm_mlp_forward(self.h, dx.data_ptr(), n, y.data_ptr(), None),
                   what="mlp_forward")
        return y

    def status(self) -> None:
        _lib.check(self.L.qpsdm_mlp_status(self.h), what="mlp_status")


# ---------------------------------------------------------------------------
# background and samples
# ---------------------------------------------------------------------------
def background_time(r, z, v0: float, kz: float):
    """Exact traveltime (s) of v(z) = v0 + kz z from the surface."""
    r = np.asarray(r, np.float64)
    z = np.asarray(z, np.float64)
    if kz < 1e-9:
        return np.hypot(r, z) / v0
    v = v0 + kz * z
    return np.arccosh(np.maximum(1.0 + kz * kz * (r * r + z * z) / (2.0 * v0 * v), 1.0)) / kz


def table_nodes(tab: LineTables, fci: int, line_y: float):
    """Features (px, py, x, y, z) of every value of the tables, in storage
    order ([cell][iys][ixs][ixl][izl] blocks), as float32 [n][5]."""
    out = np.empty((tab.ttt.size, 5), np.float32)
    for c in range(tab.nxg * tab.nzg):
        ixg, izg = divmod(c, tab.nzg)
        d = tab.desc[c]
        xs, ys = cell_surface_nodes(tab, ixg, izg, fci)
        x = ((tab.cdp1 - fci) + ixg * tab.nxi1 + np.arange(tab.nxi1)) * tab.dx
        z = (izg * tab.nzi1 + np.arange(tab.nzi1)) * tab.dzii
        PY, PX, X, Z = np.meshgrid(ys, xs, x, z, indexing="ij")
        blk = slice(int(d["idx"]), int(d["idx"]) + PY.size)
        out[blk, 0] = PX.ravel()
        out[blk, 1] = line_y + PY.ravel()
        out[blk, 2] = X.ravel()
        out[blk, 3] = line_y
        out[blk, 4] = Z.ravel()
    return out


@dataclass
class Background:
    v0: float
    kz: float
    q_ref: float

    def times(self, feat):
        f = np.asarray(feat, np.float64)
        r = np.hypot(f[:, 0] - f[:, 2], f[:, 1] - f[:, 3])
        t = background_time(r, f[:, 4], self.v0, self.kz)
        return t, t / self.q_ref


def training_targets(tab: LineTables, feat, bg: Background):
    """Targets (ms) of the table values: the corrections to the background."""
    t, q = bg.times(feat)
    y = np.empty((feat.shape[0], 2), np.float32)
    y[:, 0] = (tab.ttt - t) * 1e3
    y[:, 1] = (tab.qqq - q) * 1e3
    return y


def feature_scaling(feat):
    lo, hi = feat.min(0).astype(np.float64), feat.max(0).astype(np.float64)
    span = hi - lo
    scale = np.where(span > 1e-3, 2.0 / np.maximum(span, 1e-3), 1e-3)
    return (0.5 * (lo + hi)).astype(np.float32), scale.astype(np.float32)


# ---------------------------------------------------------------------------
# training
# ---------------------------------------------------------------------------
@dataclass
class Surrogate:
    mlp: Mlp
    bg: Background
    history: list

    def predict(self, feat):
        """(T, t*) in seconds at the feature rows (float64 numpy)."""
        n = feat.shape[0]
        y = np.empty((n, 2), np.float32)
        chunk = 1 << 22
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            y[a:b] = self.mlp.forward(feat[a:b]).cpu().numpy()
        self.mlp.status()
        t, q = self.bg.times(feat)
        return t + y[:, 0].astype(np.float64) * 1e-3, q + y[:, 1].astype(np.float64) * 1e-3


def train(tabs, line_ys, bg: Background, *, fci: int = 1, steps: int = 4000,
          batch: int = 8192, lr: float = 2e-3, lr_end: float = 2e-5, seed: int = 0,
          device: int = 0, log_every: int = 250, w_out=(1.0, 25.0)) -> Surrogate:
    """Fit the network to the tables `tabs` of lines at model y `line_ys`
    (Adam, cosine learning-rate decay, uniformly drawn mini-batches).  The
    t* correction is weighted up (w_out) because t* is ~Q times smaller than
    the traveltime it is learned next to."""
    import torch
    feats, targs = [], []
    for tab, ly in zip(tabs, line_ys):
        f = table_nodes(tab, fci, ly)
        feats.append(f)
        targs.append(training_targets(tab, f, bg))
    feat = np.concatenate(feats)
    targ = np.concatenate(targs)
    mlp = Mlp(device, seed)
    shift, scale = feature_scaling(feat)
    mlp.set_scaling(shift, scale, w_out)
    dev = mlp.dev
    X = torch.from_numpy(feat).to(dev)
    Y = torch.from_numpy(targ).to(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    n = X.shape[0]
    bx = torch.empty((batch, 5), dtype=torch.float32, device=dev)
    by = torch.empty((batch, 2), dtype=torch.float32, device=dev)
    hist = []
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), generator=gen, device=dev)
        torch.index_select(X, 0, idx, out=bx)
        torch.index_select(Y, 0, idx, out=by)
        a = lr_end + 0.5 * (lr - lr_end) * (1.0 + np.cos(np.pi * s / steps))
        want = log_every > 0 and (s % log_every == 0 or s == steps - 1)
        loss = mlp.train_step(bx, by, a, want_loss=want)
        if want:
            hist.append((s, loss))
    mlp.status()
    return Surrogate(mlp, bg, hist)


# ---------------------------------------------------------------------------
# densified tables with the table gate
# ---------------------------------------------------------------------------
def _layout_like(coarse: LineTables, surf_dx: int, surf_dy: int, half_x: float,
                 half_y: float) -> LineTables:
    nxs = 2 * int(np.ceil(half_x / surf_dx)) + 1
    nys = 2 * int(np.ceil(half_y / surf_dy)) + 1
    ncell = coarse.nxg * coarse.nzg
    block = nys * nxs * coarse.nxi1 * coarse.nzi1
    desc = np.zeros(ncell, DESC_DTYPE)
    for k in range(ncell):
        desc[k] = (k * block, nys, nxs, surf_dy, surf_dx)
    return LineTables(coarse.cdp1, coarse.cdp2, coarse.dx, coarse.dz, coarse.nxg, coarse.nzg,
                      coarse.nxi1, coarse.nzi1, coarse.dzii, desc,
                      np.zeros(ncell * block, np.float32), np.zeros(ncell * block, np.float32))


def _coarse_bilinear(coarse: LineTables, c: int, fci: int, xs_f, ys_f, vals):
    """Bilinear interpolation of a coarse cell block vals [nys][nxs][nxi1][nzi1]
    at fine surface nodes -> [len(ys_f)][len(xs_f)][nxi1][nzi1], and the
    coarse patch index of each fine node."""
    ixg, izg = divmod(c, coarse.nzg)
    xs_c, ys_c = cell_surface_nodes(coarse, ixg, izg, fci)
    d = coarse.desc[c]
    fx = np.clip((xs_f - xs_c[0]) / float(d["dxs"]), 0.0, len(xs_c) - 1.0)
    fy = np.clip((ys_f - ys_c[0]) / float(d["dys"]), 0.0, len(ys_c) - 1.0)
    ix = np.minimum(fx.astype(int), len(xs_c) - 2)
    iy = np.minimum(fy.astype(int), len(ys_c) - 2)
    wx = (fx - ix)[None, :, None, None]
    wy = (fy - iy)[:, None, None, None]
    v00 = vals[iy][:, ix]
    v01 = vals[iy][:, ix + 1]
    v10 = vals[iy + 1][:, ix]
    v11 = vals[iy + 1][:, ix + 1]
    out = (1 - wy) * ((1 - wx) * v00 + wx * v01) + wy * ((1 - wx) * v10 + wx * v11)
    return out, ix, iy


def densify(sur: Surrogate, coarse: LineTables, *, fci: int, line_y: float, surf_dx: int,
            surf_dy: int, half_x: float, half_y: float, gate_ms: float = 2.0):
    """Tables at surface spacing (surf_dx, surf_dy) from the network, gated
    against the coarse tables.  Returns (tables, stats)."""
    fine = _layout_like(coarse, surf_dx, surf_dy, half_x, half_y)
    fc = table_nodes(coarse, fci, line_y)
    tc, qc = sur.predict(fc)
    ff = table_nodes(fine, fci, line_y)
    tf, qf = sur.predict(ff)
    gated = total = 0
    for c in range(coarse.nxg * coarse.nzg):
        ixg, izg = divmod(c, coarse.nzg)
        dc, df = coarse.desc[c], fine.desc[c]
        shp_c = (int(dc["nys"]), int(dc["nxs"]), coarse.nxi1, coarse.nzi1)
        shp_f = (int(df["nys"]), int(df["nxs"]), fine.nxi1, fine.nzi1)
        sc = slice(int(dc["idx"]), int(dc["idx"]) + int(np.prod(shp_c)))
        sf = slice(int(df["idx"]), int(df["idx"]) + int(np.prod(shp_f)))
        ct = coarse.ttt[sc].reshape(shp_c).astype(np.float64)
        cq = coarse.qqq[sc].reshape(shp_c).astype(np.float64)
        # network error at the coarse nodes, worst over the cell's points
        err = np.abs(tc[sc].reshape(shp_c) - ct).max(axis=(2, 3)) * 1e3
        patch = np.maximum(np.maximum(err[:-1, :-1], err[:-1, 1:]),
                           np.maximum(err[1:, :-1], err[1:, 1:]))
        xs_f, ys_f = cell_surface_nodes(fine, ixg, izg, fci)
        bt, ix, iy = _coarse_bilinear(coarse, c, fci, xs_f, ys_f, ct)
        bq, _, _ = _coarse_bilinear(coarse, c, fci, xs_f, ys_f, cq)
        bad = patch[iy][:, ix] > gate_ms                     # [nys_f][nxs_f]
        nt = tf[sf].reshape(shp_f)
        nq = qf[sf].reshape(shp_f)
        fine.ttt[sf] = np.where(bad[:, :, None, None], bt, nt).astype(np.float32).ravel()
        fine.qqq[sf] = np.where(bad[:, :, None, None], bq, nq).astype(np.float32).ravel()
        gated += int(bad.sum())
        total += bad.size
    stats = dict(gated_nodes=gated, surface_nodes=total,
                 coarse_rms_ms=float(np.sqrt(np.mean((tc - coarse.ttt) ** 2)) * 1e3),
                 coarse_max_ms=float(np.abs(tc - coarse.ttt).max() * 1e3))
    return fine, stats


def coarse_to_fine(coarse: LineTables, *, fci: int, surf_dx: int, surf_dy: int,
                   half_x: float, half_y: float) -> LineTables:
    """Plain bilinear resampling of coarse tables on the fine surface grid
    (what the imaging kernel's surface interpolation does with the coarse
    tables); used to measure the table method's own error at fine nodes."""
    fine = _layout_like(coarse, surf_dx, surf_dy, half_x, half_y)
    for c in range(coarse.nxg * coarse.nzg):
        ixg, izg = divmod(c, coarse.nzg)
        dc, df = coarse.desc[c], fine.desc[c]
        shp_c = (int(dc["nys"]), int(dc["nxs"]), coarse.nxi1, coarse.nzi1)
        sc = slice(int(dc["idx"]), int(dc["idx"]) + int(np.prod(shp_c)))
        xs_f, ys_f = cell_surface_nodes(fine, ixg, izg, fci)
        n = len(xs_f) * len(ys_f) * fine.nxi1 * fine.nzi1
        sf = slice(int(df["idx"]), int(df["idx"]) + n)
        for src, dst in ((coarse.ttt, fine.ttt), (coarse.qqq, fine.qqq)):
            v, _, _ = _coarse_bilinear(coarse, c, fci, xs_f, ys_f,
                                       src[sc].reshape(shp_c).astype(np.float64))
            dst[sf] = v.astype(np.float32).ravel()
    return fine
