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


# ---------------------------------------------------------------------------
# on the device: training samples from eikonal grids, gate and dense tables
# ---------------------------------------------------------------------------
class EikonalSamples:
    """Training samples drawn from the eikonal solver's grids while they are
    on the device: a sampler for `tables.eikonal_line_tables` (and any other
    loop over solved source batches).  Every batch of `ns` sources yields
    `per_source * ns` samples (qpsdm_eikonal_samples: uniform (source, node)
    pairs, background-corrected targets); the set of all sources x grid
    nodes is never formed."""

    def __init__(self, bg: Background, q_bg: float, per_source: int = 256, device: int = 0,
                 seed: int = 0):
        import torch
        self.torch = torch
        self.bg = bg
        self.q_bg = q_bg
        self.per_source = per_source
        self.dev = torch.device("cuda", device)
        self.seed = seed
        self.xs, self.ts = [], []
        self.sources = 0

    def __call__(self, d_T, d_S, d_Tb, d_Sb, grid, d_src, ns):
        torch = self.torch
        n = self.per_source * ns
        x = torch.empty((n, 5), dtype=torch.float32, device=self.dev)
        t = torch.empty((n, 2), dtype=torch.float32, device=self.dev)
        b = _lib.SurBackground(self.bg.v0, self.bg.kz, self.bg.q_ref, self.q_bg)
        ptr = lambda a: None if a is None else a.data_ptr()
        rc = _lib.lib().qpsdm_eikonal_samples(
            d_T.data_ptr(), d_S.data_ptr(), ptr(d_Tb), ptr(d_Sb), C.byref(grid),
            d_src.data_ptr(), ns, C.byref(b), (self.seed * 1000003 + len(self.xs)) & (2**64 - 1),
            n, x.data_ptr(), t.data_ptr(), None)
        _lib.check(rc, what="eikonal_samples")
        self.xs.append(x)
        self.ts.append(t)
        self.sources += ns

    def tensors(self):
        torch = self.torch
        return torch.cat(self.xs), torch.cat(self.ts)


def train_device(X, Y, bg: Background, *, steps: int = 4000, batch: int = 8192,
                 lr: float = 2e-3, lr_end: float = 2e-5, seed: int = 0, device: int = 0,
                 log_every: int = 500, w_out=(1.0, 25.0)) -> Surrogate:
    """`train` on samples already on the device (X [n][5], Y [n][2] torch
    float32, e.g. from EikonalSamples): Adam with cosine decay over uniformly
    drawn mini-batches, every step the library's tcgen05 kernels."""
    import torch
    mlp = Mlp(device, seed)
    lo = X.min(0).values.double().cpu().numpy()
    hi = X.max(0).values.double().cpu().numpy()
    span = hi - lo
    scale = np.where(span > 1e-3, 2.0 / np.maximum(span, 1e-3), 1e-3).astype(np.float32)
    mlp.set_scaling((0.5 * (lo + hi)).astype(np.float32), scale, w_out)
    gen = torch.Generator(device=mlp.dev)
    gen.manual_seed(seed)
    n = X.shape[0]
    bx = torch.empty((batch, 5), dtype=torch.float32, device=mlp.dev)
    by = torch.empty((batch, 2), dtype=torch.float32, device=mlp.dev)
    hist = []
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), generator=gen, device=mlp.dev)
        torch.index_select(X, 0, idx, out=bx)
        torch.index_select(Y, 0, idx, out=by)
        a = lr_end + 0.5 * (lr - lr_end) * (1.0 + np.cos(np.pi * s / steps))
        want = log_every > 0 and (s % log_every == 0 or s == steps - 1)
        loss = mlp.train_step(bx, by, a, want_loss=want)
        if want:
            hist.append((s, loss))
    mlp.status()
    return Surrogate(mlp, bg, hist)


def layout(nxg: int, nzg: int, nxi1: int, nzi1: int, *, surf_dx: int, surf_dy: int,
           half_x: float, half_y: float):
    """Descriptors (DESC_DTYPE [nxg*nzg]) and total length of tables whose
    cells all have the surface grid +-half_x, +-half_y at (surf_dx, surf_dy)."""
    nxs = 2 * int(np.ceil(half_x / surf_dx)) + 1
    nys = 2 * int(np.ceil(half_y / surf_dy)) + 1
    block = nys * nxs * nxi1 * nzi1
    desc = np.zeros(nxg * nzg, DESC_DTYPE)
    for k in range(nxg * nzg):
        desc[k] = (k * block, nys, nxs, surf_dy, surf_dx)
    return desc, nxg * nzg * block


def _sur_line(sur: Surrogate, tab: LineTables, fci: int, line_y: float):
    return _lib.SurLine(tab.nxg, tab.nzg, tab.nxi1, tab.nzi1, tab.cdp1 - fci, tab.dx, tab.dzii,
                        line_y, sur.bg.v0, sur.bg.kz, sur.bg.q_ref)


def gate_errors(sur: Surrogate, tabs, line_ys, *, fci: int = 1):
    """Node errors (ms, torch on the device) of the network against the
    tables of the given lines (all with the same layout), the maximum over
    the lines: qpsdm_surrogate_gate.  Table data from tab.dev when present."""
    import torch
    t0 = tabs[0]
    nodes = int(sum(int(d["nys"]) * int(d["nxs"]) for d in t0.desc))
    err = torch.zeros(nodes, dtype=torch.float32, device=sur.mlp.dev)
    for tab, ly in zip(tabs, line_ys):
        ttt = tab.dev["ttt"] if tab.dev is not None else torch.from_numpy(tab.ttt).to(sur.mlp.dev)
        ln = _sur_line(sur, tab, fci, ly)
        d = np.ascontiguousarray(tab.desc)
        rc = _lib.lib().qpsdm_surrogate_gate(sur.mlp.h, C.byref(ln), d.ctypes.data,
                                             ttt.data_ptr(), int(ttt.numel()), err.data_ptr(),
                                             None)
        _lib.check(rc, what="surrogate_gate")
    return err


def dense_tables_device(sur: Surrogate, coarse: LineTables, coarse_ttt, coarse_qqq, node_err,
                        *, fci: int, line_y: float, surf_dx: int, surf_dy: int, half_x: float,
                        half_y: float, gate_ms: float = 2.0):
    """Tables of the line at model y `line_y` on the surface grid (surf_dx,
    surf_dy, +-half_x, +-half_y) from the network, on the device
    (qpsdm_surrogate_tables): returns (engine table dict with torch data,
    gated fine nodes).  coarse_ttt / coarse_qqq (torch, device): the plain
    method's tables of this line in coarse's layout -- the fallback in the
    patches whose corner nodes the network missed by more than gate_ms."""
    import torch
    fdesc, flen = layout(coarse.nxg, coarse.nzg, coarse.nxi1, coarse.nzi1, surf_dx=surf_dx,
                         surf_dy=surf_dy, half_x=half_x, half_y=half_y)
    dev = sur.mlp.dev
    ft = torch.empty(flen, dtype=torch.float32, device=dev)
    fq = torch.empty(flen, dtype=torch.float32, device=dev)
    ln = _sur_line(sur, coarse, fci, line_y)
    cd = np.ascontiguousarray(coarse.desc)
    gated = C.c_int64()
    rc = _lib.lib().qpsdm_surrogate_tables(
        sur.mlp.h, C.byref(ln), cd.ctypes.data, coarse_ttt.data_ptr(), coarse_qqq.data_ptr(),
        int(coarse_ttt.numel()), node_err.data_ptr(), float(gate_ms), fdesc.ctypes.data,
        ft.data_ptr(), fq.data_ptr(), int(flen), C.byref(gated), None)
    _lib.check(rc, what="surrogate_tables")
    d = fdesc.view(np.uint8).reshape(-1, 16).copy()
    return (dict(nxg=coarse.nxg, nzg=coarse.nzg, nxi1=coarse.nxi1, nzi1=coarse.nzi1,
                 cdp1=coarse.cdp1, cdp2=coarse.cdp2, ttt_desc=d, qqq_desc=d, ttt=ft, qqq=fq),
            int(gated.value))


def lerp_device(lo, hi, line: int, line_lo: int, line_hi: int):
    """Device copy of the tables of `line` interpolated between two lines'
    device tables, as get_ttt_all does (qpsdm_tables_lerp)."""
    import torch
    out = torch.empty_like(lo)
    rc = _lib.lib().qpsdm_tables_lerp(lo.data_ptr(), hi.data_ptr(), int(lo.numel()), int(line),
                                      int(line_lo), int(line_hi), out.data_ptr(), None)
    _lib.check(rc, what="tables_lerp")
    return out


def brick_tables(model, background, *, q_bg: float, table_lines, brick_lines, line_y_of,
                 fci: int, nxi: int, dxi: float, zmax: float, dzii: float, nxi1: int = 16,
                 coarse_dx: int, coarse_dy: int, fine_dx: int, fine_dy: int, half_x: float,
                 half_y: float, h: float, per_source: int = 512, steps: int = 4000,
                 batch: int = 8192, gate_ms: float = 2.0, device: int = 0, seed: int = 0,
                 batch_sources: int = 128):
    """The learned part end to end for a brick of image lines, on one GPU.

    1. Eikonal / t* tables (background-corrected) of the `table_lines` at the
       coarse surface spacing -- the table files the reference would read --
       while EikonalSamples draws training samples from every solved batch.
    2. The network trained on those samples (tcgen05 kernels).
    3. Its gate errors against the coarse tables of the table lines.
    4. For every brick line: the plain method's tables (coarse, interpolated
       between the bracketing table lines as get_ttt_all does, on the device)
       and the surrogate's tables at the fine surface spacing, gated.

    line_y_of(line) gives the model y of a line.  Returns a dict with the
    coarse LineTables (with device copies), per brick line the engine table
    dicts 'plain' and 'dense' (torch data), the trained Surrogate and timings."""
    import time

    import torch

    from . import tables as T
    dev = torch.device("cuda", device)
    bg = Background(background.v0, background.kz, q_bg)
    sampler = EikonalSamples(bg, q_bg, per_source=per_source, device=device, seed=seed)
    kw = dict(fci=fci, nxi=nxi, dxi=dxi, zmax=zmax, dzii=dzii, nxi1=nxi1, surf_dx=coarse_dx,
              surf_dy=coarse_dy, half_x=half_x, half_y=half_y, h=h, batch=batch_sources,
              device=device, background=background, q_background=q_bg, sampler=sampler,
              keep_device=True)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    coarse = [T.eikonal_line_tables(model, line_y=line_y_of(L), **kw) for L in table_lines]
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    X, Y = sampler.tensors()
    sur = train_device(X, Y, bg, steps=steps, batch=batch, seed=seed, device=device)
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()
    err = gate_errors(sur, coarse, [line_y_of(L) for L in table_lines], fci=fci)
    plain, dense, gated = [], [], 0
    for L in brick_lines:
        lo = max([t for t in table_lines if t <= L], default=None)
        hi = min([t for t in table_lines if t >= L], default=None)
        if lo is None or hi is None:
            raise ValueError(f"no table line brackets line {L}")
        a, b = coarse[table_lines.index(lo)], coarse[table_lines.index(hi)]
        ct = lerp_device(a.dev["ttt"], b.dev["ttt"], L, lo, hi)
        cq = lerp_device(a.dev["qqq"], b.dev["qqq"], L, lo, hi)
        d = a.as_engine_dict()
        d["ttt"], d["qqq"] = ct, cq
        plain.append(d)
        dd, g = dense_tables_device(sur, a, ct, cq, err, fci=fci, line_y=line_y_of(L),
                                    surf_dx=fine_dx, surf_dy=fine_dy, half_x=half_x,
                                    half_y=half_y, gate_ms=gate_ms)
        dense.append(dd)
        gated += g
    torch.cuda.synchronize(dev)
    t3 = time.perf_counter()
    fd = np.frombuffer(dense[0]["ttt_desc"].tobytes(), DESC_DTYPE)
    fine_nodes = int((fd["nys"].astype(np.int64) * fd["nxs"]).sum())
    return dict(coarse=coarse, plain=plain, dense=dense, surrogate=sur,
                stats=dict(eikonal_s=t1 - t0, train_s=t2 - t1, densify_s=t3 - t2,
                           sources=sampler.sources, samples=int(X.shape[0]),
                           train_steps=steps, train_batch=batch,
                           loss_first_last=[sur.history[0][1], sur.history[-1][1]],
                           gated_fine_nodes=gated,
                           fine_nodes=fine_nodes * len(brick_lines),
                           gated_fraction=gated / max(1, fine_nodes * len(brick_lines)),
                           max_gate_err_ms=float(err.max().item())))


def truth_error_sample(sur: Surrogate, model, background, *, q_bg: float, line_y: float,
                       plain_tables, fci: int, dxi: float, zmax: float, dzii: float,
                       fine_dx: int, fine_dy: int, half_x: float, half_y: float, h: float,
                       ncells: int = 32, seed: int = 0, device: int = 0):
    """Traveltime error (ms) of the surrogate and of the plain method's
    tables against the eikonal solver itself: in `ncells` seeded table cells
    of the line, one seeded node of the cell's fine surface grid is solved on
    its own local grid (background-corrected as the tables are) and compared
    at every table point of the cell with the network and with the plain
    tables (plain_tables: the engine dict of this line's coarse tables,
    bilinear in surface position as the kernels read them)."""
    from . import tables as T
    nxg, nzg = plain_tables["nxg"], plain_tables["nzg"]
    nxi1, nzi1 = plain_tables["nxi1"], plain_tables["nzi1"]
    cdesc = np.frombuffer(np.ascontiguousarray(plain_tables["ttt_desc"]).tobytes(), DESC_DTYPE)
    fdesc, _ = layout(nxg, nzg, nxi1, nzi1, surf_dx=fine_dx, surf_dy=fine_dy, half_x=half_x,
                      half_y=half_y)
    geo = LineTables(plain_tables["cdp1"], plain_tables["cdp2"], dxi, 8.0, nxg, nzg, nxi1, nzi1,
                     dzii, fdesc, np.zeros(0, np.float32), np.zeros(0, np.float32))
    rng = np.random.default_rng(seed)
    cells = np.sort(rng.choice(nxg * nzg, min(ncells, nxg * nzg), replace=False))
    srcs = []
    for c in cells:
        xs, ys = cell_surface_nodes(geo, int(c) // nzg, int(c) % nzg, fci)
        srcs.append((float(rng.choice(xs)), float(line_y + rng.choice(ys))))
    truth = T.eikonal_cell_values(model, background, q_bg=q_bg, sources=srcs, cells=cells,
                                  nxg=nxg, nzg=nzg, nxi1=nxi1, nzi1=nzi1,
                                  x_cdp1=(plain_tables["cdp1"] - fci) * dxi, dxi=dxi,
                                  dzii=dzii, zmax=zmax, line_y=line_y, h=h, half_x=half_x,
                                  half_y=half_y, device=device)
    ttt = plain_tables["ttt"]
    ttt = ttt.cpu().numpy() if hasattr(ttt, "cpu") else np.asarray(ttt)
    en, ep = [], []
    for c, (sx, sy), tt in zip(cells, srcs, truth):
        ixg, izg = divmod(int(c), nzg)
        x = ((plain_tables["cdp1"] - fci) + ixg * nxi1 + np.arange(nxi1)) * dxi
        z = (izg * nzi1 + np.arange(nzi1)) * dzii
        X, Z = np.meshgrid(x, z, indexing="ij")
        F = np.stack([np.full(X.size, sx), np.full(X.size, sy), X.ravel(),
                      np.full(X.size, line_y), Z.ravel()], 1).astype(np.float32)
        Tn, _ = sur.predict(F)
        en.append(Tn.reshape(nxi1, nzi1) - tt)
        # plain tables: bilinear between the cell's coarse surface nodes
        d = cdesc[c]
        xc = ((plain_tables["cdp1"] - fci) + ixg * nxi1 + 0.5 * (nxi1 - 1)) * dxi
        fx = (sx - xc) / float(d["dxs"]) + 0.5 * (int(d["nxs"]) - 1)
        fy = (sy - line_y) / float(d["dys"]) + 0.5 * (int(d["nys"]) - 1)
        if not (0 <= fx <= int(d["nxs"]) - 1 and 0 <= fy <= int(d["nys"]) - 1):
            continue
        ix, iy = min(int(fx), int(d["nxs"]) - 2), min(int(fy), int(d["nys"]) - 2)
        wx, wy = fx - ix, fy - iy
        blk = ttt[int(d["idx"]):int(d["idx"]) + int(d["nys"]) * int(d["nxs"]) * nxi1 * nzi1]
        blk = blk.reshape(int(d["nys"]), int(d["nxs"]), nxi1, nzi1).astype(np.float64)
        v = ((1 - wy) * ((1 - wx) * blk[iy, ix] + wx * blk[iy, ix + 1])
             + wy * ((1 - wx) * blk[iy + 1, ix] + wx * blk[iy + 1, ix + 1]))
        ep.append(v - tt)
    en = np.concatenate([e.ravel() for e in en]) * 1e3
    ep = np.concatenate([e.ravel() for e in ep]) * 1e3
    return dict(cells=len(cells), values=int(en.size),
                surrogate_rms_ms=float(np.sqrt(np.mean(en ** 2))),
                surrogate_max_ms=float(np.abs(en).max()),
                tables_rms_ms=float(np.sqrt(np.mean(ep ** 2))),
                tables_max_ms=float(np.abs(ep).max()))


# ---------------------------------------------------------------------------
# configuration 4: the network trained on source positions x volume points
# ---------------------------------------------------------------------------
def source_grid(n_side: int, spacing: float, x0: float = 0.0, y0: float = 0.0):
    """n_side x n_side surface source positions (model x, y) every `spacing` m."""
    g = x0 + np.arange(n_side) * spacing
    gy = y0 + np.arange(n_side) * spacing
    X, Y = np.meshgrid(g, gy, indexing="xy")
    return np.stack([X.ravel(), Y.ravel()], 1).astype(np.float32)


def _local_origin(src, n: int, h: float):
    """(ox, oy) of each source's n x n horizontal grid, centred on it (a
    source on the h lattice gets a grid on the same lattice)."""
    return np.asarray(src, np.float32) - np.float32(((n - 1) // 2) * h)


def _solve_grids(L, d_models, src, n: int, nz: int, h: float, max_batch: int, dev, on_batch):
    """Solves every source on its own n x n x nz grid (spacing h, centred on
    it), model and background, in batches; on_batch(d_T, d_S, d_Tb, d_Sb,
    grid, d_sp, s0, ns) sees each batch while it is on the device."""
    import ctypes as C

    import torch
    grid = _lib.EikGrid(n, n, nz, h)
    npt = n * n * nz
    nb = min(max_batch, len(src))
    d_T = [torch.empty(nb * npt, dtype=torch.float32, device=dev) for _ in d_models]
    d_S = [torch.empty(nb * npt, dtype=torch.float32, device=dev) for _ in d_models]
    d_w = torch.empty(4 * nb * npt + 4, dtype=torch.float32, device=dev)
    for s0 in range(0, len(src), nb):
        ns = min(nb, len(src) - s0)
        sp = np.zeros((ns, 4), np.float32)
        sp[:, 0:2] = src[s0:s0 + ns]
        sp[:, 2:4] = _local_origin(src[s0:s0 + ns], n, h)
        d_sp = torch.from_numpy(sp).to(dev)
        for k, (dv, dq, mdl) in enumerate(d_models):
            rc = L.qpsdm_eikonal_solve(dv.data_ptr(), dq.data_ptr(), C.byref(mdl),
                                       d_sp.data_ptr(), ns, C.byref(grid), 3.0 * h,
                                       4 * (2 * n + nz), d_w.data_ptr(), d_T[k].data_ptr(),
                                       d_S[k].data_ptr(), None)
            _lib.check(rc, what="eikonal_solve")
        on_batch(d_T[0], d_S[0], d_T[1], d_S[1], grid, d_sp, s0, ns)


def config4_eval_points(*, n_side: int, spacing: float, stride: int, n: int, nz: int,
                        h: float, held: int, held_nodes: int, seed: int):
    """Where configuration 4's network is evaluated: `held` seeded source
    positions on the h lattice between the solved sources (every `stride`-th
    of the n_side x n_side grid every `spacing` m), away from the grid's
    edge; the four solved sources around each (corners [4*held] in the order
    (0,0), (1,0), (0,1), (1,1)); and `held_nodes` seeded volume nodes per
    position, on the h lattice, inside the position's own n x n x nz grid and
    the corners' grids (grids centred on their source by _local_origin).
    Returns hx, hy, ix, iy (the lower corner's grid indices), step, corners,
    nodes [held][held_nodes][3] (x, y, z)."""
    rng = np.random.default_rng([seed, 4])
    step = spacing * stride
    lim = (n_side - 1) // stride * step
    hx = (np.round(rng.uniform(step, lim - step, held) / h) * h).astype(np.float32)
    hy = (np.round(rng.uniform(step, lim - step, held) / h) * h).astype(np.float32)
    ix = np.floor(hx / step).astype(int)
    iy = np.floor(hy / step).astype(int)
    corners = []
    for dy in (0, 1):
        for dx in (0, 1):
            corners.append(np.stack([(ix + dx) * step, (iy + dy) * step], 1))
    corners = np.concatenate(corners).astype(np.float32)
    half = ((n - 1) // 2) * h - step - h
    nodes = np.empty((held, held_nodes, 3), np.float64)
    for k in range(held):
        px = np.round((hx[k] + rng.uniform(-half, half, held_nodes)) / h) * h
        py = np.round((hy[k] + rng.uniform(-half, half, held_nodes)) / h) * h
        pz = rng.integers(1, nz, held_nodes) * h
        nodes[k] = np.stack([px, py, pz], 1)
    return hx, hy, ix, iy, step, corners, nodes


def config4_training(model, background, *, q_bg: float, n_side: int = 64,
                     spacing: float = 80.0, stride: int = 1, n: int = 256, nz: int = 201,
                     h: float = 20.0, per_source: int = 4096, steps: int = 4000,
                     batch: int = 8192, held: int = 16, held_nodes: int = 4096,
                     gate_ms: float = 2.0, max_batch: int = 16, device: int = 0,
                     seed: int = 0):
    """Configuration 4 end to end on one GPU: the network trained on the
    traveltimes and t* of a grid of surface source positions (n_side x
    n_side every `spacing` m; every `stride`-th in x and y is solved) to
    every node of an n x n x nz volume around each source (spacing h), from
    the eikonal / t* solver on `model` (background-corrected), then evaluated
    against the solver itself at `held` seeded source positions between the
    grid's sources, `held_nodes` seeded volume nodes each:

    * the network: T and t* predicted from (source, point);
    * the tables, as the imaging kernels read them: bilinear interpolation
      in source position between the four surrounding solved sources (the
      same grids, so the node lies on all five grids);
    * the gate: the share of evaluated nodes where the network misses by more
      than gate_ms (those would keep the tables).

    Samples (per_source per solved source, uniform over its volume) are drawn
    while each batch of grids is on the device; the set of sources x nodes
    (n_side^2 x n^2 nz) is never formed.  Returns the trained Surrogate and
    a dict of sizes, timings and errors (ms)."""
    import time

    import torch
    L = _lib.lib()
    dev = torch.device("cuda", device)
    src_all = source_grid(n_side, spacing)
    sel = np.zeros((n_side, n_side), bool)
    sel[::stride, ::stride] = True
    src = src_all[sel.ravel()]
    d_models = []
    for m in (model, background):
        d_models.append((torch.from_numpy(np.ascontiguousarray(m.vel, np.float32)).to(dev),
                         torch.from_numpy(np.ascontiguousarray(m.invq, np.float32)).to(dev),
                         _lib.EikModel(m.vel.shape[2], m.vel.shape[1], m.vel.shape[0], m.h,
                                       m.ox, m.oy, m.v0, m.kz)))
    bg = Background(background.v0, background.kz, q_bg)
    sampler = EikonalSamples(bg, q_bg, per_source=per_source, device=device, seed=seed)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    _solve_grids(L, d_models, src, n, nz, h, max_batch, dev,
                 lambda T, S, Tb, Sb, grid, sp, s0, ns: sampler(T, S, Tb, Sb, grid, sp, ns))
    torch.cuda.synchronize(dev)
    t1 = time.perf_counter()
    X, Y = sampler.tensors()
    sur = train_device(X, Y, bg, steps=steps, batch=batch, seed=seed, device=device)
    torch.cuda.synchronize(dev)
    t2 = time.perf_counter()

    hx, hy, ix, iy, step, corners, nodes = config4_eval_points(
        n_side=n_side, spacing=spacing, stride=stride, n=n, nz=nz, h=h, held=held,
        held_nodes=held_nodes, seed=seed)
    hsrc = np.stack([hx, hy], 1)

    def values(points_src, grids_T, grids_S, grids_Tb, grids_Sb, s0, ns, which):
        """Background-corrected (T, t*) of sources s0..s0+ns-1 at the evaluated
        nodes of `which[s]` (index into nodes)."""
        out_t, out_q = [], []
        Tm = grids_T.view(-1)
        for j in range(ns):
            s = points_src[s0 + j]
            k = which[s0 + j]
            o = _local_origin(s[None], n, h)[0]
            p = nodes[k]
            li = np.rint((p[:, 0] - o[0]) / h).astype(np.int64)
            lj = np.rint((p[:, 1] - o[1]) / h).astype(np.int64)
            lk = np.rint(p[:, 2] / h).astype(np.int64)
            idx = torch.from_numpy(j * n * n * nz + (lk * n + lj) * n + li).to(dev)
            T = Tm.index_select(0, idx).double().cpu().numpy()
            S = grids_S.view(-1).index_select(0, idx).double().cpu().numpy()
            Tb = grids_Tb.view(-1).index_select(0, idx).double().cpu().numpy()
            Sb = grids_Sb.view(-1).index_select(0, idx).double().cpu().numpy()
            r = np.hypot(p[:, 0] - s[0], p[:, 1] - s[1])
            te = background_time(r, p[:, 2], bg.v0, bg.kz)
            out_t.append(te + T - Tb)
            out_q.append(S * (te / q_bg) / np.where(Sb > 0, Sb, 1.0))
        return out_t, out_q

    pts = np.concatenate([hsrc, corners])
    which = np.concatenate([np.arange(held), np.tile(np.arange(held), 4)])
    got_t, got_q = [], []

    def on_batch(T, S, Tb, Sb, grid, sp, s0, ns):
        a, b = values(pts, T, S, Tb, Sb, s0, ns, which)
        got_t.extend(a)
        got_q.extend(b)
    _solve_grids(L, d_models, pts, n, nz, h, max_batch, dev, on_batch)
    truth_t, truth_q = got_t[:held], got_q[:held]
    c_t = [got_t[held * (1 + c):held * (2 + c)] for c in range(4)]
    c_q = [got_q[held * (1 + c):held * (2 + c)] for c in range(4)]
    wx = (hx - ix * step) / step
    wy = (hy - iy * step) / step
    en_t, en_q, et_t, et_q = [], [], [], []
    for k in range(held):
        p = nodes[k]
        F = np.stack([np.full(held_nodes, hx[k]), np.full(held_nodes, hy[k]), p[:, 0], p[:, 1],
                      p[:, 2]], 1).astype(np.float32)
        Tn, Qn = sur.predict(F)
        tab_t = ((1 - wy[k]) * ((1 - wx[k]) * c_t[0][k] + wx[k] * c_t[1][k])
                 + wy[k] * ((1 - wx[k]) * c_t[2][k] + wx[k] * c_t[3][k]))
        tab_q = ((1 - wy[k]) * ((1 - wx[k]) * c_q[0][k] + wx[k] * c_q[1][k])
                 + wy[k] * ((1 - wx[k]) * c_q[2][k] + wx[k] * c_q[3][k]))
        en_t.append(Tn - truth_t[k])
        en_q.append(Qn - truth_q[k])
        et_t.append(tab_t - truth_t[k])
        et_q.append(tab_q - truth_q[k])
    torch.cuda.synchronize(dev)
    t3 = time.perf_counter()
    ms = lambda e: np.concatenate(e) * 1e3
    en_t, en_q, et_t, et_q = ms(en_t), ms(en_q), ms(et_t), ms(et_q)
    rms = lambda e: float(np.sqrt(np.mean(e ** 2)))
    full = n_side * n_side * 256 * 256 * 201   # the configuration: 256^3 points (z: 4 km at 20 m)
    return sur, dict(
        sources=int(len(src)), sources_full=n_side * n_side, source_spacing_m=float(step),
        volume_nodes_per_source=n * n * nz, volume=f"{n} x {n} x {nz} nodes at {h:g} m",
        pairs_solved=int(len(src)) * n * n * nz, pairs_full=full,
        samples=int(X.shape[0]), train_steps=steps, train_batch=batch,
        eikonal_s=t1 - t0, train_s=t2 - t1, eval_s=t3 - t2,
        train_samples_per_s=steps * batch / (t2 - t1),
        loss_first_last=[sur.history[0][1], sur.history[-1][1]],
        evaluated=dict(sources=held, nodes=int(en_t.size)),
        traveltime_ms=dict(surrogate_rms=rms(en_t), surrogate_max=float(np.abs(en_t).max()),
                           tables_rms=rms(et_t), tables_max=float(np.abs(et_t).max())),
        tstar_ms=dict(surrogate_rms=rms(en_q), tables_rms=rms(et_q)),
        gated_fraction=float(np.mean(np.abs(en_t) > gate_ms)), gate_ms=gate_ms)
