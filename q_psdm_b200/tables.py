"""Traveltime (ttt) and t* (qqq) tables in the reference's layout.

Format (src/q-psdm.cu:103-109, :2382-2627, example examples/traveltime/Lxxx.tidx):

* index file ``Lxxx.tidx`` / ``Lxxx.qidx``: header ``cdp1, cdp2 (int32),
  dx, dz (float32), nzg, nxg, nzi1, nxi1 (int32)``, then ``nxg*nzg``
  16-byte descriptors ``{int64 idx; uint16 nys, nxs, dys, dxs}``,
  descriptor of cell (ixg, izg) at ``ixg*nzg + izg`` (depth fastest, as the
  shipped index shows: apertures grow along each run of nzg records).
* data file ``L<line>.ttt`` / ``.qqq``: native float32; the block of a cell
  starts at ``idx`` and holds ``nys*nxs*nxi1*nzi1`` values.

The reference never states the order inside a block nor where a cell's
surface grid sits (its kernel stub never reads the tables).  This engine
fixes both, and the writer below follows them:

* block order ``[iys][ixs][ixl][izl]`` (depth fastest: "in each grid the z is
  contiguous", src/q-psdm.cu:1112-1114);
* the local surface grid is centred on the cell: node (iys, ixs) lies at
  ``x = xc + (ixs - (nxs-1)/2) * dxs``, ``y = (iys - (nys-1)/2) * dys``
  relative to the image line, with ``xc`` the x of the cell's middle cdp;
* image depth z maps to table node ``z / dzii`` (dzii the table depth
  spacing), cell ``izg = node / nzi1`` (src/q-psdm.cu:2344-2349), linear
  between nodes; surface positions are bilinear between grid nodes; a
  surface position outside a cell's grid has no table value (masked).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

DESC_DTYPE = np.dtype([("idx", "<i8"), ("nys", "<u2"), ("nxs", "<u2"),
                       ("dys", "<u2"), ("dxs", "<u2")])


@dataclass
class LineTables:
    cdp1: int          # absolute first cdp of the tables
    cdp2: int
    dx: float          # cdp spacing (m)
    dz: float          # stored in the header (velocity dz of the reference)
    nxg: int
    nzg: int
    nxi1: int          # cdps per cell
    nzi1: int          # depth nodes per cell
    dzii: float        # depth-node spacing (m)
    desc: np.ndarray   # DESC_DTYPE [nxg*nzg]
    ttt: np.ndarray    # float32
    qqq: np.ndarray    # float32 (t*, s), same layout and descriptors
    dev: dict | None = None  # device copies (torch tensors ttt, qqq), when kept

    def as_engine_dict(self):
        d = self.desc.view(np.uint8).reshape(-1, 16).copy()
        return dict(nxg=self.nxg, nzg=self.nzg, nxi1=self.nxi1, nzi1=self.nzi1,
                    cdp1=self.cdp1, cdp2=self.cdp2, ttt_desc=d, qqq_desc=d,
                    ttt=self.ttt, qqq=self.qqq)


def cell_surface_nodes(tab: LineTables, ixg: int, izg: int, fci: int):
    """(x, y) of every node of a cell's surface grid, relative to (fxi, line)."""
    d = tab.desc[ixg * tab.nzg + izg]
    xc = ((tab.cdp1 - fci) + ixg * tab.nxi1 + 0.5 * (tab.nxi1 - 1)) * tab.dx
    xs = xc + (np.arange(d["nxs"]) - 0.5 * (d["nxs"] - 1)) * d["dxs"]
    ys = (np.arange(d["nys"]) - 0.5 * (d["nys"] - 1)) * d["dys"]
    return xs, ys


def build_line_tables(time_fn, tstar_fn, *, fci: int, nxi: int, dxi: float, zmax: float,
                      dzii: float, nxi1: int, nzi1: int, surf_dx: int, surf_dy: int,
                      half_x: float, half_y: float, cdp1: int | None = None,
                      cdp2: int | None = None, dz_header: float = 8.0,
                      nz_cells: int | None = None) -> LineTables:
    """Tables of one image line.

    time_fn(px, py, x, z) / tstar_fn(...) give traveltime and t* from surface
    point (px, py) to image point (x, line, z); coordinates relative to the
    first image cdp and the line; broadcastable numpy arrays.  Each cell's
    surface grid spans +-half_x, +-half_y around the cell at surf_dx/surf_dy
    spacing (odd node counts)."""
    cdp1 = fci if cdp1 is None else cdp1
    cdp2 = fci + nxi - 1 if cdp2 is None else cdp2
    ncdp = cdp2 - cdp1 + 1
    nxg = -(-ncdp // nxi1)
    nnodes = int(np.floor(zmax / dzii)) + 2          # node below zmax for the lerp
    nzg = nz_cells or -(-nnodes // nzi1)
    nxs = 2 * int(np.ceil(half_x / surf_dx)) + 1
    nys = 2 * int(np.ceil(half_y / surf_dy)) + 1
    desc = np.zeros(nxg * nzg, DESC_DTYPE)
    block = nys * nxs * nxi1 * nzi1
    ttt = np.zeros(nxg * nzg * block, np.float32)
    qqq = np.zeros_like(ttt)
    tab = LineTables(cdp1, cdp2, dxi, dz_header, nxg, nzg, nxi1, nzi1, dzii, desc, ttt, qqq)
    off = 0
    for ixg in range(nxg):
        for izg in range(nzg):
            k = ixg * nzg + izg
            desc[k] = (off, nys, nxs, surf_dy, surf_dx)
            xs, ys = cell_surface_nodes(tab, ixg, izg, fci)
            x = ((cdp1 - fci) + ixg * nxi1 + np.arange(nxi1)) * dxi
            z = (izg * nzi1 + np.arange(nzi1)) * dzii
            PY, PX, X, Z = np.meshgrid(ys, xs, x, z, indexing="ij")
            ttt[off:off + block] = time_fn(PX, PY, X, Z).astype(np.float32).ravel()
            qqq[off:off + block] = tstar_fn(PX, PY, X, Z).astype(np.float32).ravel()
            off += block
    return tab


def linear_gradient_tables(sv, *, fci: int, nxi: int, dxi: float, zmax: float,
                           sub: int = 4, nxi1: int = 16, half_x: float = 900.0,
                           half_y: float = 900.0, line_y: float | None = None) -> LineTables:
    """Analytic v(z) = v0 + k z tables, subsampled `sub` times in depth and
    surface position relative to the 10 m grid; t* of the survey's Q model
    along the straight path (`synth.tstar`: t / Q for constant Q).  line_y:
    absolute y of the line (needed by a Q model that is not layered)."""
    from .synth import traveltime, tstar

    def tfn(px, py, x, z):
        return traveltime(sv, np.hypot(px - x, py), z)

    ly = sv.fyv if line_y is None else line_y

    def qfn(px, py, x, z):
        t = traveltime(sv, np.hypot(px - x, py), z)
        if sv.q_model is None:
            return t / sv.q
        return tstar(sv, sv.fxv + px, ly + py, sv.fxv + x, ly, z, t)

    dzii = sub * sv.dzi
    nnodes = int(np.floor(zmax / dzii)) + 2
    return build_line_tables(tfn, qfn, fci=fci, nxi=nxi, dxi=dxi, zmax=zmax, dzii=dzii,
                             nxi1=nxi1, nzi1=nnodes, surf_dx=int(sub * sv.dxi),
                             surf_dy=int(sub * sv.dyi), half_x=half_x, half_y=half_y)


# ---------------------------------------------------------------------------
# file I/O in the reference's format
# ---------------------------------------------------------------------------
def write_index(path: str, tab: LineTables) -> None:
    hdr = np.array([tab.cdp1, tab.cdp2], "<i4").tobytes()
    hdr += np.array([tab.dx, tab.dz], "<f4").tobytes()
    hdr += np.array([tab.nzg, tab.nxg, tab.nzi1, tab.nxi1], "<i4").tobytes()
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(tab.desc.tobytes())


def read_index(path: str):
    b = open(path, "rb").read()
    cdp1, cdp2 = np.frombuffer(b[:8], "<i4")
    dx, dz = np.frombuffer(b[8:16], "<f4")
    nzg, nxg, nzi1, nxi1 = np.frombuffer(b[16:32], "<i4")
    n = int(nxg) * int(nzg)
    if len(b) < 32 + 16 * n:
        raise ValueError(f"{path}: index size error ({len(b)} bytes for {n} cells)")
    desc = np.frombuffer(b[32:32 + 16 * n], DESC_DTYPE).copy()
    return dict(cdp1=int(cdp1), cdp2=int(cdp2), dx=float(dx), dz=float(dz), nzg=int(nzg),
                nxg=int(nxg), nzi1=int(nzi1), nxi1=int(nxi1), desc=desc)


def write_line(ttpath: str, line: int, tab: LineTables) -> None:
    os.makedirs(ttpath, exist_ok=True)
    write_index(os.path.join(ttpath, "Lxxx.tidx"), tab)
    write_index(os.path.join(ttpath, "Lxxx.qidx"), tab)
    tab.ttt.astype("=f4").tofile(os.path.join(ttpath, f"L{line}.ttt"))
    tab.qqq.astype("=f4").tofile(os.path.join(ttpath, f"L{line}.qqq"))


def load_line(ttpath: str, line: int, line1: int, line2: int, torq: str = "t") -> np.ndarray:
    """Data of `line`, linearly interpolated between the nearest existing line
    files below and above it within [line1, line2] (src/q-psdm.cu:2488-2600)."""
    suff = "ttt" if torq == "t" else "qqq"
    lo = next((l for l in range(line, line1 - 1, -1)
               if os.path.exists(os.path.join(ttpath, f"L{l}.{suff}"))), -1)
    hi = next((l for l in range(line, line2 + 1)
               if os.path.exists(os.path.join(ttpath, f"L{l}.{suff}"))), -1)
    if lo == -1 or hi == -1:
        raise FileNotFoundError(f"no {suff} table brackets line {line} in {ttpath}")
    a = np.fromfile(os.path.join(ttpath, f"L{lo}.{suff}"), "=f4")
    if lo == hi:
        return a
    b = np.fromfile(os.path.join(ttpath, f"L{hi}.{suff}"), "=f4")
    if b.size != a.size:
        raise ValueError("table sizes of the bracketing lines differ")
    c2 = np.float32(1.0 * (line - lo) / (hi - lo))
    c1 = np.float32(1.0 - c2)
    return (a * c1 + b * c2).astype(np.float32)


# ---------------------------------------------------------------------------
# tables from the eikonal / t* generator (GPU)
# ---------------------------------------------------------------------------
@dataclass
class GridModel:
    """Velocity (m/s) and 1/Q on [nz][ny][nx] nodes of spacing h, origin
    (ox, oy) at the surface, coordinates relative to the first image cdp (x)
    and the first image line (y).  (v0, kz) is the linear-gradient background
    that starts every source analytically."""
    vel: np.ndarray
    invq: np.ndarray
    h: float
    ox: float
    oy: float
    v0: float
    kz: float


def _layout(nxi, nxi1, nzi1, nxs, nys, surf_dx, surf_dy, nzg=1):
    ncdp = nxi
    nxg = -(-ncdp // nxi1)
    desc = np.zeros(nxg * nzg, DESC_DTYPE)
    block = nys * nxs * nxi1 * nzi1
    for k in range(nxg * nzg):
        desc[k] = (k * block, nys, nxs, surf_dy, surf_dx)
    return nxg, nzg, desc, block


def eikonal_line_tables(model: GridModel, *, fci: int, nxi: int, dxi: float, zmax: float,
                        line_y: float, dzii: float, nxi1: int = 16, surf_dx: int,
                        surf_dy: int, half_x: float, half_y: float, h: float | None = None,
                        batch: int = 128, init_radius: float | None = None,
                        device: int = 0, background: GridModel | None = None,
                        q_background: float | None = None, sampler=None,
                        keep_device: bool = False) -> LineTables:
    """Tables of the image line at model y = line_y, computed by the GPU
    eikonal / t* generator (qpsdm_eikonal_solve + qpsdm_eikonal_fill) in the
    reference layout; every distinct surface node of the cells' grids is one
    source, solved on its own local grid.

    With `background` (the linear-gradient model v0 + kz z of `model`, with
    constant Q = q_background) the first-order scheme's systematic error is
    cancelled: T = T_exact(bg) + T(model) - T(bg) and
    t* = t*(model) * t*_exact(bg) / t*(bg), the background solved on the same
    grids (batch by batch, next to the model's solve) and the correction
    applied on the device (qpsdm_eikonal_correct).

    sampler(d_T, d_S, d_Tb, d_Sb, grid, d_src, ns): called for every batch
    of sources while its solved grids are on the device (training samples of
    the surrogate; d_Tb, d_Sb are None without a background).  keep_device:
    the returned tables also carry the device copies (tab.dev = dict(ttt=,
    qqq=) as torch tensors)."""
    import ctypes as C

    import torch

    from . import _lib
    L = _lib.lib()
    h = h or model.h
    r0 = init_radius if init_radius is not None else 3.0 * h
    nnodes = int(np.floor(zmax / dzii)) + 2
    nxs = 2 * int(np.ceil(half_x / surf_dx)) + 1
    nys = 2 * int(np.ceil(half_y / surf_dy)) + 1
    nxg, nzg, desc, block = _layout(nxi, nxi1, nnodes, nxs, nys, surf_dx, surf_dy)
    tab = LineTables(fci, fci + nxi - 1, dxi, 8.0, nxg, nzg, nxi1, nnodes, dzii, desc,
                     np.zeros(nxg * nzg * block, np.float32),
                     np.zeros(nxg * nzg * block, np.float32))
    # distinct surface nodes -> sources
    pos, node_src = {}, []
    for c in range(nxg * nzg):
        xs, ys = cell_surface_nodes(tab, c // nzg, c % nzg, fci)
        for y in ys:
            for x in xs:
                key = (round(float(x), 3), round(float(line_y + y), 3))
                if key not in pos:
                    pos[key] = len(pos)
                node_src.append(pos[key])
    src_xy = np.array(list(pos.keys()), np.float32)
    nsrc = len(src_xy)
    node_base = np.arange(0, nxg * nzg + 1, dtype=np.int32) * (nys * nxs)
    cell_base = np.arange(0, nxg * nzg + 1, dtype=np.int64) * block
    # local grid of each source: the cells that use it and the line
    gx = int(np.ceil((2 * (half_x + nxi1 * dxi) + 4 * h) / h)) + 1
    gy = int(np.ceil((2 * half_y + 4 * h) / h)) + 1
    gz = int(np.ceil(zmax / h)) + 3
    grid = _lib.EikGrid(gx, gy, gz, h)
    oy = line_y - half_y - 2 * h
    fg = _lib.EikFillGeom(nxi1, nnodes, nzg, dxi, dzii, 0.0, line_y)
    dev = torch.device("cuda", device)
    models = [model] + ([background] if background is not None else [])
    d_models = []
    for m in models:
        d_models.append((torch.from_numpy(np.ascontiguousarray(m.vel, np.float32)).to(dev),
                         torch.from_numpy(np.ascontiguousarray(m.invq, np.float32)).to(dev),
                         _lib.EikModel(m.vel.shape[2], m.vel.shape[1], m.vel.shape[0], m.h,
                                       m.ox, m.oy, m.v0, m.kz)))
    d_desc = torch.from_numpy(desc.view(np.uint8).copy()).to(dev)
    d_cb = torch.from_numpy(cell_base).to(dev)
    d_nb = torch.from_numpy(node_base).to(dev)
    d_ns = torch.from_numpy(np.array(node_src, np.int32)).to(dev)
    n = gx * gy * gz
    nb = min(batch, nsrc)
    # per model: solved grids and the line's tables
    d_T = [torch.empty(nb * n, dtype=torch.float32, device=dev) for _ in models]
    d_S = [torch.empty(nb * n, dtype=torch.float32, device=dev) for _ in models]
    d_tab = [(torch.zeros(tab.ttt.size, dtype=torch.float32, device=dev),
              torch.zeros(tab.qqq.size, dtype=torch.float32, device=dev)) for _ in models]
    d_w = torch.empty(4 * nb * n + 4, dtype=torch.float32, device=dev)  # QPSDM_EIK_WORK_FLOATS
    for s0 in range(0, nsrc, nb):
        ns = min(nb, nsrc - s0)
        sp = np.zeros((ns, 4), np.float32)
        sp[:, 0:2] = src_xy[s0:s0 + ns]
        sp[:, 2] = sp[:, 0] - 0.5 * (gx - 1) * h
        sp[:, 3] = oy
        d_sp = torch.from_numpy(sp).to(dev)
        for k, (dv, dq, mdl) in enumerate(d_models):
            rc = L.qpsdm_eikonal_solve(dv.data_ptr(), dq.data_ptr(), C.byref(mdl),
                                       d_sp.data_ptr(), ns, C.byref(grid), r0,
                                       4 * (gx + gy + gz), d_w.data_ptr(), d_T[k].data_ptr(),
                                       d_S[k].data_ptr(), None)
            _lib.check(rc, what="eikonal_solve")
            rc = L.qpsdm_eikonal_fill(d_T[k].data_ptr(), d_S[k].data_ptr(), C.byref(grid),
                                      d_sp.data_ptr(), s0, ns, d_desc.data_ptr(),
                                      d_cb.data_ptr(), d_nb.data_ptr(), d_ns.data_ptr(),
                                      nxg * nzg, C.byref(fg), d_tab[k][0].data_ptr(),
                                      d_tab[k][1].data_ptr(), None)
            _lib.check(rc, what="eikonal_fill")
        if sampler is not None:
            bgT = d_T[1] if background is not None else None
            bgS = d_S[1] if background is not None else None
            sampler(d_T[0], d_S[0], bgT, bgS, grid, d_sp, ns)
    d_ttt, d_qqq = d_tab[0]
    if background is not None:
        ln = _lib.SurLine(nxg, nzg, nxi1, nnodes, 0, dxi, dzii, line_y, background.v0,
                          background.kz, q_background)
        dsc = np.ascontiguousarray(desc)
        rc = L.qpsdm_eikonal_correct(C.byref(ln), dsc.ctypes.data, d_ttt.data_ptr(),
                                     d_qqq.data_ptr(), d_tab[1][0].data_ptr(),
                                     d_tab[1][1].data_ptr(), int(tab.ttt.size),
                                     float(q_background), None)
        _lib.check(rc, what="eikonal_correct")
    torch.cuda.synchronize(dev)
    tab.ttt[:] = d_ttt.cpu().numpy()
    tab.qqq[:] = d_qqq.cpu().numpy()
    if keep_device:
        tab.dev = dict(ttt=d_ttt, qqq=d_qqq)
    return tab


def eikonal_cell_values(model: GridModel, background: GridModel, *, q_bg: float, sources,
                        cells, nxg: int, nzg: int, nxi1: int, nzi1: int, x_cdp1: float,
                        dxi: float, dzii: float, zmax: float, line_y: float, h: float,
                        half_x: float, half_y: float, device: int = 0):
    """Traveltime (s) from surface point sources[k] (model x, y) to every
    table point of cell cells[k] (distinct cells of a line's tables, nxg x nzg
    cells of nxi1 cdps x nzi1 depth nodes), background-corrected as the
    tables are: T = T_exact(bg) + T(model) - T(bg).  Returns [k][nxi1][nzi1]
    float64.  The solves run on local grids as in eikonal_line_tables (one
    batch), read back through qpsdm_eikonal_fill with one surface node per
    cell."""
    import ctypes as C

    import torch

    from . import _lib
    L = _lib.lib()
    dev = torch.device("cuda", device)
    ns = len(sources)
    ncell = nxg * nzg
    gx = int(np.ceil((2 * (half_x + nxi1 * dxi) + 4 * h) / h)) + 1
    gy = int(np.ceil((2 * half_y + 4 * h) / h)) + 1
    gz = int(np.ceil(zmax / h)) + 3
    grid = _lib.EikGrid(gx, gy, gz, h)
    n = gx * gy * gz
    sp = np.zeros((ns, 4), np.float32)
    sp[:, 0:2] = np.asarray(sources, np.float32)
    sp[:, 2] = sp[:, 0] - 0.5 * (gx - 1) * h   # local grids as eikonal_line_tables'
    sp[:, 3] = line_y - half_y - 2 * h
    block = nxi1 * nzi1
    desc = np.zeros(ncell, DESC_DTYPE)
    for c in range(ncell):
        desc[c] = (c * block, 1, 1, 1, 1)
    node_src = np.full(ncell, -(1 << 30), np.int32)
    node_src[np.asarray(cells, int)] = np.arange(ns, dtype=np.int32)
    d_sp = torch.from_numpy(sp).to(dev)
    d_desc = torch.from_numpy(desc.view(np.uint8).copy()).to(dev)
    d_cb = torch.from_numpy(np.arange(ncell + 1, dtype=np.int64) * block).to(dev)
    d_nb = torch.from_numpy(np.arange(ncell + 1, dtype=np.int32)).to(dev)
    d_ns = torch.from_numpy(node_src).to(dev)
    fg = _lib.EikFillGeom(nxi1, nzi1, nzg, dxi, dzii, x_cdp1, line_y)
    d_w = torch.empty(4 * ns * n + 4, dtype=torch.float32, device=dev)  # QPSDM_EIK_WORK_FLOATS
    out = []
    for m in (model, background):
        dv = torch.from_numpy(np.ascontiguousarray(m.vel, np.float32)).to(dev)
        dq = torch.from_numpy(np.ascontiguousarray(m.invq, np.float32)).to(dev)
        mdl = _lib.EikModel(m.vel.shape[2], m.vel.shape[1], m.vel.shape[0], m.h, m.ox, m.oy,
                            m.v0, m.kz)
        d_T = torch.empty(ns * n, dtype=torch.float32, device=dev)
        d_S = torch.empty(ns * n, dtype=torch.float32, device=dev)
        _lib.check(L.qpsdm_eikonal_solve(dv.data_ptr(), dq.data_ptr(), C.byref(mdl),
                                         d_sp.data_ptr(), ns, C.byref(grid), 3.0 * h,
                                         4 * (gx + gy + gz), d_w.data_ptr(), d_T.data_ptr(),
                                         d_S.data_ptr(), None), what="eikonal_solve")
        tt = torch.zeros(ncell * block, dtype=torch.float32, device=dev)
        qq = torch.zeros(ncell * block, dtype=torch.float32, device=dev)
        _lib.check(L.qpsdm_eikonal_fill(d_T.data_ptr(), d_S.data_ptr(), C.byref(grid),
                                        d_sp.data_ptr(), 0, ns, d_desc.data_ptr(),
                                        d_cb.data_ptr(), d_nb.data_ptr(), d_ns.data_ptr(), ncell,
                                        C.byref(fg), tt.data_ptr(), qq.data_ptr(), None),
                   what="eikonal_fill")
        out.append(tt.cpu().numpy().reshape(ncell, nxi1, nzi1).astype(np.float64))
    from .surrogate import background_time
    res = []
    for k, c in enumerate(cells):
        ixg, izg = divmod(int(c), nzg)
        x = x_cdp1 + (ixg * nxi1 + np.arange(nxi1)) * dxi
        z = (izg * nzi1 + np.arange(nzi1)) * dzii
        X, Z = np.meshgrid(x, z, indexing="ij")
        r = np.hypot(X - sources[k][0], line_y - sources[k][1])
        ana = background_time(r, Z, background.v0, background.kz)
        res.append(ana + out[0][int(c)] - out[1][int(c)])
    return res
