"""Seeded reference-compat cases shared by the tests and the golden generator.

A case is a config-1 survey line imaged with the reference's stub kernel:
geometry, trace samples, aperture and dip fields, plus the derived
parameters computed by the oracle (whose sizes are pinned against the
reference's compiled npfar).  Extra traces exercise every gate branch:
outside the velocity-grid box, outside the y aperture, zero offset (azimuth
0) and columns outside the image block.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from q_psdm_b200 import synth  # noqa: E402

NTL, DT = 1000, np.float32(0.002)
THRESHOLD, CONTRACT, TAPERZONE = 600.0, 3.0, 8.0
F1, F4, FC = 1.0, 140.0, 40.0
DZII = 48.0


def _extra_traces(sv, rng):
    """Traces that hit the gate's reject and edge branches (SU cm integers)."""
    s = 1.0 / sv.scaled
    X, Y = synth.X0, synth.Y0
    rows = [
        (X - 5000, Y + 600, X + 600, Y + 600),      # source outside bbox (x)
        (X + 600, Y + 600, X + 600, Y + 9000),      # receiver outside bbox (y)
        (X + 600, Y + 200, X + 700, Y + 220),       # midpoint far from the line
        (X + 641.5, Y + 643, X + 641.5, Y + 643),   # zero offset -> azimuth 0
        (X + 640.3, Y + 640, X + 640.9, Y + 640),   # offset < 1 m
        (X + 1260, Y + 630, X + 1300, Y + 650),     # columns at the right edge
        (X - 200, Y + 640, X - 100, Y + 645),       # columns left of the image
    ]
    for _ in range(9):
        a = rng.uniform(0, 2 * np.pi)
        o = rng.uniform(10, 600)
        mx, my = rng.uniform(X + 100, X + 1200), rng.uniform(Y + 560, Y + 720)
        rows.append((mx - o * np.cos(a) / 2, my - o * np.sin(a) / 2,
                     mx + o * np.cos(a) / 2, my + o * np.sin(a) / 2))
    return np.rint(np.array(rows) * s).astype(np.int32)


def make_case(name: str = "small", seed: int = 7):
    """name: "small" (full line), "block" (an x block, wider aperture) or
    "singular" (a zero-offset trace exactly above image nodes: the
    ray-direction formula divides 0 by 0 at z = 0; the NaN tangent is
    rejected like any tangent outside the dip limits)."""
    sv = synth.config1(seed)
    rng = np.random.default_rng(seed)
    line = 64
    if name == "small":
        shots = [5, 10]
        ixstart, ixend = 0, sv.nxi
        half_x, half_y = 30, 20
        tcdp = (5, 120)
    elif name == "singular":
        shots = [5]
        ixstart, ixend = 0, sv.nxi
        half_x, half_y = 30, 20
        tcdp = (1, 128)
    elif name == "block":
        shots = [0, 15]
        ixstart, ixend = 40, 90
        half_x, half_y = 45, 60
        tcdp = (1, 128)
    else:
        raise ValueError(name)
    sx, sy, gx, gy = synth.trace_geometry(sv, shots)
    hdr = np.stack([sx, sy, gx, gy], axis=1).astype(np.int32)
    hdr = np.concatenate([hdr, _extra_traces(sv, rng)], axis=0)
    if name == "singular":
        s = 1.0 / sv.scaled
        X, Y = synth.X0, synth.Y0
        hdr = np.concatenate([hdr[:64], np.rint(np.array(
            [(X + 640, Y + 640, X + 640, Y + 640)]) * s).astype(np.int32), hdr[64:128]])
    ntr = hdr.shape[0]
    traces = rng.standard_normal((ntr, NTL)).astype(np.float32)

    st = O.derive_static(NTL, DT, THRESHOLD, CONTRACT, TAPERZONE)
    w = O.window_split(NTL, DT, F1, F4)
    iaz = O.iaztab(0.001)
    az = np.stack(synth.aperture_tables(half_x, half_y)).astype(np.int32)
    dips = np.stack([d.ravel() for d in synth.dip_fields(sv.nxi, sv.nzi, float(st["contract"]))])
    fxv, fyv = sv.fxv, sv.fyv
    fxi = fxv + (sv.fci - sv.fci) * sv.dxi
    cyi = sv.line_y(line)
    bbox = dict(fxv1=np.float32(fxv - 2000.0), exv1=np.float32(fxv + sv.nxi * sv.dxi + 2000.0),
                fyv1=np.float32(fyv - 1000.0), eyv1=np.float32(fyv + sv.nyi * sv.dyi + 1000.0))
    nxb = ixend - ixstart
    ref_args = dict(
        dyi=sv.dyi, dxi=sv.dxi, nxi=sv.nxi, nzi=sv.nzi, ntl=NTL, scaled=sv.scaled,
        fci=sv.fci, dzi=sv.dzi, dt=DT, fc=FC, eps=0.001, **bbox,
        nfft=st["nfft"], nffti=st["nffti"], dt1=st["dt1"], taperzone=st["taperzone"],
        lnG=st["lnG"], coef1=st["coef1"], coef2=st["coef2"], coef3=st["coef3"],
        coef4=st["coef4"], dzii=DZII, fxi=fxi, cyi=cyi, dw=w["dw"], itb1=w["itb1"],
        itb2=w["itb2"], nsb=w["nsb"], tdstart1=w["tdstart1"], tdstart2=w["tdstart2"],
        nf1=w["nf1"], tdmid=w["tdmid"], nww=w["nww"], ncoef1=w["ncoef1"],
        ixstart=ixstart, ixend=ixend, nxb=nxb, ttt_cdp1=tcdp[0], ttt_cdp2=tcdp[1])
    return dict(name=name, sv=sv, line=line, hdr=hdr, traces=traces, iaztab=iaz, az=az,
                dips=dips, nxb=nxb, nzi=sv.nzi, ixstart=ixstart, ixend=ixend,
                static=st, window=w, ref_args=ref_args, fxi=fxi, cyi=cyi, tcdp=tcdp,
                bbox=bbox)


def oracle_gate_params(case):
    a = case["ref_args"]
    az = case["az"]
    keep = [np.ascontiguousarray(case["iaztab"], np.int32)] + [
        np.ascontiguousarray(az[i], np.int32) for i in range(4)]
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    gp = O.GateParams(scaled=a["scaled"], fxv1=a["fxv1"], fyv1=a["fyv1"], exv1=a["exv1"],
                      eyv1=a["eyv1"], fxi=a["fxi"], cyi=a["cyi"], dxi=a["dxi"],
                      dyi=a["dyi"], eps=a["eps"], nzi=a["nzi"], ixstart=a["ixstart"],
                      ixend=a["ixend"], iaztab=ip(keep[0]), aznx1=ip(keep[1]),
                      aznx2=ip(keep[2]), azny1=ip(keep[3]), azny2=ip(keep[4]))
    gp._keep = keep
    return gp


def oracle_image_params(case):
    a = case["ref_args"]
    return O.ImageParams(nzi=a["nzi"], nxb=a["nxb"], ixstart=a["ixstart"], nt=a["nffti"],
                         dt1=a["dt1"], dxi=a["dxi"], dzi=a["dzi"], taperzone=a["taperzone"],
                         tcdp1=a["ttt_cdp1"] - a["fci"], tcdp2=a["ttt_cdp2"] - a["fci"])


def oracle_run(case):
    """Gate + stub image of the whole case through the C oracle.
    Returns (gate ints [ntr,8], geom [ntr,4], image [nxb,nzi] before /nsb, npt)."""
    gp = oracle_gate_params(case)
    ints, geom = O.gate_traces(gp, case["hdr"])
    ok = ints[:, 0] == 3
    ints3 = np.ascontiguousarray(ints[ok][:, [4, 5, 7]])
    img, npt = O.image_compat(oracle_image_params(case), geom[ok], ints3,
                              [case["dips"][i] for i in range(4)])
    return ints, geom, img.reshape(case["nxb"], case["nzi"]), npt


def engine_run(case, device=0, batches=None, big_endian=True, max_batch=4096):
    """Run the case through the C ABI (host records).  Returns (engine, image
    before /nsb, gate ints, geom, spectra re/im of the last batch)."""
    from q_psdm_b200 import engine as E
    import torch

    a = case["ref_args"]
    sv = case["sv"]
    p = E.static_params(nxi=sv.nxi, nzi=sv.nzi, ntl=NTL, dt=float(DT), dxi=sv.dxi,
                        dyi=sv.dyi, dzi=sv.dzi, fci=sv.fci, scaled=sv.scaled, fxv=sv.fxv,
                        fyv=sv.fyv, nxv=sv.nxi, nyv=sv.nyi, fc=FC, f1=F1, f4=F4,
                        threshold=THRESHOLD, contract=CONTRACT, taperzone=TAPERZONE,
                        dzii=DZII, max_batch=max_batch)
    eng = E.Engine(p, device=device)
    d = case["dips"].reshape(4, sv.nxi, sv.nzi)
    eng.set_line(fxi=case["fxi"], cyi=case["cyi"], dips=d, ttt_cdp1=case["tcdp"][0],
                 ttt_cdp2=case["tcdp"][1])
    az = case["az"]
    o = E.offset_params(p, case["ixstart"], case["ixend"], aznx1=az[0], aznx2=az[1],
                        azny1=az[2], azny2=az[3])
    eng.begin_offset(o)
    hdr = case["hdr"]
    rec = E.encode_su(hdr[:, 0], hdr[:, 1], hdr[:, 2], hdr[:, 3], case["traces"],
                      dt_us=int(round(float(DT) * 1e6)), scalco=sv.scalco,
                      big_endian=big_endian)
    ntr = rec.shape[0]
    if batches is None:
        batches = [ntr]
    c0 = 0
    for b in batches:
        eng.submit(rec[c0:c0 + b], big_endian=big_endian)
        c0 += b
    assert c0 == ntr
    img = eng.get_image(apply_nsb_scale=False)
    # device-side per-trace outputs hold the last launched batch only
    last = batches[-1] if batches[-1] <= max_batch else batches[-1] % max_batch or max_batch
    di, dg = eng.gate_device_ptrs()
    dre, dim = eng.spectra_device_ptrs()
    nww = o.nww
    ints = _d2h(di, (last, 8), torch.int32)
    geom = _d2h(dg, (last, 4), torch.float32)
    re = _d2h(dre, (last, 2 * nww), torch.float32)
    im = _d2h(dim, (last, 2 * nww), torch.float32)
    return eng, img, ints, geom, re, im


def _d2h(ptr, shape, dtype):
    """Copy engine-owned device memory into a numpy array."""
    import torch
    from tests.cuda_util import d2h
    npdt = {torch.int32: np.int32, torch.float32: np.float32}[dtype]
    return d2h(ptr, shape, npdt)
