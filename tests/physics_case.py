"""Seeded physics-mode cases: config-1 geometry and data, analytic v(z)
tables (constant Q), run through the engine and through the FP64 oracle."""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from q_psdm_b200 import synth, tables  # noqa: E402

NTL, DT = 1000, np.float32(0.002)
THRESHOLD, CONTRACT, TAPERZONE = 600.0, 3.0, 8.0
F1, F3, F4 = 1.0, 130.0, 140.0
NBINS, DTSTAR = 16, 0.0015


def make_case(nshots: int = 2, seed: int = 3, shots=None, line: int = 64,
              half_x: int = 40, half_y: int = 30, ixstart: int = 0, ixend: int = 128,
              rstep: int = 1):
    """rstep > 1 keeps every rstep-th receiver of the spread (smaller cases
    with many shots)."""
    sv = synth.config1(seed)
    if rstep > 1:
        sv.receivers = sv.receivers[::rstep].copy()
    shots = list(range(5, 5 + nshots)) if shots is None else list(shots)
    sx, sy, gx, gy = synth.trace_geometry(sv, shots)
    hdr = np.stack([sx, sy, gx, gy], axis=1).astype(np.int32)
    traces = synth.make_traces(sv, shots)
    tab = tables.linear_gradient_tables(sv, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi,
                                        zmax=(sv.nzi - 1) * sv.dzi, sub=4, nxi1=16,
                                        half_x=1000.0, half_y=500.0)
    st = O.derive_static(NTL, DT, THRESHOLD, CONTRACT, TAPERZONE)
    az = np.stack(synth.aperture_tables(half_x, half_y)).astype(np.int32)
    dips = np.stack([d.ravel() for d in synth.dip_fields(sv.nxi, sv.nzi, float(st["contract"]))])
    return dict(sv=sv, line=line, hdr=hdr, traces=traces, tab=tab, static=st, az=az,
                dips=dips, fxi=sv.fxv, cyi=sv.line_y(line), ixstart=ixstart, ixend=ixend,
                nxb=ixend - ixstart, fc=sv.fpeak)


def gate(case):
    sv = case["sv"]
    az = case["az"]
    keep = [np.ascontiguousarray(O.iaztab(), np.int32)] + [np.ascontiguousarray(az[i]) for i in range(4)]
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    # the data scale: the survey's, or a caller's (the driver takes it from
    # getscale in single precision, as the reference)
    gp = O.GateParams(scaled=case.get("scaled", sv.scaled), fxv1=np.float32(sv.fxv - 2000.0),
                      fyv1=np.float32(sv.fyv - 1000.0),
                      exv1=np.float32(sv.fxv + sv.nxi * sv.dxi + 2000.0),
                      eyv1=np.float32(sv.fyv + sv.nyi * sv.dyi + 1000.0), fxi=case["fxi"],
                      cyi=case["cyi"], dxi=sv.dxi, dyi=sv.dyi, eps=0.001, nzi=sv.nzi,
                      ixstart=case["ixstart"], ixend=case["ixend"], iaztab=ip(keep[0]),
                      aznx1=ip(keep[1]), aznx2=ip(keep[2]), azny1=ip(keep[3]),
                      azny2=ip(keep[4]))
    return O.gate_traces(gp, case["hdr"])


def oracle_run(case, nbins=NBINS, dtstar=DTSTAR):
    """FP64 image [nxb, nzi] and point-trace count."""
    sv = case["sv"]
    st = case["static"]
    ints, geom = gate(case)
    ok = ints[:, 0] == 3
    filt = O.physics_filter(st["nfft"], DT, F3, F4, case["fc"], THRESHOLD, nbins, dtstar)
    panels = O.physics_panels(case["traces"][ok], DT, st["nfft"], st["nffti"], filt)
    tab = case["tab"]
    pp = O.PhysParams(nzi=sv.nzi, nxb=case["nxb"], ixstart=case["ixstart"], nt=st["nffti"],
                      nbins=nbins, dt1=float(st["dt1"]), dxi=sv.dxi, dzi=sv.dzi,
                      taperzone=float(st["taperzone"]), dtstar=float(np.float32(dtstar)),
                      dzii=tab.dzii, tcdp1=tab.cdp1 - sv.fci, tcdp2=tab.cdp2 - sv.fci,
                      nxg=tab.nxg, nzg=tab.nzg, nxi1=tab.nxi1, nzi1=tab.nzi1)
    img, npt = O.physics_image(pp, geom[ok], ints[ok][:, [4, 5, 7]], panels,
                               [case["dips"][i] for i in range(4)], tab.as_engine_dict())
    return img.reshape(case["nxb"], sv.nzi), npt, ints


def engine(case, *, panel_dtype=0, kahan=0, nbins=NBINS, dtstar=DTSTAR, max_batch=4096,
           device=0, form=0, tile=(0, 0), use_graph=0, variant=0):
    from q_psdm_b200 import engine as E
    sv = case["sv"]
    p = E.static_params(nxi=sv.nxi, nzi=sv.nzi, ntl=NTL, dt=float(DT), dxi=sv.dxi, dyi=sv.dyi,
                        dzi=sv.dzi, fci=sv.fci, scaled=sv.scaled, fxv=sv.fxv, fyv=sv.fyv,
                        nxv=sv.nxi, nyv=sv.nyi, fc=case["fc"], f1=F1, f3=F3, f4=F4,
                        threshold=THRESHOLD, contract=CONTRACT, taperzone=TAPERZONE,
                        dzii=case["tab"].dzii, mode=1, panel_dtype=panel_dtype,
                        nbins=nbins, dtstar=dtstar, max_batch=max_batch, kahan=kahan,
                        form=form, tile_z=tile[0], tile_x=tile[1], use_graph=use_graph,
                        variant=variant)
    eng = E.Engine(p, device=device)
    d = case["dips"].reshape(4, sv.nxi, sv.nzi)
    eng.set_line(fxi=case["fxi"], cyi=case["cyi"], dips=d, tables=case["tab"].as_engine_dict())
    az = case["az"]
    o = E.offset_params(p, case["ixstart"], case["ixend"], aznx1=az[0], aznx2=az[1],
                        azny1=az[2], azny2=az[3])
    eng.begin_offset(o)
    return eng, p, o


def records(case, big_endian=True):
    from q_psdm_b200 import engine as E
    h = case["hdr"]
    return E.encode_su(h[:, 0], h[:, 1], h[:, 2], h[:, 3], case["traces"], dt_us=2000,
                       scalco=case["sv"].scalco, big_endian=big_endian)


def nrmse(a, ref):
    a = np.asarray(a, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.sqrt(np.mean((a - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))
