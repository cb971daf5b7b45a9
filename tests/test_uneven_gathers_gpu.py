"""Shot gathers of uneven size and aperture in one persistent launch.

Configuration 3's geometry (nt 2500, smooth random Q layers): the smallest
and the largest gather near one image line (591 and 11,856 traces), each
with its own aperture (3.6 km and 1.4 km), submitted together through
qpsdm_submit_gathers: one gate launch and one persistent k_image_batched
launch for the 12,447 traces.  The image equals the FP64 oracle's (gate
with the same per-trace apertures; the oracle image summed over trace
chunks, since the image is additive over traces) within the configuration
bounds of the other tests (FP16 panels 4e-4, FP32 plain 1.5e-4), and the
point-trace counts are exact.  Without the per-trace apertures the count is
larger: the caps are what bounds the gathers.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from q_psdm_b200 import synth, tables

pytestmark = pytest.mark.gpu

LINE = 384
IX0, IX1 = 100, 580           # image block (columns) spanning both shots (columns 180, 468)
AP_M = {"small": 3600.0, "big": 1400.0}
DTSTAR = 0.0025


@pytest.fixture(scope="module")
def case():
    sv = synth.config3(seed=0)
    ly = sv.line_y(LINE)
    sizes = np.array([len(g) for g in sv.gathers])
    near = np.nonzero(np.abs(sv.shots[:, 1] - ly) < 600.0)[0]
    small = int(near[np.argmin(sizes[near])])
    big = int(near[np.argmax(sizes[near])])
    assert sizes[small] < 1000 and sizes[big] > 11000
    ids = [small, big]
    sx, sy, gx, gy = synth.trace_geometry(sv, ids)
    hdr = np.stack([sx, sy, gx, gy], 1).astype(np.int32)
    spos = np.stack([sx, sy], 1).astype(np.float64) * sv.scaled
    gpos = np.stack([gx, gy], 1).astype(np.float64) * sv.scaled
    traces = synth.pair_traces_device(sv, spos, gpos, device=0, seed=17)
    ap = []
    for name, sid in (("small", small), ("big", big)):
        a = AP_M[name]
        ap.append(np.repeat([[int(round(a / sv.dxi)), int(round(0.5 * a / sv.dyi))]],
                            sizes[sid], axis=0))
    ap = np.concatenate(ap).astype(np.int32)
    tab = tables.linear_gradient_tables(sv, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi,
                                        zmax=(sv.nzi - 1) * sv.dzi, sub=16, nxi1=16,
                                        half_x=2500.0, half_y=1500.0, line_y=ly)
    from q_psdm_b200.engine import encode_su
    rec = encode_su(sx, sy, gx, gy, traces, dt_us=2000, scalco=sv.scalco)
    return dict(sv=sv, ly=ly, hdr=hdr, traces=traces, ap=ap, tab=tab, rec=rec,
                sizes=(int(sizes[small]), int(sizes[big])))


def _gate_params(sv, ly, az):
    keep = [O.iaztab()] + [np.ascontiguousarray(az[i]) for i in range(4)]
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    gp = O.GateParams(scaled=sv.scaled, fxv1=np.float32(sv.fxv - 2000.0),
                      fyv1=np.float32(sv.fyv - 1000.0),
                      exv1=np.float32(sv.fxv + sv.nxi * sv.dxi + 2000.0),
                      eyv1=np.float32(sv.fyv + sv.nyi * sv.dyi + 1000.0), fxi=sv.fxv, cyi=ly,
                      dxi=sv.dxi, dyi=sv.dyi, eps=0.001, nzi=sv.nzi, ixstart=IX0, ixend=IX1,
                      iaztab=ip(keep[0]), aznx1=ip(keep[1]), aznx2=ip(keep[2]),
                      azny1=ip(keep[3]), azny2=ip(keep[4]))
    gp._keep = keep
    return gp


def _az():
    # the offset group's tables: the largest aperture (4 km), so that the
    # per-trace apertures are what bound the gathers
    return np.stack(synth.aperture_tables(400, 200)).astype(np.int32)


@pytest.fixture(scope="module")
def oracle_image(case):
    sv, tab = case["sv"], case["tab"]
    st = O.derive_static(sv.ntl, np.float32(sv.dt), sv.threshold, 3.0, 8.0)
    ints, geom = O.gate_traces(_gate_params(sv, case["ly"], _az()), case["hdr"], case["ap"])
    ok = np.nonzero(ints[:, 0] == 3)[0]
    filt = O.physics_filter(st["nfft"], np.float32(sv.dt), 130.0, 140.0, sv.fpeak,
                            sv.threshold, 16, DTSTAR)
    pp = O.PhysParams(nzi=sv.nzi, nxb=IX1 - IX0, ixstart=IX0, nt=st["nffti"], nbins=16,
                      dt1=float(st["dt1"]), dxi=sv.dxi, dzi=sv.dzi,
                      taperzone=float(st["taperzone"]), dtstar=float(np.float32(DTSTAR)),
                      dzii=tab.dzii, tcdp1=tab.cdp1 - sv.fci, tcdp2=tab.cdp2 - sv.fci,
                      nxg=tab.nxg, nzg=tab.nzg, nxi1=tab.nxi1, nzi1=tab.nzi1)
    dips = [d.ravel() for d in synth.dip_fields(sv.nxi, sv.nzi, float(st["contract"]))]
    img = np.zeros((IX1 - IX0) * sv.nzi, np.float64)
    npt = 0
    for c0 in range(0, ok.size, 1000):   # the image is additive over traces
        sel = ok[c0:c0 + 1000]
        pan = O.physics_panels(case["traces"][sel], np.float32(sv.dt), st["nfft"],
                               st["nffti"], filt)
        part, n = O.physics_image(pp, geom[sel], ints[sel][:, [4, 5, 7]], pan, dips,
                                  tab.as_engine_dict())
        img += np.asarray(part, np.float64)
        npt += n
    assert npt > 0
    return img.reshape(IX1 - IX0, sv.nzi), npt, int(ok.size)


def _engine(case, form, dtype, use_graph=0):
    from q_psdm_b200 import engine as E
    sv, tab = case["sv"], case["tab"]
    p = E.static_params(nxi=sv.nxi, nzi=sv.nzi, ntl=sv.ntl, dt=float(sv.dt), dxi=sv.dxi,
                        dyi=sv.dyi, dzi=sv.dzi, fci=sv.fci, scaled=sv.scaled, fxv=sv.fxv,
                        fyv=sv.fyv, nxv=sv.nxi, nyv=sv.nyi, fc=sv.fpeak,
                        threshold=sv.threshold, mode=1, panel_dtype=dtype, nbins=16,
                        dtstar=DTSTAR, form=form, dzii=tab.dzii, max_batch=len(case["hdr"]),
                        variant=1 if form == 1 else 0, use_graph=use_graph)
    eng = E.Engine(p, device=0)
    eng.set_lines([dict(fxi=sv.fxv, cyi=case["ly"],
                        dips=synth.dip_fields(sv.nxi, sv.nzi, p.contract),
                        tables=tab.as_engine_dict())])
    az = _az()
    eng.begin_offset(E.offset_params(p, IX0, IX1, aznx1=az[0], aznx2=az[1], azny1=az[2],
                                     azny2=az[3]))
    return eng


def _nrmse(a, ref):
    a = np.asarray(a, np.float64).reshape(ref.shape)
    return float(np.sqrt(np.mean((a - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))


@pytest.mark.parametrize("form,dtype,tol", [(1, 2, 4e-4), (0, 0, 1.5e-4)])
def test_uneven_gathers_one_launch_match_fp64(cuda, case, oracle_image, form, dtype, tol):
    from q_psdm_b200 import _lib
    ref, npt_ref, nacc_ref = oracle_image
    eng = _engine(case, form, dtype)
    try:
        eng.profile(True)
        eng.submit_gathers(case["rec"], case["ap"])
        img = eng.get_image(False)
        st = eng.stats()
        launches = eng.kernel_time(_lib.K_IMAGE)[1]
    finally:
        eng.close()
    print(f"form {form}: gathers {case['sizes']}, accepted {st['accepted']}, "
          f"point-traces {st['point_traces']}, image launches {launches}, "
          f"NRMSE {_nrmse(img, ref):.3e}")
    assert st["accepted"] == nacc_ref
    assert st["point_traces"] == npt_ref
    if form == 1:
        assert launches == 1   # both gathers in one persistent launch
    assert _nrmse(img, ref) <= tol


def test_apertures_bound_the_gathers(cuda, case, oracle_image):
    """The same traces without their apertures: the offset group's 4 km
    tables alone accept more pairs."""
    _, npt_ref, _ = oracle_image
    eng = _engine(case, 1, 2)
    try:
        eng.submit(case["rec"])
        eng.fence()
        n = eng.stats()["point_traces"]
    finally:
        eng.close()
    assert n > npt_ref


def test_device_apertures_under_graph_replay(cuda, case, oracle_image):
    """Records and apertures resident on the device, the batch captured into
    a CUDA graph and replayed: every replay adds the same image."""
    import torch
    ref, npt_ref, _ = oracle_image
    eng = _engine(case, 1, 2, use_graph=1)
    try:
        drec = torch.from_numpy(case["rec"]).cuda()
        dap = torch.from_numpy(case["ap"]).cuda()
        for _ in range(3):   # eager, captured, replayed
            eng.submit_gathers_device(drec.data_ptr(), dap.data_ptr(), len(case["hdr"]))
        img = eng.get_image(False)
        st = eng.stats()
    finally:
        eng.close()
    assert st["point_traces"] == 3 * npt_ref
    assert _nrmse(np.asarray(img, np.float64) / 3.0, ref) <= 4e-4
