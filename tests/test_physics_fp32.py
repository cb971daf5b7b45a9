"""The FP32 restatement of the plain physics kernel (oracle/physics_fp32.c)
against the FP64 oracle (oracle/physics_oracle.c), on the CPU: the same
point-trace count (both use the engine's FP32 surface-grid test), and the
image within the FP32 tolerance of the GPU tests (5e-5) when both image the
same FP64 panels (rounded to float for the FP32 path)."""
import numpy as np

from oracle import oracle as O
from tests.physics_case import DT, DTSTAR, F3, F4, NBINS, THRESHOLD, gate, make_case, nrmse


def test_fp32_restatement_against_fp64():
    case = make_case(nshots=1, rstep=2)
    sv, st, tab = case["sv"], case["static"], case["tab"]
    ints, geom = gate(case)
    ok = ints[:, 0] == 3
    filt = O.physics_filter(st["nfft"], DT, F3, F4, case["fc"], THRESHOLD, NBINS, DTSTAR)
    pan = O.physics_panels(case["traces"][ok], DT, st["nfft"], st["nffti"], filt)
    pp = O.PhysParams(nzi=sv.nzi, nxb=case["nxb"], ixstart=case["ixstart"], nt=st["nffti"],
                      nbins=NBINS, dt1=float(st["dt1"]), dxi=sv.dxi, dzi=sv.dzi,
                      taperzone=float(st["taperzone"]), dtstar=float(np.float32(DTSTAR)),
                      dzii=tab.dzii, tcdp1=tab.cdp1 - sv.fci, tcdp2=tab.cdp2 - sv.fci,
                      nxg=tab.nxg, nzg=tab.nzg, nxi1=tab.nxi1, nzi1=tab.nzi1)
    ref, npt = O.physics_image(pp, geom[ok], ints[ok][:, [4, 5, 7]], pan,
                               [case["dips"][i] for i in range(4)], tab.as_engine_dict())
    # FP32 path: panels of every trace (zeros for rejected ones, never read)
    pan32 = np.zeros((ints.shape[0], NBINS, st["nffti"]), np.float32)
    pan32[ok] = pan
    a = O.P32(nzi=sv.nzi, nxb=case["nxb"], ixstart=case["ixstart"], nt=st["nffti"],
              nbins=NBINS, dt1=st["dt1"], dxi=sv.dxi, dzi=sv.dzi, taperzone=st["taperzone"],
              dtstar=DTSTAR, dzii=tab.dzii, tcdp1=tab.cdp1 - sv.fci, tcdp2=tab.cdp2 - sv.fci,
              nxg=tab.nxg, nzg=tab.nzg, nxi1=tab.nxi1, nzi1=tab.nzi1)
    img, n32, nimg = O.image_plain_fp32(a, ints, geom, pan32, case["dips"], tab.as_engine_dict())
    assert n32 == npt and 0 < nimg <= npt
    assert nrmse(img, ref) <= 5e-5
