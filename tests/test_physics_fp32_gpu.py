"""Physics mode, plain form, FP32 panels: the engine's image against the FP32
restatement of its kernel (oracle/physics_fp32.c), bit for bit.

Given the engine's own panels (qpsdm_panels_device_ptr) and the gate's
results (bit-exact against the oracle, tests/test_compat_gpu.py), the
restatement repeats every IEEE operation of the kernel: so the image, the
point-trace count and the count of imaged pairs must be identical.  That
pins the integer picks of the physics method (it1 = (int)(t / dt1), the t*
bin, the dip mask and the table-coverage test) exactly, the way the compat
path is pinned against the reference's own kernel.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.cuda_util import d2h
from tests.physics_case import engine, gate, make_case, records

pytestmark = pytest.mark.gpu


def _varied(case, lo_hi, seed):
    c = dict(case)
    rng = np.random.default_rng(seed)
    n = case["dips"].shape[1]
    lo = -rng.uniform(*lo_hi, size=(2, n)).astype(np.float32)
    hi = rng.uniform(*lo_hi, size=(2, n)).astype(np.float32)
    c["dips"] = np.stack([lo[0], hi[0], lo[1], hi[1]])
    return c


CASES = {
    "reference": lambda: make_case(nshots=2),
    "varied": lambda: _varied(make_case(nshots=2), (0.05, 0.35), 5),
    "steep": lambda: _varied(make_case(nshots=1, rstep=2), (2.0, 3.0), 6),
    "block": lambda: make_case(nshots=1, shots=[10], ixstart=30, ixend=100, half_x=60,
                               half_y=40),
}


@pytest.mark.parametrize("name", list(CASES))
def test_plain_fp32_bit_exact(cuda, name):
    case = CASES[name]()
    sv = case["sv"]
    rec = records(case)
    eng, p, o = engine(case, panel_dtype=0, form=0, max_batch=rec.shape[0])
    try:
        eng.submit(rec)
        img = np.asarray(eng.get_image(False), np.float32).ravel()
        st = eng.stats()
        d_pan, _ = eng.panels_device_ptrs()
        pan = d2h(d_pan, (rec.shape[0], p.nbins, p.nffti), np.float32)
    finally:
        eng.close()
    ints, geom = gate(case)
    tab = case["tab"]
    a = O.P32(nzi=sv.nzi, nxb=case["nxb"], ixstart=case["ixstart"], nt=p.nffti,
              nbins=p.nbins, dt1=p.dt1, dxi=p.dxi, dzi=p.dzi, taperzone=p.taperzone,
              dtstar=p.dtstar, dzii=p.dzii, tcdp1=tab.cdp1 - sv.fci, tcdp2=tab.cdp2 - sv.fci,
              nxg=tab.nxg, nzg=tab.nzg, nxi1=tab.nxi1, nzi1=tab.nzi1)
    ref, npt, nimg = O.image_plain_fp32(a, ints, geom, pan, case["dips"], tab.as_engine_dict())
    assert npt > 0 and nimg > 0
    assert st["point_traces"] == npt
    assert st["imaged"] == nimg
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32)), \
        f"{int((img != ref).sum())} points differ"
