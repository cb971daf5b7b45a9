"""The q-psdm driver end to end on the GPU: a reference-layout project on
disk in, the reference-named SU image and checkpoint markers out.

* compat (the reference's stub kernel): the image traces equal the oracle's
  image / nsb bit for bit, for the traces in the order the driver reads them
  (data-line files ascending); headers as the reference's fputtr block
  (src/q-psdm.cu:1766-1806);
* physics, batched FP16 panels, tables interpolated between two line files:
  image NRMSE against the FP64 oracle within the FP16 tolerance;
* markers: <offspath>/break_point.txt = last line, <infopath>/<node>_<line>,
  <projpath>/0/<task>/<node>.
"""
import ctypes as C
import ctypes.util
import os

import numpy as np
import pytest

from oracle import oracle as O
from q_psdm_b200 import synth, tables
from tests import compat_case, physics_case
from tests.driver_case import DRIVER, check_params, make_project, read_su, run_driver

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")]
LINE = 65  # 1-based image line = the cases' 0-based line 64


def _tanf(x):
    """The C library's single-precision tangent (what the driver calls)."""
    libm = C.CDLL(ctypes.util.find_library("m"))
    libm.tanf.restype = C.c_float
    libm.tanf.argtypes = [C.c_float]
    return np.float32(libm.tanf(C.c_float(x)))


def _reorder(case, order):
    c = dict(case)
    c["hdr"] = np.ascontiguousarray(case["hdr"][order])
    c["traces"] = np.ascontiguousarray(case["traces"][order])
    return c


def test_compat_bit_exact_and_layout(cuda, tmp_path):
    case = compat_case.make_case("small")
    sv = case["sv"]
    tab = tables.build_line_tables(lambda px, py, x, z: np.zeros_like(x),
                                   lambda px, py, x, z: np.zeros_like(x), fci=1, nxi=sv.nxi,
                                   dxi=sv.dxi, zmax=100.0, dzii=48.0, nxi1=16, nzi1=4,
                                   surf_dx=200, surf_dy=200, half_x=200.0, half_y=200.0,
                                   cdp1=case["tcdp"][0], cdp2=case["tcdp"][1])
    paths, order = make_project(str(tmp_path), case, image_line=LINE, tab=tab,
                                par_extra="aperx=30\napery=20\nfc=40")
    p = check_params(paths)
    run_driver(paths)
    out = os.path.join(paths["proj"], "0", "mig", "result", f"node_0.off0.L{LINE}.su")
    hdr, img = read_su(out, sv.nzi)

    # the oracle on the same traces in the same order, same gate parameters
    c = _reorder(case, order)
    a = c["ref_args"]
    uni = [np.full(18, v, np.int32) for v in (30, 30, 20, 20)]
    keep = [np.ascontiguousarray(c["iaztab"], np.int32)] + uni
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    fxi = p["fxv"] + float(np.float32(0.0))
    cyi = p["fyv"] + float(np.float32((LINE - 1) * np.float32(p["dyi"])))
    assert p["scaled"] == float(np.float32(0.01))   # getscale(-100) in float
    gp = O.GateParams(scaled=p["scaled"], fxv1=np.float32(p["fxv"] - 2000.0),
                      fyv1=np.float32(p["fyv"] - 1000.0),
                      exv1=np.float32(p["fxv"] + sv.nxi * p["dxi"] + 2000.0),
                      eyv1=np.float32(p["fyv"] + sv.nyi * p["dyi"] + 1000.0), fxi=fxi, cyi=cyi,
                      dxi=p["dxi"], dyi=p["dyi"], eps=0.001, nzi=sv.nzi, ixstart=0,
                      ixend=sv.nxi, iaztab=ip(keep[0]), aznx1=ip(keep[1]), aznx2=ip(keep[2]),
                      azny1=ip(keep[3]), azny2=ip(keep[4]))
    ints, geom = O.gate_traces(gp, c["hdr"])
    ok = ints[:, 0] == 3
    assert ok.sum() > 100
    # the driver's dip limits: tanf of the double sum rounded to float
    crad = float(c["static"]["contract"])
    lo = _tanf(np.float32(-10 * 0.0174532925199 + crad))
    hi = _tanf(np.float32(10 * 0.0174532925199 - crad))
    n = sv.nxi * sv.nzi
    dips = [np.full(n, lo, np.float32), np.full(n, hi, np.float32),
            np.full(n, lo, np.float32), np.full(n, hi, np.float32)]
    ref, npt = O.image_compat(compat_case.oracle_image_params(c), geom[ok],
                              np.ascontiguousarray(ints[ok][:, [4, 5, 7]]), dips)
    ref = ref.reshape(sv.nxi, sv.nzi) / np.float32(c["window"]["nsb"])
    assert np.abs(ref).max() > 0
    assert np.array_equal(img, ref.astype(np.float32))

    # headers of the reference's output block
    assert list(hdr["tracl"]) == list(range(1, sv.nxi + 1))
    assert list(hdr["cdp"]) == list(range(1, sv.nxi + 1))
    assert (hdr["fldr"] == LINE).all() and (hdr["offset"] == 0).all()
    assert (hdr["ns"] == sv.nzi).all() and (hdr["dt"] == int(sv.dzi * 1000)).all()
    assert (hdr["trid"] == 1).all() and (hdr["nvs"] == 1).all() and (hdr["counit"] == 1).all()
    assert (hdr["scalco"] == sv.scalco).all()
    gx = np.rint((sv.fxv + np.arange(sv.nxi) * sv.dxi) / sv.scaled)
    assert np.array_equal(hdr["sx"], gx.astype(np.int32))
    assert np.array_equal(hdr["gx"], hdr["sx"]) and np.array_equal(hdr["gy"], hdr["sy"])

    # checkpoint markers
    bp = os.path.join(paths["proj"], "data0", "break_point.txt")
    assert open(bp).read().strip() == str(LINE)
    assert os.path.exists(os.path.join(paths["path"], f"node_0_{LINE}"))
    assert os.path.exists(os.path.join(paths["proj"], "0", "mig", "node"))
    # a second run replaces (not appends to) the output of the line
    run_driver(paths)
    hdr2, img2 = read_su(out, sv.nzi)
    assert img2.shape == img.shape and np.array_equal(img2, img)
    # resume=1 after the last line: nothing is imaged again
    r = run_driver(paths, "resume=1")
    assert "Start Image Line" not in r.stderr


def test_physics_batched_fp16_with_interpolated_tables(cuda, tmp_path):
    case = physics_case.make_case(nshots=2, half_x=40, half_y=30)
    sv = case["sv"]
    case["az"] = np.stack(synth.aperture_tables(40, 30, vary=False)).astype(np.int32)
    paths, order = make_project(
        str(tmp_path), case, image_line=LINE, tab=case["tab"], tables_at=[LINE - 4, LINE + 4],
        par_extra=(f"aperx=40\napery=30\nfc={case['fc']:g}\nengine=physics\nform=batched\n"
                   f"panels=fp16\nnbins={physics_case.NBINS}\ndtstar={physics_case.DTSTAR:g}\n"
                   f"dzii={case['tab'].dzii:g}"))
    run_driver(paths)
    out = os.path.join(paths["proj"], "0", "mig", "result", f"node_0.off0.L{LINE}.su")
    _, img = read_su(out, sv.nzi)
    c = _reorder(case, order)
    c["scaled"] = float(np.float32(0.01))   # getscale(-100) in float, as the driver
    ref, npt, _ = physics_case.oracle_run(c)
    nsb = O.window_split(physics_case.NTL, physics_case.DT, physics_case.F1,
                         physics_case.F4)["nsb"]
    ref = ref / np.float32(nsb)
    assert np.abs(ref).max() > 0 and np.isfinite(img).all()
    e = physics_case.nrmse(img, ref)
    print(f"driver physics batched FP16 NRMSE {e:.3e}")
    assert e <= 2.5e-4


@pytest.mark.parametrize("engine_args", [(), ("engine=physics", "form=batched", "panels=fp16")])
def test_brick_equals_line_by_line(cuda, tmp_path, engine_args):
    """brick=3 images lines 61, 65, 69 in one pass over the data; with
    extxline=3 each data line feeds only the image lines within 3 lines of it
    (the engine's per-submit line mask), so every line's output equals the
    line-by-line run's."""
    case = physics_case.make_case(nshots=2, half_x=40, half_y=30)
    paths, _ = make_project(
        str(tmp_path), case, image_line="61,65,69", tab=case["tab"], tables_at=[57, 73],
        extxline=3,
        par_extra=(f"aperx=40\napery=30\nfc={case['fc']:g}\nnbins={physics_case.NBINS}\n"
                   f"dtstar={physics_case.DTSTAR:g}\ndzii={case['tab'].dzii:g}"))
    res = os.path.join(paths["proj"], "0", "mig", "result")
    outs = {}
    for brick in (1, 3):
        run_driver(paths, f"brick={brick}", *engine_args)
        outs[brick] = {L: read_su(os.path.join(res, f"node_0.off0.L{L}.su"), case["sv"].nzi)[1]
                       for L in (61, 65, 69)}
    for L in (61, 65, 69):
        a, b = outs[1][L], outs[3][L]
        assert np.abs(a).max() > 0
        if not engine_args:
            assert np.array_equal(a, b), L            # compat: bit for bit
        else:
            assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max(), L
