"""The C ABI library on the CPU: it loads, exports every symbol the header
declares, derives the reference's parameters exactly, and refuses to run
without a GPU (no CPU fallback)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from q_psdm_b200 import _lib
from q_psdm_b200 import engine as E

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(qpsdm_\w+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = header_functions()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers them all
    bound = {s[0] for s in _lib.SYMBOLS}
    assert set(names) <= bound, set(names) - bound


def test_struct_sizes_match_c_layout():
    # offsets fixed by the header (x86-64 SysV): a change here breaks callers
    assert C.sizeof(_lib.TttDesc) == 16
    assert C.sizeof(_lib.OffsetParams) == 4 * 14 + 4 * 18 * 4 + 4
    assert _lib.StaticParams.scaled.offset == 24


def test_npfar_matches_oracle():
    for n in list(range(1, 20000, 7)) + [720720, 10 ** 6]:
        assert E.npfar(n) == O.npfar(n)


def test_iaztab_matches_oracle():
    assert np.array_equal(E.build_iaztab(0.001), O.iaztab(0.001))


@pytest.mark.parametrize("ntl,dt", [(1000, 0.002), (2000, 0.002), (2500, 0.002),
                                    (3000, 0.002), (1250, 0.004), (777, 0.001)])
def test_static_and_offset_params_match_oracle(ntl, dt):
    p = E.static_params(nxi=64, nzi=50, ntl=ntl, dt=dt, dxi=10, dyi=10, dzi=10,
                        fxv=0.0, fyv=0.0, nxv=64, nyv=64, threshold=800.0,
                        contract=8.0, taperzone=10.0)
    s = O.derive_static(ntl, np.float32(dt), 800.0, 8.0, 10.0)
    assert (p.nfft, p.nffti) == (s["nfft"], s["nffti"])
    for k in ("dt1", "lnG", "coef1", "coef2", "coef3", "coef4", "df", "dw"):
        assert np.float32(getattr(p, k)) == s[k], k
    assert np.float32(p.taperzone) == s["taperzone"]
    o = E.offset_params(p, 0, 64, aznx1=10, aznx2=10, azny1=5, azny2=5)
    w = O.window_split(ntl, np.float32(dt), 1.0, float(np.float32(p.f4)))
    for k in ("itb1", "itb2", "nsb", "nf1", "nww", "ncoef1"):
        assert getattr(o, k) == w[k], k
    for k in ("tdstart1", "tdstart2", "tdmid", "df", "dw"):
        assert np.float32(getattr(o, k)) == w[k], k


def test_nyquist_clamps_of_main():
    # src/q-psdm.cu:711-723: f3 <= nyq-10, f4 <= nyq-5, f4-f3 > 5
    p = E.static_params(nxi=8, nzi=20, ntl=500, dt=0.004, dxi=10, dyi=10, dzi=10,
                        fxv=0.0, fyv=0.0, nxv=8, nyv=8, f3=130.0, f4=140.0)
    assert np.isclose(p.f3, 115.0) and np.isclose(p.f4, 120.0)


def test_encode_su_header_fields():
    tr = np.arange(12, dtype=np.float32).reshape(2, 6)
    for be in (True, False):
        rec = E.encode_su([1, -2], [3, 4], [5, 6], [70000, -8], tr, dt_us=2000,
                          scalco=-100, big_endian=be)
        e = ">" if be else "<"
        assert rec.shape == (2, 240 + 24)
        assert rec[1, 72:76].view(e + "i4")[0] == -2
        assert rec[0, 84:88].view(e + "i4")[0] == 70000
        assert rec[0, 70:72].view(e + "i2")[0] == -100
        assert rec[0, 114:116].view(e + "u2")[0] == 6
        assert np.array_equal(rec[1, 240:].view(e + "f4"), tr[1])


def test_engine_refuses_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = E.static_params(nxi=8, nzi=20, ntl=100, dt=0.002, dxi=10, dyi=10, dzi=10,
                        fxv=0.0, fyv=0.0, nxv=8, nyv=8)
    with pytest.raises(E.QpsdmError):
        E.Engine(p)


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "q_psdm_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                src = open(os.path.join(dirpath, f)).read()
                for pat in (r"\bimport\s+oracle", r"\bfrom\s+oracle", r"liboracle",
                            r"libqpsdm_ref", r"oracle/_ref", r"orc_\w+\("):
                    assert not re.search(pat, src), (f, pat)
