"""ctypes front-end of the C oracle and of the reference's compiled CPU code.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` leg of ``bench.py`` as the checker.  The product
path (``q_psdm_b200``) never imports this module.

* ``liboracle.so``  -- C restatement of the reference path (qpsdm_oracle.c,
  physics_oracle.c), built by ``oracle/Makefile``.
* ``_ref/libqpsdm_refcpu.so`` -- the reference's own fft.cc / psdmpkg.cc /
  segy.cc compiled in place (present only where the reference sources were
  available when ``build()`` ran).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def ref_src() -> str:
    """Directory of the reference's sources: $QPSDM_REF_SRC, else the
    checkout's usual place."""
    return os.environ.get("QPSDM_REF_SRC", "/root/reference/src")


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so (and oracle/_ref when the reference is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
    src = ref_src()
    if ref is None:
        ref = os.path.isdir(src)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, f"REF={src}", "ref", "ref-gpu"], check=True)


class GateParams(C.Structure):
    _fields_ = [
        ("scaled", C.c_double),
        ("fxv1", C.c_float), ("fyv1", C.c_float),
        ("exv1", C.c_float), ("eyv1", C.c_float),
        ("fxi", C.c_double), ("cyi", C.c_double),
        ("dxi", C.c_float), ("dyi", C.c_float), ("eps", C.c_float),
        ("nzi", C.c_int), ("ixstart", C.c_int), ("ixend", C.c_int),
        ("iaztab", C.POINTER(C.c_int)),
        ("aznx1", C.POINTER(C.c_int)), ("aznx2", C.POINTER(C.c_int)),
        ("azny1", C.POINTER(C.c_int)), ("azny2", C.POINTER(C.c_int)),
    ]


class ImageParams(C.Structure):
    _fields_ = [
        ("nzi", C.c_int), ("nxb", C.c_int), ("ixstart", C.c_int), ("nt", C.c_int),
        ("dt1", C.c_float), ("dxi", C.c_float), ("dzi", C.c_float),
        ("taperzone", C.c_float),
        ("tcdp1", C.c_int), ("tcdp2", C.c_int),
    ]


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.orc_npfa.argtypes = [C.c_int]
        L.orc_npfar.argtypes = [C.c_int]
        L.orc_pfa_table.argtypes = [_i32p, C.c_int]
        L.orc_build_iaztab.argtypes = [C.c_float, _i32p, C.c_int]
        L.orc_derive_static.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float,
                                        C.c_float, _i32p, _f32p]
        L.orc_derive_static.restype = None
        L.orc_window_split.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float,
                                       _i32p, _f32p]
        L.orc_window_split.restype = None
        L.orc_gate_trace.argtypes = [C.POINTER(GateParams), C.c_int, C.c_int,
                                     C.c_int, C.c_int, _i32p, _f32p]
        L.orc_gate_trace_cap.argtypes = [C.POINTER(GateParams), C.c_int, C.c_int,
                                         C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _f32p]
        L.orc_gain.argtypes = [_f32p, C.c_int, C.c_float]
        L.orc_gain.restype = None
        L.orc_fetch_and_taper.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_fetch_and_taper.restype = None
        L.orc_rdft.argtypes = [_f32p, C.c_int, _f64p, _f64p]
        L.orc_rdft.restype = None
        L.orc_preprocess_trace.argtypes = [_f32p, C.c_int, C.c_float, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_float, _f32p, _f32p]
        L.orc_preprocess_trace.restype = None
        L.orc_image_compat.argtypes = [C.POINTER(ImageParams), C.c_int, _f32p,
                                       _i32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                       C.POINTER(C.c_longlong)]
        L.orc_image_compat.restype = None
        L.orc_scale_image.argtypes = [_f32p, C.c_longlong, C.c_int]
        L.orc_scale_image.restype = None
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def ref_cpu():
    """The reference's compiled CPU code, or None when it was not built."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libqpsdm_refcpu.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_npfar.argtypes = [C.c_int]
        R.ref_npfa.argtypes = [C.c_int]
        R.ref_pfarc.argtypes = [C.c_int, C.c_int, _f32p, _f32p]
        R.ref_pfarc.restype = None
        R.ref_fetch_and_taper.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p]
        R.ref_getscale.argtypes = [C.c_short]
        R.ref_getscale.restype = C.c_float
        R.ref_preprocess_traces.argtypes = [_f32p, C.c_int, C.c_int, C.c_float,
                                            C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_float, _f32p, _f32p,
                                            C.c_int]
        R.ref_preprocess_traces.restype = None
        _ref = R
    return _ref


# --------------------------------------------------------------------------
# thin numpy helpers
# --------------------------------------------------------------------------
def npfar(n: int) -> int:
    return lib().orc_npfar(int(n))


def iaztab(eps: float = 0.001) -> np.ndarray:
    tab = np.zeros(4096, np.int32)
    n = lib().orc_build_iaztab(eps, tab, tab.size)
    return tab[:n].copy()


def derive_static(ntl, dt, threshold=600.0, contract=3.0, taperzone=8.0):
    oi = np.zeros(2, np.int32)
    of = np.zeros(10, np.float32)
    lib().orc_derive_static(ntl, dt, threshold, contract, taperzone, oi, of)
    keys_f = ["df", "dw", "dt1", "lnG", "coef1", "coef2", "coef3", "coef4",
              "contract", "taperzone"]
    d = {"nfft": int(oi[0]), "nffti": int(oi[1])}
    d.update({k: np.float32(v) for k, v in zip(keys_f, of)})
    return d


def window_split(ntl, dt, f1=1.0, f4=140.0):
    oi = np.zeros(7, np.int32)
    of = np.zeros(5, np.float32)
    lib().orc_window_split(ntl, dt, f1, f4, oi, of)
    keys_i = ["itb1", "itb2", "nsb", "nf1", "nf4", "nww", "ncoef1"]
    keys_f = ["tdstart1", "tdstart2", "tdmid", "df", "dw"]
    d = {k: int(v) for k, v in zip(keys_i, oi)}
    d.update({k: np.float32(v) for k, v in zip(keys_f, of)})
    return d


def fetch_and_taper(data, it1, it2):
    data = np.ascontiguousarray(data, np.float32)
    out = np.zeros(it2 - it1 + 1, np.float32)
    lib().orc_fetch_and_taper(data, data.size, it1, it2, out)
    return out


def rdft(x):
    x = np.ascontiguousarray(x, np.float32)
    n = x.size
    re = np.zeros(n // 2 + 1)
    im = np.zeros(n // 2 + 1)
    lib().orc_rdft(x, n, re, im)
    return re + 1j * im


def preprocess_trace(trace, dt, w):
    """w: window_split() dict.  Returns (re, im) float32 [2*nww]."""
    trace = np.ascontiguousarray(trace, np.float32)
    nww = w["nww"]
    re = np.zeros(2 * nww, np.float32)
    im = np.zeros(2 * nww, np.float32)
    lib().orc_preprocess_trace(trace, trace.size, dt, w["itb1"], w["itb2"],
                               w["nsb"], w["nf1"], nww, w["dw"], re, im)
    return re, im


def gate_traces(gp: GateParams, hdr: np.ndarray, aperture: np.ndarray | None = None):
    """hdr [ntr,4] int32 (sx, sy, gx, gy); aperture: optional int32 [ntr,2]
    per-trace half-widths (cdps, lines) capping the azimuth tables.  Returns
    (ints [ntr,8], geom [ntr,4])."""
    hdr = np.ascontiguousarray(hdr, np.int32)
    ntr = hdr.shape[0]
    ints = np.zeros((ntr, 8), np.int32)
    geom = np.zeros((ntr, 4), np.float32)
    oi = np.zeros(8, np.int32)
    of = np.zeros(4, np.float32)
    L = lib()
    big = 2 ** 31 - 1
    for i in range(ntr):
        cx, cy = (big, big) if aperture is None else (int(aperture[i, 0]), int(aperture[i, 1]))
        L.orc_gate_trace_cap(C.byref(gp), int(hdr[i, 0]), int(hdr[i, 1]),
                             int(hdr[i, 2]), int(hdr[i, 3]), cx, cy, oi, of)
        ints[i] = oi
        geom[i] = of
    return ints, geom


def image_compat(ip: ImageParams, geom, ints3, dips, img=None):
    """Accumulate accepted traces.  geom [n,4] f32, ints3 [n,3] i32
    (ixi1, ixi2, izimin), dips (dipx1, dipx2, dipy1, dipy2) each [nxi*nzi]."""
    geom = np.ascontiguousarray(geom, np.float32)
    ints3 = np.ascontiguousarray(ints3, np.int32)
    if img is None:
        img = np.zeros(ip.nxb * ip.nzi, np.float32)
    npt = C.c_longlong(0)
    d = [np.ascontiguousarray(x, np.float32).ravel() for x in dips]
    lib().orc_image_compat(C.byref(ip), geom.shape[0], geom.ravel(), ints3.ravel(),
                           d[0], d[1], d[2], d[3], img, C.byref(npt))
    return img, int(npt.value)


# --------------------------------------------------------------------------
# physics mode (FP64)
# --------------------------------------------------------------------------
class PhysParams(C.Structure):
    _fields_ = [
        ("nzi", C.c_int), ("nxb", C.c_int), ("ixstart", C.c_int), ("nt", C.c_int),
        ("nbins", C.c_int),
        ("dt1", C.c_double), ("dxi", C.c_double), ("dzi", C.c_double),
        ("taperzone", C.c_double), ("dtstar", C.c_double), ("dzii", C.c_double),
        ("tcdp1", C.c_int), ("tcdp2", C.c_int),
        ("nxg", C.c_int), ("nzg", C.c_int), ("nxi1", C.c_int), ("nzi1", C.c_int),
    ]


def physics_filter(nfft, dt, f3, f4, fc, threshold, nbins, dtstar):
    """[nbins, nfft/2+1] complex128: (-i ww_k) A(pi f t*_b) e^{-2i f t*_b ln(f/fc)} / nfft.

    ww is the -i*w band ramp of qpsdm() (src/q-psdm.cu:1207-1250: w below
    n3, w(n3) cos^2 taper from n3 to n4, zero from n4); A is the gain-limited
    exponential whose constants qpsdm() derives from the threshold G
    (src/q-psdm.cu:1277-1283): e^x up to ln G, the quadratic
    G(1 + u - 2.5 u^2), u = x - ln G, up to ln G + 0.2, then 1.1 G."""
    nk = nfft // 2 + 1
    df = 1.0 / (nfft * float(dt))
    dw = 2 * np.pi * df
    n3 = int(float(np.float32(f3)) / df + 0.5)
    n4 = int(float(np.float32(f4)) / df + 0.5)
    k = np.arange(nk)
    ww = np.where(k < n3, k * dw,
                  np.where(k < n4, n3 * dw * np.cos((k - n3) / max(n4 - n3, 1) * np.pi / 2) ** 2,
                           0.0))
    G = float(threshold)
    lnG = np.log(G)
    f = k * df
    out = np.zeros((nbins, nk), np.complex128)
    with np.errstate(divide="ignore", invalid="ignore"):
        lnf = np.where(f > 0, np.log(np.where(f > 0, f, 1.0) / fc), 0.0)
    for b in range(nbins):
        ts = b * float(dtstar)
        x = np.pi * f * ts
        u = x - lnG
        a = np.where(x <= lnG, np.exp(np.minimum(x, lnG)),
                     np.where(x <= lnG + 0.2, G * (1 + u - 2.5 * u * u), 1.1 * G))
        out[b] = (-1j * ww) * a * np.exp(-2j * f * ts * lnf) / nfft
    out[:, 0] = 0.0
    return out


def physics_panels(traces, dt, nfft, nffti, filt, fp32: bool = False):
    """[ntr, nbins, nffti] compensated panels of float32 traces: float64, or
    with fp32 the same computation in single precision (float32 FFTs and a
    complex64 filter; the CPU baseline's panels)."""
    traces = np.ascontiguousarray(traces, np.float32)
    ntr, ntl = traces.shape
    x = np.empty_like(traces)
    L = lib()
    g = np.empty(ntl, np.float32)
    for i in range(ntr):
        g[:] = traces[i]
        L.orc_gain(g, ntl, dt)
        L.orc_fetch_and_taper(g, ntl, 0, ntl - 1, x[i])
    if fp32:
        X = np.fft.rfft(x, n=nfft, axis=1)
        f32 = filt.astype(np.complex64) * np.float32(nffti)
        out = np.empty((ntr, filt.shape[0], nffti), np.float32)
        for b in range(filt.shape[0]):
            out[:, b, :] = np.fft.irfft(X * f32[b][None, :], n=nffti, axis=1)
        return out
    X = np.fft.rfft(x.astype(np.float64), n=nfft, axis=1)
    out = np.empty((ntr, filt.shape[0], nffti))
    for b in range(filt.shape[0]):
        out[:, b, :] = np.fft.irfft(X * filt[b][None, :], n=nffti, axis=1) * nffti
    return out


def physics_image(pp: PhysParams, geom, ints3, panels, dips, tables, img=None):
    """FP64 image [nxb*nzi] of accepted traces; tables: dict with ttt_desc,
    qqq_desc (uint8 [n,16] or structured), ttt, qqq (float32)."""
    L = lib()
    if not hasattr(L, "_phys_bound"):
        L.orc_physics_image.argtypes = [C.POINTER(PhysParams), C.c_int, _f32p, _i32p, _f64p,
                                        _f32p, _f32p, _f32p, _f32p, C.c_void_p, _f32p,
                                        C.c_void_p, _f32p, _f64p, C.POINTER(C.c_longlong)]
        L.orc_physics_image.restype = None
        L._phys_bound = True
    if img is None:
        img = np.zeros(pp.nxb * pp.nzi)
    dtab = np.ascontiguousarray(tables["ttt_desc"]).view(np.uint8)
    qtab = np.ascontiguousarray(tables["qqq_desc"]).view(np.uint8)
    npt = C.c_longlong(0)
    d = [np.ascontiguousarray(x, np.float32).ravel() for x in dips]
    L.orc_physics_image(C.byref(pp), int(np.asarray(geom).shape[0]),
                        np.ascontiguousarray(geom, np.float32).ravel(),
                        np.ascontiguousarray(ints3, np.int32).ravel(),
                        np.ascontiguousarray(panels, np.float64).ravel(),
                        d[0], d[1], d[2], d[3], dtab.ctypes.data,
                        np.ascontiguousarray(tables["ttt"], np.float32), qtab.ctypes.data,
                        np.ascontiguousarray(tables["qqq"], np.float32), img, C.byref(npt))
    return img, int(npt.value)


class P32(C.Structure):
    """Parameters of orc_image_plain_fp32 (oracle/physics_fp32.c)."""
    _fields_ = [
        ("nzi", C.c_int), ("nxb", C.c_int), ("ixstart", C.c_int), ("nt", C.c_int),
        ("nbins", C.c_int),
        ("dt1", C.c_float), ("dxi", C.c_float), ("dzi", C.c_float),
        ("taperzone", C.c_float), ("dtstar", C.c_float), ("dzii", C.c_float),
        ("tcdp1", C.c_int), ("tcdp2", C.c_int),
        ("nxg", C.c_int), ("nzg", C.c_int), ("nxi1", C.c_int), ("nzi1", C.c_int),
    ]


def image_plain_fp32(p: P32, ints, geom, panels, dips, tables, img=None):
    """The FP32 restatement of the engine's plain physics kernel
    (physics_fp32.c): image [nxb*nzi] float32 accumulated in place, and the
    (point-traces, imaged) counts.  ints [ntr][8] and geom [ntr][4] are the
    gate's results of every trace; panels [ntr][nbins][nt] float32."""
    L = lib()
    if not hasattr(L, "_p32_bound"):
        L.orc_image_plain_fp32.argtypes = [C.POINTER(P32), C.c_int, _i32p, _f32p, _f32p,
                                           _f32p, C.c_size_t, C.c_void_p, _f32p, C.c_void_p,
                                           _f32p, _f32p, C.POINTER(C.c_longlong)]
        L.orc_image_plain_fp32.restype = None
        L._p32_bound = True
    if img is None:
        img = np.zeros(p.nxb * p.nzi, np.float32)
    dtab = np.ascontiguousarray(tables["ttt_desc"]).view(np.uint8)
    qtab = np.ascontiguousarray(tables["qqq_desc"]).view(np.uint8)
    dips = np.ascontiguousarray(np.stack([np.asarray(d, np.float32).ravel() for d in dips]))
    counts = (C.c_longlong * 2)(0, 0)
    L.orc_image_plain_fp32(C.byref(p), int(np.asarray(geom).shape[0]),
                           np.ascontiguousarray(ints, np.int32).ravel(),
                           np.ascontiguousarray(geom, np.float32).ravel(),
                           np.ascontiguousarray(panels, np.float32).ravel(), dips.ravel(),
                           dips.shape[1], dtab.ctypes.data,
                           np.ascontiguousarray(tables["ttt"], np.float32), qtab.ctypes.data,
                           np.ascontiguousarray(tables["qqq"], np.float32), img, counts)
    return img, int(counts[0]), int(counts[1])
