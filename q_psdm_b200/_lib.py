"""ctypes binding of include/qpsdm_engine.h (libqpsdm_b200.so).

The structures below mirror the C header field by field.  Loading fails
loudly when the shared library is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libqpsdm_b200.so")

NAZ = 18
SU_HDR = 240
MODE_COMPAT, MODE_PHYSICS = 0, 1
K_GATE, K_PRE, K_IMAGE, K_OTHER = 0, 1, 2, 3
PANEL_FP32, PANEL_BF16, PANEL_FP16 = 0, 1, 2
ERRORS = {0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "ESTATE",
          5: "ETIMEOUT", 6: "ENOTSUP", 7: "ENOKERNEL", 8: "ESIZE"}


class TttDesc(C.Structure):
    _fields_ = [("idx", C.c_int64), ("nys", C.c_uint16), ("nxs", C.c_uint16),
                ("dys", C.c_uint16), ("dxs", C.c_uint16)]


class StaticParams(C.Structure):
    _fields_ = [
        ("dyi", C.c_float), ("dxi", C.c_float),
        ("nxi", C.c_int), ("nzi", C.c_int), ("ntl", C.c_int),
        ("scaled", C.c_double), ("fci", C.c_int), ("dzi", C.c_float),
        ("dt", C.c_float), ("fc", C.c_float),
        ("f1", C.c_float), ("f3", C.c_float), ("f4", C.c_float),
        ("threshold", C.c_float), ("contract", C.c_float), ("taperzone", C.c_float),
        ("fxv1", C.c_float), ("fyv1", C.c_float), ("exv1", C.c_float), ("eyv1", C.c_float),
        ("dzii", C.c_float),
        ("eps", C.c_float), ("nfft", C.c_int), ("nffti", C.c_int), ("dt1", C.c_float),
        ("df", C.c_float), ("dw", C.c_float),
        ("lnG", C.c_float), ("coef1", C.c_float), ("coef2", C.c_float),
        ("coef3", C.c_float), ("coef4", C.c_float),
        ("mode", C.c_int), ("panel_dtype", C.c_int), ("nbins", C.c_int),
        ("dtstar", C.c_float), ("max_batch", C.c_int), ("kahan", C.c_int),
        ("form", C.c_int), ("use_graph", C.c_int), ("tile_z", C.c_int), ("tile_x", C.c_int),
        ("variant", C.c_int), ("reserved", C.c_int * 3),
    ]


class LineParams(C.Structure):
    _fields_ = [
        ("fxi", C.c_double), ("cyi", C.c_double),
        ("dipx1", C.c_void_p), ("dipx2", C.c_void_p),
        ("dipy1", C.c_void_p), ("dipy2", C.c_void_p),
        ("nf3", C.c_void_p), ("q", C.c_void_p),
        ("nxg", C.c_int), ("nzg", C.c_int), ("nxi1", C.c_int), ("nzi1", C.c_int),
        ("ttt_cdp1", C.c_int), ("ttt_cdp2", C.c_int),
        ("ttt_desc", C.c_void_p), ("qqq_desc", C.c_void_p),
        ("ttt", C.c_void_p), ("qqq", C.c_void_p),
        ("ttt_len", C.c_int64), ("qqq_len", C.c_int64),
    ]


class OffsetParams(C.Structure):
    _fields_ = [
        ("ioffs", C.c_int), ("ixstart", C.c_int), ("ixend", C.c_int),
        ("itb1", C.c_int), ("itb2", C.c_int), ("nsb", C.c_int),
        ("tdstart1", C.c_float), ("tdstart2", C.c_float), ("tdmid", C.c_float),
        ("nf1", C.c_int), ("nww", C.c_int), ("ncoef1", C.c_int),
        ("df", C.c_float), ("dw", C.c_float),
        ("aznx1", C.c_int * NAZ), ("aznx2", C.c_int * NAZ),
        ("azny1", C.c_int * NAZ), ("azny2", C.c_int * NAZ),
        ("zero_image", C.c_int),
    ]


class EikModel(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("h", C.c_float),
                ("ox", C.c_float), ("oy", C.c_float), ("v0", C.c_float), ("kz", C.c_float)]


class EikGrid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("h", C.c_float)]


class EikFillGeom(C.Structure):
    _fields_ = [("nxi1", C.c_int), ("nzi1", C.c_int), ("nzg", C.c_int), ("dxi", C.c_float),
                ("dzii", C.c_float), ("x_cdp1", C.c_float), ("line_y", C.c_float)]


class SurBackground(C.Structure):
    _fields_ = [("v0", C.c_float), ("kz", C.c_float), ("q_ref", C.c_float), ("q_bg", C.c_float)]


class SurLine(C.Structure):
    _fields_ = [("nxg", C.c_int), ("nzg", C.c_int), ("nxi1", C.c_int), ("nzi1", C.c_int),
                ("tcdp1", C.c_int), ("dxi", C.c_float), ("dzii", C.c_float),
                ("line_y", C.c_float), ("v0", C.c_float), ("kz", C.c_float),
                ("q_ref", C.c_float)]


# (name, restype, argtypes) of every symbol include/qpsdm_engine.h declares.
_P, _I, _F, _V = C.c_void_p, C.c_int, C.c_float, C.c_void_p
SYMBOLS = [
    ("qpsdm_npfar", _I, [_I]),
    ("qpsdm_static_params_init", _I, [C.POINTER(StaticParams)]),
    ("qpsdm_build_iaztab", _I, [_F, _P, _I]),
    ("qpsdm_offset_params_init", _I, [C.POINTER(StaticParams), _I, _I, C.POINTER(OffsetParams)]),
    ("qpsdm_engine_create", _I, [C.POINTER(StaticParams), _P, _I, _I, C.POINTER(C.c_void_p)]),
    ("qpsdm_engine_destroy", _I, [_P]),
    ("qpsdm_last_error", C.c_char_p, [_P]),
    ("qpsdm_set_line", _I, [_P, C.POINTER(LineParams)]),
    ("qpsdm_set_lines", _I, [_P, C.POINTER(LineParams), _I]),
    ("qpsdm_begin_offset", _I, [_P, C.POINTER(OffsetParams)]),
    ("qpsdm_submit_traces", _I, [_P, _P, _I, _I, _I]),
    ("qpsdm_submit_traces_device", _I, [_P, _P, _I, _I, _I]),
    ("qpsdm_submit_gathers", _I, [_P, _P, _P, _I, _I, _I]),
    ("qpsdm_submit_gathers_device", _I, [_P, _P, _P, _I, _I, _I]),
    ("qpsdm_fence", _I, [_P]),
    ("qpsdm_set_line_mask", _I, [_P, C.c_ulonglong]),
    ("qpsdm_get_image", _I, [_P, _P, _I]),
    ("qpsdm_get_image_async", _I, [_P, _P, _I, C.POINTER(C.c_int64)]),
    ("qpsdm_image_wait", _I, [_P, C.c_int64]),
    ("qpsdm_image_device_ptr", _I, [_P, C.POINTER(C.c_void_p)]),
    ("qpsdm_set_stream", _I, [_P, _P]),
    ("qpsdm_tuning_info", _I, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.c_int), _P, _I]),
    ("qpsdm_profile_enable", _I, [_P, _I]),
    ("qpsdm_profile_get", _I, [_P, _I, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("qpsdm_get_counters", _I, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("qpsdm_get_stats", _I, [_P, _P, _I]),
    ("qpsdm_panels_device_ptr", _I, [_P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    ("qpsdm_spectra_device_ptr", _I, [_P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    ("qpsdm_gate_device_ptr", _I, [_P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    ("qpsdm_fft_r2c", _I, [_P, _I, _I, _P, _P]),
    ("qpsdm_fft_c2r", _I, [_P, _I, _I, _P, _P]),
    ("qpsdm_fft_r2c_noalloc", _I, [_P, _I, _I, _P, _P]),
    ("qpsdm_eikonal_solve", _I, [_P, _P, C.POINTER(EikModel), _P, _I, C.POINTER(EikGrid),
                                 _F, _I, _P, _P, _P, _P]),
    ("qpsdm_eikonal_fill", _I, [_P, _P, C.POINTER(EikGrid), _P, _I, _I, _P, _P, _P, _P, _I,
                                C.POINTER(EikFillGeom), _P, _P, _P]),
    ("qpsdm_mlp_create", _I, [_I, C.POINTER(C.c_void_p)]),
    ("qpsdm_mlp_destroy", _I, [_P]),
    ("qpsdm_mlp_param_count", _I, []),
    ("qpsdm_mlp_set_params", _I, [_P, _P]),
    ("qpsdm_mlp_get_params", _I, [_P, _P]),
    ("qpsdm_mlp_set_scaling", _I, [_P, _P, _P, _P]),
    ("qpsdm_mlp_gradients", _I, [_P, _P, _P, _I, _P, C.POINTER(C.c_float), _P]),
    ("qpsdm_mlp_train_step", _I, [_P, _P, _P, _I, _F, C.POINTER(C.c_float), _P]),
    ("qpsdm_mlp_forward", _I, [_P, _P, _I, _P, _P]),
    ("qpsdm_mlp_status", _I, [_P]),
    ("qpsdm_eikonal_samples", _I, [_P, _P, _P, _P, C.POINTER(EikGrid), _P, _I,
                                   C.POINTER(SurBackground), C.c_uint64, _I, _P, _P, _P]),
    ("qpsdm_tables_lerp", _I, [_P, _P, C.c_int64, _I, _I, _I, _P, _P]),
    ("qpsdm_eikonal_correct", _I, [C.POINTER(SurLine), _P, _P, _P, _P, _P, C.c_int64, _F, _P]),
    ("qpsdm_surrogate_gate", _I, [_P, C.POINTER(SurLine), _P, _P, C.c_int64, _P, _P]),
    ("qpsdm_surrogate_tables", _I, [_P, C.POINTER(SurLine), _P, _P, _P, C.c_int64, _P, _F, _P,
                                    _P, _P, C.c_int64, C.POINTER(C.c_int64), _P]),
]
FFT_NOALLOC_MAX_N = 8192
ETIMEOUT = 5
ESIZE = 8

_lib = None


def lib() -> C.CDLL:
    """Load libqpsdm_b200.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m q_psdm_b200.build` "
                "(the engine has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SYMBOLS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class QpsdmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def check(rc: int, handle=None, what: str = "") -> None:
    if rc != 0:
        msg = ""
        if handle:
            m = lib().qpsdm_last_error(handle)
            msg = m.decode() if m else ""
        raise QpsdmError(rc, f"{what} {msg}".strip())
