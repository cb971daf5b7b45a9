"""Host-side mirror of the reference's imaging interface over the C ABI.

The reference drives its path from ``qpsdm()`` (src/q-psdm.cu:1070-1860):
line set-up (tables, dip/Q fields), block and offset set-up (window split,
aperture), then every trace through ``psdm_kernel`` (src/q-psdm.cu:2063),
then the image is read back and divided by ``nsb``.  ``Engine`` exposes the
same steps: ``set_line``, ``begin_offset``, ``submit``, ``get_image``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import LineParams, OffsetParams, StaticParams, TttDesc, check, lib

__all__ = ["Engine", "static_params", "offset_params", "build_iaztab", "npfar",
           "encode_su", "StaticParams", "OffsetParams", "LineParams", "TttDesc",
           "QpsdmError"]

QpsdmError = _lib.QpsdmError


def npfar(n: int) -> int:
    """get_opt_n_fftw (src/fft.cc:3721): smallest valid real PFA length >= n."""
    return lib().qpsdm_npfar(int(n))


def build_iaztab(eps: float = 0.001) -> np.ndarray:
    tab = np.zeros(4096, np.int32)
    n = lib().qpsdm_build_iaztab(eps, tab.ctypes.data, tab.size)
    if n < 0:
        raise ValueError("bad eps")
    return tab[:n].copy()


def static_params(*, nxi, nzi, ntl, dt, dxi, dyi, dzi, fci=1, scaled=1.0,
                  fxv, fyv, nxv, nyv, fc=40.0, f1=1.0, f3=130.0, f4=140.0,
                  threshold=600.0, contract=3.0, taperzone=8.0, dzii=48.0,
                  mode=_lib.MODE_COMPAT, panel_dtype=_lib.PANEL_FP32, nbins=16,
                  dtstar=0.002, max_batch=4096, kahan=0, form=0, use_graph=0,
                  tile_z=0, tile_x=0, variant=0) -> StaticParams:
    """Build line-independent parameters the way main()/qpsdm() do.

    The velocity-grid bounding box is padded by 2 km in x and 1 km in y
    (src/q-psdm.cu:1380-1383); contract/taperzone are given in degrees.
    """
    p = StaticParams()
    p.dyi, p.dxi, p.nxi, p.nzi, p.ntl = dyi, dxi, nxi, nzi, ntl
    p.scaled, p.fci, p.dzi, p.dt, p.fc = scaled, fci, dzi, dt, fc
    p.f1, p.f3, p.f4, p.threshold = f1, f3, f4, threshold
    p.contract, p.taperzone = contract, taperzone
    p.fxv1 = fxv - 2000.0
    p.exv1 = fxv + nxv * dxi + 2000.0
    p.fyv1 = fyv - 1000.0
    p.eyv1 = fyv + nyv * dyi + 1000.0
    p.dzii = dzii
    p.mode, p.panel_dtype, p.nbins, p.dtstar = mode, panel_dtype, nbins, dtstar
    p.max_batch, p.kahan = max_batch, kahan
    p.form, p.use_graph, p.tile_z, p.tile_x = form, use_graph, tile_z, tile_x
    p.variant = variant
    check(lib().qpsdm_static_params_init(C.byref(p)), what="static_params_init")
    return p


def offset_params(p: StaticParams, ixstart: int, ixend: int, *, aznx1, aznx2,
                  azny1, azny2, ioffs: int = 0, zero_image: int = 1) -> OffsetParams:
    o = OffsetParams()
    check(lib().qpsdm_offset_params_init(C.byref(p), ixstart, ixend, C.byref(o)),
          what="offset_params_init")
    for name, v in (("aznx1", aznx1), ("aznx2", aznx2), ("azny1", azny1), ("azny2", azny2)):
        a = np.broadcast_to(np.asarray(v, np.int32), (_lib.NAZ,))
        getattr(o, name)[:] = [int(x) for x in a]
    o.ioffs, o.zero_image = ioffs, zero_image
    return o


def encode_su(sx, sy, gx, gy, traces: np.ndarray, *, dt_us: int, scalco: int = 0,
              big_endian: bool = True) -> np.ndarray:
    """SU records (240-byte header + ns float32) as a uint8 array [ntr, 240+4ns].

    Header offsets follow src/segy.cc:53-80 (scalco@70, sx@72, sy@76, gx@80,
    gy@84, ns@114, dt@116)."""
    traces = np.ascontiguousarray(traces, np.float32)
    ntr, ns = traces.shape
    e = ">" if big_endian else "<"
    rec = np.zeros((ntr, 240 + 4 * ns), np.uint8)
    hdr = rec[:, :240]
    def put(off, vals, dt):
        hdr[:, off:off + np.dtype(dt).itemsize] = (
            np.asarray(vals).astype(e + dt).reshape(-1, 1).view(np.uint8).reshape(ntr, -1))
    put(70, np.full(ntr, scalco), "i2")
    put(72, sx, "i4")
    put(76, sy, "i4")
    put(80, gx, "i4")
    put(84, gy, "i4")
    put(114, np.full(ntr, ns), "u2")
    put(116, np.full(ntr, dt_us), "u2")
    rec[:, 240:] = traces.astype(e + "f4").view(np.uint8).reshape(ntr, 4 * ns)
    return rec


@dataclass
class _LineKeep:
    """Host arrays referenced by a LineParams while set_line runs."""
    arrays: list


class Engine:
    """One imaging engine bound to one CUDA device (a consumer of qpsdm())."""

    def __init__(self, params: StaticParams, device: int = 0, iaztab=None):
        self.p = params
        tab = build_iaztab(params.eps) if iaztab is None else np.ascontiguousarray(iaztab, np.int32)
        self._iaz = tab
        h = C.c_void_p()
        check(lib().qpsdm_engine_create(C.byref(params), tab.ctypes.data, tab.size,
                                        device, C.byref(h)), what="engine_create")
        self.h = h
        self.off: OffsetParams | None = None

    # -- lifetime --------------------------------------------------------
    def close(self) -> None:
        if self.h:
            lib().qpsdm_engine_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc, what):
        check(rc, self.h, what)

    # -- line / offset -----------------------------------------------------
    def set_line(self, *, fxi: float, cyi: float, dips, nf3=None, q=None,
                 tables=None, ttt_cdp1=None, ttt_cdp2=None) -> None:
        """dips: (dipx1, dipx2, dipy1, dipy2), each [nxi, nzi] float32.
        tables: None or dict(nxg, nzg, nxi1, nzi1, cdp1, cdp2, ttt_desc,
        ttt, qqq_desc, qqq) in the reference layout; ttt and qqq may be numpy
        arrays or float32 torch tensors on the engine's device."""
        self.set_lines([dict(fxi=fxi, cyi=cyi, dips=dips, nf3=nf3, q=q, tables=tables,
                             ttt_cdp1=ttt_cdp1, ttt_cdp2=ttt_cdp2)])

    def set_lines(self, lines) -> None:
        """An image brick: a list of set_line keyword dicts, one per line."""
        keep = []
        arr = (LineParams * len(lines))()
        for i, ln in enumerate(lines):
            arr[i] = self._line_params(keep, **ln)
        self._ck(lib().qpsdm_set_lines(self.h, arr, len(lines)), "set_lines")
        self.nlines = len(lines)

    def _line_params(self, keep, *, fxi, cyi, dips, nf3=None, q=None, tables=None,
                     ttt_cdp1=None, ttt_cdp2=None) -> LineParams:
        def fptr(a, dt=np.float32):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt)
            keep.append(a)
            return a.ctypes.data
        lp = LineParams()
        lp.fxi, lp.cyi = fxi, cyi
        lp.dipx1, lp.dipx2, lp.dipy1, lp.dipy2 = (fptr(d) for d in dips)
        lp.nf3 = fptr(nf3, np.int32)
        lp.q = fptr(q)
        if tables is not None:
            lp.nxg, lp.nzg = tables["nxg"], tables["nzg"]
            lp.nxi1, lp.nzi1 = tables["nxi1"], tables["nzi1"]
            lp.ttt_cdp1, lp.ttt_cdp2 = tables["cdp1"], tables["cdp2"]
            for k in ("ttt_desc", "qqq_desc"):
                d = np.ascontiguousarray(tables[k])
                keep.append(d)
                setattr(lp, k, d.ctypes.data)
            for k in ("ttt", "qqq"):
                a = tables[k]
                if hasattr(a, "is_cuda") and a.is_cuda:  # table data on the device
                    assert a.is_contiguous() and str(a.dtype) == "torch.float32"
                    keep.append(a)
                    setattr(lp, k, a.data_ptr())
                    setattr(lp, k + "_len", int(a.numel()))
                else:
                    setattr(lp, k, fptr(a))
                    setattr(lp, k + "_len", int(np.asarray(a).size))
        else:
            lp.ttt_cdp1 = self.p.fci if ttt_cdp1 is None else ttt_cdp1
            lp.ttt_cdp2 = self.p.fci + self.p.nxi - 1 if ttt_cdp2 is None else ttt_cdp2
        return lp

    def begin_offset(self, o: OffsetParams) -> None:
        self._ck(lib().qpsdm_begin_offset(self.h, C.byref(o)), "begin_offset")
        self.off = o

    # -- traces --------------------------------------------------------------
    def submit(self, records: np.ndarray, big_endian: bool = True) -> None:
        """records: uint8 [ntr, 240 + 4*ntl] host SU records."""
        records = np.ascontiguousarray(records, np.uint8)
        ntr = records.shape[0]
        ns = (records.shape[1] - 240) // 4
        self._ck(lib().qpsdm_submit_traces(self.h, records.ctypes.data, ntr, ns,
                                           int(big_endian)), "submit_traces")

    def submit_device(self, d_records: int, ntr: int, big_endian: bool = True) -> None:
        """d_records: device pointer (e.g. a torch uint8 tensor's data_ptr())."""
        self._ck(lib().qpsdm_submit_traces_device(self.h, C.c_void_p(d_records), ntr,
                                                  self.p.ntl, int(big_endian)),
                 "submit_traces_device")

    def submit_gathers(self, records: np.ndarray, aperture: np.ndarray,
                       big_endian: bool = True) -> None:
        """Gathers of uneven sizes and apertures: records uint8 [ntr, 240 + 4*ntl],
        aperture int32 [ntr, 2] = each trace's half-width in cdps and in lines
        (capping the offset group's azimuth tables)."""
        records = np.ascontiguousarray(records, np.uint8)
        aperture = np.ascontiguousarray(aperture, np.int32)
        ntr = records.shape[0]
        if aperture.shape != (ntr, 2):
            raise ValueError("aperture must be int32 [ntr, 2]")
        ns = (records.shape[1] - 240) // 4
        self._ck(lib().qpsdm_submit_gathers(self.h, records.ctypes.data, aperture.ctypes.data,
                                            ntr, ns, int(big_endian)), "submit_gathers")

    def submit_gathers_device(self, d_records: int, d_aperture: int, ntr: int,
                              big_endian: bool = True) -> None:
        """Device pointers: records and int32 [ntr, 2] apertures."""
        self._ck(lib().qpsdm_submit_gathers_device(self.h, C.c_void_p(d_records),
                                                   C.c_void_p(d_aperture), ntr, self.p.ntl,
                                                   int(big_endian)), "submit_gathers_device")

    def fence(self) -> None:
        self._ck(lib().qpsdm_fence(self.h), "fence")

    def set_line_mask(self, mask: int) -> None:
        """Lines of the brick (bit il = line il) the following submits feed."""
        self._ck(lib().qpsdm_set_line_mask(self.h, int(mask) & (2 ** 64 - 1)), "set_line_mask")

    def get_image(self, apply_nsb_scale: bool = True) -> np.ndarray:
        """[nxb, nzi] for one line, [nlines, nxb, nzi] for a brick."""
        nxb = self.off.ixend - self.off.ixstart
        nl = getattr(self, "nlines", 1)
        img = np.zeros((nl, nxb, self.p.nzi), np.float32)
        self._ck(lib().qpsdm_get_image(self.h, img.ctypes.data, int(apply_nsb_scale)),
                 "get_image")
        return img[0] if nl == 1 else img

    def image_shape(self):
        """Shape of the full image buffer: (nlines, nxb, nzi)."""
        return (getattr(self, "nlines", 1), self.off.ixend - self.off.ixstart, self.p.nzi)

    def get_image_async(self, host_img: np.ndarray, apply_nsb_scale: bool = True) -> int:
        """Enqueue the image read into host_img (a page-locked float32 array
        of image_shape(), e.g. a pinned torch tensor's numpy view); returns
        the ticket for image_wait.  host_img must stay untouched until then."""
        assert host_img.dtype == np.float32 and host_img.flags.c_contiguous
        assert host_img.size == int(np.prod(self.image_shape()))
        t = C.c_int64(-1)
        self._ck(lib().qpsdm_get_image_async(self.h, host_img.ctypes.data,
                                             int(apply_nsb_scale), C.byref(t)),
                 "get_image_async")
        return t.value

    def image_wait(self, ticket: int) -> None:
        self._ck(lib().qpsdm_image_wait(self.h, int(ticket)), "image_wait")

    def set_stream(self, stream_handle: int | None) -> None:
        """Run engine kernels on a caller stream (e.g. torch's
        ``torch.cuda.current_stream().cuda_stream``); None = the engine's own."""
        self._ck(lib().qpsdm_set_stream(self.h, C.c_void_p(stream_handle or 0)), "set_stream")

    def profile(self, on: bool = True) -> None:
        """Start (or stop) per-launch CUDA-event timing; resets the sums."""
        self._ck(lib().qpsdm_profile_enable(self.h, int(on)), "profile_enable")

    def kernel_time(self, cls: int):
        """(total device ms, launches) of one kernel class since profile()."""
        ms, n = C.c_double(), C.c_int64()
        self._ck(lib().qpsdm_profile_get(self.h, cls, C.byref(ms), C.byref(n)), "profile_get")
        return ms.value, n.value

    def tuning(self) -> dict:
        """The batched form's autotuned image-kernel variant and timings."""
        v, tz, tx, mb = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        ms = np.zeros(32, np.float32)
        n = lib().qpsdm_tuning_info(self.h, C.byref(v), C.byref(tz), C.byref(tx),
                                    C.byref(mb), ms.ctypes.data, ms.size)
        if n < 0:
            raise QpsdmError(-n, "tuning_info")
        return {"variant": v.value, "tile": [tz.value, tx.value], "min_blocks": mb.value,
                "variant_ms": [float(x) for x in ms[:n]]}

    def image_device_ptr(self) -> int:
        p = C.c_void_p()
        self._ck(lib().qpsdm_image_device_ptr(self.h, C.byref(p)), "image_device_ptr")
        return p.value

    def counters(self):
        a, n = C.c_int64(), C.c_int64()
        self._ck(lib().qpsdm_get_counters(self.h, C.byref(a), C.byref(n)), "get_counters")
        return a.value, n.value

    def stats(self):
        """dict(accepted, point_traces, tile_decided, imaged) since begin_offset."""
        a = np.zeros(4, np.int64)
        rc = lib().qpsdm_get_stats(self.h, a.ctypes.data, 4)
        if rc < 0 or rc != 4:
            self._ck(rc if rc else 1, "get_stats")
        return dict(accepted=int(a[0]), point_traces=int(a[1]), tile_decided=int(a[2]),
                    imaged=int(a[3]))

    def panels_device_ptrs(self):
        """(d_panels, d_pscale) device pointers of the last submit's panels."""
        a, b = C.c_void_p(), C.c_void_p()
        self._ck(lib().qpsdm_panels_device_ptr(self.h, C.byref(a), C.byref(b)), "panels")
        return a.value, b.value

    def spectra_device_ptrs(self):
        r, i = C.c_void_p(), C.c_void_p()
        self._ck(lib().qpsdm_spectra_device_ptr(self.h, C.byref(r), C.byref(i)), "spectra")
        return r.value, i.value

    def gate_device_ptrs(self):
        r, i = C.c_void_p(), C.c_void_p()
        self._ck(lib().qpsdm_gate_device_ptr(self.h, C.byref(r), C.byref(i)), "gate")
        return r.value, i.value
