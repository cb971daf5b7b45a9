"""Generate the golden vectors of tests/golden/ from the reference itself.

Run from the repository root where the reference sources are available:

    make -C oracle ref            # builds oracle/_ref/libqpsdm_refcpu.so
    python tests/golden/make_golden.py cpu

The CPU vectors come from the reference's own fft.cc / psdmpkg.cc compiled in
place (oracle/_ref): npfar over a range of lengths, pfarc spectra of seeded
signals at every length the configurations use, fetch_and_taper outputs, and
the preprocessing spectra of seeded traces driven through the reference's
fetch_and_taper + pfarc.

    make -C oracle ref-gpu        # builds oracle/_ref/libqpsdm_refgpu.so
    python tests/golden/make_golden.py gpu [OUTDIR]   (on a machine with a B200)

The GPU vectors come from the reference's own psdm_kernel + image_depth_gpu
(compiled with its own -O2 --use_fast_math flags for sm_100a) run on seeded
traces: per-trace acceptance, spectra and the accumulated stub image.  They
are written to OUTDIR (default tests/golden/) and copied here by hand when
they were made on another machine.

    make -C oracle ref
    python tests/golden/make_golden.py pkg

The driver-utility transcript (pkg_cases.txt, pkg_cases.err): tests/pkg_cases.cpp
compiled with -DPKG_REF against the reference's psdmpkg.h / segy.h and its
psdmpkg.cc / segy.cc objects in oracle/_ref, run in an empty directory;
stdout and stderr as printed.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
FFT_LENGTHS = [2, 16, 720, 728, 1008, 1232, 1260, 1540, 1716, 2002, 2520, 3080,
               4004, 5040, 6006]


def cpu() -> None:
    R = O.ref_cpu()
    if R is None:
        raise SystemExit("oracle/_ref/libqpsdm_refcpu.so missing: make -C oracle ref")
    out = {}
    ns = np.concatenate([np.arange(1, 20001), [30000, 100000, 360361, 720720, 800000]])
    out["npfar_n"] = ns.astype(np.int32)
    out["npfar"] = np.array([R.ref_npfar(int(n)) for n in ns], np.int32)
    rng = np.random.default_rng(20240601)
    for n in FFT_LENGTHS:
        x = rng.standard_normal(n).astype(np.float32)
        cz = np.zeros(n + 2, np.float32)
        R.ref_pfarc(-1, n, x.copy(), cz)
        out[f"pfarc_in_{n}"] = x
        out[f"pfarc_out_{n}"] = cz
    x = rng.standard_normal(1000).astype(np.float32)
    out["taper_in"] = x
    for (a, b) in [(0, 999), (-5, 300), (280, 999), (0, 100), (500, 1300), (0, 0)]:
        o = np.zeros(b - a + 1, np.float32)
        R.ref_fetch_and_taper(x, 1000, a, b, o)
        out[f"taper_{a}_{b}"] = o
    # preprocessing of psdm_kernel for ntl=1000, dt=2 ms (c1 windows)
    ntl, dt = 1000, np.float32(0.002)
    w = O.window_split(ntl, dt, 1.0, 140.0)
    tr = rng.standard_normal((8, ntl)).astype(np.float32)
    re = np.zeros((8, 2 * w["nww"]), np.float32)
    im = np.zeros_like(re)
    R.ref_preprocess_traces(tr, 8, ntl, dt, w["itb1"], w["itb2"], w["nsb"], w["nf1"],
                            w["nww"], w["dw"], re, im, 1)
    out["pre_traces"] = tr
    out["pre_re"] = re
    out["pre_im"] = im
    out["pre_window"] = np.array([w[k] for k in ("itb1", "itb2", "nsb", "nf1", "nww")], np.int32)
    np.savez_compressed(os.path.join(HERE, "ref_cpu_vectors.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_cpu_vectors.npz"))


class RefGpuArgs(C.Structure):
    _fields_ = [
        ("dyi", C.c_float), ("dxi", C.c_float),
        ("nxi", C.c_int), ("nzi", C.c_int), ("ntl", C.c_int),
        ("scaled", C.c_double), ("fci", C.c_int),
        ("dzi", C.c_float), ("dt", C.c_float), ("fc", C.c_float), ("eps", C.c_float),
        ("fxv1", C.c_float), ("fyv1", C.c_float), ("exv1", C.c_float), ("eyv1", C.c_float),
        ("nfft", C.c_int), ("nffti", C.c_int),
        ("dt1", C.c_float), ("taperzone", C.c_float), ("lnG", C.c_float),
        ("coef1", C.c_float), ("coef2", C.c_float), ("coef3", C.c_float),
        ("coef4", C.c_float), ("dzii", C.c_float),
        ("fxi", C.c_double), ("cyi", C.c_double), ("dw", C.c_float),
        ("itb1", C.c_int), ("itb2", C.c_int), ("nsb", C.c_int),
        ("tdstart1", C.c_float), ("tdstart2", C.c_float), ("nf1", C.c_int),
        ("tdmid", C.c_float), ("nww", C.c_int), ("ncoef1", C.c_int),
        ("ixstart", C.c_int), ("ixend", C.c_int), ("nxb", C.c_int),
        ("ttt_cdp1", C.c_int), ("ttt_cdp2", C.c_int),
    ]


def gpu_case(name: str):
    """Seeded compat case shared by the GPU golden run and the tests."""
    from tests.compat_case import make_case  # noqa: E402
    return make_case(name)


def gpu(outdir: str | None = None) -> None:
    path = os.path.join(ROOT, "oracle", "_ref", "libqpsdm_refgpu.so")
    L = C.CDLL(path)
    f32 = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
    i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    L.ref_gpu_run.argtypes = [C.POINTER(RefGpuArgs), C.c_int, i32, f32, i32, i32, f32,
                              f32, i32, f32, f32]
    outdir = outdir or os.path.join(ROOT, "tests", "golden")
    os.makedirs(outdir, exist_ok=True)
    for name in ("small", "block"):
        case = gpu_case(name)
        a = RefGpuArgs()
        for k, v in case["ref_args"].items():
            setattr(a, k, v)
        ntr = case["hdr"].shape[0]
        img = np.zeros(case["nxb"] * case["nzi"], np.float32)
        acc = np.zeros(ntr, np.int32)
        nww = case["ref_args"]["nww"]
        re = np.zeros((ntr, 2 * nww), np.float32)
        im = np.zeros_like(re)
        rc = L.ref_gpu_run(C.byref(a), ntr, np.ascontiguousarray(case["hdr"], np.int32),
                           np.ascontiguousarray(case["traces"], np.float32),
                           np.ascontiguousarray(case["iaztab"], np.int32),
                           np.ascontiguousarray(case["az"], np.int32),
                           np.ascontiguousarray(case["dips"], np.float32),
                           img, acc, re, im)
        if rc != 0:
            raise SystemExit(f"ref_gpu_run failed: {rc}")
        np.savez_compressed(os.path.join(outdir, f"ref_gpu_{name}.npz"),
                            img=img.reshape(case["nxb"], case["nzi"]), accepted=acc,
                            re=re[acc == 1], im=im[acc == 1])
        print(name, "accepted", int(acc.sum()), "of", ntr, "img max", float(np.abs(img).max()))


def pkg() -> None:
    import subprocess
    import tempfile
    ref = os.path.join(ROOT, "oracle", "_ref")
    objs = [os.path.join(ref, o) for o in ("psdmpkg.o", "segy.o", "fft.o")]
    if not all(os.path.exists(o) for o in objs):
        raise SystemExit("oracle/_ref objects missing: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
        exe = os.path.join(tmp, "pkg_cases_ref")
        subprocess.run(["g++", "-O2", "-std=c++17", "-DPKG_REF", "-w", "-I" + O.ref_src(),
                        os.path.join(ROOT, "tests", "pkg_cases.cpp")] + objs
                       + ["-fopenmp", "-o", exe], check=True)
        run = os.path.join(tmp, "run")
        os.mkdir(run)
        r = subprocess.run([exe], cwd=run, capture_output=True, text=True, check=True)
    with open(os.path.join(HERE, "pkg_cases.txt"), "w") as f:
        f.write(r.stdout)
    with open(os.path.join(HERE, "pkg_cases.err"), "w") as f:
        f.write(r.stderr)
    print(f"pkg_cases: {len(r.stdout.splitlines())} lines")


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "cpu"
    if what == "pkg":
        pkg()
    elif what == "gpu":
        gpu(sys.argv[2] if len(sys.argv) > 2 else None)
    else:
        cpu()
