"""libqpsdm_pkg.so -- the driver's utility API (include/qpsdm_psdmpkg.h,
include/qpsdm_segy.h) against the reference's psdmpkg.cc / segy.cc.

tests/pkg_cases.cpp exercises every function (par.dat records, the command
line, lists, tuples, the end taper, the mute, coordinate scales, project
paths, SU trace readers and writers, velocity-file coordinates) and prints a
transcript with floats as bit patterns.  Built against this library it must
print, byte for byte, the transcript the reference's own objects printed
(tests/golden/pkg_cases.txt, made by tests/golden/make_golden.py pkg), and,
where oracle/_ref holds the reference's objects, the transcript they print
now.
"""
from __future__ import annotations

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "q_psdm_b200")
CASES = os.path.join(ROOT, "tests", "pkg_cases.cpp")
GOLDEN = os.path.join(ROOT, "tests", "golden")
REF_OBJS = [os.path.join(ROOT, "oracle", "_ref", o) for o in ("psdmpkg.o", "segy.o", "fft.o")]

# every function the two headers declare, by the name the library exports
DECLARED = [
    "malloc1c", "malloc2c", "malloc1i", "malloc2i", "malloc3i", "malloc1f", "malloc2f",
    "malloc3f", "malloc4f", "malloc1d", "malloc2d", "free1c", "free2c", "free1i", "free2i",
    "free3i", "free1f", "free2f", "free3f", "free4f", "free1d", "free2d", "parseint",
    "initargs_inner", "getparint", "getparfloat", "getpardouble", "getparstr(char const*, char**)",
    "getparstr(char const*, char const**)", "readparfile", "fetch_and_taper", "fsize", "fexist",
    "strrev1", "strrtrim", "parsepath", "parsetuple", "time_offset_mute_santity", "getscale",
    "get_vel_coor", "time_offset_mute", "fgettr", "fputtr", "sgettr", "sputtr",
]
C_LINKAGE = {"getscale", "get_vel_coor", "time_offset_mute"}


@pytest.fixture(scope="module")
def pkg_lib():
    from q_psdm_b200.build import build_pkg
    return build_pkg()


def _run(exe: str, tmp) -> subprocess.CompletedProcess:
    run = tmp / ("run_" + os.path.basename(exe))
    run.mkdir()
    return subprocess.run([exe], cwd=run, capture_output=True, text=True, timeout=120)


def _first_difference(a: str, b: str) -> str:
    la, lb = a.splitlines(), b.splitlines()
    for i, (x, y) in enumerate(zip(la, lb)):
        if x != y:
            return f"line {i + 1}:\n  got  {x[:300]}\n  want {y[:300]}"
    return f"line counts {len(la)} vs {len(lb)}"


@pytest.fixture(scope="module")
def transcript(pkg_lib, tmp_path_factory):
    tmp = tmp_path_factory.mktemp("pkg")
    exe = str(tmp / "pkg_cases")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), CASES,
                    "-L" + PKG, "-lqpsdm_pkg", "-Wl,-rpath," + PKG, "-o", exe], check=True)
    r = _run(exe, tmp)
    assert r.returncode == 0, r.stderr
    return r


def test_library_exports_every_declared_function(pkg_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", pkg_lib], capture_output=True,
                         text=True, check=True).stdout
    names = {ln.split(" ", 2)[2] for ln in out.splitlines() if " T " in ln}
    for f in DECLARED:
        if f in C_LINKAGE:
            assert f in names, f"{f} not exported with C linkage"
        elif "(" in f:
            assert f in names, f"{f} not exported"
        else:
            assert any(n.startswith(f + "(") for n in names), f"{f} not exported"
    for g in ("xargc", "xargv", "inited"):
        assert f" {g}" in out or any(ln.endswith(" " + g) for ln in out.splitlines())


def test_transcript_matches_golden(transcript):
    with open(os.path.join(GOLDEN, "pkg_cases.txt")) as f:
        want = f.read()
    with open(os.path.join(GOLDEN, "pkg_cases.err")) as f:
        want_err = f.read()
    assert transcript.stdout == want, _first_difference(transcript.stdout, want)
    assert transcript.stderr == want_err


def test_transcript_matches_reference_objects(transcript, tmp_path):
    from oracle import oracle as O
    src = O.ref_src()
    if not (all(os.path.exists(o) for o in REF_OBJS) and os.path.isdir(src)):
        pytest.skip("reference objects not built here (make -C oracle ref)")
    exe = str(tmp_path / "pkg_cases_ref")
    subprocess.run(["g++", "-O2", "-std=c++17", "-DPKG_REF", "-w", "-I" + src, CASES]
                   + REF_OBJS + ["-fopenmp", "-o", exe], check=True)
    r = _run(exe, tmp_path)
    assert r.returncode == 0
    assert transcript.stdout == r.stdout, _first_difference(transcript.stdout, r.stdout)
    assert transcript.stderr == r.stderr


def test_transcript_covers_every_function(transcript):
    heads = {ln.split(" ", 1)[0] for ln in transcript.stdout.splitlines()}
    for h in ("parseint", "parsetuple", "readpar", "initargs", "getparint", "getparfloat",
              "getpardouble", "getparstr", "taper", "mute", "getscale", "parsepath", "strrtrim",
              "fsize", "fgettr", "sgettr", "sputtr", "fputtr", "get_vel_coor", "arrays"):
        assert h in heads, h


def test_single_tuple_and_signed_numbers(pkg_lib):
    """Where the reference fails (one tuple: it writes past an empty block and
    returns NULL; a '-' sign: it never returns), the library parses."""
    import ctypes as C
    L = C.CDLL(pkg_lib)
    f = L._Z10parsetuplePKcPiS1_
    f.restype = C.POINTER(C.c_float)
    f.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    nt, ne = C.c_int(), C.c_int()
    p = f(b"(100,-2.5e1)", C.byref(nt), C.byref(ne))
    assert (nt.value, ne.value) == (1, 2)
    assert (p[0], p[1]) == (100.0, -25.0)
    p = f(b"(-1,2),(3,+4)", C.byref(nt), C.byref(ne))
    assert (nt.value, ne.value) == (2, 2)
    assert [p[i] for i in range(4)] == [-1.0, 2.0, 3.0, 4.0]
