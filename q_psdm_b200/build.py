"""Build the engine's shared library for sm_100a (in-tree).

``python -m q_psdm_b200.build`` compiles every ``csrc/*.cu`` / ``csrc/*.cpp``
with nvcc (``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``) into
``q_psdm_b200/libqpsdm_b200.so``, the driver's utility library
(``pkg/*.cpp``: psdmpkg and the SU trace I/O, host C++ with g++) into
``q_psdm_b200/libqpsdm_pkg.so``, then the ``q-psdm`` command-line driver
(``driver/q_psdm.cpp``) into ``q_psdm_b200/bin/q-psdm``.  Objects go to ``q_psdm_b200/_build/``;
a source is recompiled only when it, or a header, is newer than its object.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libqpsdm_b200.so")
PKGSRC = os.path.join(PKG, "pkg")
PKGLIB = os.path.join(PKG, "libqpsdm_pkg.so")
CXX = os.environ.get("CXX", "g++")
DRIVER = os.path.join(PKG, "driver")
DRIVER_BIN = os.path.join(PKG, "bin", "q-psdm")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
         "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
         "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs += glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max((os.path.getmtime(h) for h in hs), default=0.0)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OUT, os.path.basename(src) + ".o")
    if (os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
            and os.path.getmtime(obj) >= _headers_mtime()):
        return obj
    cmd = [NVCC, "-c", src, "-o", obj] + ARCH + FLAGS
    if src.endswith(".cpp"):
        cmd += ["-x", "c++"]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build_pkg() -> str:
    """libqpsdm_pkg.so: psdmpkg (parameters, lists, mute, taper, paths) and
    the SU trace readers/writers.  No contraction: float arithmetic exactly as
    written (-ffp-contract=off), so results match the reference's bit for bit."""
    srcs = sorted(glob.glob(os.path.join(PKGSRC, "*.cpp")))
    if (os.path.exists(PKGLIB)
            and all(os.path.getmtime(PKGLIB) >= os.path.getmtime(s) for s in srcs)
            and os.path.getmtime(PKGLIB) >= _headers_mtime()):
        return PKGLIB
    cmd = [CXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
           "-fno-fast-math", "-Wall", "-I" + os.path.join(ROOT, "include"),
           "-o", PKGLIB] + srcs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"libqpsdm_pkg build failed:\n{r.stdout}\n{r.stderr}")
    return PKGLIB


def build_driver() -> str:
    """The q-psdm command-line driver (host C++ over the C ABI), linked
    against the in-tree libraries (rpath $ORIGIN/..)."""
    src = os.path.join(DRIVER, "q_psdm.cpp")
    os.makedirs(os.path.dirname(DRIVER_BIN), exist_ok=True)
    if (os.path.exists(DRIVER_BIN) and os.path.getmtime(DRIVER_BIN) >= os.path.getmtime(src)
            and os.path.getmtime(DRIVER_BIN) >= os.path.getmtime(LIB)
            and os.path.getmtime(DRIVER_BIN) >= os.path.getmtime(PKGLIB)
            and os.path.getmtime(DRIVER_BIN) >= _headers_mtime()):
        return DRIVER_BIN
    cmd = [NVCC, "-O2", "-std=c++17", "-x", "c++", src, "-o", DRIVER_BIN,
           "-I" + os.path.join(ROOT, "include"), "-L" + PKG, "-lqpsdm_b200", "-lqpsdm_pkg", "-lpthread",
           "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/.."]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    return DRIVER_BIN


def build(verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if (not os.path.exists(LIB)
            or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs)):
        cmd = [NVCC, "-shared", "-o", LIB] + objs + ARCH + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_pkg()
    build_driver()
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
