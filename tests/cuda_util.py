"""Minimal CUDA runtime access for tests: copies between host and engine-owned
device memory (the engine hands out raw device pointers)."""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np

_rt = None


def cudart():
    global _rt
    if _rt is None:
        cands = glob.glob("/usr/local/cuda/lib64/libcudart.so*")
        import torch  # noqa: F401  (makes sure the primary context exists first)
        cands += glob.glob(os.path.join(os.path.dirname(os.path.dirname(torch.__file__)),
                                        "nvidia", "cuda_runtime", "lib", "libcudart.so*"))
        for c in cands:
            try:
                _rt = C.CDLL(c)
                break
            except OSError:
                continue
        if _rt is None:
            raise RuntimeError("libcudart not found")
        _rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        _rt.cudaMemcpy.restype = C.c_int
        _rt.cudaDeviceSynchronize.restype = C.c_int
    return _rt


def d2h(ptr: int, shape, dtype) -> np.ndarray:
    out = np.empty(shape, dtype)
    rt = cudart()
    rc = rt.cudaMemcpy(out.ctypes.data, C.c_void_p(ptr), out.nbytes, 2)
    if rc != 0:
        raise RuntimeError(f"cudaMemcpy D2H failed: {rc}")
    return out
