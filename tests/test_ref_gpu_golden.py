"""The compat oracle against the reference's own GPU engine (CPU test).

tests/golden/ref_gpu_{small,block}.npz were produced on a B200 by the
reference's psdm_kernel + image_depth_gpu, compiled from its sources with its
own -O2 --use_fast_math flags (tests/golden/make_golden.py gpu), on the cases
of tests/compat_case.py.  The engine's compat kernel equals the oracle bit
for bit (tests/test_compat_gpu.py), so these bounds hold for the engine too.

The reference divides and takes square roots with fast-math approximations;
the oracle (and engine) use IEEE rounding.  Measured differences: identical
acceptance and masks, image NRMSE ~1e-6, largest deviation ~2e-6 of the image
peak; the bounds below leave a factor ~5.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.compat_case import make_case, oracle_run

HERE = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["small", "block"])
def test_oracle_matches_reference_binary(name):
    g = np.load(os.path.join(HERE, f"ref_gpu_{name}.npz"))
    c = make_case(name)
    ints, geom, img, npt = oracle_run(c)
    acc = (ints[:, 0] == 3).astype(np.int32)
    assert np.array_equal(acc, g["accepted"])
    ref = g["img"]
    assert np.array_equal(img == 0, ref == 0), "mask differs"
    d = np.abs(img.astype(np.float64) - ref)
    assert d.max() <= 1e-5 * np.abs(ref).max()
    assert np.sqrt(np.mean(d ** 2)) / np.sqrt(np.mean(ref.astype(np.float64) ** 2)) <= 5e-6
    # spectra of the accepted traces
    w = c["window"]
    ok = np.nonzero(acc)[0]
    for k in range(0, len(ok), max(1, len(ok) // 16)):
        ore, oim = O.preprocess_trace(c["traces"][ok[k]], np.float32(0.002), w)
        s = max(np.abs(ore).max(), np.abs(oim).max())
        assert np.abs(g["re"][k] - ore).max() <= 1e-6 * s
        assert np.abs(g["im"][k] - oim).max() <= 1e-6 * s
