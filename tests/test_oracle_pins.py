"""The oracle against the reference's own outputs (CPU only).

Golden vectors (tests/golden/ref_cpu_vectors.npz) were produced by the
reference's fft.cc / psdmpkg.cc compiled from its sources
(tests/golden/make_golden.py).  When oracle/_ref is present the same checks
also run live against the compiled reference.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_cpu_vectors.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_npfar_matches_reference(gold):
    ns, want = gold["npfar_n"], gold["npfar"]
    got = np.array([O.npfar(int(n)) for n in ns], np.int32)
    assert np.array_equal(got, want)


def test_pfa_table_is_the_reference_set(gold):
    tab = np.zeros(240, np.int32)
    assert O.lib().orc_pfa_table(tab, 240) == 240
    # every npfar result is twice a table entry, and every small entry occurs
    halves = set((gold["npfar"] // 2).tolist())
    assert halves <= set(tab.tolist())
    assert {t for t in tab.tolist() if t <= 10000} <= halves


@pytest.mark.parametrize("n", [2, 16, 720, 728, 1008, 1232, 1260, 1540, 1716, 2002,
                               2520, 3080, 4004, 5040, 6006])
def test_rdft_matches_pfarc(gold, n):
    x = gold[f"pfarc_in_{n}"]
    cz = gold[f"pfarc_out_{n}"]
    ref = cz[0::2].astype(np.float64) + 1j * cz[1::2]
    mine = O.rdft(x)
    # pfarc is single precision; the oracle is a double DFT
    assert np.abs(ref - mine).max() <= 1e-6 * np.abs(mine).max() * max(1, np.log2(n) / 4)


def test_fetch_and_taper_bit_exact(gold):
    x = gold["taper_in"]
    for key in gold.files:
        if key.startswith("taper_") and key != "taper_in":
            a, b = (int(v) for v in key.split("_")[1:])
            assert np.array_equal(O.fetch_and_taper(x, a, b), gold[key]), key


def test_preprocess_matches_reference(gold):
    tr = gold["pre_traces"]
    w = O.window_split(1000, np.float32(0.002), 1.0, 140.0)
    assert [w[k] for k in ("itb1", "itb2", "nsb", "nf1", "nww")] == gold["pre_window"].tolist()
    for i in range(tr.shape[0]):
        re, im = O.preprocess_trace(tr[i], np.float32(0.002), w)
        scale = max(np.abs(gold["pre_re"][i]).max(), np.abs(gold["pre_im"][i]).max())
        assert np.abs(re - gold["pre_re"][i]).max() <= 2e-6 * scale
        assert np.abs(im - gold["pre_im"][i]).max() <= 2e-6 * scale


# Derived sizes per configuration, evaluated by the reference's formulas
# with its compiled npfar (dt = 2 ms, f1 = 1, f4 = 140).
SIZES = {1000: (1008, 2002, 720, 280, 1, 201), 2000: (2002, 4004, 1232, 768, 2, 343),
         2500: (2520, 5040, 1540, 960, 3, 429), 3000: (3080, 6006, 1716, 1284, 3, 478)}


@pytest.mark.parametrize("ntl", sorted(SIZES))
def test_derived_sizes(ntl):
    s = O.derive_static(ntl, np.float32(0.002))
    w = O.window_split(ntl, np.float32(0.002), 1.0, 140.0)
    assert (s["nfft"], s["nffti"], w["nsb"], w["itb2"], w["nf1"], w["nww"]) == SIZES[ntl]


def test_iaztab_sectors():
    t = O.iaztab(0.001)
    assert t.size == 2001
    assert set(np.unique(t).tolist()) == set(range(18))
    # sectors are contiguous and increase with (1 - cos)
    nz = t[t > 0]
    assert np.all(np.diff(nz) >= 0)


@pytest.mark.skipif(O.ref_cpu() is None, reason="reference not compiled here")
def test_live_reference_agrees():
    R = O.ref_cpu()
    for n in list(range(1, 5000, 3)) + [720720, 800000]:
        assert O.npfar(n) == R.ref_npfar(n)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(1000).astype(np.float32)
    for a, b in [(3, 700), (-10, 1200)]:
        o = np.zeros(b - a + 1, np.float32)
        R.ref_fetch_and_taper(x, 1000, a, b, o)
        assert np.array_equal(o, O.fetch_and_taper(x, a, b))
