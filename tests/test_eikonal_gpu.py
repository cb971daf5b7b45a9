"""The GPU eikonal / t* table generator.

* With the background correction a linear-gradient model reproduces the
  analytic linear-gradient tables (same layout) to 0.1 ms.
* A fast velocity anomaly under the line makes traveltimes earlier, never
  later, by roughly the time saved along the ray (~15 ms for +15 % over
  ~300 m at 2 km/s).
* Grid refinement (40 m -> 20 m) changes the corrected tables by well under
  the 2 ms surrogate gate (RMS) and t* by under 1 %.
"""
import numpy as np
import pytest

from q_psdm_b200 import synth, tables

pytestmark = pytest.mark.gpu
KW = dict(fci=1, nxi=128, dxi=10.0, zmax=990.0, line_y=640.0, dzii=40.0, nxi1=16, surf_dx=40,
          surf_dy=40, half_x=600.0, half_y=600.0)
BOX = dict(xr=(-900, 2300), yr=(-900, 2200), zmax=1100, v0=2000.0, kz=0.6, q=60.0)


def _anomalous(h):
    m = synth.config2_model(h=h, anomalies=False, layered_q=False, **BOX)
    Z, Y, X = np.meshgrid(np.arange(m.vel.shape[0]) * h, m.oy + np.arange(m.vel.shape[1]) * h,
                          m.ox + np.arange(m.vel.shape[2]) * h, indexing="ij")
    m.vel *= (1 + 0.15 * np.exp(-((X - 640) ** 2 + (Y - 640) ** 2 + (Z - 500) ** 2)
                                / 150.0 ** 2)).astype(np.float32)
    return m


@pytest.fixture(scope="module")
def analytic():
    sv = synth.config1()
    return tables.linear_gradient_tables(sv, fci=1, nxi=128, dxi=10.0, zmax=990.0, sub=4,
                                         nxi1=16, half_x=600.0, half_y=600.0)


def test_background_reproduces_analytic(cuda, analytic):
    bg = synth.config2_model(h=40.0, anomalies=False, layered_q=False, **BOX)
    t = tables.eikonal_line_tables(bg, h=40.0, init_radius=200.0, background=bg,
                                   q_background=60.0, **KW)
    assert np.abs(t.ttt - analytic.ttt).max() < 1e-4
    assert np.abs(t.qqq - analytic.qqq).max() < 1e-6


def test_anomaly_and_refinement(cuda, analytic):
    out = {}
    for h in (40.0, 20.0):
        bg = synth.config2_model(h=h, anomalies=False, layered_q=False, **BOX)
        out[h] = tables.eikonal_line_tables(_anomalous(h), h=h, init_radius=200.0,
                                            background=bg, q_background=60.0, **KW)
    d = (out[40.0].ttt - analytic.ttt) * 1e3
    assert d.max() < 0.1 and -25.0 < d.min() < -5.0
    r = (out[40.0].ttt - out[20.0].ttt) * 1e3
    assert np.sqrt(np.mean(r ** 2)) < 1.0 and np.abs(r).max() < 4.0
    q = np.abs(out[40.0].qqq - out[20.0].qqq) / np.maximum(out[20.0].qqq, 1e-6)
    assert np.sqrt(np.mean(q ** 2)) < 0.01


def test_unbiased_solve_is_first_order(cuda, analytic):
    # without the correction the first-order scheme overestimates (tens of ms
    # at 40 m); the generator reports that honestly rather than hiding it
    bg = synth.config2_model(h=40.0, anomalies=False, layered_q=False, **BOX)
    t = tables.eikonal_line_tables(bg, h=40.0, init_radius=200.0, **KW)
    d = (t.ttt - analytic.ttt) * 1e3
    assert d.mean() > 0.0 and np.abs(d).max() < 40.0
