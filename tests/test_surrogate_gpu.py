"""What the trained surrogate gains over the method without it.

Model: v(z) = 2000 + 0.6 z with a +15 % and a -12 % Gaussian velocity
anomaly under the line and two Q layers (200 above 600 m, 120 below).  The
GPU eikonal generator writes the line's tables at a 160 m surface spacing
(the coarse tables the method would store) and at 40 m (the fine truth).
The network is trained on the coarse tables only, by the library's
tensor-core kernels, and densifies them to 40 m.

Against the 40 m truth, at the fine surface nodes:
* bilinear interpolation of the coarse tables (what the imaging kernel does
  with them) is off by milliseconds where the traveltime curves in the
  source position;
* the linear-gradient background alone misses the anomalies;
* background + network is several times better than either.
The image built with the densified tables is closer to the truth-table image
than the image built with the coarse tables.  With an untrained network every
patch fails the 2 ms gate and the result is exactly the table fallback.
"""
import numpy as np
import pytest

from q_psdm_b200 import synth, tables
from tests.physics_case import engine, make_case, nrmse, records

pytestmark = pytest.mark.gpu

LINE_Y = 640.0
KW = dict(fci=1, nxi=128, dxi=10.0, zmax=990.0, line_y=LINE_Y, dzii=40.0, nxi1=16,
          half_x=960.0, half_y=480.0)
BOX = dict(xr=(-1300, 2600), yr=(-700, 2000), zmax=1100, v0=2000.0, kz=0.6, q=60.0)
ANOMALIES = ((500.0, 700.0, 450.0, 200.0, 0.15), (900.0, 560.0, 700.0, 250.0, -0.12))


def _model(h):
    m = synth.config2_model(h=h, anomalies=False, layered_q=True, **BOX)
    nz, ny, nx = m.vel.shape
    Z, Y, X = np.meshgrid(np.arange(nz) * h, m.oy + np.arange(ny) * h, m.ox + np.arange(nx) * h,
                          indexing="ij")
    for ax, ay, az, rad, amp in ANOMALIES:
        m.vel *= (1 + amp * np.exp(-((X - ax) ** 2 + (Y - ay) ** 2 + (Z - az) ** 2)
                                   / rad ** 2)).astype(np.float32)
    return m


@pytest.fixture(scope="module")
def setup():
    from q_psdm_b200 import surrogate as S
    h = 40.0
    model = _model(h)
    bg = synth.config2_model(h=h, anomalies=False, layered_q=False, **BOX)
    common = dict(h=h, init_radius=200.0, background=bg, q_background=BOX["q"], **KW)
    coarse = tables.eikonal_line_tables(model, surf_dx=160, surf_dy=160, **common)
    truth = tables.eikonal_line_tables(model, surf_dx=40, surf_dy=40, **common)
    back = S.Background(BOX["v0"], BOX["kz"], 100.0)
    sur = S.train([coarse], [LINE_Y], back, fci=1, steps=3000, batch=8192, seed=0)
    fine, stats = S.densify(sur, coarse, fci=1, line_y=LINE_Y, surf_dx=40, surf_dy=40,
                            half_x=KW["half_x"], half_y=KW["half_y"])
    interp = S.coarse_to_fine(coarse, fci=1, surf_dx=40, surf_dy=40, half_x=KW["half_x"],
                              half_y=KW["half_y"])
    feat = S.table_nodes(truth, 1, LINE_Y)
    t_bg, q_bg = back.times(feat)
    return dict(S=S, coarse=coarse, truth=truth, fine=fine, stats=stats, interp=interp,
                t_bg=t_bg, q_bg=q_bg, sur=sur, back=back)


def _ms(a, b):
    d = (np.asarray(a, np.float64) - np.asarray(b, np.float64)) * 1e3
    return float(np.sqrt(np.mean(d ** 2))), float(np.abs(d).max())


def test_training_converged(cuda, setup):
    h = setup["sur"].history
    assert h[-1][1] < 1e-2 * h[0][1], h


def test_surrogate_gains_over_tables_and_background(cuda, setup):
    truth = setup["truth"]
    tab_rms, tab_max = _ms(setup["interp"].ttt, truth.ttt)
    bg_rms, bg_max = _ms(setup["t_bg"], truth.ttt)
    sur_rms, sur_max = _ms(setup["fine"].ttt, truth.ttt)
    q_tab, _ = _ms(setup["interp"].qqq, truth.qqq)
    q_sur, _ = _ms(setup["fine"].qqq, truth.qqq)
    st = setup["stats"]
    print(f"traveltime error at 40 m nodes (ms, rms/max): coarse tables {tab_rms:.3f}/"
          f"{tab_max:.2f}, background {bg_rms:.3f}/{bg_max:.2f}, surrogate {sur_rms:.3f}/"
          f"{sur_max:.2f}; t* rms tables {q_tab:.4f} surrogate {q_sur:.4f}; gated "
          f"{st['gated_nodes']}/{st['surface_nodes']}; fit at coarse nodes "
          f"{st['coarse_rms_ms']:.3f}/{st['coarse_max_ms']:.2f}")
    assert tab_max > 2.0 and bg_max > 5.0            # both plain methods miss by ms
    assert sur_rms < 0.5 * tab_rms and sur_rms < 0.2 * bg_rms
    assert sur_max < 0.5 * tab_max
    assert q_sur < q_tab
    assert st["coarse_max_ms"] < 2.0 and st["gated_nodes"] == 0


def test_image_gain(cuda, setup):
    case = make_case(nshots=2, half_x=40, half_y=30)
    imgs = {}
    for name in ("truth", "interp", "coarse", "fine"):
        case["tab"] = setup[name]
        eng, _, _ = engine(case, panel_dtype=0)
        try:
            eng.submit(records(case))
            imgs[name] = eng.get_image(False)
        finally:
            eng.close()
    assert np.abs(imgs["truth"]).max() > 0
    e_coarse = nrmse(imgs["coarse"], imgs["truth"])
    e_interp = nrmse(imgs["interp"], imgs["truth"])
    e_fine = nrmse(imgs["fine"], imgs["truth"])
    print(f"image NRMSE vs truth tables: coarse {e_coarse:.3e} (resampled {e_interp:.3e}), "
          f"surrogate {e_fine:.3e}")
    # the kernel's own surface interpolation of coarse tables equals resampling them
    assert abs(e_interp - e_coarse) < 0.1 * e_coarse + 1e-6
    assert e_fine < 0.5 * e_coarse


def test_gate_falls_back_to_tables(cuda, setup):
    S = setup["S"]
    raw = S.Surrogate(S.Mlp(0, params=S.init_params(9, out_scale=1e3)), setup["back"], [])
    raw.mlp.set_scaling(setup["sur"].mlp.shift, setup["sur"].mlp.scale)
    # the untrained network misses the coarse nodes by far more than 2 ms
    fine, st = S.densify(raw, setup["coarse"], fci=1, line_y=LINE_Y, surf_dx=40, surf_dy=40,
                         half_x=KW["half_x"], half_y=KW["half_y"])
    assert st["gated_nodes"] == st["surface_nodes"]
    assert np.array_equal(fine.ttt, setup["interp"].ttt)
    assert np.array_equal(fine.qqq, setup["interp"].qqq)
