"""Configurations 3 and 5 as synthesised (no GPU): uneven gathers, Q models,
and the seeded accuracy samples the GPU tests image."""
import numpy as np

from q_psdm_b200 import synth


def test_config3_gathers_and_layered_q():
    sv = synth.config3(0)
    n = np.array([len(g) for g in sv.gathers])
    assert len(sv.shots) == 1024 and n.min() >= 500 and n.max() <= 12000
    assert sv.ntraces == n.sum()
    # each gather: the nearest receivers of its shot
    s = sv.shots[7]
    d = np.hypot(*(sv.receivers - s).T)
    assert d[sv.gathers[7]].max() <= np.sort(d)[len(sv.gathers[7]) - 1] + 1e-9
    qn = sv.q_model[2]
    assert qn.min() >= 25.0 and qn.max() <= 150.0
    # t* / t is the vertical-time average of 1/Q: between the extremes
    r = synth.tstar(sv, synth.X0, synth.Y0, synth.X0, synth.Y0, np.array([300.0, 2500.0]),
                    np.ones(2))
    assert (r >= 1 / qn.max() - 1e-12).all() and (r <= 1 / qn.min() + 1e-12).all()


def test_config5_gas_cloud():
    sv = synth.config5(0)
    assert sv.ntraces == 3_500_000 and sv.threshold == 100.0
    cx, cy = synth.X0 + 5120.0, synth.Y0 + 5120.0
    # vertical path through the whole ellipsoid (2 x 450 m) against one beside it
    through = synth.tstar(sv, cx, cy, cx, cy, 3000.0, 1.0)
    beside = synth.tstar(sv, cx + 3000.0, cy, cx + 3000.0, cy, 3000.0, 1.0)
    assert abs(beside - 0.01) < 1e-12
    assert abs(through - (0.01 + 900.0 / 2550.0 * (1 / 20 - 1 / 100))) < 1e-9
    ax = synth.CLOUD_AXES[0]
    # a straight path from (cx - L, 0) down to (cx + L, 3000): the chord through
    # the cloud follows from the ellipsoid's equation, here checked numerically
    L = 1500.0
    a, b = np.array([cx - L, cy, 0.0]), np.array([cx + L, cy, 3000.0])
    s = np.linspace(0, 1, 400001)
    p = a + s[:, None] * (b - a)
    inside = (((p[:, 0] - cx) / ax) ** 2 + ((p[:, 2] - 1500.0) / synth.CLOUD_AXES[2]) ** 2) <= 1
    chord = inside.mean() * np.linalg.norm(b - a)
    got = synth.tstar(sv, a[0], a[1], b[0], b[1], b[2], 1.0)
    assert abs(got - (0.01 + chord / 2550.0 * (1 / 20 - 1 / 100))) < 2e-6


def test_config5_model_cloud():
    m = synth.config5_model(h=100.0)
    iz, iy, ix = int(1500 / 100), int((5120 - m.oy) / 100), int((5120 - m.ox) / 100)
    v_in, q_in = m.vel[iz, iy, ix], 1.0 / m.invq[iz, iy, ix]
    assert abs(v_in - 0.8 * (1800 + 0.5 * 1500)) < 1.0 and abs(q_in - 20.0) < 1e-3
    far = m.vel[iz, iy, 0], 1.0 / m.invq[iz, iy, 0]
    assert abs(far[0] - (1800 + 0.5 * 1500)) < 1e-3 and abs(far[1] - 100.0) < 1e-3


def test_accuracy_samples_build():
    for name in ("c1", "c3"):
        smp = synth.accuracy_sample(name, ntr=64)
        sv = smp["sv"]
        assert smp["traces"].shape == (64, sv.ntl)
        assert smp["records"].shape == (64, 240 + 4 * sv.ntl)
        assert np.isfinite(smp["tab"].qqq).all() and (smp["tab"].qqq > 0).any()
