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
    # vertical path through the whole cloud (1600 m) against one beside it
    through = synth.tstar(sv, cx, cy, cx, cy, 3000.0, 1.0)
    beside = synth.tstar(sv, cx + 3000.0, cy, cx + 3000.0, cy, 3000.0, 1.0)
    assert abs(beside - 0.01) < 1e-12
    assert abs(through - (0.01 + 1600.0 / 2550.0 * (1 / 20 - 1 / 100))) < 1e-9


def test_accuracy_samples_build():
    for name in ("c1", "c3"):
        smp = synth.accuracy_sample(name, ntr=64)
        sv = smp["sv"]
        assert smp["traces"].shape == (64, sv.ntl)
        assert smp["records"].shape == (64, 240 + 4 * sv.ntl)
        assert np.isfinite(smp["tab"].qqq).all() and (smp["tab"].qqq > 0).any()
