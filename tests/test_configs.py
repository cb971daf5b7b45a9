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


def test_oracle_gate_aperture_cap():
    """A per-trace aperture caps the azimuth tables: a cap at or above the
    tables changes nothing; a smaller one narrows the columns to
    cdpx - cap .. cdpx + cap - 1 and rejects traces whose midpoint line lies
    beyond the cap."""
    import ctypes as C
    from oracle import oracle as O
    sv = synth.config3(seed=0)
    line = 384
    ly = sv.line_y(line)
    az = np.stack(synth.aperture_tables(200, 100)).astype(np.int32)
    keep = [O.iaztab()] + [np.ascontiguousarray(az[i]) for i in range(4)]
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    gp = O.GateParams(scaled=sv.scaled, fxv1=np.float32(sv.fxv - 2000.0),
                      fyv1=np.float32(sv.fyv - 1000.0),
                      exv1=np.float32(sv.fxv + sv.nxi * sv.dxi + 2000.0),
                      eyv1=np.float32(sv.fyv + sv.nyi * sv.dyi + 1000.0), fxi=sv.fxv, cyi=ly,
                      dxi=sv.dxi, dyi=sv.dyi, eps=0.001, nzi=sv.nzi, ixstart=0, ixend=sv.nxi,
                      iaztab=ip(keep[0]), aznx1=ip(keep[1]), aznx2=ip(keep[2]),
                      azny1=ip(keep[3]), azny2=ip(keep[4]))
    sx, sy, gx, gy = synth.trace_geometry(sv, [int(np.argmin(np.abs(sv.shots[:, 1] - ly)))])
    hdr = np.stack([sx, sy, gx, gy], 1).astype(np.int32)[::7]
    base, _ = O.gate_traces(gp, hdr)
    same, _ = O.gate_traces(gp, hdr, np.full((len(hdr), 2), 1000, np.int32))
    assert (same == base).all()
    cap = np.tile(np.array([[60, 25]], np.int32), (len(hdr), 1))
    capped, _ = O.gate_traces(gp, hdr, cap)
    acc_b, acc_c = base[:, 0] == 3, capped[:, 0] == 3
    assert acc_c.sum() < acc_b.sum() and not (acc_c & ~acc_b).any()
    assert (np.abs(capped[acc_c, 2]) <= 25).all()
    cdpx = capped[acc_c, 1]
    assert (capped[acc_c, 4] >= np.maximum(cdpx - 60, 0)).all()
    assert (capped[acc_c, 5] <= cdpx + 59).all()
