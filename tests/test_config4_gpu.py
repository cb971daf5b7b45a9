"""Configuration 4 at a reduced, stated scale: the network trained on the
eikonal / t* solver's traveltimes from a grid of surface source positions to
every node of a volume around each (config-2 model: velocity anomalies and
5 Q layers), then evaluated against the solver at seeded source positions
between the grid's sources.  Scale here: 64 of the 4096 source positions
(every 8th in x and y, 640 m apart) x 64 x 64 x 51 nodes at 40 m (of 256^3),
so about 0.08 % of the configuration's (source, point) pairs; the bench's
`surrogate.config4` section runs a larger fraction.

The network must learn (loss down by 10x), and at positions between the
solved sources it must beat the tables -- bilinear interpolation between the
four surrounding solved sources, as the imaging kernels read tables -- in
traveltime RMS error."""
import pytest

pytestmark = pytest.mark.gpu


def test_config4_reduced(cuda):
    from q_psdm_b200 import surrogate as S
    from q_psdm_b200 import synth
    wide = dict(xr=(-2800.0, 7900.0), yr=(-2800.0, 7900.0))
    model = synth.config2_model(h=40.0, **wide)
    bg = synth.config2_model(h=40.0, anomalies=False, layered_q=False, q=80.0, **wide)
    sur, r = S.config4_training(model, bg, q_bg=80.0, n_side=64, spacing=80.0, stride=8,
                                n=64, nz=51, h=40.0, per_source=4096, steps=1500,
                                batch=8192, held=12, held_nodes=2048, max_batch=32, seed=1)
    sur.mlp.close()
    print(r)
    assert r["sources"] == 64 and r["samples"] == 64 * 4096
    first, last = r["loss_first_last"]
    assert last < 0.1 * first
    tt = r["traveltime_ms"]
    assert tt["surrogate_rms"] < tt["tables_rms"]
    assert tt["surrogate_rms"] < 5.0
    assert 0.0 <= r["gated_fraction"] <= 1.0
