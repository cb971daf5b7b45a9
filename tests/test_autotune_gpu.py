"""The batch-shape autotuner (q_psdm_b200.autotune) on a small physics case:
every candidate that fits is built and timed on the caller's gathers, the
choice is the fastest measured one, a candidate whose estimated footprint
exceeds the free-memory share is skipped without being built, and the
estimate of the engine's footprint is close to what the engine allocates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
    import torch

    from q_psdm_b200 import engine as E
    from q_psdm_b200 import parallel
    from tests import physics_case as P
    case = P.make_case(nshots=4, rstep=2)
    rec = P.records(case)
    shot = parallel.source_runs(rec)
    per = int(np.bincount(shot).max())
    stream = torch.cuda.Stream()
    line = dict(fxi=case["fxi"], cyi=case["cyi"],
                dips=case["dips"].reshape(4, case["sv"].nxi, case["sv"].nzi),
                tables=case["tab"].as_engine_dict())

    def make_engine(g, nl):
        eng, p, o = P.engine(case, panel_dtype=2, form=1, max_batch=g * per)
        eng.set_stream(stream.cuda_stream)
        eng.set_lines([line] * nl)
        eng.begin_offset(o)
        return eng, stream

    def batches_of(g):
        out = []
        for k in range(3):   # shots first .. first + g - 1, whole gathers
            first = (k * g) % 4
            idx = np.nonzero((shot >= first) & (shot < first + g))[0]
            out.append((torch.from_numpy(np.ascontiguousarray(rec[idx])).cuda(), idx.size))
        return out

    return case, per, make_engine, batches_of


def test_tuner_picks_the_fastest_fitting_shape(cuda):
    from q_psdm_b200 import autotune as A
    case, per, make_engine, batches_of = _setup()
    st = case["static"]
    sv = case["sv"]

    def estimate(g, nl):
        if (g, nl) == (4, 4):
            return 1 << 60        # cannot fit: must be skipped unbuilt
        return A.footprint_bytes(max_batch=g * per, nlines=nl, ns=1000, nfft=int(st["nfft"]),
                                 nffti=int(st["nffti"]), nbins=16, panel_bytes=2, nxi=sv.nxi,
                                 nzi=sv.nzi, table_bytes_per_line=0)

    ch = A.tune_batch_shape(make_engine, batches_of, estimate,
                            [(1, 1), (2, 2), (4, 1), (4, 4)], steps=2)
    d = ch.as_dict()
    print(d)
    byshape = {(c.gathers, c.lines): c for c in ch.candidates}
    assert byshape[(4, 4)].skipped and byshape[(4, 4)].measured_bytes == 0
    done = [c for c in ch.candidates if not c.skipped]
    assert len(done) == 3 and all(c.gpt_per_s > 0 and c.point_traces > 0 for c in done)
    best = max(done, key=lambda c: c.gpt_per_s)
    assert (ch.gathers, ch.lines) == (best.gathers, best.lines)
    # panels dominate the footprint: the estimate is within 2x of the measured
    c4 = byshape[(4, 1)]
    assert 0.5 * c4.measured_bytes <= c4.estimate_bytes <= 2.0 * c4.measured_bytes
