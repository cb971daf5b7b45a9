"""The batch-shape autotuner's host logic on the CPU (q_psdm_b200.autotune),
with a fake engine and a fake CUDA clock: the fastest candidate that fits is
chosen, a candidate whose estimate exceeds the free-memory share is not
built, a candidate whose engine cannot be built is skipped with the reason,
the measured footprint is free memory before less after, and the kernel-
variant timings of the engine that ran them are reported.  The footprint
estimate grows with traces and lines as the engine's buffers do."""
import pytest

from q_psdm_b200 import autotune as A


class _Clock:
    t = 0.0       # ms
    free = 100e9  # bytes


class _Event:
    def __init__(self, enable_timing=False):
        self.at = None

    def record(self, stream=None):
        self.at = _Clock.t

    def elapsed_time(self, other):
        return other.at - self.at


class _Engine:
    """ms per batch and point-traces per batch from the shape."""

    def __init__(self, g, nl, tuned):
        self.g, self.nl = g, nl
        self.npt = 0
        self.tuned = tuned
        _Clock.free -= 1e8 * g * nl   # what the engine "allocates"

    def submit_device(self, ptr, ntr):
        # throughput rises with lines per pass and with gathers up to 8,
        # falls past 8 gathers
        self.npt += ntr * self.nl * 1000
        per = 1.0 + 0.1 * (8 - self.g) if self.g <= 8 else 1.5
        _Clock.t += ntr * self.nl * per / (1.0 + 0.05 * self.nl)

    def stats(self):
        return {"point_traces": self.npt}

    def tuning(self):
        return {"variant": 3, "variant_ms": [1.5, 1.0] if self.tuned else [0.0, 0.0]}

    def close(self):
        _Clock.free += 1e8 * self.g * self.nl


class _Rec:
    def data_ptr(self):
        return 0


@pytest.fixture
def fake_cuda(monkeypatch):
    import torch
    _Clock.t, _Clock.free = 0.0, 100e9
    monkeypatch.setattr(torch.cuda, "set_device", lambda d: None)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a: None)
    monkeypatch.setattr(torch.cuda, "empty_cache", lambda: None)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda *a: (_Clock.free, 200e9))
    monkeypatch.setattr(torch.cuda, "Event", _Event)


def test_tuner_picks_fastest_fitting_shape(fake_cuda):
    built = []

    def make_engine(g, nl):
        if (g, nl) == (4, 4):
            raise RuntimeError("engine_create: out of memory")
        built.append((g, nl))
        return _Engine(g, nl, tuned=len(built) == 1), None

    def batches_of(g):
        return [(_Rec(), 100 * g) for _ in range(3)]

    def estimate(g, nl):
        return 1e12 if (g, nl) == (16, 16) else 1e8 * g * nl

    cands = [(8, 16), (4, 16), (4, 4), (16, 16), (16, 8), (8, 8)]
    ch = A.tune_batch_shape(make_engine, batches_of, estimate, cands, steps=2)
    by = {(c.gathers, c.lines): c for c in ch.candidates}
    assert (16, 16) not in built and by[(16, 16)].skipped.startswith("estimated")
    assert by[(4, 4)].skipped.startswith("not built") and "out of memory" in by[(4, 4)].skipped
    done = [c for c in ch.candidates if not c.skipped]
    assert len(done) == 4
    best = max(done, key=lambda c: c.gpt_per_s)
    assert (ch.gathers, ch.lines) == (best.gathers, best.lines) == (8, 16)
    assert by[(8, 16)].measured_bytes == int(1e8 * 8 * 16)
    assert by[(16, 8)].gpt_per_s < by[(8, 8)].gpt_per_s * 1.0001  # slower past 8 gathers
    d = ch.as_dict()
    assert d["kernel_variants"]["tuned_on"] == "8 x 16"
    assert d["kernel_variants"]["variant_ms"] == [1.5, 1.0]
    assert _Clock.free == 100e9   # every built engine closed


def test_tuner_fails_when_nothing_fits(fake_cuda):
    with pytest.raises(RuntimeError, match="no candidate fits"):
        A.tune_batch_shape(lambda g, nl: (_Engine(g, nl, False), None),
                           lambda g: [(_Rec(), 10)] * 3, lambda g, nl: 1e15, [(8, 16)])


def test_footprint_grows_with_traces_and_lines():
    kw = dict(ns=3000, nfft=3080, nffti=6006, nbins=16, panel_bytes=2, nxi=1024, nzi=600,
              table_bytes_per_line=50_000_000)
    a = A.footprint_bytes(max_batch=80_000, nlines=16, **kw)
    assert A.footprint_bytes(max_batch=160_000, nlines=16, **kw) > a
    assert A.footprint_bytes(max_batch=80_000, nlines=32, **kw) > a
    # the panels dominate: 80,000 traces x 16 bins x 6006 x 2 bytes
    assert a > 80_000 * 16 * 6006 * 2
