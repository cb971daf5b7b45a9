"""Asynchronous image reads (qpsdm_get_image_async / qpsdm_image_wait): each
read lands the image as it stood after the submits before it -- the next
submit's kernels do not leak in, though that submit is enqueued before the
read is waited for -- equal to the synchronous qpsdm_get_image at the same
point, with or without the /nsb scale; more reads than the ring holds are
waited for in order; pageable host memory is refused."""
import numpy as np
import pytest

from q_psdm_b200 import parallel

pytestmark = pytest.mark.gpu


def _pinned(shape):
    import torch
    return torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()


def _batches(case, records):
    shot = parallel.source_runs(records)
    return [np.ascontiguousarray(records[shot == s]) for s in np.unique(shot)]


def test_async_reads_match_sync_reads(cuda):
    from tests import physics_case as P
    case = P.make_case(nshots=3, rstep=2)
    bats = _batches(case, P.records(case))
    # the synchronous reads after each batch
    eng, _, _ = P.engine(case, panel_dtype=2, form=1)
    try:
        want = []
        for b in bats:
            eng.submit(b)
            want.append(eng.get_image(False).copy())
        want_scaled = eng.get_image(True).copy()
    finally:
        eng.close()
    # the same batches, each read enqueued before the next submit
    eng, _, _ = P.engine(case, panel_dtype=2, form=1)
    try:
        shape = eng.image_shape()
        bufs = [_pinned(shape) for _ in bats]
        tickets = []
        for b, buf in zip(bats, bufs):
            eng.submit(b)
            tickets.append(eng.get_image_async(buf, apply_nsb_scale=False))
        scaled = _pinned(shape)
        ts = eng.get_image_async(scaled, apply_nsb_scale=True)
        for t in tickets:
            eng.image_wait(t)
        eng.image_wait(ts)
        eng.image_wait(tickets[0])   # waiting twice is harmless
        for got, w in zip(bufs, want):
            assert np.array_equal(got.reshape(w.shape), w)
        assert np.array_equal(scaled.reshape(want_scaled.shape), want_scaled)
        # more outstanding reads than the ring's 4 slots
        more = [_pinned(shape) for _ in range(6)]
        tk = [eng.get_image_async(m, apply_nsb_scale=False) for m in more]
        for t in reversed(tk):
            eng.image_wait(t)
        for m in more:
            assert np.array_equal(m.reshape(want[-1].shape), want[-1])
        # pageable memory is refused
        with pytest.raises(Exception):
            eng.get_image_async(np.zeros(shape, np.float32))
    finally:
        eng.close()
