"""Batch-shape autotuner: shot gathers per batch and image lines per pass.

The reference sizes its work to device memory by hand: it splits the image
into `nblock` x-blocks (src/q-psdm.cu:1147-1148, :1518-1528) and images one
line per pass, each trace preprocessed again for every line.  The batched
form instead images a batch of whole shot gathers into a brick of lines in
one pass (each trace's t* panels computed once for the brick), so two sizes
decide its throughput:

* the brick (lines per pass): more lines share each trace's panels, and the
  lines of a brick are launched back to back from one captured graph;
* the gathers per batch: more gathers give each tile more members to walk
  per receiver group and fewer launches, but more sources per tile (shared
  memory per block) and more panel memory.

`tune_batch_shape` measures each candidate (gathers, lines) on the caller's
own data: it builds an engine of that shape, runs one untimed batch (which
also runs the kernel-variant autotuner of the engine for the image shape),
times `steps` batches with CUDA events on the engine's stream, reads the
point-traces the device counted, and keeps the shape with the most
point-traces per second.  A candidate whose estimated device footprint
(panels, records, spectra and per-line buffers, `footprint_bytes`) exceeds
the given share of the free HBM is not built; the measured footprint of
those that are (free memory before and after) is reported beside the
estimate.
"""
from __future__ import annotations

from dataclasses import dataclass, field

SU_HDR = 240


def footprint_bytes(*, max_batch: int, nlines: int, ns: int, nfft: int, nffti: int,
                    nbins: int, panel_bytes: int, nxi: int, nzi: int,
                    table_bytes_per_line: int) -> int:
    """Estimated device bytes of a batched physics engine: per trace the t*
    panels (nbins x nffti samples), two staged SU records, the forward
    spectrum and the grouping buffers; per line the gate outputs of every
    trace, the image (and its Kahan term), the dip fields and the tables."""
    rec = SU_HDR + 4 * ns
    per_trace = (nbins * nffti * panel_bytes + 2 * rec + 8 * (nfft // 2 + 1) + 96)
    per_line = (2 * 4 * nxi * nzi + 4 * 4 * nxi * nzi + table_bytes_per_line
                + max_batch * (8 * 4 + 4 * 4))
    return max_batch * per_trace + nlines * per_line


@dataclass
class Candidate:
    gathers: int
    lines: int
    estimate_bytes: int = 0
    measured_bytes: int = 0
    traces: float = 0.0
    ms_per_batch: float = 0.0
    point_traces: float = 0.0
    gpt_per_s: float = 0.0
    skipped: str = ""
    kernel_tuning: dict = None  # the engine's kernel-variant autotuner, if it ran here


@dataclass
class Choice:
    gathers: int
    lines: int
    candidates: list = field(default_factory=list)
    kernel_tuning: dict = None

    def as_dict(self):
        return {"gathers": self.gathers, "lines": self.lines,
                "candidates": [
                    {"gathers": c.gathers, "lines": c.lines, "gpt_per_s": round(c.gpt_per_s, 2),
                     "ms_per_batch": round(c.ms_per_batch, 3),
                     "estimate_gb": round(c.estimate_bytes / 1e9, 2),
                     "measured_gb": round(c.measured_bytes / 1e9, 2),
                     **({"skipped": c.skipped} if c.skipped else {})}
                    for c in self.candidates],
                **({"kernel_variants": {
                    "tuned_on": next(f"{c.gathers} x {c.lines}" for c in self.candidates
                                     if c.kernel_tuning),
                    "variant": self.kernel_tuning["variant"],
                    "variant_ms": [round(x, 3) for x in self.kernel_tuning["variant_ms"]]}}
                   if self.kernel_tuning else {})}


def tune_batch_shape(make_engine, batches_of, estimate, candidates, *, steps: int = 2,
                     hbm_share: float = 0.8, device: int = 0) -> Choice:
    """Pick (gathers per batch, lines per pass) among `candidates`.

    make_engine(gathers, lines) -> (engine, stream): an engine of that shape,
        lines set and offset group begun, bound to `stream`;
    batches_of(gathers) -> list of (device SU records tensor, ntr), at least
        steps + 1 batches of whole gathers;
    estimate(gathers, lines) -> estimated device bytes (`footprint_bytes`).
    """
    import torch
    torch.cuda.set_device(device)
    out = []
    for g, nl in candidates:
        c = Candidate(g, nl)
        out.append(c)
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        free0, _ = torch.cuda.mem_get_info()
        c.estimate_bytes = int(estimate(g, nl))
        if c.estimate_bytes > hbm_share * free0:
            c.skipped = (f"estimated {c.estimate_bytes / 1e9:.1f} GB > {hbm_share:.0%} of "
                         f"{free0 / 1e9:.1f} GB free")
            continue
        bats = None
        try:
            bats = batches_of(g)
            eng, stream = make_engine(g, nl)
        except Exception as exc:  # e.g. out of device memory despite the estimate
            c.skipped = f"not built: {exc}"
            del bats
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            continue
        try:
            eng.submit_device(bats[0][0].data_ptr(), bats[0][1])
            torch.cuda.synchronize()
            c.measured_bytes = int(free0 - torch.cuda.mem_get_info()[0])
            tu = eng.tuning()
            if any(x > 0 for x in tu["variant_ms"]):
                c.kernel_tuning = tu
            s0 = eng.stats()["point_traces"]
            ev = []
            ntr = 0
            for k in range(steps):
                rec, n = bats[1 + k % (len(bats) - 1)] if len(bats) > 1 else bats[0]
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                eng.submit_device(rec.data_ptr(), n)
                e1.record(stream)
                ev.append((e0, e1))
                ntr += n
            torch.cuda.synchronize()
            ms = sum(a.elapsed_time(b) for a, b in ev)
            npt = eng.stats()["point_traces"] - s0
        finally:
            eng.close()
            del bats
        c.traces = ntr / steps
        c.ms_per_batch = ms / steps
        c.point_traces = npt / steps
        c.gpt_per_s = npt / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    done = [c for c in out if not c.skipped and c.gpt_per_s > 0]
    if not done:
        raise RuntimeError("batch-shape autotuner: no candidate fits the device")
    best = max(done, key=lambda c: c.gpt_per_s)
    ch = Choice(best.gathers, best.lines, out)
    ch.kernel_tuning = next((c.kernel_tuning for c in out if c.kernel_tuning), None)
    return ch
