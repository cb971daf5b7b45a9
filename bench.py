"""Benchmark of the imaging path: Gpoint-traces/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c5|c2] [--form batched|plain|compat]

A point-trace is one (image point, trace) pair inside the trace's aperture
whose source and receiver both have table values at the point -- the pairs
the imaging kernel evaluates; the engine counts them on the device, the
oracle the same way.

Workload (--config c5, the default): configuration 5, the full combined
form.  Image 1024 x 1024 x 600 at 10 m, 350 shots x 100 x 100 receivers
(3.5 M traces), nt = 3000, dt = 2 ms, 25 Hz; v(z) = 1800 + 0.5 z with a
low-velocity gas-cloud ellipsoid of Q = 20 in Q = 100; 40 dB gain limit.
The brick: 16 image lines 504..519.  Tables: the project's eikonal / t*
solver on the config-5 model (50 m grid, background-corrected) writes the
table files of lines 504 and 520 at surface nodes every 320 m (depth nodes
every 80 m) -- what the reference reads; the plain form interpolates them
between lines as get_ttt_all does; the batched form images through the
surrogate's tables: the MLP, trained on samples drawn from those solves,
evaluated at surface nodes every 160 m for every brick line, gated at 2 ms
against the eikonal tables.  Data: seeded synthetic gathers of the shots
whose sources lie within the tables' reach of the brick (|y| <= 1.5 km),
in a seeded order; each step is 8 whole gathers (80,000 traces).
--config c2 keeps configuration 2's geometry with analytic v(z) tables.

Forms (a step = one pass over one batch):
  batched  8 shot gathers into the brick of 16 image lines; FP16 t* panels
           (each trace scaled by a power of two into FP16's range), computed
           once per trace and shared by the brick; receiver-grouped
           persistent kernel; each batch replayed from a captured CUDA graph.
           The headline.
  plain    1 shot gather into 1 image line, FP32 panels, launch per shot and
           per line, as the reference organises its work; timed in the same
           run, reported under "forms" with the batched-over-plain ratio.
  compat   the reference's own (stub) kernel semantics, 1 shot into 1 line.

`value`: records resident in HBM, CUDA events on the engine's stream around
each step, L2 flushed (256 MiB write) before each step.  `e2e`: the host API
with records in pinned host memory (qpsdm_submit_traces) and the image read
back (qpsdm_get_image) every step, wall clock.

Multi-GPU (torchrun): every rank images its own shots into its own image
brick (weak scaling, no data-path collective); timings are reduced with max.

--impl reference times the reference's own CPU path for the imaging step on
the host cores: its preprocessing compiled from its sources (oracle/_ref) plus
the CPU restatement of its imaging kernel (oracle/), bounded samples.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpoint-traces/s, plain vs batched+BF16+surrogate form, at NRMSE<=1e-3 vs FP64"
# FP32 operations per point-trace.  Physics: 42 table
# interpolation, 14 ray geometry and weights, 6 time/t* pick, 2 accumulate.
# Compat: the stub body of image_depth_gpu (src/q-psdm.cu:2303-2378).
F_PT = {"batched": 64, "plain": 64, "compat": 35}
# DRAM bytes (read + write) per point-trace of the image kernel, from one ncu
# capture each (profiles/): scaled to a launch by its point-traces.
TRAFFIC_B_PER_PT = {
    "batched": (212.7e6 + 7.9e6) / 5.892e8,   # config 5, 2 gathers x 1 line capture
    "plain": (229.7e6 + 4.9e6) / 9.58e8,      # the plain form's own step
    "compat": 4.55e6 / 9.83e8,                # the compat form's own step
}
FORMS = {  # shots per step, lines per step, panel dtype, physics form
    "batched": (8, 16, 2, 1),
    "plain": (1, 1, 0, 0),
    "compat": (1, 1, 0, None),
}
DTYPE_NAME = {0: "fp32", 1: "bf16", 2: "fp16"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c5", choices=["c5", "c3", "c2"])
    ap.add_argument("--form", default="batched", choices=list(FORMS))
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-shape-tune", action="store_true",
                    help="keep the default batch shape (8 gathers x 16 lines) instead of "
                         "autotuning it")
    ap.add_argument("--no-config4", action="store_true",
                    help="skip the configuration-4 surrogate training beside the headline")
    ap.add_argument("--config4-full", action="store_true",
                    help="configuration 4 at full scale (4096 sources x 256^2 x 201 nodes; "
                         "tens of minutes) instead of the default reduced scale")
    ap.add_argument("--no-c3", action="store_true",
                    help="skip configuration 3 (uneven gathers) beside the headline")
    ap.add_argument("--only-surrogate", action="store_true",
                    help="time only the surrogate network's kernels (for profiling)")
    ap.add_argument("--only-eikonal", action="store_true",
                    help="time only the eikonal / t* table generator (one image line)")
    ap.add_argument("--eik-half", type=float, default=2000.0,
                    help="half aperture in x (m) of the eikonal tables (y: half of it)")
    ap.add_argument("--shots", type=int, default=0,
                    help="shot gathers per step of the chosen form (default: the form's own)")
    ap.add_argument("--lines", type=int, default=0,
                    help="image lines per step of the chosen form (default: the form's own)")
    ap.add_argument("--batches", type=int, default=0,
                    help="distinct batches held in HBM and cycled by the steps")
    ap.add_argument("--tile", default="",
                    help="batched kernel tile 'Z,X' instead of autotuning (for profiling)")
    ap.add_argument("--variant", type=int, default=0,
                    help="batched kernel variant (1-based, the engine's autotuner list) "
                         "instead of autotuning (for profiling)")
    ap.add_argument("--train-steps", type=int, default=4000,
                    help="training steps of the surrogate (config 5)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
class Workload:
    """Common part: static parameters, image lines, aperture, batches."""

    HALF_CDPS, HALF_LINES = 200, 100  # aperture: +-2 km in x, +-1 km in y
    LINE0 = 0
    nbatch = 2

    def __init__(self, rank: int = 0, tile=(0, 0), variant: int = 0):
        from q_psdm_b200 import synth
        self.synth = synth
        self.tile = tile
        self.variant = variant
        self.rank = rank
        self._rec = {}

    # the static parameters of a form
    def static(self, form: str, max_batch: int, use_graph: int = 0):
        from q_psdm_b200 import engine as E
        sv = self.sv
        _, _, dtype, pform = FORMS[form]
        tz, tx = self.tile if form == "batched" else (0, 0)
        kw = dict(nxi=sv.nxi, nzi=sv.nzi, ntl=sv.ntl, dt=float(sv.dt), dxi=sv.dxi, dyi=sv.dyi,
                  dzi=sv.dzi, fci=sv.fci, scaled=sv.scaled, fxv=sv.fxv, fyv=sv.fyv,
                  nxv=sv.nxi, nyv=sv.nyi, fc=sv.fpeak, threshold=sv.threshold,
                  max_batch=max_batch)
        if pform is None:
            return E.static_params(**kw)
        return E.static_params(**kw, mode=1, panel_dtype=dtype, nbins=16, dtstar=self.DTSTAR,
                               form=pform, dzii=self.dzii, tile_z=tz, tile_x=tx,
                               variant=self.variant if form == "batched" else 0,
                               use_graph=use_graph)

    def lines(self, form: str, contract_rad: float):
        sv = self.sv
        nl = FORMS[form][1]
        dips = self.synth.dip_fields(sv.nxi, sv.nzi, contract_rad)
        return [dict(fxi=sv.fxv, cyi=sv.line_y(L), dips=dips,
                     tables=None if FORMS[form][3] is None else self.tables_for(form, L))
                for L in self.form_lines(form)[:nl]]

    def aperture(self):
        return self.synth.aperture_tables(self.HALF_CDPS, self.HALF_LINES)

    def form_batches(self, form: str, nbatch: int):
        """The distinct batches a form's steps cycle through: (SU records,
        per-trace apertures or None)."""
        ns = FORMS[form][0]
        return [(self.batch(k, ns), None) for k in range(nbatch)]

    def batch(self, k: int, nshots: int) -> np.ndarray:
        """SU records (big-endian) of shots k*nshots .. k*nshots+nshots-1."""
        from q_psdm_b200 import engine as E
        out = []
        for j in range(k * nshots, k * nshots + nshots):
            sid = self.shot(j)
            if sid not in self._rec:
                sx, sy, gx, gy = self.synth.trace_geometry(self.sv, [sid])
                tr = self.traces(sid, sx, sy, gx, gy)
                self._rec[sid] = E.encode_su(sx, sy, gx, gy, tr, dt_us=2000,
                                             scalco=self.sv.scalco)
            out.append(self._rec[sid])
        return np.concatenate(out)


class Config5(Workload):
    """Configuration 5: the full combined form (batched + panels + surrogate
    tables against plain FP32 tables)."""

    LINE0 = 504
    TABLE_LINES = (504, 520)
    NLINES = 16
    DTSTAR = 0.005          # t* bins of 5 ms: 16 bins reach 80 ms (Q = 20 below the cloud)
    COARSE, FINE = 320, 160  # surface-node spacing (m) of the eikonal and surrogate tables
    HALF_X, HALF_Y = 2500.0, 1500.0  # surface reach of every table cell (m)
    H = 50.0                # eikonal grid (m)
    dzii = 80.0
    nbatch = 6

    def __init__(self, rank=0, tile=(0, 0), variant=0, train_steps=4000):
        super().__init__(rank, tile, variant)
        self.sv = self.synth.config5(seed=11)
        self.train_steps = train_steps
        sv = self.sv
        y0, y1 = sv.line_y(self.LINE0), sv.line_y(self.LINE0 + self.NLINES - 1)
        near = np.nonzero((sv.shots[:, 1] >= y0 - self.HALF_Y)
                          & (sv.shots[:, 1] <= y1 + self.HALF_Y))[0]
        rng = np.random.default_rng([11, 5])
        self.shot_ids = near[rng.permutation(near.size)]
        self.ntr_shot = len(sv.receivers)
        self.tabs = None
        self.device = 0

    def shot(self, k: int) -> int:
        return int(self.shot_ids[(self.rank * 7 + k) % len(self.shot_ids)])

    def traces(self, sid, sx, sy, gx, gy):
        sv = self.sv
        spos = np.stack([sx, sy], 1).astype(np.float64) * sv.scaled
        gpos = np.stack([gx, gy], 1).astype(np.float64) * sv.scaled
        return self.synth.pair_traces_device(sv, spos, gpos, device=self.device,
                                             seed=1000 + sid)

    def line_y_model(self, L):
        return L * self.sv.dyi

    def setup(self, dev):
        """Eikonal tables of the table lines, the surrogate and every brick
        line's plain and surrogate tables (q_psdm_b200.surrogate.brick_tables)."""
        from q_psdm_b200 import surrogate as S
        sv = self.sv
        self.device = dev
        model = self.synth.config5_model(h=self.H)
        bg = self.synth.config5_model(h=self.H, cloud=False)
        self.model, self.bg = model, bg
        self.tabs = S.brick_tables(
            model, bg, q_bg=100.0, table_lines=list(self.TABLE_LINES),
            brick_lines=list(range(self.LINE0, self.LINE0 + self.NLINES)),
            line_y_of=self.line_y_model, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi,
            zmax=(sv.nzi - 1) * sv.dzi, dzii=self.dzii, nxi1=16, coarse_dx=self.COARSE,
            coarse_dy=self.COARSE, fine_dx=self.FINE, fine_dy=self.FINE, half_x=self.HALF_X,
            half_y=self.HALF_Y, h=self.H, steps=self.train_steps, device=dev, seed=0)

    def form_lines(self, form):
        if form == "batched":
            return list(range(self.LINE0, self.LINE0 + self.NLINES))
        return [self.LINE0 + self.NLINES // 2]   # plain / compat: the brick's middle line

    def tables_for(self, form, L):
        k = L - self.LINE0
        return self.tabs["dense" if form == "batched" else "plain"][k]

    def config(self, form):
        sv = self.sv
        ns, nl, dtype, pf = FORMS[form]
        st = self.tabs["stats"] if self.tabs else {}
        return {"workload": f"config5 (image {sv.nxi}x{sv.nyi}x{sv.nzi} @10m, "
                            f"{len(sv.shots)} shots x 100x100 receivers = 3.5M traces, "
                            f"nt={sv.ntl}, dt=2ms, v(z) + gas-cloud ellipsoid Q=20 in Q=100, "
                            f"40 dB gain limit), form {form}: {ns} shot gather(s) "
                            f"({ns * self.ntr_shot} traces) x {nl} image line(s) of "
                            f"{sv.nxi}x{sv.nzi} per step",
                "form": form, "shots_per_step": ns, "lines_per_step": nl,
                "traces_per_step": ns * self.ntr_shot,
                "shots": f"{len(self.shot_ids)} shots whose sources lie within the tables' "
                         f"reach of the brick (|y - brick| <= {self.HALF_Y:.0f} m), seeded "
                         f"order; {self.nbatch} distinct batches of {ns} resident in HBM, "
                         f"cycled by the steps",
                "panels": DTYPE_NAME[dtype] if pf is not None else "none (stub kernel)",
                "tables": ("surrogate: the MLP at surface nodes every 160 m for each brick "
                           "line, gated at 2 ms against the eikonal tables"
                           if form == "batched" else
                           "eikonal tables of lines 504 and 520 (surface nodes every 320 m, "
                           "depth 80 m), interpolated between the lines as get_ttt_all does"),
                "eikonal": "config-5 model on a 50 m grid, background-corrected, t* in FP64",
                "surrogate": st,
                "aperture_cdps": self.HALF_CDPS, "aperture_lines": self.HALF_LINES,
                "dtstar_s": self.DTSTAR,
                "l2": "flushed (256 MiB write) before every timed step (inputs ~1 GB/batch)"}


class Config3(Workload):
    """Configuration 3: shot gathers of uneven size and aperture through one
    persistent imaging launch per batch."""

    LINE0 = 376
    NLINES = 16
    TABLE_LINES = (376, 392)
    DTSTAR = 0.0025
    SURF = 320               # surface-node spacing (m) of the eikonal tables
    HALF_X, HALF_Y = 2500.0, 1500.0
    H = 50.0
    dzii = 80.0
    nbatch = 4
    BATCH_TRACES = 81920     # a batched step: whole gathers up to this many traces
    HALF_CDPS, HALF_LINES = 400, 200  # the offset group's tables: the largest aperture

    def __init__(self, rank=0, tile=(0, 0), variant=0, train_steps=0):
        super().__init__(rank, tile, variant)
        sv = self.sv = self.synth.config3(seed=11)
        y0, y1 = sv.line_y(self.LINE0), sv.line_y(self.LINE0 + self.NLINES - 1)
        near = np.nonzero((sv.shots[:, 1] >= y0 - self.HALF_Y)
                          & (sv.shots[:, 1] <= y1 + self.HALF_Y))[0]
        rng = np.random.default_rng([11, 3])
        self.shot_ids = near[rng.permutation(near.size)]
        # each gather's aperture, seeded uniform in [1, 4] km: half-widths
        # in cdps (x) and lines (y, half of x) as the accuracy samples use
        ap = np.random.default_rng([11, 33]).uniform(1000.0, 4000.0, size=len(sv.shots))
        self.ap_m = ap
        self.ap_half = np.stack([np.rint(ap / sv.dxi), np.rint(0.5 * ap / sv.dyi)],
                                1).astype(np.int32)
        self.ntr_shot = int(np.mean([len(sv.gathers[i]) for i in self.shot_ids]))
        self.tabs = None
        self.device = 0
        self._packed = None

    def shot(self, k: int) -> int:
        return int(self.shot_ids[(self.rank * 7 + k) % len(self.shot_ids)])

    def traces(self, sid, sx, sy, gx, gy):
        sv = self.sv
        spos = np.stack([sx, sy], 1).astype(np.float64) * sv.scaled
        gpos = np.stack([gx, gy], 1).astype(np.float64) * sv.scaled
        return self.synth.pair_traces_device(sv, spos, gpos, device=self.device,
                                             seed=3000 + sid)

    def line_y_model(self, L):
        return L * self.sv.dyi

    def setup(self, dev):
        """Eikonal / t* tables of the two table lines (config 3's v(z) with its
        smooth random Q layers) and, per brick line, their interpolation
        between the lines on the device."""
        from q_psdm_b200 import surrogate as S
        from q_psdm_b200 import tables as T
        import torch
        sv = self.sv
        self.device = dev
        model, bg, qb = self.synth.config_models("c3", h=self.H)
        t0 = time.perf_counter()
        coarse = [T.eikonal_line_tables(
            model, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi, zmax=(sv.nzi - 1) * sv.dzi,
            line_y=self.line_y_model(L), dzii=self.dzii, nxi1=16, surf_dx=self.SURF,
            surf_dy=self.SURF, half_x=self.HALF_X, half_y=self.HALF_Y, h=self.H, background=bg,
            q_background=qb, device=dev, keep_device=True) for L in self.TABLE_LINES]
        lo, hi = self.TABLE_LINES
        plain = []
        for L in range(self.LINE0, self.LINE0 + self.NLINES):
            d = coarse[0].as_engine_dict()
            d["ttt"] = S.lerp_device(coarse[0].dev["ttt"], coarse[1].dev["ttt"], L, lo, hi)
            d["qqq"] = S.lerp_device(coarse[0].dev["qqq"], coarse[1].dev["qqq"], L, lo, hi)
            plain.append(d)
        torch.cuda.synchronize()
        self.tabs = {"plain": plain, "coarse": coarse, "eikonal_s": time.perf_counter() - t0}

    def form_lines(self, form):
        if form == "batched":
            return list(range(self.LINE0, self.LINE0 + self.NLINES))
        return [self.LINE0 + self.NLINES // 2]

    def tables_for(self, form, L):
        return self.tabs["plain"][L - self.LINE0]

    def gather(self, k: int):
        """SU records and per-trace apertures of the k-th gather (seeded order)."""
        recs = self.batch(k, 1)
        sid = self.shot(k)
        return recs, np.repeat(self.ap_half[sid][None], recs.shape[0], axis=0)

    def form_batches(self, form: str, nbatch: int):
        """batched: whole gathers packed in order up to BATCH_TRACES traces a
        batch; plain: one gather a step (launch per shot)."""
        if form != "batched":
            return [self.gather(k) for k in range(nbatch)]
        out, k, self._packed = [], 0, []
        for _ in range(nbatch):
            rs, aps, n = [], [], 0
            while True:
                r, a = self.gather(k)
                if rs and n + r.shape[0] > self.BATCH_TRACES:
                    break
                rs.append(r)
                aps.append(a)
                n += r.shape[0]
                k += 1
            out.append((np.concatenate(rs), np.concatenate(aps)))
            self._packed.append((len(rs), n))   # (gathers, traces) of each batch
        return out

    def sample_batch(self):
        """The first two gathers (records, apertures) for the accuracy sample."""
        (r0, a0), (r1, a1) = self.gather(0), self.gather(1)
        return np.concatenate([r0, r1]), np.concatenate([a0, a1])

    def config(self, form):
        sv = self.sv
        _, nl, dtype, pf = FORMS[form]
        sizes = [len(sv.gathers[i]) for i in self.shot_ids]
        return {"workload": f"config3 (image {sv.nxi}x{sv.nyi}x{sv.nzi} @10m, "
                            f"{len(sv.shots)} shot gathers of U[500,12000] traces with "
                            f"apertures U[1,4] km, nt={sv.ntl}, dt=2ms, v(z) with smooth random "
                            f"Q layers 25-150), form {form}: "
                            + (f"whole gathers packed up to {self.BATCH_TRACES} traces "
                               f"x {nl} image lines per step (one persistent launch per "
                               f"batch, replayed from a CUDA graph)" if form == "batched" else
                               "1 gather x 1 image line per step (launch per shot)"),
                "form": form, "lines_per_step": nl,
                "gathers": f"{len(self.shot_ids)} gathers whose shots lie within "
                           f"{self.HALF_Y:.0f} m of the brick, seeded order; sizes "
                           f"{min(sizes)}..{max(sizes)} (mean {np.mean(sizes):.0f}); each "
                           f"trace carries its gather's aperture (qpsdm_submit_gathers)",
                "panels": DTYPE_NAME[dtype],
                "tables": f"eikonal / t* tables of config 3's model (50 m grid) for lines "
                          f"{self.TABLE_LINES[0]} and {self.TABLE_LINES[1]} (surface nodes "
                          f"every {self.SURF} m, depth 80 m), interpolated between the lines on "
                          f"the device for every brick line",
                "dtstar_s": self.DTSTAR,
                "l2": "flushed (256 MiB write) before every timed step"}


class Config2(Workload):
    """Configuration 2's geometry with analytic v(z) tables (the previous
    headline, kept for comparison)."""

    LINE0 = 252
    DTSTAR = 0.002
    dzii = 80.0
    nbatch = 2

    def __init__(self, rank=0, tile=(0, 0), variant=0, train_steps=0):
        super().__init__(rank, tile, variant)
        self.sv = self.synth.config2(seed=11)
        ly = self.sv.line_y(self.LINE0 + 4)
        self.shot_ids = np.argsort(np.abs(self.sv.shots[:, 1] - ly), kind="stable")
        self.ntr_shot = len(self.sv.receivers)
        self._tab = None
        self.tabs = None

    def shot(self, k: int) -> int:
        return int(self.shot_ids[(self.rank * 7 + k) % len(self.shot_ids)])

    def traces(self, sid, sx, sy, gx, gy):
        return self.synth.make_traces(self.sv, [sid])

    def setup(self, dev):
        from q_psdm_b200 import tables as T
        sv = self.sv
        self._tab = T.linear_gradient_tables(
            sv, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi, zmax=(sv.nzi - 1) * sv.dzi, sub=8,
            nxi1=16, half_x=2500.0, half_y=1200.0)

    def form_lines(self, form):
        return list(range(self.LINE0, self.LINE0 + 16))

    def tables_for(self, form, L):
        return self._tab.as_engine_dict()

    def config(self, form):
        sv = self.sv
        ns, nl, dtype, pf = FORMS[form]
        return {"workload": f"config2 ({len(sv.shots)} shots x 96x96 receivers, nt={sv.ntl}, "
                            f"dt=2ms, image {sv.nxi}x{sv.nyi}x{sv.nzi} @10m), form {form}: "
                            f"{ns} shot gather(s) x {nl} image line(s) of {sv.nxi}x{sv.nzi} "
                            f"per step",
                "form": form, "shots_per_step": ns, "lines_per_step": nl,
                "traces_per_step": ns * self.ntr_shot,
                "panels": DTYPE_NAME[dtype] if pf is not None else "none (stub kernel)",
                "tables": "analytic v(z)=1800+0.5z traveltime and t* (Q=80), surface and depth "
                          "subsampled 8x, reference ttt/qqq layout",
                "aperture_cdps": self.HALF_CDPS, "aperture_lines": self.HALF_LINES,
                "l2": "flushed (256 MiB write) before every timed step"}


WORKLOADS = {"c5": Config5, "c3": Config3, "c2": Config2}


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp32_peak_tflops(torch):
    """Measured FP32 (non-tensor) throughput: cuBLAS SGEMM 8192^3, TF32 off."""
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, device="cuda")
    b = torch.randn(n, n, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def fma_peak_tflops(torch):
    """Measured FP32 FMA rate: the library's k_fma_rate (16 independent FMA
    chains per thread, 4 blocks of 512 threads per SM), best of 5 launches
    timed with CUDA events on the launching stream."""
    from q_psdm_b200 import _lib
    L = _lib.lib()
    f = L.qpsdm_internal_fma_rate
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_void_p]
    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    blocks = 4 * nsm
    out = torch.empty(blocks * 512, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    flop = C.c_double(0.0)
    best = 1e9
    for k in range(7):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = f(blocks, 4096, out.data_ptr(), C.byref(flop), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if rc != 0:
            raise RuntimeError(f"qpsdm_internal_fma_rate: {_lib.ERRORS.get(rc, rc)}")
        if k >= 2:
            best = min(best, e0.elapsed_time(e1))
    return flop.value / (best * 1e-3) / 1e12


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def _kernel_times(eng, _lib):
    return {name: eng.kernel_time(c) for name, c in
            (("gate", _lib.K_GATE), ("panels", _lib.K_PRE), ("image", _lib.K_IMAGE),
             ("grouping", _lib.K_OTHER))}


def _submit(eng, batch):
    """One batch of resident records (and per-trace apertures, if any)."""
    d, a, n = batch
    if a is None:
        eng.submit_device(d.data_ptr(), n)
    else:
        eng.submit_gathers_device(d.data_ptr(), a.data_ptr(), n)


def _eager_kernel_times(form, wl, dev, stream, dbat, max_batch, flush, nsteps=2):
    """Per-kernel CUDA-event times of `nsteps` steps of a second engine that
    runs the batches eagerly (an engine replaying CUDA graphs records no
    events inside them): the per-kernel breakdown and the image kernel's time
    per launch of a graph-timed run."""
    from q_psdm_b200 import _lib
    from q_psdm_b200 import engine as E
    import torch
    p = wl.static(form, max_batch=max_batch)
    eng = E.Engine(p, device=dev)
    try:
        eng.set_stream(stream.cuda_stream)
        eng.set_lines(wl.lines(form, p.contract))
        az = wl.aperture()
        eng.begin_offset(E.offset_params(p, 0, p.nxi, aznx1=az[0], aznx2=az[1], azny1=az[2],
                                         azny2=az[3]))
        _submit(eng, dbat[0])
        torch.cuda.synchronize()
        eng.profile(True)
        ev = []
        for k in range(nsteps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _submit(eng, dbat[k % len(dbat)])
            e1.record(stream)
            ev.append((e0, e1))
        torch.cuda.synchronize()
        kt = _kernel_times(eng, _lib)
        kt["step_wall"] = (sum(a.elapsed_time(b) for a, b in ev), nsteps)
        eng.profile(False)
    finally:
        eng.close()
    return kt, nsteps


def run_form(form, wl, args, dev, dist, *, steps, warmup, e2e=True, clocks=True):
    import torch
    from q_psdm_b200 import _lib
    from q_psdm_b200 import engine as E

    # the batched form replays each batch from a captured CUDA graph
    graph = form == "batched"
    nbatch = wl.nbatch if form == "batched" else 2
    bats = wl.form_batches(form, nbatch)   # [(records, apertures or None)]
    max_batch = max(r.shape[0] for r, _ in bats)
    p = wl.static(form, max_batch=max_batch, use_graph=int(graph))
    eng = E.Engine(p, device=dev)
    stream = torch.cuda.Stream()  # non-default: its handle is never 0
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    eng.set_lines(wl.lines(form, p.contract))
    az = wl.aperture()
    o = E.offset_params(p, 0, p.nxi, aznx1=az[0], aznx2=az[1], azny1=az[2], azny2=az[3])
    eng.begin_offset(o)
    dbat = [(torch.from_numpy(r).cuda(), None if a is None else torch.from_numpy(a).cuda(),
             r.shape[0]) for r, a in bats]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    for k in range(max(warmup, nbatch + 1)):   # every batch eager once, then captured
        _submit(eng, dbat[k % nbatch])
    torch.cuda.synchronize()
    st0 = eng.stats()
    nacc0, npt0 = st0["accepted"], st0["point_traces"]
    eng.profile(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(dev)
    if clocks:
        clk.start()
    ev = []
    for k in range(steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _submit(eng, dbat[k % nbatch])
        e1.record(stream)
        ev.append((e0, e1))
    torch.cuda.synchronize()
    ck = clk.stop() if clocks else None
    ms = sum(a.elapsed_time(b) for a, b in ev)
    st1 = eng.stats()
    nacc1, npt1 = st1["accepted"], st1["point_traces"]
    npt = npt1 - npt0
    pairs = {k: (st1[k] - st0[k]) / steps for k in ("tile_decided", "imaged")}
    kt = _kernel_times(eng, _lib)  # launch counts (graph replays included)
    eng.profile(False)
    kms = {k: v[0] / steps for k, v in kt.items()}
    img_launch = kt["image"][0] / max(kt["image"][1], 1)
    img_effective = None
    if graph:  # kernel times from eager steps of the same batches
        kte, nst = _eager_kernel_times(form, wl, dev, stream, dbat, max_batch, flush)
        wall = kte.pop("step_wall")[0] / nst
        kms = {k: v[0] / nst for k, v in kte.items()}
        img_launch = kte["image"][0] / max(kte["image"][1], 1)
        # consecutive lines run on two streams, so launch durations overlap:
        # the image kernel's share of a timed step is the step's time less
        # the gate and the panels (the grouping kernels, 1-3 % of it, run
        # beside the other stream's image launch and stay in)
        img_effective = ((ms / steps - kms["gate"] - kms["panels"])
                         / max(kte["image"][1] / nst, 1))
        kms["eager_step_wall"] = wall
    t = torch.tensor([ms, float(npt)], dtype=torch.float64, device="cuda")
    if dist:
        tm, tn = t[0:1].clone(), t[1:2].clone()
        dist.all_reduce(tm, op=dist.ReduceOp.MAX)
        dist.all_reduce(tn, op=dist.ReduceOp.SUM)
        ms_max, npt_all = float(tm.item()), float(tn.item())
    else:
        ms_max, npt_all = ms, float(npt)
    out = {"value": npt_all / (ms_max * 1e-3) / 1e9, "ms_per_step": ms_max / steps,
           "point_traces_per_step": npt_all / steps, "clocks": ck,
           "kernel_ms_per_step": kms,
           "gate_accepted_per_step": (nacc1 - nacc0) / steps,
           "pairs_per_step": dict(pairs, point_traces=npt / steps,
                                  kept_fraction=1.0 - pairs["tile_decided"] / max(npt / steps, 1),
                                  imaged_fraction=pairs["imaged"] / max(npt / steps, 1)),
           "launches": int(sum(v[1] for v in kt.values())),
           "traces_per_step": sum(dbat[k % nbatch][2] for k in range(steps)) / steps,
           "image_ms_per_launch": img_launch if img_effective is None else img_effective,
           "image_ms_per_launch_overlapped": img_launch,
           "image_launches": kt["image"][1], "npt": npt}
    if form == "batched":
        tu = eng.tuning()
        out["tuning"] = {"variant": tu["variant"], "tile_depths_cdps": tu["tile"],
                         "min_blocks_per_sm": tu["min_blocks"],
                         "variant_ms": [round(x, 3) for x in tu["variant_ms"]]}

    if e2e:
        eng.set_stream(None)
        eng.begin_offset(o)
        pinned = [torch.empty(r.shape, dtype=torch.uint8).pin_memory() for r, _ in bats]
        for pr, (r, _) in zip(pinned, bats):
            pr.numpy()[:] = r
        hosts = [(pr.numpy(), a) for pr, (_, a) in zip(pinned, bats)]

        def host_submit(h):
            if h[1] is None:
                eng.submit(h[0])
            else:
                eng.submit_gathers(h[0], h[1])
        host_submit(hosts[0])
        img = eng.get_image(True)
        shape = eng.image_shape()
        imgbuf = [torch.empty(shape, dtype=torch.float32).pin_memory().numpy()
                  for _ in range(2)]

        def timed_loop(pipelined):
            """steps x (H2D of the step's records + the step's kernels + D2H of
            the step's image), wall clock.  Pipelined: each step's image read
            is enqueued behind its kernels (qpsdm_get_image_async) and waited
            for after the next step's records are copied, so that copy
            overlaps the previous step's kernels; otherwise qpsdm_get_image
            waits after every submit."""
            _, n0 = eng.counters()
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            h2d = 0
            pending = None
            for k in range(steps):
                h = hosts[k % nbatch]
                host_submit(h)
                h2d += h[0].nbytes + (0 if h[1] is None else h[1].nbytes)
                if pipelined:
                    t = eng.get_image_async(imgbuf[k % 2], True)
                    if pending is not None:
                        eng.image_wait(pending)
                    pending = t
                else:
                    eng.get_image(True)
            if pending is not None:
                eng.image_wait(pending)
            t1 = time.perf_counter()
            _, n1 = eng.counters()
            te = torch.tensor([t1 - t0], dtype=torch.float64, device="cuda")
            nn = torch.tensor([float(n1 - n0)], dtype=torch.float64, device="cuda")
            if dist:
                dist.all_reduce(te, op=dist.ReduceOp.MAX)
                dist.all_reduce(nn, op=dist.ReduceOp.SUM)
            return float(nn.item()) / float(te.item()) / 1e9, h2d // steps

        v_sync, _ = timed_loop(False)
        v, h2d = timed_loop(True)
        out["e2e"] = {"value": v, "unit": "Gpoint-traces/s", "h2d_bytes_per_step": int(h2d),
                      "d2h_bytes_per_step": int(imgbuf[0].nbytes),
                      "path": "qpsdm_submit_traces from pinned host SU records (DMA) every "
                              "step, and every step's image read back: "
                              "qpsdm_get_image_async behind the step's kernels, "
                              "qpsdm_image_wait after the next step's records are copied",
                      "value_synchronous_reads": v_sync}
    eng.close()
    del dbat
    torch.cuda.set_stream(torch.cuda.default_stream())
    return out


# the first candidate is the default shape: the kernel-variant autotuner, which
# runs once per image shape, times its variants on that shape's first batch
SHAPE_CANDIDATES = ((8, 16), (4, 16), (8, 8), (16, 8), (16, 16))


def tune_shape(wl, dev, steps=2):
    """Gathers per batch and lines per pass of the batched form, chosen by the
    project's batch-shape autotuner (q_psdm_b200.autotune) on this workload's
    own gathers and brick lines; FORMS["batched"] takes the choice."""
    import torch
    from q_psdm_b200 import autotune as A
    from q_psdm_b200 import engine as E
    _, _, dt, pf = FORMS["batched"]
    sv = wl.sv
    stream = torch.cuda.Stream()
    cands = [(g, nl) for g, nl in SHAPE_CANDIDATES
             if nl <= wl.NLINES and g * (steps + 1) <= len(wl.shot_ids)]
    tab_bytes = {}

    def make_engine(g, nl):
        FORMS["batched"] = (g, nl, dt, pf)
        p = wl.static("batched", max_batch=g * wl.ntr_shot)
        eng = E.Engine(p, device=dev)
        eng.set_stream(stream.cuda_stream)
        eng.set_lines(wl.lines("batched", p.contract))
        az = wl.aperture()
        eng.begin_offset(E.offset_params(p, 0, p.nxi, aznx1=az[0], aznx2=az[1],
                                         azny1=az[2], azny2=az[3]))
        return eng, stream

    def batches_of(g):
        return [(torch.from_numpy(wl.batch(k, g)).cuda(), g * wl.ntr_shot)
                for k in range(steps + 1)]

    def estimate(g, nl):
        if not tab_bytes:
            t = wl.tables_for("batched", wl.LINE0)
            # t, t* and the (t, t*) pairs on the device
            tab_bytes["line"] = 4 * (int(t["ttt"].numel()) * 2 + int(t["qqq"].numel()))
        p = wl.static("batched", max_batch=g * wl.ntr_shot)
        return A.footprint_bytes(max_batch=g * wl.ntr_shot, nlines=nl, ns=sv.ntl, nfft=p.nfft,
                                 nffti=p.nffti, nbins=16, panel_bytes=2, nxi=sv.nxi,
                                 nzi=sv.nzi, table_bytes_per_line=tab_bytes["line"])

    ch = A.tune_batch_shape(make_engine, batches_of, estimate, cands, steps=steps, device=dev)
    FORMS["batched"] = (ch.gathers, ch.lines, dt, pf)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return ch.as_dict()


def run_ours(args, rank, world, dist):
    import torch
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    if args.shots or args.lines:
        ns, nl, dt, pf = FORMS[args.form]
        FORMS[args.form] = (args.shots or ns, args.lines or nl, dt, pf)
    tile = tuple(int(v) for v in args.tile.split(",")) if args.tile else (0, 0)
    wl = WORKLOADS[args.config](rank, tile, args.variant, args.train_steps)
    if args.batches:
        wl.nbatch = args.batches
    if args.lines and hasattr(wl, "NLINES"):
        wl.NLINES = args.lines
    t0 = time.perf_counter()
    wl.setup(dev)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()   # the table generator's scratch
    setup_s = time.perf_counter() - t0
    shape = None
    if (args.form == "batched" and args.config == "c5" and not (args.shots or args.lines)
            and not args.no_shape_tune):
        t1 = time.perf_counter()
        shape = tune_shape(wl, dev)
        shape["tune_s"] = time.perf_counter() - t1
        if dist:  # every rank runs rank 0's shape
            import torch
            t = torch.tensor([shape["gathers"], shape["lines"]], dtype=torch.int64,
                             device="cuda")
            dist.broadcast(t, 0)
            g, nl = (int(v) for v in t.tolist())
            FORMS["batched"] = (g, nl) + FORMS["batched"][2:]
            shape["gathers"], shape["lines"] = g, nl
    head = run_form(args.form, wl, args, dev, dist, steps=args.steps, warmup=args.warmup,
                    e2e=not args.no_e2e)
    keys = ("value", "ms_per_step", "point_traces_per_step", "kernel_ms_per_step",
            "gate_accepted_per_step", "pairs_per_step")
    forms = {args.form: {k: head[k] for k in keys}}
    if args.form == "batched":
        pl = run_form("plain", wl, args, dev, dist, steps=max(3, args.steps // 2),
                      warmup=2, e2e=False, clocks=False)
        forms["plain"] = {k: pl[k] for k in keys}
        forms["batched_over_plain"] = head["value"] / pl["value"]
    if rank != 0:
        return None, wl
    sgemm = fp32_peak_tflops(torch)
    fp32 = fma_peak_tflops(torch)
    npt_launch = head["npt"] / max(head["image_launches"], 1)
    achieved = npt_launch * F_PT[args.form] / (head["image_ms_per_launch"] * 1e-3) / 1e12
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    roof = {"bound": "fp32", "kernel": {"batched": "k_image_batched", "plain": "k_image_plain",
                                        "compat": "k_image_compat"}[args.form],
            "achieved": achieved, "peak": fp32, "unit": "TFLOP/s", "frac": achieved / fp32,
            "traffic": TRAFFIC_B_PER_PT[args.form] * npt_launch,
            "traffic_note": "DRAM bytes per launch: ncu dram__bytes_read+write per point-trace "
                            "of a smaller capture (profiles/) x this launch's point-traces",
            "flop_per_point_trace": F_PT[args.form],
            "point_traces_per_launch": npt_launch,
            "kept_fraction": head["pairs_per_step"]["kept_fraction"],
            "imaged_fraction": head["pairs_per_step"]["imaged_fraction"],
            "flop_note": "64 flop credited per point-trace; pairs decided for a whole tile "
                         "(1 - kept_fraction) execute none of them, pairs that fail the dip "
                         "test or the time window (kept - imaged) about half",
            "kernel_ms_per_launch": head["image_ms_per_launch"],
            "kernel_ms_note": "effective time per launch: the timed step's time less the "
                              "gate and panel kernels, over the step's image launches "
                              "(consecutive lines run on two streams and their launches "
                              "overlap; each launch's own duration is "
                              "kernel_ms_per_launch_overlapped)",
            "kernel_ms_per_launch_overlapped": head.get("image_ms_per_launch_overlapped"),
            "peak_source": "measured in this run: the library's FP32 FMA-chain kernel "
                           "(k_fma_rate, of measured)",
            "sgemm_tflops_measured": sgemm,
            "frac_of_sgemm": achieved / sgemm,
            "hbm_peak_gbs_measured": peaks.get("hbm_gbs"),
            "note": "imaging is a data-dependent FP32 gather/accumulate (not a dense "
                    "contraction, not HBM-bound); DRAM traffic per launch from ncu is in "
                    "profiles/"}
    res = {"metric": METRIC, "value": head["value"], "unit": "Gpoint-traces/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f32 (fp16 panels)" if args.form == "batched" else "f32",
           "data": "synthetic", "config": wl.config(args.form), "roofline": roof,
           "e2e": head.get("e2e"), "gpu_launches": head["launches"], "clocks": head["clocks"],
           "point_traces_per_step": head["point_traces_per_step"],
           "kernel_ms_per_step": head["kernel_ms_per_step"], "forms": forms,
           "setup_s": setup_s}
    if "tuning" in head:
        res["config"]["autotuned"] = head["tuning"]
    if shape is not None:
        res["config"]["batch_shape_autotuned"] = shape
    if args.form == "batched":
        res["config"]["cuda_graph"] = ("each batch replayed from a captured CUDA graph (captured "
                                       "in the warm-up steps); per-kernel times from eager steps")
    return res, wl


def run_config3(args, rank, dev, dist):
    """Configuration 3 beside the headline: uneven gathers with their own
    apertures, batched (one persistent launch per packed batch, graph
    replay) against plain (launch per shot), with e2e and an accuracy sample."""
    import torch
    wl = Config3(rank)
    t0 = time.perf_counter()
    wl.setup(dev)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    steps = max(4, args.steps // 2)
    b = run_form("batched", wl, args, dev, dist, steps=steps, warmup=args.warmup,
                 e2e=not args.no_e2e, clocks=False)
    pl = run_form("plain", wl, args, dev, dist, steps=max(4, steps), warmup=2, e2e=False,
                  clocks=False)
    keys = ("value", "ms_per_step", "traces_per_step", "point_traces_per_step",
            "kernel_ms_per_step", "gate_accepted_per_step", "pairs_per_step")
    out = {"config": wl.config("batched"),
           "forms": {"batched": {k: b[k] for k in keys}, "plain": {k: pl[k] for k in keys},
                     "batched_over_plain": b["value"] / pl["value"]},
           "e2e": b.get("e2e"), "tuning": b.get("tuning"), "image_launches": b["image_launches"],
           "batches": [{"gathers": g, "traces": n} for g, n in wl._packed],
           "steps": steps, "setup_s": setup_s, "eikonal_s": wl.tabs["eikonal_s"]}
    if rank == 0 and not (args.no_cpu or args.no_accuracy):
        out["accuracy"] = accuracy_vs_fp64(wl, dev)
    return out


# ---------------------------------------------------------------------------
# configuration 4: the surrogate trained on source positions x volume nodes
# ---------------------------------------------------------------------------
def run_config4(dev, full=False):
    """The network trained on the eikonal / t* solver's output for a grid of
    surface source positions over configuration 2's model (anomalies, 5 Q
    layers) and evaluated against the solver between the grid's sources
    (q_psdm_b200.surrogate.config4_training).  Default scale: 1024 of the
    4096 positions (every 2nd in x and y, 160 m apart) x 128 x 128 x 101
    nodes at 40 m; --config4-full: all 4096 x 256 x 256 x 201 at 20 m."""
    import torch
    from q_psdm_b200 import surrogate as S
    from q_psdm_b200 import synth
    h = 20.0 if full else 40.0
    wide = dict(xr=(-2800.0, 7900.0), yr=(-2800.0, 7900.0))
    model = synth.config2_model(h=h, **wide)
    bg = synth.config2_model(h=h, anomalies=False, layered_q=False, q=80.0, **wide)
    kw = (dict(stride=1, n=256, nz=201, h=20.0, max_batch=8) if full else
          dict(stride=2, n=128, nz=101, h=40.0, max_batch=32))
    sur, r = S.config4_training(model, bg, q_bg=80.0, n_side=64, spacing=80.0,
                                per_source=4096, steps=4000, batch=8192, held=16,
                                held_nodes=4096, device=dev, seed=0, **kw)
    sur.mlp.close()
    torch.cuda.empty_cache()
    r["scale"] = ("full" if full else
                  f"reduced: {r['pairs_solved'] / r['pairs_full']:.4f} of the configuration's "
                  f"(source, point) pairs solved")
    r["model"] = "config 2: v(z) = 1800 + 0.5 z with two seeded anomalies, 5 Q layers"
    return r


# ---------------------------------------------------------------------------
# the surrogate network (tcgen05 kernels)
# ---------------------------------------------------------------------------
# algorithmic multiply-adds per query: 5x128 + 3 x 128x128 + 128x2
MLP_MAC = 5 * 128 + 3 * 128 * 128 + 128 * 2


def run_surrogate(dev, steps, warmup, n_query=1 << 22, batch=1 << 16):
    """Inference (one launch over n_query points) and one Adam training step
    over `batch` samples, CUDA events around each on the launching stream.
    Training FLOPs are counted as 3x the forward (forward, data gradient and
    weight gradient); the kernel's recomputation of activations is extra work
    not counted."""
    import torch
    from q_psdm_b200 import surrogate as S
    torch.cuda.set_device(dev)
    net = S.Mlp(dev, seed=0)
    net.set_scaling(np.zeros(5), np.ones(5), (1.0, 25.0))
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.rand((n_query, 5), generator=g, device="cuda") * 2 - 1
    y = torch.empty((n_query, 2), device="cuda")
    xb = torch.rand((batch, 5), generator=g, device="cuda") * 2 - 1
    tb = torch.sin(3 * xb[:, :2]).contiguous()
    stream = torch.cuda.current_stream()

    def timed(fn, k):
        evs = []
        for _ in range(k):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            evs.append((e0, e1))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in evs]

    for _ in range(warmup):
        net.forward(x, out=y)
        net.train_step(xb, tb, 1e-3)
    torch.cuda.synchronize()
    inf = timed(lambda: net.forward(x, out=y), steps)
    trn = timed(lambda: net.train_step(xb, tb, 1e-3), steps)
    net.status()
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    peak = peaks.get("bf16_tflops")
    src = "MEASURED_PEAKS.json bf16_tflops (burst, of measured)"
    if peak is None:
        peak, src = 1590.0, "fallback 1.59 PFLOP/s (of fallback)"
    ms_i = statistics.median(inf)
    ms_t = statistics.median(trn)
    tf_i = 2.0 * MLP_MAC * n_query / (ms_i * 1e-3) / 1e12
    tf_t = 3 * 2.0 * MLP_MAC * batch / (ms_t * 1e-3) / 1e12
    net.close()
    return {"network": "5 -> 128x4 (SiLU) -> 2, BF16 operands, FP32 accumulation (tcgen05)",
            "inference": {"kernel": "k_mlp_forward", "queries_per_launch": n_query,
                          "ms_per_launch": ms_i, "gqueries_per_s": n_query / ms_i / 1e6,
                          "roofline": {"bound": "tensor", "achieved": tf_i, "peak": peak,
                                       "unit": "TFLOP/s", "frac": tf_i / peak,
                                       "flop_per_query": 2 * MLP_MAC, "peak_source": src}},
            "training": {"kernels": "k_mlp_grad + k_mlp_reduce + k_mlp_adam + k_mlp_pack",
                         "batch": batch, "ms_per_step": ms_t,
                         "msamples_per_s": batch / ms_t / 1e3,
                         "roofline": {"bound": "tensor", "achieved": tf_t, "peak": peak,
                                      "unit": "TFLOP/s", "frac": tf_t / peak,
                                      "flop_per_sample": 6 * MLP_MAC, "peak_source": src}}}


# ---------------------------------------------------------------------------
# the eikonal / t* table generator
# ---------------------------------------------------------------------------
def run_eikonal(dev, half_x=2000.0):
    """Tables of one config-2 image line (512 cdps, depth to 3990 m at 80 m
    nodes, 160 m surface nodes over +-half_x, +-half_x/2) from the config-2
    model (v = 1800 + 0.5 z with two +-15 % anomalies, 5 Q layers) on a 40 m
    grid, background-corrected (two solves per source).  Wall time of the
    whole generator, device synchronised at both ends."""
    import torch
    from q_psdm_b200 import synth
    from q_psdm_b200 import tables as T
    torch.cuda.set_device(dev)
    sv = synth.config2(seed=11)
    h = 40.0
    model = synth.config2_model(h=h)
    bg = synth.config2_model(h=h, anomalies=False, layered_q=False)
    line_y = Config2.LINE0 * sv.dyi
    kw = dict(fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi, zmax=(sv.nzi - 1) * sv.dzi, line_y=line_y,
              dzii=80.0, nxi1=16, surf_dx=160, surf_dy=160, half_x=half_x,
              half_y=half_x / 2, h=h, init_radius=200.0, background=bg, q_background=80.0)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tab = T.eikonal_line_tables(model, **kw)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    nsrc = len({(round(float(x), 3), round(float(y), 3))
                for c in range(tab.nxg * tab.nzg)
                for x in T.cell_surface_nodes(tab, c // tab.nzg, c % tab.nzg, sv.fci)[0]
                for y in T.cell_surface_nodes(tab, c // tab.nzg, c % tab.nzg, sv.fci)[1]})
    return {"generator": "Godunov relaxation of the eikonal and the t* transport on a local "
                         "grid per surface node, background-corrected (2 solves per source)",
            "model": "config-2: 1800+0.5z, two +-15% Gaussian anomalies (300 m), Q layers "
                     "200/120/80/50/30, 40 m grid",
            "line_tables": {"cells": tab.nxg * tab.nzg, "surface_nodes": nsrc,
                            "values": int(tab.ttt.size), "half_x_m": half_x},
            "seconds": el, "surface_nodes_per_s": nsrc / el,
            "finite": bool(np.isfinite(tab.ttt).all() and np.isfinite(tab.qqq).all())}


# ---------------------------------------------------------------------------
# CPU legs and accuracy
# ---------------------------------------------------------------------------
def _gate_params(O, wl, line):
    sv = wl.sv
    az = np.stack(wl.aperture()).astype(np.int32)
    keep = [O.iaztab()] + [np.ascontiguousarray(az[i]) for i in range(4)]
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    gp = O.GateParams(scaled=sv.scaled, fxv1=np.float32(sv.fxv - 2000.0),
                      fyv1=np.float32(sv.fyv - 1000.0),
                      exv1=np.float32(sv.fxv + sv.nxi * sv.dxi + 2000.0),
                      eyv1=np.float32(sv.fyv + sv.nyi * sv.dyi + 1000.0), fxi=sv.fxv,
                      cyi=sv.line_y(line), dxi=sv.dxi, dyi=sv.dyi, eps=0.001, nzi=sv.nzi,
                      ixstart=0, ixend=sv.nxi, iaztab=ip(keep[0]), aznx1=ip(keep[1]),
                      aznx2=ip(keep[2]), azny1=ip(keep[3]), azny2=ip(keep[4]))
    gp._keep = keep
    return gp


def _hdr_traces(rec):
    hdr = np.stack([rec[:, o:o + 4].copy().view(">i4").ravel() for o in (72, 76, 80, 84)],
                   axis=1).astype(np.int32)
    return hdr, rec[:, 240:].copy().view(">f4").astype(np.float32)


def _host_tables(t):
    """An engine table dict with host (numpy) data."""
    d = dict(t)
    for k in ("ttt", "qqq"):
        if hasattr(d[k], "cpu"):
            d[k] = d[k].cpu().numpy()
    return d


def _phys_params(O, wl, st, tab):
    sv = wl.sv
    return O.PhysParams(nzi=sv.nzi, nxb=sv.nxi, ixstart=0, nt=st["nffti"], nbins=16,
                        dt1=float(st["dt1"]), dxi=sv.dxi, dzi=sv.dzi,
                        taperzone=float(st["taperzone"]), dtstar=float(np.float32(wl.DTSTAR)),
                        dzii=wl.dzii, tcdp1=tab["cdp1"] - sv.fci, tcdp2=tab["cdp2"] - sv.fci,
                        nxg=tab["nxg"], nzg=tab["nzg"], nxi1=tab["nxi1"], nzi1=tab["nzi1"])


def _cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_compat_rate(wl, budget_s=10.0, line=None):
    """The reference's CPU path of one image line: gate, its preprocessing
    (compiled reference code when oracle/_ref exists, else the oracle) and the
    C restatement of its imaging kernel, all host threads."""
    from oracle import oracle as O
    sv = wl.sv
    line = wl.form_lines("plain")[0] if line is None else line
    st = O.derive_static(sv.ntl, np.float32(sv.dt), sv.threshold, 3.0, 8.0)
    w = O.window_split(sv.ntl, np.float32(sv.dt), 1.0, 140.0)
    gp = _gate_params(O, wl, line)
    ipar = O.ImageParams(nzi=sv.nzi, nxb=sv.nxi, ixstart=0, nt=st["nffti"], dt1=st["dt1"],
                         dxi=sv.dxi, dzi=sv.dzi, taperzone=st["taperzone"], tcdp1=0,
                         tcdp2=sv.nxi - 1)
    dips = [d.ravel() for d in wl.synth.dip_fields(sv.nxi, sv.nzi, float(st["contract"]))]
    hdr, traces = _hdr_traces(wl.batch(0, 1))
    R = O.ref_cpu()
    nthr = os.cpu_count() or 1
    img = np.zeros(sv.nxi * sv.nzi, np.float32)
    n, t_tot, npt_tot, ntr_tot, i0 = 256, 0.0, 0, 0, 0
    while True:
        sl = slice(i0 % hdr.shape[0], i0 % hdr.shape[0] + n)
        h, tr = hdr[sl], traces[sl]
        t0 = time.perf_counter()
        ints, geom = O.gate_traces(gp, h)
        ok = ints[:, 0] == 3
        nok = int(ok.sum())
        npt = 0
        if nok:
            re = np.zeros((nok, 2 * w["nww"]), np.float32)
            im = np.zeros_like(re)
            if R is not None:
                R.ref_preprocess_traces(np.ascontiguousarray(tr[ok]), nok, sv.ntl,
                                        np.float32(sv.dt), w["itb1"], w["itb2"], w["nsb"],
                                        w["nf1"], w["nww"], w["dw"], re, im, nthr)
            else:
                for k, j in enumerate(np.nonzero(ok)[0]):
                    re[k], im[k] = O.preprocess_trace(tr[j], np.float32(sv.dt), w)
            _, npt = O.image_compat(ipar, geom[ok], np.ascontiguousarray(ints[ok][:, [4, 5, 7]]),
                                    dips, img)
        t_tot += time.perf_counter() - t0
        npt_tot += npt
        ntr_tot += n
        i0 += n
        if t_tot >= budget_s or ntr_tot >= 8 * hdr.shape[0]:
            break
        if t_tot < budget_s / 8:
            n = min(hdr.shape[0], n * 2)
    kind = "reference" if R is not None else "port"
    return {"value": npt_tot / t_tot / 1e9, "unit": "Gpoint-traces/s", "cores": nthr,
            "kind": kind, "cpu_model": _cpu_model(),
            "sample": f"{ntr_tot} traces of a {wl.sv.name} shot gather into one "
                      f"{sv.nxi}x{sv.nzi} line ({npt_tot} point-traces, {t_tot:.1f} s): gate + "
                      f"the reference's preprocessing "
                      f"({'compiled from its sources' if R is not None else 'oracle'}) + C "
                      f"restatement of its image_depth_gpu (the stub body, ts = tg = 1: the "
                      f"reference has no other imaging), {nthr} threads"}


def cpu_physics_rate(wl, budget_s=12.0):
    """The physics method on the CPU in FP32: the oracle's FP32 restatement of
    the engine's plain kernel (oracle/physics_fp32.c, OpenMP over image
    points, all host threads) on panels computed in single precision by
    numpy, with the plain form's tables, on a bounded sample of one shot
    gather into one line.  Gate, panels and imaging are timed together."""
    from oracle import oracle as O
    sv = wl.sv
    line = wl.form_lines("plain")[0]
    st = O.derive_static(sv.ntl, np.float32(sv.dt), sv.threshold, 3.0, 8.0)
    gp = _gate_params(O, wl, line)
    tab = _host_tables(wl.tables_for("plain", line))
    a = O.P32(nzi=sv.nzi, nxb=sv.nxi, ixstart=0, nt=st["nffti"], nbins=16, dt1=st["dt1"],
              dxi=sv.dxi, dzi=sv.dzi, taperzone=st["taperzone"], dtstar=wl.DTSTAR,
              dzii=wl.dzii, tcdp1=tab["cdp1"] - sv.fci, tcdp2=tab["cdp2"] - sv.fci,
              nxg=tab["nxg"], nzg=tab["nzg"], nxi1=tab["nxi1"], nzi1=tab["nzi1"])
    filt = O.physics_filter(st["nfft"], np.float32(sv.dt), 130.0, 140.0, sv.fpeak,
                            sv.threshold, 16, wl.DTSTAR)
    dips = np.stack([d.ravel() for d in wl.synth.dip_fields(sv.nxi, sv.nzi,
                                                            float(st["contract"]))])
    hdr, traces = _hdr_traces(wl.batch(0, 1))
    nthr = os.cpu_count() or 1
    img = np.zeros(sv.nxi * sv.nzi, np.float32)
    rng = np.random.default_rng(1)
    n, t_tot, npt_tot, ntr_tot = 16, 0.0, 0, 0
    while True:
        idx = np.sort(rng.choice(hdr.shape[0], n, replace=False))
        t0 = time.perf_counter()
        ints, geom = O.gate_traces(gp, hdr[idx])
        ok = ints[:, 0] == 3
        npt = 0
        if ok.any():
            pan = np.zeros((n, 16, st["nffti"]), np.float32)
            pan[ok] = O.physics_panels(traces[idx][ok], np.float32(sv.dt), st["nfft"],
                                       st["nffti"], filt, fp32=True)
            _, npt, _ = O.image_plain_fp32(a, ints, geom, pan, dips, tab, img)
        t_tot += time.perf_counter() - t0
        npt_tot += npt
        ntr_tot += n
        if t_tot >= budget_s or ntr_tot >= 4096:
            break
        if t_tot < budget_s / 8:
            n = min(512, n * 2)
    return {"value": npt_tot / t_tot / 1e9, "unit": "Gpoint-traces/s", "cores": nthr,
            "kind": "port", "cpu_model": _cpu_model(),
            "sample": f"{ntr_tot} random traces of a {sv.name} shot into one {sv.nxi}x{sv.nzi} "
                      f"line ({npt_tot} point-traces, {t_tot:.1f} s): the physics method in "
                      f"FP32 on the CPU -- the FP32 C restatement of the engine's plain kernel "
                      f"(OpenMP over image points, {nthr} threads) on numpy FP32 panels, gate "
                      f"included"}


def accuracy_vs_fp64(wl, dev, ntr=1200, seed=2):
    """NRMSE of the batched-form image and of the plain FP32 image against the
    FP64 oracle on the same input and the same tables each form uses: a
    seeded sample of `ntr` traces of the step's first two shot gathers,
    imaged into the plain form's line (the brick's middle line)."""
    from oracle import oracle as O
    from q_psdm_b200 import engine as E
    sv = wl.sv
    line = wl.form_lines("plain")[0]
    rec, ap = wl.sample_batch() if hasattr(wl, "sample_batch") else (wl.batch(0, 2), None)
    rng = np.random.default_rng(seed)
    pick = np.sort(rng.choice(rec.shape[0], ntr, replace=False))
    rec = np.ascontiguousarray(rec[pick])
    ap = None if ap is None else np.ascontiguousarray(ap[pick])
    hdr, traces = _hdr_traces(rec)
    st = O.derive_static(sv.ntl, np.float32(sv.dt), sv.threshold, 3.0, 8.0)
    filt = O.physics_filter(st["nfft"], np.float32(sv.dt), 130.0, 140.0, sv.fpeak,
                            sv.threshold, 16, wl.DTSTAR)
    dips = [d.ravel() for d in wl.synth.dip_fields(sv.nxi, sv.nzi, float(st["contract"]))]
    ints, geom = O.gate_traces(_gate_params(O, wl, line), hdr, ap)
    ok = ints[:, 0] == 3
    pan = O.physics_panels(traces[ok], np.float32(sv.dt), st["nfft"], st["nffti"], filt)
    out = {"sample": f"{ntr} seeded traces of 2 {sv.name} shot gathers into line {line}"
                     + ("" if ap is None else " (each with its gather's aperture)")
                     + "; FP64 oracle: numpy float64 panels + C imaging with the form's own "
                       "tables"}
    refs = {}
    # the batched form with its FP16 panels, the plain form, and the batched
    # form with BF16 panels (the panel type the metric names) for comparison
    for form, dtype in (("batched", None), ("plain", None), ("batched", 1)):
        tab = wl.tables_for(form, line)
        if form not in refs:
            ref, npt = O.physics_image(_phys_params(O, wl, st, tab), geom[ok],
                                       ints[ok][:, [4, 5, 7]], pan, dips, _host_tables(tab))
            refs[form] = (np.asarray(ref, np.float64).reshape(sv.nxi, sv.nzi), npt)
        ref, npt = refs[form]
        saved = FORMS[form]
        if dtype is not None:
            FORMS[form] = saved[:2] + (dtype,) + saved[3:]
        try:
            p = wl.static(form, max_batch=ntr)
        finally:
            FORMS[form] = saved
        eng = E.Engine(p, device=dev)
        try:
            eng.set_lines([dict(fxi=sv.fxv, cyi=sv.line_y(line),
                                dips=wl.synth.dip_fields(sv.nxi, sv.nzi, p.contract),
                                tables=tab)])
            az = wl.aperture()
            eng.begin_offset(E.offset_params(p, 0, p.nxi, aznx1=az[0], aznx2=az[1],
                                             azny1=az[2], azny2=az[3]))
            if ap is None:
                eng.submit(rec)
            else:
                eng.submit_gathers(rec, ap)
            img = np.asarray(eng.get_image(False), np.float64).reshape(sv.nxi, sv.nzi)
            _, n = eng.counters()
        finally:
            eng.close()
        e = float(np.sqrt(np.mean((img - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))
        dt_name = DTYPE_NAME[FORMS[form][2] if dtype is None else dtype]
        out[f"nrmse_{form}_{dt_name}_panels_vs_fp64"] = e
        out[f"point_traces_{form}"] = int(n)
        if n != npt:
            out[f"point_trace_mismatch_{form}"] = [int(n), int(npt)]
    return out


def accuracy_config(name, dev, ntr=1200, eikonal=True):
    """Image NRMSE of the batched (FP16 panels) and plain (FP32 panels) forms
    against the FP64 oracle on a seeded sample of configuration `name`
    (`synth.accuracy_sample`: its own geometry, trace length, Q model, gain
    limit and image size; eikonal tables of its own model), one line."""
    from oracle import oracle as O
    from q_psdm_b200 import engine as E
    from q_psdm_b200 import synth
    smp = synth.accuracy_sample(name, ntr=ntr, eikonal=eikonal, device=dev)
    sv, tab = smp["sv"], smp["tab"]
    st = O.derive_static(sv.ntl, np.float32(sv.dt), sv.threshold, 3.0, 8.0)
    az = np.stack(smp["az"]).astype(np.int32)
    keep = [O.iaztab()] + [np.ascontiguousarray(az[i]) for i in range(4)]
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    gp = O.GateParams(scaled=sv.scaled, fxv1=np.float32(sv.fxv - 2000.0),
                      fyv1=np.float32(sv.fyv - 1000.0),
                      exv1=np.float32(sv.fxv + sv.nxi * sv.dxi + 2000.0),
                      eyv1=np.float32(sv.fyv + sv.nyi * sv.dyi + 1000.0), fxi=sv.fxv,
                      cyi=smp["cyi"], dxi=sv.dxi, dyi=sv.dyi, eps=0.001, nzi=sv.nzi,
                      ixstart=0, ixend=sv.nxi, iaztab=ip(keep[0]), aznx1=ip(keep[1]),
                      aznx2=ip(keep[2]), azny1=ip(keep[3]), azny2=ip(keep[4]))
    ints, geom = O.gate_traces(gp, smp["hdr"])
    ok = ints[:, 0] == 3
    dts = float(np.float32(smp["dtstar"]))
    filt = O.physics_filter(st["nfft"], np.float32(sv.dt), 130.0, 140.0, sv.fpeak,
                            sv.threshold, 16, smp["dtstar"])
    pan = O.physics_panels(smp["traces"][ok], np.float32(sv.dt), st["nfft"], st["nffti"], filt)
    pp = O.PhysParams(nzi=sv.nzi, nxb=sv.nxi, ixstart=0, nt=st["nffti"], nbins=16,
                      dt1=float(st["dt1"]), dxi=sv.dxi, dzi=sv.dzi,
                      taperzone=float(st["taperzone"]), dtstar=dts, dzii=tab.dzii,
                      tcdp1=tab.cdp1 - sv.fci, tcdp2=tab.cdp2 - sv.fci, nxg=tab.nxg,
                      nzg=tab.nzg, nxi1=tab.nxi1, nzi1=tab.nzi1)
    dips = [d.ravel() for d in synth.dip_fields(sv.nxi, sv.nzi, float(st["contract"]))]
    ref, npt = O.physics_image(pp, geom[ok], ints[ok][:, [4, 5, 7]], pan, dips,
                               tab.as_engine_dict())
    ref = np.asarray(ref, np.float64).reshape(sv.nxi, sv.nzi)
    out = {"sample": smp["describe"] + f" ({npt} point-traces, nt {sv.ntl}, "
                                       f"nffti {st['nffti']}, gain limit {sv.threshold:g})"}
    for form, dtype in (("batched", 2), ("plain", 0)):
        p = E.static_params(nxi=sv.nxi, nzi=sv.nzi, ntl=sv.ntl, dt=float(sv.dt), dxi=sv.dxi,
                            dyi=sv.dyi, dzi=sv.dzi, fci=sv.fci, scaled=sv.scaled, fxv=sv.fxv,
                            fyv=sv.fyv, nxv=sv.nxi, nyv=sv.nyi, fc=sv.fpeak,
                            threshold=sv.threshold, mode=1, panel_dtype=dtype, nbins=16,
                            dtstar=smp["dtstar"], form=1 if form == "batched" else 0,
                            dzii=tab.dzii, max_batch=len(smp["hdr"]))
        eng = E.Engine(p, device=dev)
        try:
            eng.set_lines([dict(fxi=sv.fxv, cyi=smp["cyi"],
                                dips=synth.dip_fields(sv.nxi, sv.nzi, p.contract),
                                tables=tab.as_engine_dict())])
            eng.begin_offset(E.offset_params(p, 0, sv.nxi, aznx1=az[0], aznx2=az[1],
                                             azny1=az[2], azny2=az[3]))
            eng.submit(smp["records"])
            img = np.asarray(eng.get_image(False), np.float64).reshape(sv.nxi, sv.nzi)
            _, n = eng.counters()
        finally:
            eng.close()
        if n != npt:
            raise RuntimeError(f"{name} {form}: point-traces {n} != oracle {npt}")
        e = float(np.sqrt(np.mean((img - ref) ** 2)) / np.sqrt(np.mean(ref ** 2)))
        out[f"nrmse_{form}_{'fp16' if dtype == 2 else 'fp32'}_panels_vs_fp64"] = e
    return out


def surrogate_truth(wl, dev):
    """Traveltime error of the surrogate's and of the plain tables against
    the eikonal solver at the plain form's line (config 5)."""
    from q_psdm_b200 import surrogate as S
    sv = wl.sv
    line = wl.form_lines("plain")[0]
    return S.truth_error_sample(
        wl.tabs["surrogate"], wl.model, wl.bg, q_bg=100.0, line_y=wl.line_y_model(line),
        plain_tables=wl.tables_for("plain", line), fci=sv.fci, dxi=sv.dxi,
        zmax=(sv.nzi - 1) * sv.dzi, dzii=wl.dzii, fine_dx=wl.FINE, fine_dy=wl.FINE,
        half_x=wl.HALF_X, half_y=wl.HALF_Y, h=wl.H, ncells=32, seed=3, device=dev)


def run_reference(args, rank, world):
    if rank != 0:
        return None
    wl = WORKLOADS[args.config](0)
    for _ in range(args.warmup):
        cpu_compat_rate(wl, budget_s=0.3)
    vals = []
    t0 = time.perf_counter()
    info = None
    for _ in range(args.steps):
        info = cpu_compat_rate(wl, budget_s=max(1.0, 60.0 / max(args.steps, 1)))
        vals.append(info["value"])
    el = time.perf_counter() - t0
    v = float(np.mean(vals))
    info = dict(info, value=v)
    sv = wl.sv
    cfg = {"workload": f"{sv.name} geometry (image {sv.nxi}x{sv.nyi}x{sv.nzi} @10m, "
                       f"nt={sv.ntl}), the reference's own CPU path: one shot gather of the "
                       f"benchmark's brick into one {sv.nxi}x{sv.nzi} image line per sample",
           "form": "reference (per trace, per line)", "shots_per_step": 1, "lines_per_step": 1,
           "computation": "gate + the reference's preprocessing compiled from its sources "
                          "(oracle/_ref: t^2 gain, tapers, two PFA r2c windows, -i w) + the C "
                          "restatement of image_depth_gpu, whose body is a stub (ts = tg = 1, "
                          "src/q-psdm.cu:2350-2351): the reference has no physics imaging, "
                          "on the CPU or elsewhere",
           "aperture_cdps": wl.HALF_CDPS, "aperture_lines": wl.HALF_LINES}
    return {"metric": METRIC, "impl": "reference", "value": v, "unit": "Gpoint-traces/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": cfg, "cpu_baseline": info,
            "e2e": {"value": v, "unit": "Gpoint-traces/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1 and args.impl != "reference":
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    if args.only_surrogate:
        res = run_surrogate(int(os.environ.get("LOCAL_RANK", "0")), args.steps, args.warmup)
    elif args.only_eikonal:
        res = run_eikonal(int(os.environ.get("LOCAL_RANK", "0")), args.eik_half)
    elif args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        res, wl = run_ours(args, rank, world, dist)
        dev = int(os.environ.get("LOCAL_RANK", "0"))
        if args.config == "c5" and args.form == "batched" and not args.no_c3:
            c3 = run_config3(args, rank, dev, dist)
            if res is not None:
                res["config3"] = c3
        if res is not None and not args.no_surrogate:
            res["surrogate"] = run_surrogate(dev, args.steps, args.warmup)
            if not args.no_config4:
                res["surrogate"]["config4"] = run_config4(dev, full=args.config4_full)
        if res is not None and not args.no_cpu:
            # the CPU leg: the oracle timed on a host sample and, unless
            # --no-accuracy, the oracle's FP64 images of seeded samples (this
            # workload's and one of configurations 1, 3 and 5 each) against
            # the engine's images of the same traces
            res["cpu_baseline"] = (cpu_compat_rate(wl) if args.form == "compat"
                                   else cpu_physics_rate(wl))
            if not args.no_accuracy:
                res["accuracy"] = accuracy_vs_fp64(wl, dev)
                if args.config == "c5":
                    res["accuracy"]["surrogate_traveltime_vs_eikonal"] = surrogate_truth(wl, dev)
                res["accuracy"]["configs"] = {n: accuracy_config(n, dev)
                                              for n in ("c1", "c2", "c3", "c5")}
    if res is not None:
        print(json.dumps(res), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
