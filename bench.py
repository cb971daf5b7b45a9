"""Benchmark of the imaging path: Gpoint-traces/s on one or more B200s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form compat|plain|batched]

A step images one shot gather (config 2 geometry: 96x96 receivers, nt=2000,
dt=2 ms) into one 512-cdp x 400-depth image line.  A point-trace is one
(image point, trace) pair inside the trace's aperture; the engine counts
them on the device.  `value` is measured with the records already resident
in HBM (qpsdm_submit_traces_device); `e2e` goes through the host API
(qpsdm_submit_traces from host records, get_image every step).  L2 is
flushed (a 256 MiB write) before every timed step; only the step is timed.

Multi-GPU (torchrun): every rank images its own shots into its own image
(weak scaling, no data-path collective); timings are reduced with max.

--impl reference times the reference's own CPU path on the host cores: the
reference's preprocessing (fetch_and_taper + pfarc compiled from its sources
into oracle/_ref, when present) plus the CPU restatement of image_depth_gpu
(oracle/), on a bounded sample of each step's traces.
"""
from __future__ import annotations

import argparse
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
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# Floating-point operations of one point-trace of the stub kernel
# (src/q-psdm.cu:2303-2378): 2 sub, 2x(3 mul/add + sqrt), 3x(2 div + add),
# 2 div, 7 mul/div (ds/dg ratio), 3 double (div, add, mul), 2 (v*tr, +=).
F_PT_COMPAT = 35


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="compat", choices=["compat"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
class Workload:
    """Config 2 geometry, one image line, shot gathers as steps."""

    LINE = 256
    HALF_CDPS, HALF_LINES = 200, 100   # aperture: +-2 km in x, +-1 km in y

    def __init__(self, rank: int = 0):
        from q_psdm_b200 import synth
        self.synth = synth
        self.sv = synth.config2(seed=11)
        self.rank = rank
        sv = self.sv
        # shots whose midpoints reach the line (|sy - line| small), per rank
        ly = sv.line_y(self.LINE)
        order = np.argsort(np.abs(sv.shots[:, 1] - ly), kind="stable")
        self.shot_ids = order
        self.ntr = len(sv.receivers)
        self.nt = sv.ntl
        self.dt = np.float32(sv.dt)
        self._rec = {}

    def records(self, k: int, big_endian=True):
        """SU records of the k-th shot of this rank (cached)."""
        from q_psdm_b200 import engine as E
        sid = int(self.shot_ids[(self.rank * 7 + k) % len(self.shot_ids)])
        key = (sid, big_endian)
        if key not in self._rec:
            sx, sy, gx, gy = self.synth.trace_geometry(self.sv, [sid])
            tr = self.synth.make_traces(self.sv, [sid])
            self._rec[key] = E.encode_su(sx, sy, gx, gy, tr, dt_us=2000,
                                         scalco=self.sv.scalco, big_endian=big_endian)
        return self._rec[key]

    def static(self, form: str, max_batch: int):
        from q_psdm_b200 import engine as E
        sv = self.sv
        return E.static_params(nxi=sv.nxi, nzi=sv.nzi, ntl=sv.ntl, dt=float(sv.dt),
                               dxi=sv.dxi, dyi=sv.dyi, dzi=sv.dzi, fci=sv.fci,
                               scaled=sv.scaled, fxv=sv.fxv, fyv=sv.fyv, nxv=sv.nxi,
                               nyv=sv.nyi, fc=30.0, max_batch=max_batch)

    def line_args(self, contract_rad):
        sv = self.sv
        dips = self.synth.dip_fields(sv.nxi, sv.nzi, contract_rad)
        return dict(fxi=sv.fxv, cyi=sv.line_y(self.LINE), dips=dips)

    def aperture(self):
        return self.synth.aperture_tables(self.HALF_CDPS, self.HALF_LINES)

    def config(self, form):
        sv = self.sv
        return {"workload": f"config2 {form}: one shot gather ({self.ntr} traces, "
                            f"nt={sv.ntl}, dt=2ms) per step into a {sv.nxi}x{sv.nzi} image "
                            f"line ({sv.nxi}x{sv.nyi}x{sv.nzi} volume, 10 m)",
                "form": form, "traces_per_step": self.ntr, "image_line": [sv.nxi, sv.nzi],
                "aperture_cdps": [self.HALF_CDPS, self.HALF_CDPS],
                "aperture_lines": [self.HALF_LINES, self.HALF_LINES],
                "l2": "flushed (256 MiB write) before every timed step",
                "data": "synthetic, seeded"}


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
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def fp32_peak_tflops(torch):
    """Measured FP32 (non-tensor) throughput: cuBLAS SGEMM with TF32 off."""
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
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def run_ours(args, rank, world, dist):
    import torch
    from q_psdm_b200 import engine as E
    from q_psdm_b200 import _lib

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    wl = Workload(rank)
    p = wl.static(args.form, max_batch=wl.ntr)
    eng = E.Engine(p, device=dev)
    # a dedicated stream: the engine runs on it and the step events are
    # recorded on it (torch's default stream handle is 0, which the C ABI
    # reads as "the engine's own stream")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    eng.set_line(**wl.line_args(p.contract))
    az = wl.aperture()
    o = E.offset_params(p, 0, p.nxi, aznx1=az[0], aznx2=az[1], azny1=az[2], azny2=az[3])
    eng.begin_offset(o)

    nsteps = args.warmup + args.steps
    nshots = min(nsteps, 4)
    recs = [wl.records(k) for k in range(nshots)]
    drecs = [torch.from_numpy(r).cuda() for r in recs]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step(k):
        eng.submit_device(drecs[k % nshots].data_ptr(), wl.ntr)

    for k in range(args.warmup):
        step(k)
    torch.cuda.synchronize()
    _, npt0 = eng.counters()
    eng.profile(True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    times = []
    for k in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step(args.warmup + k)
        e1.record(stream)
        times.append((e0, e1))
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in times)
    _, npt1 = eng.counters()
    npt = npt1 - npt0
    img_ms, img_launches = eng.kernel_time(_lib.K_IMAGE)
    launches = sum(eng.kernel_time(c)[1] for c in range(4))
    eng.profile(False)

    tot = torch.tensor([ms, float(npt)], dtype=torch.float64, device="cuda")
    if dist:
        t_max = tot[0:1].clone()
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        n_sum = tot[1:2].clone()
        dist.all_reduce(n_sum, op=dist.ReduceOp.SUM)
        ms_max, npt_all = float(t_max.item()), float(n_sum.item())
    else:
        ms_max, npt_all = ms, float(npt)
    value = npt_all / (ms_max * 1e-3) / 1e9

    # ---- end to end through the host API ---------------------------------
    e2e = None
    if not args.no_e2e:
        host_recs = recs
        eng.set_stream(None)
        eng.begin_offset(o)
        img_host = None
        eng.submit(host_recs[0])
        img_host = eng.get_image(True)
        _, n0 = eng.counters()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for k in range(args.steps):
            eng.submit(host_recs[k % nshots])
            img_host = eng.get_image(True)
        t1 = time.perf_counter()
        _, n1 = eng.counters()
        t = torch.tensor([t1 - t0], dtype=torch.float64, device="cuda")
        n = torch.tensor([float(n1 - n0)], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dist.all_reduce(n, op=dist.ReduceOp.SUM)
        e2e = {"value": float(n.item()) / float(t.item()) / 1e9, "unit": "Gpoint-traces/s",
               "h2d_bytes_per_step": int(host_recs[0].nbytes),
               "d2h_bytes_per_step": int(img_host.nbytes),
               "path": "qpsdm_submit_traces (host SU records -> pinned staging -> H2D) + "
                       "qpsdm_get_image every step"}

    result = None
    if rank == 0:
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        fp32 = fp32_peak_tflops(torch)
        peak_note = "fp32 peak measured in this run: cuBLAS SGEMM 8192^3, TF32 off"
        achieved = npt / args.steps * F_PT_COMPAT / (img_ms / max(img_launches, 1) * 1e-3) / 1e12 \
            if img_launches else None
        per_launch_npt = npt / max(img_launches, 1)
        roof = {"bound": "fp32", "kernel": "k_image_compat",
                "achieved": achieved, "peak": fp32, "unit": "TFLOP/s",
                "frac": (achieved / fp32) if achieved else None,
                "traffic": None,
                "flop_per_point_trace": F_PT_COMPAT,
                "point_traces_per_launch": per_launch_npt,
                "kernel_ms_per_launch": img_ms / max(img_launches, 1),
                "peak_source": peak_note,
                "note": "imaging is an FP32 CUDA-core gather/accumulate, not HBM or "
                        "tensor bound; traffic per launch from ncu is in profiles/"}
        if os.path.exists(peaks_path):
            roof["hbm_peak_gbs_measured"] = json.load(open(peaks_path)).get("hbm_gbs")
        result = {
            "metric": METRIC, "value": value, "unit": "Gpoint-traces/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": wl.config(args.form),
            "roofline": roof, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
            "point_traces_per_step": npt_all / args.steps,
        }
    eng.close()
    return result, wl


# ---------------------------------------------------------------------------
# CPU arm (reference CPU path / cpu_baseline)
# ---------------------------------------------------------------------------
def cpu_path_rate(wl: Workload, ntrace_sample: int, budget_s: float = 12.0):
    """Reference CPU path on a bounded sample of one shot: preprocessing by the
    reference's compiled code (or the oracle when oracle/_ref is absent) and
    the stub imaging by the C restatement, all host threads."""
    from oracle import oracle as O
    sv = wl.sv
    st = O.derive_static(sv.ntl, np.float32(sv.dt), 600.0, 3.0, 8.0)
    w = O.window_split(sv.ntl, np.float32(sv.dt), 1.0, 140.0)
    iaz = O.iaztab()
    az = np.stack(wl.aperture()).astype(np.int32)
    ly = sv.line_y(wl.LINE)
    keep = [iaz] + [np.ascontiguousarray(az[i]) for i in range(4)]
    import ctypes as C
    ip = lambda x: x.ctypes.data_as(C.POINTER(C.c_int))
    gp = O.GateParams(scaled=sv.scaled, fxv1=np.float32(sv.fxv - 2000.0),
                      fyv1=np.float32(sv.fyv - 1000.0),
                      exv1=np.float32(sv.fxv + sv.nxi * sv.dxi + 2000.0),
                      eyv1=np.float32(sv.fyv + sv.nyi * sv.dyi + 1000.0), fxi=sv.fxv, cyi=ly,
                      dxi=sv.dxi, dyi=sv.dyi, eps=0.001, nzi=sv.nzi, ixstart=0, ixend=sv.nxi,
                      iaztab=ip(keep[0]), aznx1=ip(keep[1]), aznx2=ip(keep[2]),
                      azny1=ip(keep[3]), azny2=ip(keep[4]))
    ipar = O.ImageParams(nzi=sv.nzi, nxb=sv.nxi, ixstart=0, nt=st["nffti"], dt1=st["dt1"],
                         dxi=sv.dxi, dzi=sv.dzi, taperzone=st["taperzone"], tcdp1=0,
                         tcdp2=sv.nxi - 1)
    dips = [d.ravel() for d in wl.synth.dip_fields(sv.nxi, sv.nzi, float(st["contract"]))]
    rec = wl.records(0)
    hdr = np.stack([rec[:, o:o + 4].copy().view(">i4").ravel() for o in (72, 76, 80, 84)],
                   axis=1).astype(np.int32)
    traces = rec[:, 240:].copy().view(">f4").astype(np.float32)
    R = O.ref_cpu()
    kind = "reference" if R is not None else "port"
    nthr = os.cpu_count() or 1
    img = np.zeros(sv.nxi * sv.nzi, np.float32)
    # grow the sample until it costs ~budget_s
    n = min(ntrace_sample, hdr.shape[0])
    t_total, npt_total, ntr_total = 0.0, 0, 0
    idx0 = 0
    while True:
        sl = slice(idx0 % hdr.shape[0], idx0 % hdr.shape[0] + n)
        h, tr = hdr[sl], traces[sl]
        t0 = time.perf_counter()
        ints, geom = O.gate_traces(gp, h)
        ok = ints[:, 0] == 3
        nok = int(ok.sum())
        re = np.zeros((max(nok, 1), 2 * w["nww"]), np.float32)
        im = np.zeros_like(re)
        if nok:
            if R is not None:
                R.ref_preprocess_traces(np.ascontiguousarray(tr[ok]), nok, sv.ntl,
                                        np.float32(sv.dt), w["itb1"], w["itb2"], w["nsb"],
                                        w["nf1"], w["nww"], w["dw"], re, im, nthr)
            else:
                for i, j in enumerate(np.nonzero(ok)[0]):
                    re[i], im[i] = O.preprocess_trace(tr[j], np.float32(sv.dt), w)
            _, npt = O.image_compat(ipar, geom[ok], np.ascontiguousarray(ints[ok][:, [4, 5, 7]]),
                                    dips, img)
        else:
            npt = 0
        t_total += time.perf_counter() - t0
        npt_total += npt
        ntr_total += n
        idx0 += n
        if t_total >= budget_s or ntr_total >= 4 * hdr.shape[0]:
            break
        if t_total < budget_s / 8:
            n = min(hdr.shape[0], n * 2)
    return {"value": npt_total / t_total / 1e9, "unit": "Gpoint-traces/s", "cores": nthr,
            "kind": kind,
            "sample": f"{ntr_total} traces of a config-2 shot gather into the 512x400 line "
                      f"({npt_total} point-traces, {t_total:.1f} s): gate + reference "
                      f"preprocessing ({'oracle/_ref' if R is not None else 'oracle port'}) "
                      f"+ C restatement of image_depth_gpu, {nthr} threads"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    wl = Workload(0)
    for _ in range(args.warmup):
        cpu_path_rate(wl, 64, budget_s=0.5)
    vals = []
    t0 = time.perf_counter()
    info = None
    for _ in range(args.steps):
        info = cpu_path_rate(wl, 256, budget_s=max(1.0, 60.0 / max(args.steps, 1)))
        vals.append(info["value"])
    el = time.perf_counter() - t0
    v = float(np.mean(vals))
    info = dict(info, value=v)
    return {"metric": METRIC, "impl": "reference", "value": v, "unit": "Gpoint-traces/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": wl.config("compat"), "cpu_baseline": info,
            "e2e": {"value": v, "unit": "Gpoint-traces/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = tdist
    if args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        res, wl = run_ours(args, rank, world, dist)
        if res is not None and not args.no_cpu:
            res["cpu_baseline"] = cpu_path_rate(wl, 256)
    if res is not None:
        print(json.dumps(res), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
