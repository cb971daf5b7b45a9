"""Seeded synthetic surveys for the benchmark configurations.

The reference ships no runnable example (its data and table blobs are
missing), so every test and benchmark input is generated here: survey
geometry (shots, receivers, image grid, velocity-grid box), SU trace content
(Ricker reflections attenuated by exp(-pi f t*) with Kjartansson constant-Q
dispersion, plus seeded Gaussian noise), aperture tables and dip fields.

Traveltime in v(z) = v0 + k z from a surface point to depth z at horizontal
distance r is  T = acosh(1 + k^2 (r^2 + z^2) / (2 v0 v(z))) / k.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

X0, Y0 = 500000.0, 4000000.0  # survey origin (m): exercises the double-precision gate


@dataclass
class Survey:
    name: str
    nxi: int
    nyi: int
    nzi: int
    dxi: float
    dyi: float
    dzi: float
    ntl: int
    dt: float
    v0: float
    k: float
    q: float
    fpeak: float
    shots: np.ndarray          # [ns, 2] absolute x, y (m)
    receivers: np.ndarray      # [nr, 2] absolute x, y (m) (same spread for every shot)
    reflector_z: float = 600.0
    diffractors: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    snr_db: float = 20.0
    scalco: int = -100         # coordinates stored in cm
    fci: int = 1
    seed: int = 0
    # per-shot receiver indices (gathers of uneven size); None: every shot
    # records the whole spread
    gathers: list | None = None
    # Q model: None (constant q), ("layers", z_nodes, q_nodes) with Q linear
    # between the nodes, or ("cloud", x, y, z, (ax, ay, az), q_cloud): an
    # ellipsoid of semi-axes ax, ay, az (m) inside a background of constant q
    q_model: tuple | None = None
    threshold: float = 600.0   # gain limit of the inverse-Q filter

    @property
    def fxv(self) -> float:     # x of image cdp fci (velocity grid = image grid)
        return X0

    @property
    def fyv(self) -> float:
        return Y0

    @property
    def scaled(self) -> float:
        return -1.0 / self.scalco if self.scalco < 0 else float(max(self.scalco, 1))

    def line_y(self, line: int) -> float:
        """cyi of image line `line` (0-based), src/q-psdm.cu:1430-1431."""
        return self.fyv + line * self.dyi

    @property
    def ntraces(self) -> int:
        if self.gathers is not None:
            return int(sum(len(g) for g in self.gathers))
        return len(self.shots) * len(self.receivers)

    def receivers_of(self, shot: int) -> np.ndarray:
        return self.receivers if self.gathers is None else self.receivers[self.gathers[shot]]


def config1(seed: int = 0) -> Survey:
    """Plain method, small: image 128x128x100 at 10 m, v(z)=2000+0.6z, Q=60,
    16 shots on a 4x4 grid, 32x32 receivers at 20 m, nt=1000, dt=2 ms."""
    xs = X0 + np.array([260.0, 520.0, 780.0, 1040.0])
    shots = np.array([(x, Y0 + (y - X0)) for y in xs for x in xs])
    rx = X0 + 325.0 + 20.0 * np.arange(32)
    receivers = np.array([(x, Y0 + (y - X0)) for y in rx for x in rx])
    diff = np.array([[X0 + 400.0, Y0 + 640.0, 350.0],
                     [X0 + 640.0, Y0 + 640.0, 450.0],
                     [X0 + 900.0, Y0 + 500.0, 800.0]])
    return Survey("c1", 128, 128, 100, 10.0, 10.0, 10.0, 1000, 0.002, 2000.0, 0.6,
                  60.0, 25.0, shots, receivers, 600.0, diff, 20.0, seed=seed)


def config2(seed: int = 0) -> Survey:
    """Plain method at scale: image 512x512x400 at 10 m, v(z)=1800+0.5z, 200
    shots x 96x96 receivers, nt=2000, dt=2 ms, 30 Hz.  (Velocity anomalies and
    the layered Q live in the table generator; the gate and imaging only need
    this geometry.)"""
    sxg = X0 + 128.0 + 256.0 * np.arange(20)
    syg = Y0 + 256.0 + 512.0 * np.arange(10)
    shots = np.array([(x, y) for y in syg for x in sxg])
    rg = 5120.0 / 96.0
    r1 = rg * (0.5 + np.arange(96))
    receivers = np.array([(X0 + x, Y0 + y) for y in r1 for x in r1])
    diff = np.array([[X0 + 1500.0, Y0 + 2560.0, 1200.0],
                     [X0 + 2560.0, Y0 + 2560.0, 2000.0],
                     [X0 + 3600.0, Y0 + 2000.0, 3000.0]])
    return Survey("c2", 512, 512, 400, 10.0, 10.0, 10.0, 2000, 0.002, 1800.0, 0.5,
                  80.0, 30.0, shots, receivers, 2000.0, diff, 20.0, seed=seed)


def config3(seed: int = 0) -> Survey:
    """Batching stress case: image 768x768x500 at 10 m, v(z)=1800+0.5z,
    nt=2500, dt=2 ms, 25 Hz; 1024 shots on a 32x32 grid, each recording the
    n nearest receivers of a 128x128 spread at 60 m, n seeded uniform in
    [500, 12000] (gathers of uneven size); smooth random Q: linear between
    seeded values in [25, 150] every 700 m of depth."""
    rng = np.random.default_rng([seed, 3])
    g = X0 + 120.0 + 240.0 * np.arange(32)
    shots = np.array([(x, Y0 + (y - X0)) for y in g for x in g])
    r1 = 30.0 + 60.0 * np.arange(128)
    receivers = np.array([(X0 + x, Y0 + y) for y in r1 for x in r1])
    counts = rng.integers(500, 12001, size=len(shots))
    gathers = []
    for (sx, sy), n in zip(shots, counts):
        d2 = (receivers[:, 0] - sx) ** 2 + (receivers[:, 1] - sy) ** 2
        gathers.append(np.sort(np.argsort(d2, kind="stable")[:n]))
    zn = np.arange(0.0, 5600.0, 700.0)
    qn = rng.uniform(25.0, 150.0, size=len(zn))
    diff = np.array([[X0 + 2000.0, Y0 + 3840.0, 1500.0],
                     [X0 + 3840.0, Y0 + 3840.0, 2600.0],
                     [X0 + 5600.0, Y0 + 3000.0, 3800.0]])
    return Survey("c3", 768, 768, 500, 10.0, 10.0, 10.0, 2500, 0.002, 1800.0, 0.5,
                  80.0, 25.0, shots, receivers, 2500.0, diff, 20.0, seed=seed,
                  gathers=gathers, q_model=("layers", zn, qn))


CLOUD_AXES = (1200.0, 900.0, 450.0)  # semi-axes (m) of the config-5 gas cloud


def config5(seed: int = 0) -> Survey:
    """Large, strongly attenuating case: image 1024x1024x600 at 10 m,
    v(z)=1800+0.5z, nt=3000, dt=2 ms, 25 Hz; 350 shots (14 x 25) x 100x100
    receivers at 102.4 m = 3.5 M traces; Q = 100 with a gas-cloud ellipsoid
    of Q = 20 (semi-axes 1200 x 900 x 450 m, centre 1500 m deep under the
    middle of the image; its low velocity is in `config5_model`); 40 dB gain
    limit of the inverse-Q filter (threshold 100)."""
    sxg = X0 + 366.0 + 731.0 * np.arange(14)
    syg = Y0 + 205.0 + 410.0 * np.arange(25)
    shots = np.array([(x, y) for y in syg for x in sxg])
    r1 = 51.2 + 102.4 * np.arange(100)
    receivers = np.array([(X0 + x, Y0 + y) for y in r1 for x in r1])
    diff = np.array([[X0 + 5120.0, Y0 + 5120.0, 2500.0],
                     [X0 + 3000.0, Y0 + 5120.0, 3500.0],
                     [X0 + 7000.0, Y0 + 4500.0, 4500.0]])
    return Survey("c5", 1024, 1024, 600, 10.0, 10.0, 10.0, 3000, 0.002, 1800.0, 0.5,
                  100.0, 25.0, shots, receivers, 3000.0, diff, 20.0, seed=seed,
                  q_model=("cloud", X0 + 5120.0, Y0 + 5120.0, 1500.0, CLOUD_AXES, 20.0),
                  threshold=100.0)


def traveltime(sv: Survey, r, z):
    """Linear-gradient traveltime from the surface (z=0)."""
    r = np.asarray(r, np.float64)
    z = np.asarray(z, np.float64)
    v = sv.v0 + sv.k * z
    arg = 1.0 + sv.k ** 2 * (r * r + z * z) / (2.0 * sv.v0 * v)
    return np.arccosh(np.maximum(arg, 1.0)) / sv.k


def ricker_spectrum(f, fpeak):
    a = (f / fpeak) ** 2
    return (2.0 / np.sqrt(np.pi)) * a / fpeak * np.exp(-a)


def trace_geometry(sv: Survey, shot_ids=None):
    """(sx, sy, gx, gy) as SU integers (scalco units) for the given shots."""
    shot_ids = np.arange(len(sv.shots)) if shot_ids is None else np.asarray(shot_ids)
    rec = [sv.receivers_of(int(i)) for i in shot_ids]
    sxy = np.concatenate([np.repeat(sv.shots[i][None], len(r), axis=0)
                          for i, r in zip(shot_ids, rec)]) if len(rec) else np.zeros((0, 2))
    gxy = np.concatenate(rec) if len(rec) else np.zeros((0, 2))
    scale = 1.0 / sv.scaled
    to_i = lambda a: np.rint(a * scale).astype(np.int64).astype(np.int32)
    return to_i(sxy[:, 0]), to_i(sxy[:, 1]), to_i(gxy[:, 0]), to_i(gxy[:, 1])


def vertical_time(sv: Survey, z):
    """One-way vertical time to depth z in v(z) = v0 + k z."""
    z = np.asarray(z, np.float64)
    return np.log1p(sv.k * z / sv.v0) / sv.k if sv.k > 1e-9 else z / sv.v0


def tstar(sv: Survey, px, py, x, y, z, t):
    """t* of the straight path from the surface point (px, py, 0) to (x, y, z)
    with traveltime t (absolute coordinates, m).

    Constant Q: t / q.  Layers: t times the vertical-time average of 1/Q over
    [0, z] (Q linear between the model's nodes; the integral by 64-point
    midpoint rule).  Cloud: t / q plus (1/q_cloud - 1/q) times the time spent
    inside the ellipsoid, the chord length over v at the cloud's centre."""
    t = np.asarray(t, np.float64)
    if sv.q_model is None:
        return t / sv.q
    kind = sv.q_model[0]
    if kind == "layers":
        zn, qn = np.asarray(sv.q_model[1], float), np.asarray(sv.q_model[2], float)
        z = np.asarray(z, np.float64)
        zu, inv = np.unique(z, return_inverse=True)  # the ratio depends on z only
        u = (np.arange(64) + 0.5) / 64.0
        zz = zu[:, None] * u
        w = 1.0 / (sv.v0 + sv.k * zz)
        num = (w / np.interp(zz, zn, qn)).sum(-1)
        den = w.sum(-1)
        ratio = np.where(zu > 0, num / np.maximum(den, 1e-30), 1.0 / np.interp(0.0, zn, qn))
        return t * ratio[inv].reshape(z.shape)
    _, cx, cy, cz, axes, qc = sv.q_model
    ax = np.broadcast_to(np.asarray(axes, float), (3,))
    a = np.stack(np.broadcast_arrays(np.asarray(px, float), np.asarray(py, float),
                                     np.zeros_like(np.asarray(px, float))), -1)
    b = np.stack(np.broadcast_arrays(np.asarray(x, float), np.asarray(y, float),
                                     np.asarray(z, float)), -1)
    L = np.linalg.norm(b - a, axis=-1)
    c = np.array([cx, cy, cz])
    # chord of the segment a + s (b - a), s in [0, 1], inside the ellipsoid:
    # in coordinates scaled by the semi-axes it is a unit sphere, and the
    # parameter interval is the same in both
    a, b, c = a / ax, b / ax, c / ax
    d = b - a
    dd = np.maximum((d * d).sum(-1), 1e-30)
    s0 = ((c - a) * d).sum(-1) / dd
    m = a + s0[..., None] * d
    h2 = 1.0 - ((m - c) ** 2).sum(-1)
    half = np.sqrt(np.maximum(h2, 0.0) / dd)
    s1, s2 = np.clip(s0 - half, 0.0, 1.0), np.clip(s0 + half, 0.0, 1.0)
    chord = np.where(h2 > 0, (s2 - s1) * L, 0.0)
    tin = chord / (sv.v0 + sv.k * cz)
    return t / sv.q + tin * (1.0 / qc - 1.0 / sv.q)


def make_traces(sv: Survey, shot_ids=None, noise: bool = True) -> np.ndarray:
    """Trace samples [ntr, ntl] float32 for the given shots.

    Events: the flat reflector (reflection time through the midpoint at the
    reflector depth) and the point diffractors.  Each event is the Ricker
    spectrum delayed by its traveltime, attenuated by exp(-pi f t*) with t*
    of the survey's Q model summed over the two legs (`tstar`) and
    phase-shifted by the Kjartansson dispersion term
    exp(+2 i f t* ln(f / fpeak)).  Gaussian noise at snr_db (seeded)."""
    sx, sy, gx, gy = (a.astype(np.float64) * sv.scaled for a in trace_geometry(sv, shot_ids))
    return pair_traces(sv, np.stack([sx, sy], 1), np.stack([gx, gy], 1), noise)


def pair_traces(sv: Survey, spos: np.ndarray, gpos: np.ndarray,
                noise: bool = True) -> np.ndarray:
    """Trace samples [ntr, ntl] float32 of the (source, receiver) position
    pairs spos[i], gpos[i] (absolute x, y in m), as make_traces synthesises
    them."""
    sx, sy = spos[:, 0].astype(np.float64), spos[:, 1].astype(np.float64)
    gx, gy = gpos[:, 0].astype(np.float64), gpos[:, 1].astype(np.float64)
    ntr = sx.size
    n = sv.ntl
    nf = n // 2 + 1
    f = np.fft.rfftfreq(n, sv.dt)
    fpos = np.maximum(f, 1e-6)
    W = ricker_spectrum(f, sv.fpeak)
    times = []
    amps = []
    qstar = []
    mx, my = 0.5 * (sx + gx), 0.5 * (sy + gy)
    h = 0.5 * np.hypot(gx - sx, gy - sy)
    tr1 = traveltime(sv, h, sv.reflector_z)
    times.append(2.0 * tr1)
    amps.append(np.full(ntr, 1.0))
    qstar.append(tstar(sv, sx, sy, mx, my, sv.reflector_z, tr1)
                 + tstar(sv, gx, gy, mx, my, sv.reflector_z, tr1))
    for (dx, dy, dz) in sv.diffractors:
        ts = traveltime(sv, np.hypot(sx - dx, sy - dy), dz)
        tg = traveltime(sv, np.hypot(gx - dx, gy - dy), dz)
        times.append(ts + tg)
        amps.append(np.full(ntr, 0.5))
        qstar.append(tstar(sv, sx, sy, dx, dy, dz, ts) + tstar(sv, gx, gy, dx, dy, dz, tg))
    out = np.zeros((ntr, n), np.float32)
    chunk = 4096
    for c0 in range(0, ntr, chunk):
        c1 = min(ntr, c0 + chunk)
        spec = np.zeros((c1 - c0, nf), np.complex128)
        for t, a, q in zip(times, amps, qstar):
            tt = t[c0:c1, None]
            ts_ = q[c0:c1, None]
            spec += (a[c0:c1, None] * W[None, :] * np.exp(-np.pi * f * ts_)
                     * np.exp(2j * fpos * ts_ * np.log(fpos / sv.fpeak))
                     * np.exp(-2j * np.pi * f * tt))
        tr = np.fft.irfft(spec, n=n, axis=1) / sv.dt
        if noise:
            rng = np.random.default_rng([sv.seed, c0])
            rms = np.sqrt(np.mean(tr ** 2, axis=1, keepdims=True)) + 1e-30
            tr = tr + rng.standard_normal(tr.shape) * rms * 10 ** (-sv.snr_db / 20.0)
        out[c0:c1] = tr.astype(np.float32)
    return out


def pair_traces_device(sv: Survey, spos: np.ndarray, gpos: np.ndarray, *, device: int = 0,
                       seed: int = 0, chunk: int = 8192) -> np.ndarray:
    """pair_traces computed with torch on a GPU (float64 spectra): the same
    events, amplitudes, t* and dispersion, noise from a seeded torch
    generator.  For benchmark batches of many traces; returns float32
    [ntr, ntl] on the host."""
    import torch
    dev = torch.device("cuda", device)
    ntr, n = spos.shape[0], sv.ntl
    nf = n // 2 + 1
    f = torch.fft.rfftfreq(n, sv.dt, device=dev, dtype=torch.float64)
    fpos = torch.clamp(f, min=1e-6)
    W = torch.from_numpy(ricker_spectrum(np.fft.rfftfreq(n, sv.dt), sv.fpeak)).to(dev)
    lnf = torch.log(fpos / sv.fpeak)
    sx, sy = spos[:, 0].astype(np.float64), spos[:, 1].astype(np.float64)
    gx, gy = gpos[:, 0].astype(np.float64), gpos[:, 1].astype(np.float64)
    mx, my = 0.5 * (sx + gx), 0.5 * (sy + gy)
    h = 0.5 * np.hypot(gx - sx, gy - sy)
    tr1 = traveltime(sv, h, sv.reflector_z)
    events = [(2.0 * tr1, np.full(ntr, 1.0),
               tstar(sv, sx, sy, mx, my, sv.reflector_z, tr1)
               + tstar(sv, gx, gy, mx, my, sv.reflector_z, tr1))]
    for (dx, dy, dz) in sv.diffractors:
        ts = traveltime(sv, np.hypot(sx - dx, sy - dy), dz)
        tg = traveltime(sv, np.hypot(gx - dx, gy - dy), dz)
        events.append((ts + tg, np.full(ntr, 0.5),
                       tstar(sv, sx, sy, dx, dy, dz, ts) + tstar(sv, gx, gy, dx, dy, dz, tg)))
    out = np.empty((ntr, n), np.float32)
    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    for c0 in range(0, ntr, chunk):
        c1 = min(ntr, c0 + chunk)
        spec = torch.zeros((c1 - c0, nf), dtype=torch.complex128, device=dev)
        for t, a, q in events:
            tt = torch.from_numpy(t[c0:c1]).to(dev)[:, None]
            qq = torch.from_numpy(q[c0:c1]).to(dev)[:, None]
            aa = torch.from_numpy(a[c0:c1]).to(dev)[:, None]
            amp = aa * W[None, :] * torch.exp(-np.pi * f * qq)
            phase = 2.0 * fpos * qq * lnf - 2.0 * np.pi * f * tt
            spec += amp * torch.polar(torch.ones_like(phase), phase)
        trc = torch.fft.irfft(spec, n=n, dim=1) / sv.dt
        rms = torch.sqrt(torch.mean(trc * trc, dim=1, keepdim=True)) + 1e-30
        trc = trc + torch.randn(trc.shape, generator=gen, device=dev, dtype=torch.float64) \
            * rms * 10 ** (-sv.snr_db / 20.0)
        out[c0:c1] = trc.float().cpu().numpy()
    return out


def aperture_tables(half_cdps: int, half_lines: int, *, vary: bool = True):
    """aznx1, aznx2, azny1, azny2 (18 azimuth sectors) in image cells.

    The reference allocates these per offset group and never fills them
    (src/q-psdm.cu:1542-1545); callers supply them here.  With vary=True the
    aperture changes slightly with azimuth so that the azimuth bin matters."""
    a = np.arange(18)
    d = (a % 5) if vary else np.zeros(18, int)
    return (np.full(18, half_cdps, np.int32) - d.astype(np.int32),
            np.full(18, half_cdps, np.int32) + d.astype(np.int32),
            np.full(18, half_lines, np.int32),
            np.full(18, half_lines, np.int32))


def dip_fields(nxi: int, nzi: int, contract_rad: float):
    """Constant dip limits tan(-10deg + contract), tan(10deg - contract)
    (src/q-psdm.cu:1463-1472)."""
    lo = np.float32(np.tan(np.float32(-10 * 0.0174532925199 + contract_rad)))
    hi = np.float32(np.tan(np.float32(10 * 0.0174532925199 - contract_rad)))
    x1 = np.full((nxi, nzi), lo, np.float32)
    x2 = np.full((nxi, nzi), hi, np.float32)
    return x1, x2, x1.copy(), x2.copy()


def config2_anomalies(seed: int = 0):
    """Two seeded Gaussian velocity anomalies (+15 % and -15 %, 300 m radius)
    inside the config-2 image volume: rows of (x, y, z, relative amplitude),
    coordinates relative to the first image cdp and line."""
    rng = np.random.default_rng([seed, 2])
    xy = rng.uniform(1200.0, 3900.0, size=(2, 2))
    z = rng.uniform(900.0, 2400.0, size=2)
    return np.array([[xy[0, 0], xy[0, 1], z[0], 0.15], [xy[1, 0], xy[1, 1], z[1], -0.15]])


Q_LAYERS = ((0.0, 200.0), (600.0, 120.0), (1300.0, 80.0), (2100.0, 50.0), (3000.0, 30.0))


def config2_model(h: float = 40.0, seed: int = 0, anomalies: bool = True,
                  layered_q: bool = True, xr=(-2800.0, 7900.0), yr=(-1400.0, 6600.0),
                  zmax: float = 4200.0, v0: float = 1800.0, kz: float = 0.5, q: float = 80.0):
    """Config-2 model on a grid: v(z) = v0 + kz z plus the two anomalies, and
    the 5-layer Q model (Q 200/120/80/50/30 below 0/600/1300/2100/3000 m)."""
    from .tables import GridModel
    xs = np.arange(xr[0], xr[1] + h, h, dtype=np.float32)
    ys = np.arange(yr[0], yr[1] + h, h, dtype=np.float32)
    zs = np.arange(0.0, zmax + h, h, dtype=np.float32)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    v = v0 + kz * Z
    if anomalies:
        for ax, ay, az, amp in config2_anomalies(seed):
            r2 = (X - ax) ** 2 + (Y - ay) ** 2 + (Z - az) ** 2
            v = v * (1.0 + amp * np.exp(-r2 / (300.0 ** 2)))
    iq = np.full(v.shape, 1.0 / q, np.float32)
    if layered_q:
        for ztop, qv in Q_LAYERS:
            iq[Z >= ztop] = 1.0 / qv
    return GridModel(v.astype(np.float32), iq.astype(np.float32), h, float(xs[0]),
                     float(ys[0]), v0, kz)


def config5_model(h: float = 50.0, cloud: bool = True, xr=(-2800.0, 13100.0),
                  yr=(-1400.0, 11700.0), zmax: float = 6200.0, v0: float = 1800.0,
                  kz: float = 0.5, q: float = 100.0, q_cloud: float = 20.0,
                  dv: float = -0.2):
    """Config-5 model on a grid (coordinates relative to the first image cdp
    and line): v(z) = v0 + kz z, and a gas cloud -- the ellipsoid of
    `config5`'s Q model (centre under the middle of the image, 1500 m deep,
    semi-axes CLOUD_AXES) -- with velocity lowered by 20 % and Q = 20 inside,
    Q = 100 outside; both blend over a shell of 0.8 to 1.2 ellipsoidal radii
    so that the eikonal grid sees a smooth model."""
    from .tables import GridModel
    xs = np.arange(xr[0], xr[1] + h, h, dtype=np.float32)
    ys = np.arange(yr[0], yr[1] + h, h, dtype=np.float32)
    zs = np.arange(0.0, zmax + h, h, dtype=np.float32)
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    v = v0 + kz * Z
    iq = np.full(v.shape, 1.0 / q, np.float32)
    if cloud:
        ax, ay, az = CLOUD_AXES
        rho = np.sqrt(((X - 5120.0) / ax) ** 2 + ((Y - 5120.0) / ay) ** 2
                      + ((Z - 1500.0) / az) ** 2)
        w = np.clip((1.2 - rho) / 0.4, 0.0, 1.0)
        w = w * w * (3.0 - 2.0 * w)          # smoothstep: 1 inside, 0 outside
        v = v * (1.0 + dv * w)
        iq = (1.0 - w) / q + w / q_cloud
    return GridModel(v.astype(np.float32), iq.astype(np.float32), h, float(xs[0]),
                     float(ys[0]), v0, kz)


# ---------------------------------------------------------------------------
# seeded accuracy samples of every configuration
# ---------------------------------------------------------------------------
SAMPLES = {
    # name: (survey, line, shots near the line, dtstar (s), aperture half-width
    # (m) or None for a seeded value in [1, 4] km, table half-widths (m))
    "c1": (config1, 64, 4, 0.0015, 400.0, (900.0, 900.0)),
    "c2": (config2, 256, 2, 0.002, 2000.0, (2500.0, 1500.0)),
    "c3": (config3, 384, 3, 0.0025, None, (2500.0, 1500.0)),
    "c5": (config5, 512, 2, 0.005, 2000.0, (2500.0, 1500.0)),
}


def config_models(name: str, h: float = 50.0):
    """(model, background, Q of the background) of a configuration on a grid
    for the eikonal table generator: c2 the anomalies and the 5 Q layers,
    c3 v(z) with its smooth random Q layers, c5 the gas cloud."""
    if name == "c2":
        return (config2_model(h=h), config2_model(h=h, anomalies=False, layered_q=False),
                80.0)
    if name == "c5":
        return config5_model(h=h), config5_model(h=h, cloud=False), 100.0
    if name == "c3":
        sv = config3()
        m = config2_model(h=h, anomalies=False, layered_q=False, xr=(-2800.0, 10500.0),
                          yr=(-1400.0, 9100.0), zmax=5200.0, v0=sv.v0, kz=sv.k, q=80.0)
        zn, qn = np.asarray(sv.q_model[1], float), np.asarray(sv.q_model[2], float)
        z = np.arange(m.vel.shape[0]) * h
        m.invq[:] = (1.0 / np.interp(z, zn, qn)).astype(np.float32)[:, None, None]
        bg = config2_model(h=h, anomalies=False, layered_q=False, xr=(-2800.0, 10500.0),
                           yr=(-1400.0, 9100.0), zmax=5200.0, v0=sv.v0, kz=sv.k, q=80.0)
        return m, bg, 80.0
    raise ValueError(f"no gridded model for {name}")


def accuracy_sample(name: str, ntr: int = 1200, seed: int = 7, eikonal: bool = False,
                    device: int = 0) -> dict:
    """A seeded sample of a configuration for image accuracy against the FP64
    oracle: `ntr` traces drawn from the shots nearest to one image line (their
    gathers as the configuration records them), the line's tables and the
    aperture tables.  Tables: with eikonal=True (configurations 2, 3, 5) the
    project's eikonal / t* generator on the configuration's gridded model
    (`config_models`: anomalies and Q layers, smooth random Q, the gas
    cloud), else analytic v(z) tables with t* of the configuration's Q model
    along straight rays; surface nodes every 160 m in both."""
    from . import tables as T
    from .engine import encode_su
    make, line, nsh, dtstar, ap, (hx, hy) = SAMPLES[name]
    sv = make(seed)
    rng = np.random.default_rng([seed, 11])
    if ap is None:
        ap = float(rng.uniform(1000.0, 4000.0))
    ly = sv.line_y(line)
    near = np.argsort(np.abs(sv.shots[:, 1] - ly) + 1e-3 * np.abs(sv.shots[:, 0] - X0
                                                                   - 0.5 * sv.nxi * sv.dxi),
                      kind="stable")[:nsh]
    sx, sy, gx, gy = trace_geometry(sv, near)
    pick = np.sort(rng.choice(sx.size, min(ntr, sx.size), replace=False))
    spos = np.stack([sx[pick], sy[pick]], 1).astype(np.float64) * sv.scaled
    gpos = np.stack([gx[pick], gy[pick]], 1).astype(np.float64) * sv.scaled
    traces = pair_traces(sv, spos, gpos)
    hdr = np.stack([sx[pick], sy[pick], gx[pick], gy[pick]], 1).astype(np.int32)
    rec = encode_su(hdr[:, 0], hdr[:, 1], hdr[:, 2], hdr[:, 3], traces,
                    dt_us=int(round(sv.dt * 1e6)), scalco=sv.scalco)
    sub_n = 16  # 160 m nodes
    if eikonal and name != "c1":
        # the configuration's own model through the eikonal / t* generator
        # (surface nodes every 160 m, depth nodes every 80 m, 50 m grid)
        model, bg, qb = config_models(name, h=50.0)
        tab = T.eikonal_line_tables(model, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi,
                                    zmax=(sv.nzi - 1) * sv.dzi, line_y=line * sv.dyi,
                                    dzii=80.0, nxi1=16, surf_dx=160, surf_dy=160, half_x=hx,
                                    half_y=hy, h=50.0, background=bg, q_background=qb,
                                    device=device)
    else:
        tab = T.linear_gradient_tables(sv, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi,
                                       zmax=(sv.nzi - 1) * sv.dzi, sub=sub_n, nxi1=16,
                                       half_x=hx, half_y=hy, line_y=ly)
    half_cdps, half_lines = int(round(ap / sv.dxi)), int(round(0.5 * ap / sv.dyi))
    return dict(name=name, sv=sv, line=line, cyi=ly, hdr=hdr, traces=traces, records=rec,
                tab=tab, az=aperture_tables(half_cdps, half_lines), dtstar=dtstar,
                aperture_m=ap,
                describe=f"{len(pick)} seeded traces of the {nsh} shot gathers nearest to "
                         f"line {line} of configuration {name[1:]}, aperture +-{ap:.0f} m, "
                         + ("eikonal tables of the configuration's model"
                            if eikonal and name != "c1" else "analytic v(z) tables"))
