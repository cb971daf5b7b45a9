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
        return len(self.shots) * len(self.receivers)


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
    s = sv.shots[shot_ids]
    nr = len(sv.receivers)
    sxy = np.repeat(s, nr, axis=0)
    gxy = np.tile(sv.receivers, (len(shot_ids), 1))
    scale = 1.0 / sv.scaled
    to_i = lambda a: np.rint(a * scale).astype(np.int64).astype(np.int32)
    return to_i(sxy[:, 0]), to_i(sxy[:, 1]), to_i(gxy[:, 0]), to_i(gxy[:, 1])


def make_traces(sv: Survey, shot_ids=None, noise: bool = True) -> np.ndarray:
    """Trace samples [ntr, ntl] float32 for the given shots.

    Events: the flat reflector (reflection time through the midpoint at the
    reflector depth) and the point diffractors.  Each event is the Ricker
    spectrum delayed by its traveltime, attenuated by exp(-pi f t*) with
    t* = t / Q and phase-shifted by the Kjartansson dispersion term
    exp(+2 i f t* ln(f / fpeak)).  Gaussian noise at snr_db (seeded)."""
    sx, sy, gx, gy = (a.astype(np.float64) * sv.scaled for a in trace_geometry(sv, shot_ids))
    ntr = sx.size
    n = sv.ntl
    nf = n // 2 + 1
    f = np.fft.rfftfreq(n, sv.dt)
    fpos = np.maximum(f, 1e-6)
    W = ricker_spectrum(f, sv.fpeak)
    times = []
    amps = []
    mx, my = 0.5 * (sx + gx), 0.5 * (sy + gy)
    h = 0.5 * np.hypot(gx - sx, gy - sy)
    times.append(2.0 * traveltime(sv, h, sv.reflector_z))
    amps.append(np.full(ntr, 1.0))
    for (dx, dy, dz) in sv.diffractors:
        ts = traveltime(sv, np.hypot(sx - dx, sy - dy), dz)
        tg = traveltime(sv, np.hypot(gx - dx, gy - dy), dz)
        times.append(ts + tg)
        amps.append(np.full(ntr, 0.5))
    out = np.zeros((ntr, n), np.float32)
    chunk = 4096
    for c0 in range(0, ntr, chunk):
        c1 = min(ntr, c0 + chunk)
        spec = np.zeros((c1 - c0, nf), np.complex128)
        for t, a in zip(times, amps):
            tt = t[c0:c1, None]
            tstar = tt / sv.q
            spec += (a[c0:c1, None] * W[None, :] * np.exp(-np.pi * f * tstar)
                     * np.exp(2j * fpos * tstar * np.log(fpos / sv.fpeak))
                     * np.exp(-2j * np.pi * f * tt))
        tr = np.fft.irfft(spec, n=n, axis=1) / sv.dt
        if noise:
            rng = np.random.default_rng([sv.seed, c0])
            rms = np.sqrt(np.mean(tr ** 2, axis=1, keepdims=True)) + 1e-30
            tr = tr + rng.standard_normal(tr.shape) * rms * 10 ** (-sv.snr_db / 20.0)
        out[c0:c1] = tr.astype(np.float32)
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
