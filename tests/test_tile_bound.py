"""The batched kernel's tile-level dip test, restated in numpy (float64).

For an image tile (a box of cdps x depths on the line, y = 0) the kernel
bounds the unit vectors from the tile's points to a source and a receiver by
interval arithmetic over the box and drops the member when an upper bound of
one of the four dip-test functions (ux - tanx1c uz, tanx2c uz - ux, and y
alike) is negative.  Here, for random tiles, sources, receivers and per-point
dip limits: wherever the bound drops a member, no point of the tile passes
the per-point test (brute force over the tile's points), and the bound drops
most members that fail everywhere.  The CUDA code evaluates the same bound in
FP32 with a margin of 1e-4 max(1, |tan|) (the largest dip-limit tangent of
the tile): the FP32 case below does the same, with dip limits up to tan 3,
against the per-point test in FP32.  (`tests/test_physics_gpu.py` checks the
kernel's images point by point against the plain form.)
"""
import numpy as np
import pytest

TZ, TX, DX, DZ = 16, 8, 10.0, 10.0


def unit_bounds(px, py, x0, x1, z0, z1, f=np.float64):
    px, py, x0, x1, z0, z1 = (f(v) if np.isscalar(v) else np.asarray(v, f)
                              for v in (px, py, x0, x1, z0, z1))
    dxl, dxh = px - x1, px - x0
    adxmin = np.where((dxl <= 0) & (dxh >= 0), 0.0, np.minimum(np.abs(dxl), np.abs(dxh)))
    adxmax = np.maximum(np.abs(dxl), np.abs(dxh))
    irmin = f(1.0) / np.sqrt(adxmin * adxmin + py * py + z0 * z0)
    irmax = f(1.0) / np.sqrt(adxmax * adxmax + py * py + z1 * z1)
    axl = np.where(dxl >= 0, dxl * irmax, dxl * irmin)
    axh = np.where(dxh >= 0, dxh * irmin, dxh * irmax)
    ayl = np.where(py >= 0, py * irmax, py * irmin)
    ayh = np.where(py >= 0, py * irmin, py * irmax)
    return axl, axh, ayl, ayh, z0 * irmax, z1 * irmin


def corner_max(tlo, thi, vlo, vhi):
    return np.maximum(np.maximum(tlo * vlo, tlo * vhi), np.maximum(thi * vlo, thi * vhi))


def tile_keep(s, g, box, lim, f=np.float64, margin=0.0):
    a, b = unit_bounds(*s, *box, f=f), unit_bounds(*g, *box, f=f)
    lim = [(f(lo), f(hi)) for lo, hi in lim]
    uxl, uxh = a[0] + b[0], a[1] + b[1]
    uyl, uyh = a[2] + b[2], a[3] + b[3]
    uzl, uzh = a[4] + b[4], a[5] + b[5]
    (t1lo, t1hi), (t2lo, t2hi), (u1lo, u1hi), (u2lo, u2hi) = lim
    fx1 = uxh + corner_max(-t1hi, -t1lo, uzl, uzh)
    fx2 = corner_max(t2lo, t2hi, uzl, uzh) - uxl
    fy1 = uyh + corner_max(-u1hi, -u1lo, uzl, uzh)
    fy2 = corner_max(u2lo, u2hi, uzl, uzh) - uyl
    m = f(margin)
    return ~((fx1 < m) | (fx2 < m) | (fy1 < m) | (fy2 < m))


@pytest.mark.parametrize("f,tan_range", [(np.float64, (0.05, 0.35)), (np.float32, (0.05, 0.35)),
                                         (np.float32, (0.5, 3.0)), (np.float64, (0.5, 3.0))])
def test_tile_bound_is_conservative(f, tan_range):
    rng = np.random.default_rng(5)
    tz = np.deg2rad(8.0)
    dropped = dropped_fail = fail_all = 0
    for _ in range(120):
        iz0 = int(rng.integers(0, 400)) // TZ * TZ
        ix0 = int(rng.integers(0, 512)) // TX * TX
        zs = (iz0 + np.arange(TZ)) * DZ
        xs = (ix0 + np.arange(TX)) * DX
        Z, X = [a.ravel() for a in np.meshgrid(zs, xs, indexing="ij")]
        # per-point dip limits and their taper-expanded values
        t = [s_ * rng.uniform(*tan_range, Z.size) for s_ in (-1, 1, -1, 1)]
        tc = [t[0] - tz * (1 + t[0] ** 2), t[1] + tz * (1 + t[1] ** 2),
              t[2] - tz * (1 + t[2] ** 2), t[3] + tz * (1 + t[3] ** 2)]
        lim = [(c.min(), c.max()) for c in tc]
        box = (xs[0], xs[-1], zs[0], zs[-1])
        n = 400
        s = (rng.uniform(-3000, 8000, n), rng.uniform(-3000, 3000, n))
        g = (rng.uniform(-3000, 8000, n), rng.uniform(-3000, 3000, n))
        if f is np.float32:  # the kernel's margin: 1e-4 max(1, largest |tan| of the tile)
            tmax = max(max(abs(lo), abs(hi)) for lo, hi in lim)
            keep = tile_keep(s, g, box, lim, f, -1e-4 * max(1.0, tmax))
        else:
            keep = tile_keep(s, g, box, lim)
        tc = [c.astype(f) for c in tc]

        def unit(px, py):
            px, py = px.astype(f), py.astype(f)
            dx = px[:, None] - X[None].astype(f)
            dy = np.broadcast_to(py[:, None], (n, Z.size))
            dz = np.broadcast_to(Z[None].astype(f), (n, Z.size))
            r = np.sqrt(dx * dx + dy * dy + dz * dz)
            return dx / r, dy / r, dz / r

        ax, ay, az = unit(*s)
        bx, by, bz = unit(*g)
        ux, uy, uz = ax + bx, ay + by, az + bz
        passes = ((ux - tc[0] * uz > 0) & (tc[1] * uz - ux > 0)
                  & (uy - tc[2] * uz > 0) & (tc[3] * uz - uy > 0))
        anyp = passes.any(1)
        assert not (anyp & ~keep).any(), "a dropped member passes at a point of the tile"
        dropped += (~keep).sum()
        fail_all += (~anyp).sum()
        dropped_fail += (~keep & ~anyp).sum()
    # the bound is close: it drops most members that fail at every point
    assert dropped_fail == dropped and dropped >= 0.8 * fail_all
