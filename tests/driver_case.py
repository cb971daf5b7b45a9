"""A reference-layout project on disk for the q-psdm driver tests.

    <tmp>/proj/vel/vel_loadin            velocity grid (SU, big-endian), 128 x 128
    <tmp>/proj/data0/nofffile.rcd        "nofffile=1"
    <tmp>/proj/data0/off0/ell_off0       "0,3000"
    <tmp>/proj/data0/off0/line<L>        the case's traces, by midpoint line
    <tmp>/proj/0/mig                     path (projpath/iproc/task)
    <tmp>/tt/Lxxx.{tidx,qidx}, L<L>.{ttt,qqq}
    <tmp>/par.dat

Image line L (1-based, fldr of the velocity grid) is the case's 0-based
line L - 1.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from q_psdm_b200 import synth, tables  # noqa: E402
from q_psdm_b200 import engine as E  # noqa: E402

DRIVER = os.path.join(ROOT, "q_psdm_b200", "bin", "q-psdm")


def _be_header(n, **fields):
    """SU headers [n, 240] big-endian with the given int fields set."""
    off = dict(tracl=(0, ">i4"), fldr=(8, ">i4"), cdp=(20, ">i4"), scalco=(70, ">i2"),
               sx=(72, ">i4"), sy=(76, ">i4"), gx=(80, ">i4"), gy=(84, ">i4"),
               ns=(114, ">u2"), dt=(116, ">u2"))
    h = np.zeros((n, 240), np.uint8)
    for k, v in fields.items():
        o, dt = off[k]
        a = np.broadcast_to(np.asarray(v), (n,)).astype(dt)
        h[:, o:o + a.itemsize] = a.view(np.uint8).reshape(n, a.itemsize)
    return h


def write_velocity(path, sv, ns=4):
    """Velocity grid = image grid: cdp 1..nxi, fldr 1..nyi, coordinates in cm."""
    cdp, fldr = np.meshgrid(np.arange(1, sv.nxi + 1), np.arange(1, sv.nyi + 1))
    cdp, fldr = cdp.ravel(), fldr.ravel()
    s = 1.0 / sv.scaled
    gx = np.rint((sv.fxv + (cdp - 1) * sv.dxi) * s).astype(np.int64)
    gy = np.rint((sv.fyv + (fldr - 1) * sv.dyi) * s).astype(np.int64)
    h = _be_header(cdp.size, cdp=cdp, fldr=fldr, scalco=sv.scalco, sx=gx, sy=gy, gx=gx, gy=gy,
                   ns=ns, dt=4000)
    data = np.full((cdp.size, ns), 2000.0, ">f4").view(np.uint8).reshape(cdp.size, 4 * ns)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.concatenate([h, data], axis=1).tofile(path)


def read_su(path, ns):
    raw = np.fromfile(path, np.uint8).reshape(-1, 240 + 4 * ns)
    h = raw[:, :240]
    get = lambda o, dt: h[:, o:o + np.dtype(dt).itemsize].copy().view(dt).ravel()
    hdr = dict(tracl=get(0, ">i4"), fldr=get(8, ">i4"), cdp=get(20, ">i4"),
               trid=get(28, ">i2"), nvs=get(30, ">i2"), offset=get(36, ">i4"),
               scalco=get(70, ">i2"), sx=get(72, ">i4"), sy=get(76, ">i4"),
               gx=get(80, ">i4"), gy=get(84, ">i4"), counit=get(88, ">i2"),
               ns=get(114, ">u2"), dt=get(116, ">u2"))
    data = raw[:, 240:].copy().view(">f4").astype(np.float32)
    return hdr, data


def make_project(tmp, case, *, image_line, par_extra="", tab=None, tables_at=None,
                 offsets="0,3000", extxline=300):
    """Lay out the project for `case` (a dict with sv, hdr [ntr,4] cm ints,
    traces [ntr,ntl]).  Returns (paths dict, trace order the driver reads)."""
    sv = case["sv"]
    proj = os.path.join(tmp, "proj")
    path = os.path.join(proj, "0", "mig")
    os.makedirs(path, exist_ok=True)
    write_velocity(os.path.join(proj, "vel", "vel_loadin"), sv)
    d0 = os.path.join(proj, "data0")
    os.makedirs(os.path.join(d0, "off0"), exist_ok=True)
    open(os.path.join(d0, "nofffile.rcd"), "w").write("nofffile=1\n")
    open(os.path.join(d0, "off0", "ell_off0"), "w").write(offsets + "\n")
    hdr = case["hdr"]
    my = 0.5 * (hdr[:, 1] + hdr[:, 3]).astype(np.float64) * sv.scaled
    dline = np.rint((my - sv.fyv) / sv.dyi).astype(int) + 1
    rec = E.encode_su(hdr[:, 0], hdr[:, 1], hdr[:, 2], hdr[:, 3], case["traces"], dt_us=2000,
                      scalco=sv.scalco)
    order = []
    for L in sorted(set(dline.tolist())):
        if not 1 <= L <= sv.nyi:   # outside line1..line2: never read by the driver
            continue
        idx = np.nonzero(dline == L)[0]
        rec[idx].tofile(os.path.join(d0, "off0", f"line{L}"))
        order.append(idx)
    order = np.concatenate(order)
    tt = os.path.join(tmp, "tt")
    if tab is not None:
        for L in (tables_at or [int(image_line)]):
            tables.write_line(tt, L, tab)
    else:
        os.makedirs(tt, exist_ok=True)
    par = os.path.join(tmp, "par.dat")
    with open(par, "w") as f:
        f.write(f"""# q-psdm parameters
ntl=1000
dt=0.002          # 2 ms
line1=1
line2={sv.nyi}
zmin=0
zmax={(sv.nzi - 1) * sv.dzi:g}
dzi={sv.dzi:g}
cdp1=1
cdp2={sv.nxi}
line={image_line}
extxline={extxline}
opcrp=1
threshold=600
contract=3
taperzone=8
f4=140 \\
   # continuation of the f4 record
ninv=5
ninv=7
{par_extra}
""")
    return dict(proj=proj, path=path, par=par, tt=tt), order


def run_driver(paths, *args, nodename="node_0", timeout=600, check=True):
    cmd = [DRIVER, f"path={paths['path']}", f"parfilepath={paths['par']}",
           f"nodename={nodename}", f"ttpath={paths['tt']}"] + list(args)
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if check and r.returncode != 0:
        raise RuntimeError(f"q-psdm failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    return r


def check_params(paths, *args, **kw):
    r = run_driver(paths, "check=1", *args, **kw)
    return json.loads(r.stdout.strip().splitlines()[-1])
