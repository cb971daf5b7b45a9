"""The q-psdm command-line driver on the CPU (check=1: keys resolved, no
imaging).  Key lookup follows the reference's getparstr/readparfile
(src/psdmpkg.cc:233-574): command line first, then par.dat records; '#'
comments, backslash continuation, a key given twice in par.dat is ignored;
defaults and derived quantities as main() (src/q-psdm.cu:383-915)."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests import compat_case
from tests.driver_case import DRIVER, check_params, make_project, run_driver

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER), reason="driver not built")


@pytest.fixture(scope="module")
def project(tmp_path_factory):
    case = compat_case.make_case("small")
    tmp = str(tmp_path_factory.mktemp("drv"))
    paths, _ = make_project(tmp, case, image_line=65,
                            par_extra="fc=30\nfc=35\nf3=300\naperx=30\napery=20")
    return case, paths


def test_paths_and_defaults(project):
    case, paths = project
    p = check_params(paths)
    proj = paths["proj"]
    assert p["projpath"] == proj and p["projname"] == "proj"
    assert p["iproc"] == 0 and p["task"] == "mig"
    assert p["offspath"] == proj + "/data0"          # default <projpath>/data<iproc>
    assert p["velfilepath"] == proj + "/vel/vel_loadin"
    assert p["infopath"] == paths["path"]
    assert p["gpu"] == 0 and p["node0"] == "node"
    assert p["fc"] == 40.0                           # given twice in par.dat: ignored
    assert p["f1"] == 1.0 and p["threshold"] == 600.0
    assert p["contract_deg"] == 3.0 and p["taperzone_deg"] == 8.0
    assert p["f4"] == 140.0                          # continued record, trailing comment
    assert p["f3"] == 135.0     # 300 -> Nyquist - 10 = 240, then f4 - f3 <= 5 -> f4 - 5
    assert p["opcrp"] == 1 and p["extxline"] == 300
    assert p["aperx"] == 30 and p["apery"] == 20
    assert p["engine"] == "compat" and p["form"] == "batched" and p["panels"] == "fp16"
    assert p["dzii"] == 48.0                         # 8 * round(50 / 8)
    assert p["noffs"] == 1 and p["offmin"] == 0.0 and p["offmax"] == 3000.0
    assert (p["nfft"], p["nffti"]) == (1008, 2002)


def test_geometry_from_velocity_and_data(project):
    case, paths = project
    sv = case["sv"]
    p = check_params(paths)
    assert (p["nxi"], p["nzi"], p["fci"]) == (sv.nxi, sv.nzi, 1)
    assert (p["fcv"], p["flv"], p["nxv"], p["nyv"]) == (1, 1, sv.nxi, sv.nyi)
    assert p["dxi"] == pytest.approx(sv.dxi) and p["dyi"] == pytest.approx(sv.dyi)
    # float arithmetic of the reference: gx (cm) * 0.01f
    assert p["fxv"] == float(np.float32(np.float32(sv.fxv * 100) * np.float32(0.01)))
    assert p["fyv"] == float(np.float32(np.float32(sv.fyv * 100) * np.float32(0.01)))
    assert p["scaled"] == pytest.approx(0.01, rel=1e-6)


def test_command_line_overrides_par(project):
    case, paths = project
    p = check_params(paths, "fc=33", "line=60,62-64,70:5:80", "engine=physics", "form=plain",
                     "nodename=ignored_9", nodename="gpuhost_3")
    assert p["fc"] == 33.0
    assert p["lines"] == [60, 62, 63, 64, 70, 75, 80]
    assert p["engine"] == "physics" and p["panels"] == "fp32"
    assert p["gpu"] == 3 and p["node0"] == "gpuhost"


def test_missing_required_keys_exit_1(project, tmp_path):
    case, paths = project
    r = subprocess.run([DRIVER, f"path={paths['path']}"], capture_output=True, text=True)
    assert r.returncode == 1 and "parfilepath must be specified" in r.stderr
    par = tmp_path / "bad.dat"
    par.write_text("ntl=1000\n")
    bad = dict(paths, par=str(par))
    r = run_driver(bad, "check=1", check=False)
    assert r.returncode == 1 and "dt must be specified" in r.stderr
    r = run_driver(paths, "check=1", nodename="nogpu", check=False)
    assert r.returncode == 1 and "Format Error" in r.stderr


def test_data_sample_mismatch_rejected(project):
    case, paths = project
    r = run_driver(paths, "check=1", "ntl=999", check=False)
    assert r.returncode == 1 and "tr.ns=1000" in r.stderr


# ---- input faults, found by the dry run of the inputs (check=2) -----------
def _small_tables(case):
    from q_psdm_b200 import tables
    sv = case["sv"]
    return tables.linear_gradient_tables(sv, fci=sv.fci, nxi=sv.nxi, dxi=sv.dxi,
                                         zmax=(sv.nzi - 1) * sv.dzi, sub=8, nxi1=16,
                                         half_x=400.0, half_y=200.0)


@pytest.fixture(scope="module")
def tabled(tmp_path_factory):
    case = compat_case.make_case("small")
    tmp = str(tmp_path_factory.mktemp("drv2"))
    paths, _ = make_project(tmp, case, image_line=65, tab=_small_tables(case),
                            tables_at=[60, 70])
    return case, paths


def _dry(paths, *args, check=True):
    r = run_driver(paths, "check=2", *args, check=check)
    return r, (json.loads(r.stdout.strip().splitlines()[-1]) if r.returncode == 0 else None)


def test_dry_run_lists_tables_and_data(tabled):
    case, paths = tabled
    _, p = _dry(paths)
    tab = _small_tables(case)
    # line 65 lies between the table files of lines 60 and 70
    assert p["tables"] == [dict(line=65, ttt=tab.ttt.size, qqq=tab.qqq.size, nxg=tab.nxg,
                                nzg=tab.nzg)]
    assert p["data"] and all(d["partial_bytes"] == 0 for d in p["data"])
    assert sum(d["traces"] for d in p["data"]) > 0


def _copy_project(paths, tmp_path):
    import shutil
    dst = dict(paths)
    for k in ("proj", "tt"):
        dst[k] = str(tmp_path / k)
        shutil.copytree(paths[k], dst[k])
    dst["path"] = paths["path"].replace(paths["proj"], dst["proj"])
    return dst


@pytest.mark.parametrize("fault", ["negative_nxg", "grid_beyond_file", "short_header",
                                   "zero_nzi1"])
def test_bad_table_index_rejected(tabled, tmp_path, fault):
    """A table index whose header does not describe the file is an index size
    error (exit 1), raised before anything is allocated for the grid."""
    case, paths = tabled
    p2 = _copy_project(paths, tmp_path)
    idx = os.path.join(p2["tt"], "Lxxx.tidx")
    b = bytearray(open(idx, "rb").read())
    if fault == "negative_nxg":
        b[20:24] = np.int32(-5).tobytes()
    elif fault == "grid_beyond_file":
        b[16:20] = np.int32(1 << 20).tobytes()     # nzg: 2^20 cells per column
    elif fault == "zero_nzi1":
        b[24:28] = np.int32(0).tobytes()
    else:
        b = b[:20]
    open(idx, "wb").write(bytes(b))
    r, _ = _dry(p2, check=False)
    assert r.returncode == 1 and "index size error" in r.stderr


def test_missing_table_line_rejected(tabled):
    """No table file brackets the image line: exit 1 naming the table."""
    case, paths = tabled
    r, _ = _dry(paths, "line=75", check=False)
    assert r.returncode == 1 and "brackets line 75" in r.stderr


def test_truncated_data_file_reported(tabled, tmp_path):
    """A data file cut inside its last trace: the whole traces are read and
    the partial one ignored, as the reference's producer does
    (src/q-psdm.cu:1909); the dry run reports the partial bytes."""
    case, paths = tabled
    p2 = _copy_project(paths, tmp_path)
    _, before = _dry(p2)
    f = before["data"][0]["file"].replace(paths["proj"], p2["proj"])
    n = os.path.getsize(f)
    with open(f, "r+b") as fh:
        fh.truncate(n - 1000)
    _, after = _dry(p2)
    d = [x for x in after["data"] if x["file"] == f][0]
    assert d["traces"] == before["data"][0]["traces"] - 1
    assert d["partial_bytes"] == 240 + 4 * 1000 - 1000
