"""The C++ drop-in (include/cpu_vh.h, libcpu-vh_lib.so) end to end on the GPU.

A reference maintainer's embedding code -- HYDRO::initialize_from_vector and
run_hydro_no_cli, reading rhic-conf/ and writing cpu-vh_output/surface.dat
(HydroWrapper.cpp:20-136, HydroPlugin.cpp:74-321) -- is compiled against this
repository's header and run.  Its surface.dat and its field dumps must be
byte-identical to the ones the reference's own run() writes for the same case
(golden hashes from tests/golden/dropin_case.py): same rows, same order, same
text."""
import hashlib
import json
import os
import shutil
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "cpu-vh_b200")
sys.path.insert(0, os.path.join(HERE, "golden"))
import dropin_case  # noqa: E402


def _driver(tmp):
    exe = os.path.join(tmp, "plugin_driver")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), os.path.join(HERE, "plugin_driver.cpp"),
                    "-L", PKG, "-lcpu-vh_lib", "-lvh_b200", f"-Wl,-rpath,{PKG}", "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("case", ["2p1d", "3p1d"])
def test_dropin_surface_matches_reference(case, tmp_path):
    """2+1D (callFOFinder2p1D) and 3+1D (callFOFinder3p1D, FreezeOut.cpp:200-280)
    runs to the reference's stop rule"""
    tmp = str(tmp_path)
    exe = _driver(tmp)
    c = dropin_case.CASES[case]
    shutil.copytree(c["conf"], os.path.join(tmp, "rhic-conf"))
    os.makedirs(os.path.join(tmp, "cpu-vh_output"))
    dropin_case.e_vector(case).tofile(os.path.join(tmp, "e.bin"))
    r = subprocess.run([exe, "e.bin"], cwd=tmp, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "All cells have dropped below freezeout energy density" in r.stdout
    with open(os.path.join(tmp, "cpu-vh_output", "surface.dat"), "rb") as f:
        data = f.read()
    with open(c["golden"]) as f:
        gold = json.load(f)
    assert data.count(b"\n") == gold["rows"]
    assert hashlib.sha256(data).hexdigest() == gold["sha256"]
    # the field dumps of outputDynamicalQuantities (HydroPlugin.cpp:40-71), byte for byte
    out = os.path.join(tmp, "cpu-vh_output")
    mine = {n: hashlib.sha256(open(os.path.join(out, n), "rb").read()).hexdigest()
            for n in os.listdir(out) if n != "surface.dat"}
    assert mine == gold["dumps"]


def test_cpu_vh_executable_runs_ideal_gubser(tmp_path):
    """The `cpu-vh -c DIR -o DIR -h` command line on IC type 3 (ideal Gubser)
    on an even grid (the reference's type-3 velocity is 0/0 at r = 0)."""
    tmp = str(tmp_path)
    conf = os.path.join(tmp, "conf")
    os.makedirs(conf)
    os.makedirs(os.path.join(tmp, "out"))
    with open(os.path.join(conf, "lattice.properties"), "w") as f:
        f.write("nx=40\nny=40\nnz=1\nnt=60\ndx=0.2\ndy=0.2\ndz=0.1\ndt=0.02\nfo=2\n")
    with open(os.path.join(conf, "hydro.properties"), "w") as f:
        f.write("t0=1.0\netas=0.2\nTF=0.155\npiNS=0\nTreg=0.1\nFO=1\n")
    with open(os.path.join(conf, "ic.properties"), "w") as f:
        f.write("type=3\nnsrc=0\nA=208\ne0=15.0\nsnn=62\nb=0\nalpha=1\nvar=0.16\nmean=5.9\nsrc=0\n")
    r = subprocess.run([os.path.join(PKG, "cpu-vh"), "-c", conf, "-o", os.path.join(tmp, "out"), "-h"], cwd=tmp,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Average time/step" in r.stdout
    surf = open(os.path.join(tmp, "out", "surface.dat")).read().splitlines()
    assert len(surf) > 0 and all(len(ln.split()) == 20 for ln in surf[:50])
    assert os.path.exists(os.path.join(tmp, "out", "e_1.000.dat"))
    for name in ("wxy", "beta_x", "beta_y"):      # the reference's vorticity dumps (HydroPlugin.cpp:66-70)
        assert os.path.exists(os.path.join(tmp, "out", f"{name}_1.000.dat")), name
