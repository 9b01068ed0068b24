"""The C++ drop-in (include/tspeed_gpu.hpp) driven like the reference's
examples, against the reference's golden seismograms (GPU)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import load_golden
from helpers import rel
from tspeed_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def build_example(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    assert cxx, "no C++ compiler"
    exe = str(tmp_path / "dropin")
    lib = os.path.join(ROOT, "tspeed_b200")
    subprocess.run([cxx, "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_example.cpp"), "-L" + lib, "-ltspeed_b200",
                    "-Wl,-rpath," + lib, "-o", exe], check=True)
    return exe


def example_args(exe, g, tmp_path, src, ricker):
    m = W.Mesh(g["xy"], g["tri"], g["region"], 0.0, 0.0)
    W.write_gmsh(str(tmp_path / "m.msh"), m)
    W.write_rcv(str(tmp_path / "m.rcv"), g["rcv"])
    regions = []
    for reg in sorted(set(g["region"].tolist())):
        e = int(np.argmax(g["region"] == reg))
        regions += [str(reg), repr(float(g["lam"][e])), repr(float(g["mu"][e])), repr(float(g["rho"][e]))]
    f0, t0, amp, sdir = (float(v) for v in ricker)
    return [exe, str(tmp_path / "m.msh"), str(tmp_path / "m.rcv"), str(tmp_path / "out"), str(int(g["N"])),
            repr(float(g["penalty"])), repr(float(g["dt"])), str(int(g["nsteps"])), repr(float(src[0])),
            repr(float(src[1])), repr(f0), repr(t0), repr(amp), str(int(sdir)), str(len(regions) // 4)] + regions


def test_cpp_dropin_config1_full_parity_and_speed(tmp_path):
    """Configuration 1 in full (2,000 steps) through the C++ drop-in, the
    loop written like the reference's examples (a step() and an
    eval_receivers() call per step, write_receivers at the end): the
    reference's seismograms within 1e-12, and the loop's wall time within
    1.5x of one tsp_run call plus one read-back on the same problem (queued
    steps run as graph replays)."""
    exe = build_example(tmp_path)
    g = load_golden("g_config1_full")
    args = example_args(exe, g, tmp_path, g["src"][0], g["ricker"][0]) + ["timing"]
    res = subprocess.run(args, check=True, capture_output=True, text=True)
    n = int(g["nsteps"])
    assert res.stdout.startswith(f"steps {n} ")
    seis = np.stack([np.loadtxt(str(tmp_path / f"out_rcv_{i}.out")) for i in range(len(g["rcv"]))], 1)
    assert rel(seis, g["seis"][0]) < 1e-12
    line = [ln for ln in res.stdout.splitlines() if ln.startswith("timing")][0].split()
    t_loop, t_run = float(line[2]), float(line[4])
    print("drop-in loop", t_loop, "s; tsp_run", t_run, "s")
    assert t_loop <= 1.5 * t_run + 2e-3


@pytest.mark.parametrize("case", ["g_n2_layers", "g_ba_n5"])
def test_cpp_dropin_matches_reference_golden(case, tmp_path):
    exe = build_example(tmp_path)
    g = load_golden(case)
    ba = "basis" in g
    # Tolerances as in test_gpu_parity.py: the BoundaryAdapted reference mass
    # (condition number 1.1e5 at N = 5) amplifies rounding.
    tol = 1e-11 if ba else 1e-12
    args = example_args(exe, g, tmp_path, g["src"], g["ricker"])
    if ba:
        args.append("ba")
    res = subprocess.run(args, check=True, capture_output=True, text=True)
    assert res.stdout.startswith(f"steps {int(g['nsteps'])} ")
    seis = np.stack([np.loadtxt(str(tmp_path / f"out_rcv_{i}.out")) for i in range(len(g["rcv"]))], 1)
    assert seis.shape == g["seis"].shape
    ok = np.isfinite(g["seis"])
    assert rel(seis[ok], g["seis"][ok]) < tol
    # FESpace::points_out / field_out / L2error, host and device forms.
    n = int(g["nsteps"])
    assert (tmp_path / "out.points").read_bytes() == bytes(g["points_txt"])
    ref = np.array([[float(v) for v in ln.split()] for ln in bytes(g["field_txt"]).decode().splitlines()])
    scale = np.abs(ref).max()
    for form in ("host", "dev"):
        got = np.loadtxt(str(tmp_path / f"out.{form}.u_{n}.field"))
        assert got.shape == ref.shape
        assert np.all(np.abs(got - ref) <= 1e-5 * np.abs(ref) + 1e-11 * scale)
    l2 = [float(v) for v in res.stdout.splitlines()[1].split()[1:]]
    assert abs(l2[0] / float(g["l2_u"]) - 1) < tol and abs(l2[1] / float(g["l2_u"]) - 1) < tol
