"""The C++ host layer under AddressSanitizer and UndefinedBehaviorSanitizer (CPU).

tests/cpp/host_sanitize.cpp drives every host routine behind the C-ABI
(reference tables, geometry, neighbour search, block pattern, point location,
the Gmsh reader on good and malformed files, quadrature, projection, force
times); it is compiled here with tspeed_b200/csrc/tsp_host.cpp under
-fsanitize=address,undefined with recovery off, so any sanitizer report or
broken invariant ends the program with a non-zero status.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "tspeed_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_host_layer_under_asan_ubsan(tmp_path):
    exe = str(tmp_path / "host_sanitize")
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=all", "-I" + CSRC, os.path.join(ROOT, "tests", "cpp", "host_sanitize.cpp"),
           os.path.join(CSRC, "tsp_host.cpp"), "-o", exe]
    subprocess.run(cmd, check=True, timeout=300)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "host layer checks passed" in r.stdout
    assert "runtime error" not in r.stderr and "AddressSanitizer" not in r.stderr, r.stderr
