"""The checked build (TSP_CHECKED: every gather index the step kernels read is
range-checked on the device) against the default build, on the GPU.

tests/checked_run.py runs one problem through every step-kernel family --
plain FP64 rows, FP64 tensor-core (DMMA) and CUDA-core batched, FP32 ring,
k-split and tensor-core fixed-point batched, matrix-free -- in a process of
its own, once per library. The checks change no arithmetic, so every field
and seismogram must be bit-identical, and the checked run must report no
index failure (a failure would make its read-backs return TSP_ERR_INDEX and
the script fail).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SCRIPT = os.path.join(ROOT, "tests", "checked_run.py")


def run(tmp_path, checked):
    out = str(tmp_path / ("checked.npz" if checked else "default.npz"))
    env = dict(os.environ, TSP_CHECKED="1" if checked else "0")
    env.pop("TSP_BATCHED_VARIANT", None)
    r = subprocess.run([sys.executable, SCRIPT, out], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    d = np.load(out)
    return {k: d[k] for k in d.files}


@pytest.mark.gpu
def test_checked_build_matches_default_build(tmp_path):
    if not os.path.exists(os.path.join(ROOT, "tspeed_b200", "libtspeed_b200_checked.so")):
        pytest.fail("checked library missing: python -m tspeed_b200.build --checked")
    a = run(tmp_path, checked=False)
    b = run(tmp_path, checked=True)
    assert int(a.pop("checked")) == 0 and int(b.pop("checked")) == 1
    assert set(a) == set(b) and len(a) == 14
    differ = [k for k in sorted(a) if not np.array_equal(a[k], b[k])]
    assert not differ, differ
    for k in sorted(a):
        assert np.isfinite(a[k]).all() and np.abs(a[k]).max() > 0, k
