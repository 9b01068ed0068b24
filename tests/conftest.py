import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


# Benchmark-size goldens (several shots, subsampled receiver traces): a
# schema of their own, used by tests/test_gpu_scale_parity.py.
SCALE_GOLDENS = ("g_config1_full", "g_config3_sample")


def golden_cases():
    return sorted(n for n in (os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))
                  if n not in SCALE_GOLDENS)


def load_golden(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(params=golden_cases())
def golden(request):
    g = load_golden(request.param)
    g["name"] = request.param
    return g
