"""The allocation-free CFL estimate (GPU).

tsp_estimate_lmax_noalloc serves callers that may not allocate device memory
when they need the estimate: its iteration vectors live in a fixed device
array inside the library instead of cudaMalloc'd buffers. This file is named
to be collected last, so that a run stopping at the first failure has run
every other test already.
"""
import ctypes as C

import numpy as np
import pytest

from tspeed_b200 import capi
from tspeed_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(sim, iters):
    out = C.c_double()
    rc = capi.lib().tsp_estimate_lmax_noalloc(sim._h, iters, C.byref(out))
    if rc != 0:
        raise capi.TspError(rc, capi.lib().tsp_last_error(sim._h).decode())
    return out.value


def _mesh():
    m = W.jittered_rect(4, 3, 400.0, 300.0, seed=5)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    return m, lam, mu, rho


# One shot (explicit FP64 / FP32 blocks, the matrix-free operator) and several
# shots (FP64 blocks at the batched pitch; FP32 blocks with the batched
# kernels' state shadow): the estimate works on the operator alone, whatever
# the handle's step kernels.
CASES = [
    (2, "fp64", "explicit", 1),
    (4, "fp32", "explicit", 1),
    (3, "fp64", "matrix_free", 1),
    (4, "fp64", "explicit", 3),
    (5, "fp32", "explicit", 3),
]


@pytest.mark.parametrize("N,precision,op,nshots", CASES)
def test_noalloc_lmax_matches_allocating_entry_point(N, precision, op, nshots):
    m, lam, mu, rho = _mesh()
    shots = [(150.0, 140.0), (250.0, 100.0), (90.0, 200.0)][:nshots]
    with capi.Simulation.create(m.xy, m.tri, N, lam, mu, rho, shots, [], penalty=10.0,
                                precision=precision, op=op) as s:
        ref = s.estimate_lmax(2000)
        first = _noalloc(s, 2000)
        second = _noalloc(s, 2000)
    # Same power iteration from another start vector: both converge to lmax.
    assert abs(first - ref) / ref < 1e-6
    assert abs(second - ref) / ref < 1e-6
    # The shared scratch is re-initialised by every call: the second call
    # repeats the first, up to the order in which the device's atomic sums
    # of the Rayleigh quotient land (last bits).
    assert abs(second - first) <= 1e-12 * abs(first)


def test_noalloc_rejects_problems_beyond_the_scratch():
    m = W.jittered_rect(300, 150, 3000.0, 1500.0, seed=2)  # 90,000 triangles, N=5: 3.78 M doubles per vector
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    with capi.Simulation.create(m.xy, m.tri, 5, lam, mu, rho, [(1500.0, 700.0)], [], penalty=10.0,
                                precision="fp32") as s:
        with pytest.raises(capi.TspError) as e:
            _noalloc(s, 3)
        assert e.value.code == -1 and "scratch" in str(e.value)
