"""Multi-mesh batch (uneven sizes and degrees, one graph for all) against
the same meshes run one by one (GPU)."""
import numpy as np
import pytest

from helpers import rel
from tspeed_b200 import capi
from tspeed_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small_batch():
    return W.mesh_batch(nmesh=6, seed=77, tri_range=(40, 160), N_range=(2, 5), nsteps=40)


@pytest.mark.parametrize("op,precision", [("explicit", "fp64"), ("matrix_free", "fp64"), ("explicit", "fp32")])
def test_batch_matches_single_meshes(op, precision):
    probs = small_batch()
    n = 40
    with capi.Batch(probs, precision=precision, op=op) as b:
        lmax = b.estimate_lmax(400)
        dt = 0.4 * 2 / np.sqrt(lmax)
        b.set_dt(dt)
        b.set_ricker(n)
        b.set_seismogram_capacity(n)
        b.first_step()
        b.run(17)
        b.run(n - 18)
        us = [b.u(m) for m in range(len(probs))]
        ss = [b.seismograms(m, 0, n) for m in range(len(probs))]
        assert b.ngroups == len(set(p.N for p in probs))
    tol = 1e-12 if precision == "fp64" else 1e-5
    for m, p in enumerate(probs):
        with capi.Simulation.from_problem(p, precision=precision, op=op) as s:
            l1 = s.estimate_lmax(400)
            assert abs(l1 - lmax[m]) / l1 < 1e-3  # different start vectors
            s.set_dt(dt[m])
            src = p.sources[0]
            s.set_ricker(0, src.f0, src.t0, src.amp, src.direction, n)
            s.first_step()
            s.run(n - 1)
            assert rel(us[m], s.u()) < tol
            assert rel(ss[m], s.seismograms(0, n)[0]) < tol
