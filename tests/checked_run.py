"""Runs one small problem through every step-kernel family and saves the
results (used by tests/test_gpu_checked.py, once with the default library and
once with the checked one, TSP_CHECKED=1, each in a process of its own since
a process loads one of the two).

    python tests/checked_run.py <out.npz>
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from tspeed_b200 import capi  # noqa: E402
from tspeed_b200 import workloads as W  # noqa: E402

# (tag, precision, operator, kernel variant or None, shots): the plain FP64
# row kernel, the FP64 tensor-core (DMMA) batched kernel, the FP32 ring
# kernel, the k-split FP32 kernel, the tensor-core fixed-point kernel, the
# CUDA-core FP64 batched kernel and the matrix-free kernel.
FORMS = [("rows", "fp64", "explicit", None, 1), ("dmma", "fp64", "explicit", 5, 70),
         ("ring", "fp32", "explicit", 8, 70), ("ksplit", "fp32", "explicit", 0, 70),
         ("fx", "fp32", "explicit", 4, 70), ("cuda64", "fp64", "explicit", 2, 70),
         ("matfree", "fp64", "matrix_free", None, 1)]


def main(out):
    m = W.jittered_rect(9, 5, 900.0, 500.0, seed=77)
    rng = np.random.default_rng(3)
    vp = 2500 + 1500 * rng.random(m.ne)
    lam, mu, rho = W.lame(vp, vp / 1.8, 2000 + 500 * rng.random(m.ne))
    shots = [(40 + 820 * rng.random(), 40 + 420 * rng.random()) for _ in range(70)]
    rcv = W.surface_receivers(m, 5)
    n = 60
    res = {"checked": np.array(capi.lib().tsp_checked_build())}
    with capi.Simulation.create(m.xy, m.tri, 5, lam, mu, rho, shots[:1], rcv, penalty=10.0) as s:
        # 0.4 of the CFL limit, rounded to 3 digits: the power iteration sums
        # with atomics, so its last bits vary from run to run, and both runs
        # must step with the same dt.
        dt = float(f"{0.4 * 2 / np.sqrt(s.estimate_lmax(60)):.3g}")
    for tag, prec, op, variant, ns in FORMS:
        if variant is None:
            os.environ.pop("TSP_BATCHED_VARIANT", None)
        else:
            os.environ["TSP_BATCHED_VARIANT"] = str(variant)
        with capi.Simulation.create(m.xy, m.tri, 5, lam, mu, rho, shots[:ns], rcv, penalty=10.0, precision=prec,
                                    op=op) as s:
            s.set_dt(dt)
            for k in range(ns):
                s.set_ricker(k, 25.0, 0.04, -1.0, k % 2, n)
            s.first_step()
            s.run(n - 1)
            res[tag + "_seis"] = s.seismograms(0, n)
            res[tag + "_u"] = s.u_all()
    np.savez(out, **res)


if __name__ == "__main__":
    main(sys.argv[1])
