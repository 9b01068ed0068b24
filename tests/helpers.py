"""Shared helpers for the tests: oracle-side problem setup from a golden case."""
import numpy as np

import tsp_oracle as O


def oracle_setup(g):
    """Oracle operator, points and force table for a golden case."""
    N = int(g["N"])
    xy, tri = g["xy"], g["tri"].astype(np.int64)
    basis = str(g["basis"]) if "basis" in g else "dubiner"
    sp = O.make_space(N, basis)
    geo = O.geometry(xy, tri)
    neigh, nedg = O.neighbours(tri)
    row_ptr, cols, blocks, minv = O.assemble(sp, geo, neigh, nedg, g["lam"], g["mu"], g["rho"], float(g["penalty"]))
    se, sphi = O.locate(N, xy, tri, geo, *g["src"], basis=basis)
    rl = [O.locate(N, xy, tri, geo, x, y, basis=basis) for (x, y) in g["rcv"]]
    f0, t0, amp, sdir = g["ricker"]
    nst = int(g["nsteps"])
    F = []
    for t in O.force_times(float(g["dt"]), nst):
        v = O.ricker(t, f0, t0, amp)
        F.append((v, 0.0) if int(sdir) == 0 else (0.0, v))
    return dict(basis=basis, minv_ref=None if basis == "dubiner" else sp.minv_ref, sp=sp, geo=geo, neigh=neigh, nedg=nedg, row_ptr=row_ptr, cols=cols, blocks=blocks, minv=minv,
                src_elem=se, src_phi=sphi, rcv_elem=[r[0] for r in rl], rcv_phi=[r[1] for r in rl], F=np.array(F))


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
