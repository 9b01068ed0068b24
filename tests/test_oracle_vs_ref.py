"""The oracle against the reference's own sources run live (CPU).

Needs oracle/_ref/tsp_ref_run (built by `make -C oracle REF=...` or
__graft_entry__.build()); skipped where it is absent.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import tsp_oracle as O
from helpers import rel
from tspeed_b200 import workloads as W

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "tsp_ref_run")
pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="reference oracle not built")


@pytest.mark.parametrize("N,nx,ny,seed", [(3, 7, 4, 5), (6, 4, 3, 8), (7, 3, 3, 2)])
def test_random_case_against_live_reference(tmp_path, N, nx, ny, seed):
    rng = np.random.default_rng(seed)
    m = W.jittered_rect(nx, ny, 100.0 * nx, 100.0 * ny, seed=seed)
    vp = 2500 + 2000 * rng.random(m.ne)
    lam, mu, rho = W.lame(vp, vp / (1.6 + 0.4 * rng.random(m.ne)), 1800 + 900 * rng.random(m.ne))
    rc = W.surface_receivers(m, 3) + [(0.5 * m.Lx + 3.3, 0.3 * m.Ly)]
    W.write_gmsh(str(tmp_path / "m.msh"), m)
    W.write_rcv(str(tmp_path / "m.rcv"), rc)
    np.stack([lam, mu, rho], 1).tofile(str(tmp_path / "m.mat"))
    dt, nst, pen = 5e-5, 25, 7.5
    src = (0.45 * m.Lx, 0.55 * m.Ly)
    out = str(tmp_path / "o")
    cmd = [REF, "--mesh", str(tmp_path / "m.msh"), "--N", str(N), "--mat", str(tmp_path / "m.mat"), "--rcv",
           str(tmp_path / "m.rcv"), "--out", out, "--dt", repr(dt), "--nsteps", str(nst), "--src", repr(src[0]),
           repr(src[1]), "--ricker", "20.0", "0.05", "1.0", "--sdir", "1", "--penalty", repr(pen), "--dump-blocks"]
    json.loads(subprocess.run(cmd, check=True, capture_output=True, text=True).stdout)
    sp = O.make_space(N)
    tri = m.tri.astype(np.int64)
    geo = O.geometry(m.xy, tri)
    nb, ned = O.neighbours(tri)
    row_ptr, cols, blocks, minv = O.assemble(sp, geo, nb, ned, lam, mu, rho, pen)
    b = open(out + ".blocks.bin", "rb").read()
    nnzb = int(np.frombuffer(b, np.int32, 3, 0)[2])
    o = 12 + 4 * (m.ne + 1) + 4 * nnzb
    ref_blocks = np.frombuffer(b, np.float64, nnzb * 4 * sp.Np ** 2, o).reshape(nnzb, 2 * sp.Np, 2 * sp.Np)
    assert np.abs(blocks - ref_blocks).max() / np.abs(ref_blocks).max() < 1e-14
    se, sphi = O.locate(N, m.xy, tri, geo, *src)
    rl = [O.locate(N, m.xy, tri, geo, x, y) for (x, y) in rc]
    F = [(0.0, O.ricker(t, 20.0, 0.05, 1.0)) for t in O.force_times(dt, nst)]
    u, seis, _ = O.leapfrog(row_ptr, cols, blocks, minv, m.ne, sp.Np, dt, nst, se, sphi, F,
                            [r[0] for r in rl], [r[1] for r in rl])
    seis_ref = np.fromfile(out + ".seis.bin", dtype=np.float64).reshape(nst, len(rc), 2)
    assert rel(seis, seis_ref) < 1e-12
