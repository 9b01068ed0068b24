"""Generates the golden fixtures in this folder from the reference itself.

Runs the reference's own leap-frog path, compiled unmodified by
oracle/Makefile against the project's Eigen-subset shim
(oracle/_ref/tsp_ref_run), on small seeded meshes, and stores inputs and
outputs as .npz. Rebuild with:

    make -C oracle && python tests/golden/make_golden.py [case ...]

(the reference sources are read from $TSPEED_REF, default /root/reference).

Cases named g_ba_* use the reference's BoundaryAdapted space
(FESpace<N, Dunavant<2N>, BoundaryAdapted<N>>, Examples/src/Lamb.cpp:26).
Each case also holds the reference's FESpace services: transform of a fixed
field (proj), L2error of that projection (l2_proj) and of the final
displacement (l2_u), and the text written by field_out / points_out for the
final step (field_txt / points_txt, bytes).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from tspeed_b200 import workloads as W  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "tsp_ref_run")

# name: (nx, ny, Lx, Ly, N, materials, penalty, dt, nsteps, src, ricker(f0,t0,amp,dir), nrcv, dump_blocks)
CASES = {
    "g_n2_layers": dict(nx=6, ny=4, Lx=600.0, Ly=400.0, N=2, mat="layers", penalty=10.0, dt=4e-4, nsteps=60,
                        src=(310.0, 190.0), ricker=(15.0, 1 / 15.0, -1.0, 1), nrcv=4, blocks=True),
    "g_n4_lognormal": dict(nx=8, ny=5, Lx=800.0, Ly=500.0, N=4, mat="lognormal", penalty=10.0, dt=1.5e-4,
                           nsteps=40, src=(400.0, 260.0), ricker=(12.0, 1 / 12.0, -1.0, 1), nrcv=5, blocks=False),
    "g_config1_small": dict(nx=10, ny=5, Lx=4000.0, Ly=2000.0, N=4, mat="config1", penalty=10.0, dt=2e-3,
                            nsteps=150, src=(2000.0, 1500.0), ricker=(8.0, 1 / 8.0, -1.0, 1), nrcv=8, blocks=False),
    "g_n1_xforce": dict(nx=4, ny=3, Lx=400.0, Ly=300.0, N=1, mat="homog", penalty=2.0, dt=1e-3, nsteps=50,
                        src=(150.0, 140.0), ricker=(10.0, 0.1, 1.0, 0), nrcv=3, blocks=True),
    "g_n8": dict(nx=3, ny=2, Lx=300.0, Ly=200.0, N=8, mat="lognormal", penalty=10.0, dt=2e-5, nsteps=20,
                 src=(140.0, 90.0), ricker=(20.0, 0.05, -1.0, 1), nrcv=2, blocks=False),
    "g_ba_n3": dict(nx=5, ny=4, Lx=500.0, Ly=400.0, N=3, mat="lognormal", penalty=10.0, dt=2e-4, nsteps=60,
                    src=(260.0, 210.0), ricker=(50.0, 0.01, -1.0, 1), nrcv=4, blocks=True, basis="ba"),
    "g_ba_n5": dict(nx=4, ny=3, Lx=400.0, Ly=300.0, N=5, mat="layers", penalty=10.0, dt=5e-5, nsteps=40,
                    src=(190.0, 160.0), ricker=(150.0, 0.0015, -1.0, 0), nrcv=3, blocks=True, basis="ba"),
}


def materials(kind, m, rng):
    ne = m.ne
    if kind == "layers":
        top = W.centroids(m)[:, 1] > 0.6 * m.Ly
        m.region = np.where(top, 1, 2).astype(np.int32)
        return W.lame(np.where(top, 1800.0, 4000.0), np.where(top, 1000.0, 2300.0), np.where(top, 1900.0, 2500.0))
    if kind == "lognormal":
        vp = 3000 * np.exp(rng.normal(0, 0.1, ne))
        return W.lame(vp, vp / np.sqrt(3), 2000 + 300 * rng.random(ne))
    if kind == "config1":
        return W.lame(np.full(ne, 3200.0), np.full(ne, 1847.0), np.full(ne, 2200.0))
    return W.lame(np.full(ne, 3000.0), np.full(ne, 1700.0), np.full(ne, 2100.0))


def run_case(name, c, tmp):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    m = W.jittered_rect(c["nx"], c["ny"], c["Lx"], c["Ly"], seed=11)
    lam, mu, rho = materials(c["mat"], m, rng)
    rcv = W.surface_receivers(m, c["nrcv"])
    msh, rcvf, matf, out = (os.path.join(tmp, name + s) for s in (".msh", ".rcv", ".mat", ""))
    W.write_gmsh(msh, m)
    W.write_rcv(rcvf, rcv)
    np.stack([lam, mu, rho], 1).astype(np.float64).tofile(matf)
    f0, t0, amp, sdir = c["ricker"]
    cmd = [REF, "--mesh", msh, "--N", str(c["N"]), "--mat", matf, "--rcv", rcvf, "--out", out, "--dt", repr(c["dt"]),
           "--nsteps", str(c["nsteps"]), "--src", repr(c["src"][0]), repr(c["src"][1]), "--ricker", repr(f0),
           repr(t0), repr(amp), "--sdir", str(sdir), "--penalty", repr(c["penalty"])]
    if c["blocks"]:
        cmd.append("--dump-blocks")
    if c.get("basis", "dubiner") != "dubiner":
        cmd += ["--basis", c["basis"]]
    info = json.loads(subprocess.run(cmd, check=True, capture_output=True, text=True).stdout)
    ne = m.ne
    raw = open(out + ".mesh.bin", "rb").read()
    off = 0
    hdr = np.frombuffer(raw, np.int32, 2, off); off += 8
    Np = int(hdr[1])
    nb = np.frombuffer(raw, np.int32, ne * 6, off).reshape(ne, 6); off += ne * 24
    geo = np.frombuffer(raw, np.float64, ne * 5, off).reshape(ne, 5); off += ne * 40
    minv = np.frombuffer(raw, np.float64, ne, off); off += ne * 8
    src_elem = int(np.frombuffer(raw, np.int32, 1, off)[0]); off += 4
    src_phi = np.frombuffer(raw, np.float64, Np, off); off += Np * 8
    nr = int(np.frombuffer(raw, np.int32, 1, off)[0]); off += 4
    rcv_elem, rcv_phi = [], []
    for _ in range(nr):
        rcv_elem.append(int(np.frombuffer(raw, np.int32, 1, off)[0])); off += 4
        rcv_phi.append(np.frombuffer(raw, np.float64, Np, off)); off += Np * 8
    minv_ref = np.frombuffer(raw, np.float64, Np * Np, off).reshape(Np, Np); off += Np * Np * 8
    u = open(out + ".u.bin", "rb").read()
    rec = 8 + 16 * ne * Np
    snaps = {int(np.frombuffer(u, np.int64, 1, i)[0]): np.frombuffer(u, np.float64, 2 * ne * Np, i + 8)
             for i in range(0, len(u), rec)}
    seis = np.fromfile(out + ".seis.bin", dtype=np.float64).reshape(c["nsteps"], nr, 2)
    proj = np.fromfile(out + ".proj.bin", dtype=np.float64)
    field_txt = np.frombuffer(open(out + ".u_%d.field" % c["nsteps"], "rb").read(), np.uint8)
    points_txt = np.frombuffer(open(out + ".points", "rb").read(), np.uint8)
    d = dict(xy=m.xy, tri=m.tri, region=m.region, lam=lam, mu=mu, rho=rho, N=c["N"], penalty=c["penalty"],
             dt=c["dt"], nsteps=c["nsteps"], src=np.array(c["src"]), ricker=np.array(c["ricker"]),
             rcv=np.array(rcv), neigh=nb[:, :3], nedge=nb[:, 3:], detJ=geo[:, 0], minv=minv, src_elem=src_elem,
             src_phi=src_phi, rcv_elem=np.array(rcv_elem), rcv_phi=np.array(rcv_phi), seis=seis,
             u_first=snaps[1], u_final=snaps[c["nsteps"]], last_time=info["last_time"],
             proj=proj, l2_proj=info["l2_proj"], l2_u=info["l2_u"], field_txt=field_txt, points_txt=points_txt)
    if c.get("basis", "dubiner") != "dubiner":
        d["basis"] = c["basis"]
        d["minv_ref"] = minv_ref
    if c["blocks"]:
        b = open(out + ".blocks.bin", "rb").read()
        h = np.frombuffer(b, np.int32, 3, 0)
        nnzb = int(h[2])
        o = 12
        d["row_ptr"] = np.frombuffer(b, np.int32, ne + 1, o); o += 4 * (ne + 1)
        d["col"] = np.frombuffer(b, np.int32, nnzb, o); o += 4 * nnzb
        d["blocks"] = np.frombuffer(b, np.float64, nnzb * 4 * Np * Np, o).reshape(nnzb, 2 * Np, 2 * Np)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
    print(name, "ne", ne, "Np", Np, "steps", c["nsteps"], "last_time", info["last_time"])


# Benchmark-size cases: the reference's stepping loop (TimeAdvance.cpp:41-59,
# driven as Examples/src/Wedge.cpp:72-81 does) over a benchmark configuration's
# full step count, one reference process per shot.
#   g_config1_full: configuration 1 in full (40x20 squares -> 1,600 triangles,
#     N=4, homogeneous, Ricker 8 Hz at (2000, 1500), 8 surface receivers,
#     2,000 steps); every receiver sample and the final displacement.
#   g_config3_sample: the 64-shot configuration's shape on its x0.2 sample
#     (40x20 squares, N=5, log-normal vp, 128 surface receivers, 3,000 steps),
#     8 seeded shots; receiver samples every SEIS_EVERY-th step (the 10 Hz
#     Ricker's band lies far below the sampling rate), the final displacement
#     of shots U_SHOTS.
# dt = 0.4 x the CFL limit 2/sqrt(lmax(M^-1 B)), lmax by power iteration on the
# oracle's operator, rounded to 3 significant digits.
SCALE_CASES = {
    "g_config1_full": dict(config=1, scale=1.0, nshots=1, seis_every=1, u_shots=(0,)),
    "g_config3_sample": dict(config=3, scale=0.2, nshots=8, shot_seed=2024, seis_every=30, u_shots=(0, 5)),
}


def oracle_lmax(prob, iters=200):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import tsp_oracle as O
    tri = prob.mesh.tri.astype(np.int64)
    sp = O.make_space(prob.N)
    geo = O.geometry(prob.mesh.xy, tri)
    nb, ned = O.neighbours(tri)
    rp, cols, blocks, minv = O.assemble(sp, geo, nb, ned, prob.lam, prob.mu, prob.rho, prob.penalty)
    ne, Np = prob.mesh.ne, prob.Np
    mi = np.concatenate([np.repeat(minv, Np), np.repeat(minv, Np)])
    x = np.random.default_rng(0).standard_normal(2 * ne * Np)
    lam = 0.0
    for _ in range(iters):
        y = mi * O.apply_B(rp, cols, blocks, x, ne, Np)
        lam = float(x @ y / (x @ x))
        x = y / np.linalg.norm(y)
    return lam


def run_scale_case(name, c, tmp):
    from concurrent.futures import ThreadPoolExecutor
    kw = dict(scale=c["scale"])
    if c["config"] == 3:
        kw.update(nshots=c["nshots"], shot_seed=c["shot_seed"])
    prob = W.config(c["config"], **kw)
    m = prob.mesh
    lmax = oracle_lmax(prob)
    dt = float(f"{0.4 * 2.0 / np.sqrt(lmax):.3g}")
    msh, rcvf, matf = (os.path.join(tmp, name + s) for s in (".msh", ".rcv", ".mat"))
    W.write_gmsh(msh, m)
    W.write_rcv(rcvf, prob.receivers)
    np.stack([prob.lam, prob.mu, prob.rho], 1).astype(np.float64).tofile(matf)
    nsteps = prob.nsteps

    def one(k):
        sr = prob.sources[k]
        out = os.path.join(tmp, f"{name}.{k}")
        cmd = [REF, "--mesh", msh, "--N", str(prob.N), "--mat", matf, "--rcv", rcvf, "--out", out, "--dt", repr(dt),
               "--nsteps", str(nsteps), "--src", repr(sr.x), repr(sr.y), "--ricker", repr(sr.f0), repr(sr.t0),
               repr(sr.amp), "--sdir", str(sr.direction), "--penalty", repr(prob.penalty)]
        info = json.loads(subprocess.run(cmd, check=True, capture_output=True, text=True).stdout)
        seis = np.fromfile(out + ".seis.bin", dtype=np.float64).reshape(nsteps, len(prob.receivers), 2)
        u = open(out + ".u.bin", "rb").read()
        rec = 8 + 16 * m.ne * prob.Np
        snaps = {int(np.frombuffer(u, np.int64, 1, i)[0]): np.frombuffer(u, np.float64, 2 * m.ne * prob.Np, i + 8)
                 for i in range(0, len(u), rec)}
        return info, seis[::c["seis_every"]].copy(), snaps[nsteps].copy()

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        res = list(ex.map(one, range(prob.nshots)))
    d = dict(xy=m.xy, tri=m.tri, region=m.region, lam=prob.lam, mu=prob.mu, rho=prob.rho, N=prob.N,
             penalty=prob.penalty, dt=dt, lmax_oracle=lmax, nsteps=nsteps,
             src=np.array([(sr.x, sr.y) for sr in prob.sources]),
             ricker=np.array([(sr.f0, sr.t0, sr.amp, sr.direction) for sr in prob.sources]),
             rcv=np.array(prob.receivers), seis_every=c["seis_every"],
             seis=np.stack([r[1] for r in res]), u_shots=np.array(c["u_shots"]),
             u_final=np.stack([res[k][2] for k in c["u_shots"]]),
             last_time=res[0][0]["last_time"], ref_loop_s=np.array([r[0]["loop_s"] for r in res]))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
    print(name, "ne", m.ne, "Np", prob.Np, "shots", prob.nshots, "steps", nsteps, "dt", dt,
          "loop_s", [round(r[0]["loop_s"], 1) for r in res])


def main():
    if not os.path.exists(REF):
        sys.exit(f"{REF} missing: run `make -C oracle` first (reference sources from $TSPEED_REF)")
    only = sys.argv[1:]
    with tempfile.TemporaryDirectory() as tmp:
        for name, c in CASES.items():
            if not only or name in only:
                run_case(name, c, tmp)
        for name, c in SCALE_CASES.items():
            if not only or name in only:
                run_scale_case(name, c, tmp)


if __name__ == "__main__":
    main()
