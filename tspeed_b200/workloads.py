"""Seeded synthetic workloads for the leap-frog path, plus Gmsh 2.2 / receiver
file writers.

The reference publishes no datasets; its examples read Gmsh 2.2 ASCII meshes
(Mesh.cpp:174-257) and "x y" receiver lists (Receivers_imp.hpp:61-82). The
benchmark meshes are jittered rectangles: an nx x ny grid of squares over
[0, Lx] x [0, Ly], each square split along its (i,j)-(i+1,j+1) diagonal into
two counter-clockwise triangles, interior vertices moved uniformly by up to
10% of the spacing per axis. Elements are numbered square by square (row by
row, two per square), so face neighbours are close in index.

Materials come from (vp, vs, rho) as mu = rho vs^2, lambda = rho vp^2 - 2 mu.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Mesh:
    xy: np.ndarray      # [nv, 2] float64
    tri: np.ndarray     # [ne, 3] int32, CCW, 0-based vertex ids
    region: np.ndarray  # [ne] int32, Gmsh elementary tag (>= 1)
    Lx: float
    Ly: float

    @property
    def ne(self) -> int:
        return int(self.tri.shape[0])


def jittered_rect(nx: int, ny: int, Lx: float, Ly: float, seed: int, jitter: float = 0.1) -> Mesh:
    rng = np.random.default_rng(seed)
    hx, hy = Lx / nx, Ly / ny
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="xy")
    x = ii.astype(np.float64) * hx
    y = jj.astype(np.float64) * hy
    jx = rng.uniform(-jitter, jitter, size=x.shape) * hx
    jy = rng.uniform(-jitter, jitter, size=y.shape) * hy
    interior = (ii > 0) & (ii < nx) & (jj > 0) & (jj < ny)
    x = np.where(interior, x + jx, x)
    y = np.where(interior, y + jy, y)
    xy = np.stack([x.ravel(), y.ravel()], 1)
    vid = lambda i, j: j * (nx + 1) + i  # noqa: E731
    tri = np.empty((2 * nx * ny, 3), dtype=np.int32)
    sj, si = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    sj, si = sj.ravel(), si.ravel()
    v00, v10 = vid(si, sj), vid(si + 1, sj)
    v11, v01 = vid(si + 1, sj + 1), vid(si, sj + 1)
    tri[0::2] = np.stack([v00, v10, v11], 1)
    tri[1::2] = np.stack([v00, v11, v01], 1)
    region = np.ones(tri.shape[0], dtype=np.int32)
    return Mesh(xy, tri, region, Lx, Ly)


def centroids(m: Mesh) -> np.ndarray:
    return m.xy[m.tri].mean(axis=1)


def lame(vp, vs, rho):
    vp, vs, rho = (np.asarray(a, dtype=np.float64) for a in (vp, vs, rho))
    mu = rho * vs * vs
    lam = rho * vp * vp - 2.0 * mu
    return lam, mu, rho


def write_gmsh(path: str, m: Mesh) -> None:
    """Gmsh 2.2 ASCII as read by Mesh::Mesh (Mesh.cpp:174-257): type-2
    triangles with two tags (physical, elementary); the elementary tag is the
    region. Coordinates are written with 17 significant digits, so the file
    reproduces the in-memory doubles exactly."""
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n")
        f.write(f"{m.xy.shape[0]}\n")
        f.write("".join(f"{i + 1} {x:.17g} {y:.17g} 0\n" for i, (x, y) in enumerate(m.xy)))
        f.write("$EndNodes\n$Elements\n")
        f.write(f"{m.ne}\n")
        f.write("".join(f"{k + 1} 2 2 {r} {r} {a + 1} {b + 1} {c + 1}\n"
                        for k, ((a, b, c), r) in enumerate(zip(m.tri.tolist(), m.region.tolist()))))
        f.write("$EndElements\n")


def write_rcv(path: str, pts) -> None:
    with open(path, "w") as f:
        for (x, y) in pts:
            f.write(f"{x:.17g} {y:.17g}\n")


def surface_receivers(m: Mesh, nr: int):
    """nr receivers evenly spaced on the top surface y = Ly, at the centres of
    nr equal intervals (so, for the benchmark grids, never on a mesh vertex)."""
    return [(m.Lx * (r + 0.5) / nr, m.Ly) for r in range(nr)]


@dataclass
class Source:
    x: float
    y: float
    f0: float
    t0: float
    amp: float = -1.0   # vertical force pointing down, as Examples/src/Lamb.cpp:37
    direction: int = 1  # 0: x, 1: y


@dataclass
class Problem:
    name: str
    mesh: Mesh
    N: int
    lam: np.ndarray
    mu: np.ndarray
    rho: np.ndarray
    sources: list           # one Source per shot
    receivers: list         # [(x, y)], shared by all shots
    nsteps: int
    penalty: float = 10.0
    cfl_fraction: float = 0.4
    seed: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def Np(self) -> int:
        return (self.N + 1) * (self.N + 2) // 2

    @property
    def nshots(self) -> int:
        return len(self.sources)

    @property
    def dofs_per_shot(self) -> int:
        return 2 * self.mesh.ne * self.Np


def _interior_points(m: Mesh, n: int, rng, margin: float = 0.05):
    xs = rng.uniform(margin * m.Lx, (1 - margin) * m.Lx, size=n)
    ys = rng.uniform(margin * m.Ly, (1 - margin) * m.Ly, size=n)
    return list(zip(xs.tolist(), ys.tolist()))


def config(k: int, scale: float = 1.0, seed: int = 1234, nshots: int | None = None,
           nsteps: int | None = None, shot_seed: int | None = None) -> Problem:
    """The five benchmark configurations, optionally shrunk by `scale` (grid
    squares per axis scale by it; materials, degree and source types are kept).

    1: 40x20 squares over 4000x2000 m, N=4, homogeneous (rho 2200, vp 3200,
       vs 1847), Ricker f0=8 Hz at (2000, 1500), 2000 steps, 8 receivers.
    2: 400x200 squares, N=6, two layers (top 30%: vp 1800 vs 1000 rho 1900;
       below: vp 4000 vs 2300 rho 2500), f0=15 Hz, 5000 steps, 64 receivers.
    3: 200x100 squares, N=5, per-element log-normal vp (mean 3000,
       sigma_log 0.1, vs = vp/sqrt(3), rho 2300), 64 shots at seeded interior
       points, 3000 steps, 128 receivers.
    5: 640x512 squares, N=6, 8 random layers (vp in [1500, 6000]), f0=20 Hz,
       10000 steps, 256 receivers.
    """
    rng = np.random.default_rng(seed + 97 * k)
    sc = lambda n: max(2, int(round(n * scale)))  # noqa: E731
    if k == 1:
        m = jittered_rect(sc(40), sc(20), 4000.0, 2000.0, seed)
        lam, mu, rho = lame(np.full(m.ne, 3200.0), np.full(m.ne, 1847.0), np.full(m.ne, 2200.0))
        src = [Source(2000.0, 1500.0, 8.0, 1.0 / 8.0)]
        return Problem("config1", m, 4, lam, mu, rho, src, surface_receivers(m, 8), nsteps or 2000, seed=seed)
    if k == 2:
        m = jittered_rect(sc(400), sc(200), 4000.0, 2000.0, seed)
        cy = centroids(m)[:, 1]
        top = cy > 0.7 * m.Ly
        m.region = np.where(top, 1, 2).astype(np.int32)
        vp = np.where(top, 1800.0, 4000.0)
        vs = np.where(top, 1000.0, 2300.0)
        rh = np.where(top, 1900.0, 2500.0)
        lam, mu, rho = lame(vp, vs, rh)
        src = [Source(2000.0, 1000.0, 15.0, 1.0 / 15.0)]
        return Problem("config2", m, 6, lam, mu, rho, src, surface_receivers(m, 64), nsteps or 5000, seed=seed)
    if k == 3:
        m = jittered_rect(sc(200), sc(100), 4000.0, 2000.0, seed)
        vp = 3000.0 * np.exp(rng.normal(0.0, 0.1, size=m.ne) - 0.5 * 0.1 ** 2)
        lam, mu, rho = lame(vp, vp / math.sqrt(3.0), np.full(m.ne, 2300.0))
        ns = 64 if nshots is None else nshots
        pts = _interior_points(m, ns, rng if shot_seed is None else np.random.default_rng(shot_seed))
        f0 = 10.0
        src = [Source(x, y, f0, 1.0 / f0) for (x, y) in pts]
        return Problem("config3", m, 5, lam, mu, rho, src, surface_receivers(m, 128), nsteps or 3000, seed=seed)
    if k == 5:
        m = jittered_rect(sc(640), sc(512), 6400.0, 5120.0, seed)
        edges = np.sort(rng.uniform(0.0, m.Ly, size=7))
        cy = centroids(m)[:, 1]
        layer = np.searchsorted(edges, cy)
        vps = rng.uniform(1500.0, 6000.0, size=8)
        vp = vps[layer]
        m.region = (layer + 1).astype(np.int32)
        lam, mu, rho = lame(vp, vp / math.sqrt(3.0), np.full(m.ne, 2300.0))
        src = [Source(m.Lx / 2, 0.6 * m.Ly, 20.0, 1.0 / 20.0)]
        return Problem("config5", m, 6, lam, mu, rho, src, surface_receivers(m, 256), nsteps or 10000, seed=seed)
    raise ValueError("config must be 1, 2, 3 or 5 (config 4 is a batch of meshes: see mesh_batch)")


def mesh_batch(nmesh: int = 256, seed: int = 4321, tri_range=(500, 20000), N_range=(3, 8),
               nsteps: int = 2000, scale: float = 1.0):
    """Config 4: independent jittered rectangles with triangle counts uniform
    in tri_range (times scale), degree uniform in N_range, one homogeneous
    material each (vp in [2000, 5000], vp/vs in [1.6, 2.0], rho in
    [1800, 2700]) and one Ricker source with f0 in [5, 20] Hz."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(nmesh):
        nt = int(rng.integers(tri_range[0], tri_range[1] + 1) * scale)
        nsq = max(2, nt // 2)
        ny = max(1, int(round(math.sqrt(nsq / 2))))
        nx = max(1, nsq // ny)
        m = jittered_rect(nx, ny, 2000.0 * nx / ny, 2000.0, seed + 7 * k + 1)
        N = int(rng.integers(N_range[0], N_range[1] + 1))
        vp = float(rng.uniform(2000.0, 5000.0))
        vs = vp / float(rng.uniform(1.6, 2.0))
        rh = float(rng.uniform(1800.0, 2700.0))
        lam, mu, rho = lame(np.full(m.ne, vp), np.full(m.ne, vs), np.full(m.ne, rh))
        f0 = float(rng.uniform(5.0, 20.0))
        (sx, sy), = _interior_points(m, 1, rng)
        out.append(Problem(f"mesh{k}", m, N, lam, mu, rho, [Source(sx, sy, f0, 1.0 / f0)],
                           surface_receivers(m, 8), nsteps, seed=seed))
    return out
