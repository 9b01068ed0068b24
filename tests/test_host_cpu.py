"""Host-side checks of the C-ABI library that need no GPU (CPU)."""
import os
import re

import numpy as np
import pytest

import tsp_oracle as O
from helpers import golden_field
from tspeed_b200 import capi
from tspeed_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            txt = open(os.path.join(inc, fn)).read()
            syms |= set(re.findall(r"^\w[\w\s\*]*?\b(tsp_\w+)\s*\(", txt, flags=re.M))
    return syms


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    syms = header_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing
    assert set(capi.SIGNATURES) == syms


def test_checked_build_exports_the_same_symbols():
    """The TSP_CHECKED library (device-side index checks) exports every
    declared entry point and reports itself as checked; the default library
    does not."""
    import ctypes
    path = os.path.join(ROOT, "tspeed_b200", "libtspeed_b200_checked.so")
    if not os.path.exists(path):
        pytest.skip("checked library not built (python -m tspeed_b200.build --checked)")
    L = ctypes.CDLL(path)
    missing = [s for s in header_symbols() if not hasattr(L, s)]
    assert not missing, missing
    assert L.tsp_checked_build() == 1
    assert capi.lib().tsp_checked_build() == (1 if os.environ.get("TSP_CHECKED") == "1" else 0)


def test_version_string():
    assert b"sm_100a" in capi.lib().tsp_version()


def test_gmsh_roundtrip(tmp_path):
    m = W.jittered_rect(5, 3, 500.0, 300.0, seed=4)
    m.region = (1 + (np.arange(m.ne) % 3)).astype(np.int32)
    p = str(tmp_path / "m.msh")
    W.write_gmsh(p, m)
    xy, tri, reg = capi.gmsh_read(p)
    assert np.array_equal(xy, m.xy) and np.array_equal(tri, m.tri) and np.array_equal(reg, m.region)


def test_gmsh_errors(tmp_path):
    with pytest.raises(capi.TspError) as e:
        capi.gmsh_read(str(tmp_path / "missing.msh"))
    assert e.value.code == -6
    bad = tmp_path / "bad.msh"
    bad.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n")
    with pytest.raises(capi.TspError):
        capi.gmsh_read(str(bad))


def test_neighbours_match_oracle_and_golden(golden):
    nb, ned = capi.mesh_neighbours(golden["tri"])
    assert np.array_equal(nb, golden["neigh"]) and np.array_equal(ned, golden["nedge"])


def test_neighbours_large_mesh_matches_oracle():
    m = W.jittered_rect(60, 40, 6000.0, 4000.0, seed=9)
    nb, ned = capi.mesh_neighbours(m.tri)
    onb, oned = O.neighbours(m.tri.astype(np.int64))
    assert np.array_equal(nb, onb) and np.array_equal(ned, oned)


def test_neighbours_reject_clockwise_duplicate():
    tri = np.array([[0, 1, 2], [0, 1, 3]], dtype=np.int32)  # both own directed edge 0->1
    with pytest.raises(capi.TspError) as e:
        capi.mesh_neighbours(tri)
    assert e.value.code == -6


def test_force_times_match_oracle():
    for dt in (1e-3, 3.7e-4, 0.1):
        assert np.array_equal(capi.force_times(dt, 500), np.array(O.force_times(dt, 500)))


def test_create_validates_before_touching_a_device():
    m = W.jittered_rect(2, 2, 200.0, 200.0, seed=1)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1700.0), np.full(m.ne, 2000.0))
    with pytest.raises(capi.TspError) as e:
        capi.Simulation.create(m.xy, m.tri, 0, lam, mu, rho, [(50.0, 50.0)], [])
    assert e.value.code == -9
    with pytest.raises(capi.TspError) as e:
        capi.Simulation.create(m.xy, m.tri, 3, lam, mu, -rho, [(50.0, 50.0)], [])
    assert e.value.code == -1
    with pytest.raises(capi.TspError) as e:  # BoundaryAdapted has no matrix-free operator
        capi.Simulation.create(m.xy, m.tri, 3, lam, mu, rho, [(50.0, 50.0)], [], op="matrix_free", basis="ba")
    assert e.value.code == -9
    capi.TSP_BASIS["bogus"] = 7  # an undefined basis value reaches the C-ABI check
    try:
        with pytest.raises(capi.TspError) as e:
            capi.Simulation.create(m.xy, m.tri, 3, lam, mu, rho, [(50.0, 50.0)], [], basis="bogus")
        assert e.value.code == -1 and "basis" in str(e.value)
    finally:
        del capi.TSP_BASIS["bogus"]


@pytest.mark.parametrize("basis", ["dubiner", "ba"])
@pytest.mark.parametrize("N", [1, 3, 5])
def test_projection_matches_oracle_transform(N, basis):
    m = W.jittered_rect(4, 3, 400.0, 300.0, seed=N)
    pts = capi.quadrature_points(N, m.xy, m.tri)
    fun = lambda x, y: (np.sin(x / 97.0) * np.cos(y / 61.0), 1e-3 * x * y)  # noqa: E731
    fx, fy = fun(pts[..., 0], pts[..., 1])
    got = capi.project(N, m.xy, m.tri, np.stack([fx, fy], -1), basis=basis)
    sp = O.make_space(N, basis)
    tri = m.tri.astype(np.int64)
    ref = O.transform(sp, m.xy, tri, O.geometry(m.xy, tri), fun)
    # The dense M_ref^-1 of BoundaryAdapted amplifies rounding by its
    # condition number (1.3e4 at N = 3, 1.1e5 at N = 5).
    tol = 1e-13 if basis == "dubiner" else 1e-11
    assert np.abs(got - ref).max() / np.abs(ref).max() < tol


@pytest.mark.parametrize("basis", ["dubiner", "ba"])
def test_projection_reproduces_polynomials_of_degree_N(basis):
    N = 3
    m = W.jittered_rect(3, 2, 300.0, 200.0, seed=3)
    pts = capi.quadrature_points(N, m.xy, m.tri)
    f = lambda x, y: (1e-6 * x ** 3 - 2e-4 * x * y, 0.5 + 1e-5 * y ** 2)  # noqa: E731
    fx, fy = f(pts[..., 0], pts[..., 1])
    uh = capi.project(N, m.xy, m.tri, np.stack([fx, fy], -1), basis=basis)
    # Evaluate the modal expansion back at the quadrature points.
    sp = O.make_space(N, basis)
    ne, Np = m.ne, sp.Np
    vx = uh[:ne * Np].reshape(ne, Np) @ sp.B.T
    vy = uh[ne * Np:].reshape(ne, Np) @ sp.B.T
    assert np.abs(vx - fx).max() < 1e-10 * max(1.0, np.abs(fx).max())
    assert np.abs(vy - fy).max() < 1e-10 * max(1.0, np.abs(fy).max())


def test_points_out_matches_reference_bytes(golden, tmp_path):
    """FESpace::points_out text of the reference, byte for byte."""
    f = tmp_path / "pts"
    capi.points_out(golden["xy"], golden["tri"], str(f))
    assert f.read_bytes() == bytes(golden["points_txt"])


def test_projection_matches_reference_golden(golden):
    """tsp_project_basis against the reference's own FESpace::transform."""
    g = golden
    basis = str(g["basis"]) if "basis" in g else "dubiner"
    N = int(g["N"])
    pts = capi.quadrature_points(N, g["xy"], g["tri"])
    fx, fy = golden_field(g)(pts[..., 0], pts[..., 1])
    got = capi.project(N, g["xy"], g["tri"], np.stack([fx, fy], -1), basis=basis)
    tol = 1e-13 if basis == "dubiner" else 1e-11  # cond(M_ref) for BoundaryAdapted
    assert np.abs(got - g["proj"]).max() / np.abs(g["proj"]).max() < tol


@pytest.mark.parametrize("basis", ["dubiner", "ba"])
@pytest.mark.parametrize("N", [1, 4, 8])
def test_eval_basis_and_quadrature_rule_match_oracle(N, basis):
    sp = O.make_space(N, basis)
    r, w = capi.quadrature_rule(N)
    assert np.abs(r - sp.rule.nodes2d).max() < 1e-15 and np.abs(w - sp.rule.w2d).max() < 1e-16
    rng = np.random.default_rng(N)
    c = rng.random(30)
    e = rng.random(30) * (1 - c)
    phi = capi.eval_basis(N, np.stack([c, e], -1), basis=basis)
    assert np.abs(phi - O.basis_phi(N, basis, c, e).T).max() < 1e-12


@pytest.mark.parametrize("basis", ["dubiner", "ba"])
def test_locate_points_matches_oracle_scan(basis):
    """The grid-accelerated point location returns what the reference's
    first-hit linear scan does (Receivers_imp.hpp:34-51): random interior
    points, points on shared edges and vertices (the lowest id wins), and
    points outside the mesh."""
    N = 3
    m = W.jittered_rect(12, 7, 1200.0, 700.0, seed=9)
    rng = np.random.default_rng(3)
    pts = [(1200 * rng.random(), 700 * rng.random()) for _ in range(200)]
    pts += [tuple(m.xy[v]) for v in rng.integers(0, m.xy.shape[0], 40)]          # vertices
    for e in rng.integers(0, m.ne, 40):                                           # edge midpoints
        a, b = m.tri[e][0], m.tri[e][1]
        pts.append(tuple(0.5 * (m.xy[a] + m.xy[b])))
    pts += [(-5.0, 100.0), (600.0, 700.5), (1300.0, -20.0)]                       # outside
    elem, phi = capi.locate_points(N, m.xy, m.tri, pts, basis=basis)
    tri = m.tri.astype(np.int64)
    geo = O.geometry(m.xy, tri)
    for k, (x, y) in enumerate(pts):
        try:
            r = O.locate(N, m.xy, tri, geo, x, y, basis=basis)
        except KeyError:
            r = None
        if r is None:
            assert elem[k] == -1
        else:
            assert elem[k] == r[0]
            ok = np.isfinite(r[1])
            assert np.allclose(phi[k][ok], r[1][ok], rtol=0, atol=1e-12)
