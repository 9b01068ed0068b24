"""The oracle restatement against the golden vectors of the reference (CPU)."""
import numpy as np
import pytest

import tsp_oracle as O
from helpers import golden_field, l2_proj_tol, oracle_setup, rel


def test_neighbours_match_reference(golden):
    nb, ned = O.neighbours(golden["tri"].astype(np.int64))
    assert (nb == golden["neigh"]).all() and (ned == golden["nedge"]).all()


def test_geometry_and_minv(golden):
    o = oracle_setup(golden)
    assert np.array_equal(o["geo"].detJ, golden["detJ"])
    # BoundaryAdapted: the reference stores 1/(rho detJ) * M_ref^-1 and the
    # golden scalar is recovered by one division, hence one rounding.
    tol = 0.0 if o["basis"] == "dubiner" else 4e-16
    assert np.max(np.abs(o["minv"] - golden["minv"]) / np.abs(golden["minv"])) <= tol


def test_points_match_reference(golden):
    o = oracle_setup(golden)
    assert o["src_elem"] == int(golden["src_elem"])
    assert np.allclose(o["src_phi"], golden["src_phi"], rtol=0, atol=1e-13)
    assert list(o["rcv_elem"]) == list(golden["rcv_elem"])
    # A receiver exactly on the collapsed vertex (eta = 1) gives NaN in the
    # reference (0/0 in ShapeFunctions_imp.hpp:34); the oracle reproduces it.
    assert np.allclose(np.array(o["rcv_phi"]), golden["rcv_phi"], rtol=0, atol=1e-13, equal_nan=True)


def test_blocks_match_reference(golden):
    if "blocks" not in golden:
        pytest.skip("case without block dump")
    o = oracle_setup(golden)
    assert np.array_equal(o["row_ptr"], golden["row_ptr"]) and np.array_equal(o["cols"], golden["col"])
    scale = np.abs(golden["blocks"]).max()
    assert np.abs(o["blocks"] - golden["blocks"]).max() / scale < 1e-14


def test_reference_inverse_mass(golden):
    """M_ref^-1 of the space (FESpace_imp.hpp:48-68): identity for Dubiner,
    dense for BoundaryAdapted, against the matrix the reference inverted."""
    o = oracle_setup(golden)
    if o["basis"] == "dubiner":
        assert np.array_equal(o["sp"].minv_ref, np.eye(o["sp"].Np))
        return
    ref = golden["minv_ref"]
    assert np.abs(o["sp"].minv_ref - ref).max() / np.abs(ref).max() < 1e-12


def test_leapfrog_matches_reference(golden):
    o = oracle_setup(golden)
    ne, Np = golden["tri"].shape[0], o["sp"].Np
    u, seis, snaps = O.leapfrog(o["row_ptr"], o["cols"], o["blocks"], o["minv"], ne, Np, float(golden["dt"]),
                                int(golden["nsteps"]), o["src_elem"], o["src_phi"], o["F"], o["rcv_elem"],
                                o["rcv_phi"], snap_steps=(1,), minv_ref=o["minv_ref"])
    assert rel(snaps[1], golden["u_first"]) < 1e-13
    assert rel(u, golden["u_final"]) < 1e-12
    assert np.array_equal(np.isnan(seis), np.isnan(golden["seis"]))
    ok = ~np.isnan(golden["seis"])
    assert rel(seis[ok], golden["seis"][ok]) < 1e-12


@pytest.mark.parametrize("N", [1, 2, 4, 5, 6, 8])
def test_dubiner_orthonormal(N):
    sp = O.make_space(N)
    M = sp.B.T @ (sp.rule.w2d[:, None] * sp.B)
    assert np.abs(M - np.eye(sp.Np)).max() < 5e-14


@pytest.mark.parametrize("n", [2, 5, 9])
def test_gauleg_integrates_polynomials(n):
    x, w = O.gauleg(n, 0.0, 1.0)
    for d in range(2 * n):
        assert abs(np.sum(w * x ** d) - 1.0 / (d + 1)) < 1e-14


def test_force_times_accumulate_like_reference():
    ts = O.force_times(1e-3, 5)
    assert ts[0] == 0.0 and ts[1] == 1e-3 + 1e-3 and ts[2] == (1e-3 + 1e-3) + 1e-3


@pytest.mark.parametrize("N", [1, 2, 3, 5, 8])
def test_boundary_adapted_spans_dubiner_space(N):
    """BoundaryAdapted<N> and Dubiner<N> span the same polynomial space P_N:
    the change of basis C (phi_BA = C phi_Dub) is exact on random points and
    its gradients follow from the same C (ShapeFunctions_imp.hpp:55-118)."""
    rng = np.random.default_rng(N)
    c = rng.random(200)
    e = rng.random(200) * (1 - c)
    D, A = O.dubiner_phi(N, c, e), O.ba_phi(N, c, e)
    C = np.linalg.lstsq(D.T, A.T, rcond=None)[0].T
    assert np.abs(C @ D - A).max() < 1e-11
    assert np.linalg.matrix_rank(C) == D.shape[0]
    gD, gA = O.dubiner_grad(N, c, e), O.ba_grad(N, c, e)
    assert np.abs(np.einsum("ij,jqk->iqk", C, gD) - gA).max() < 1e-9


def test_boundary_adapted_vertex_and_edge_modes_vanish():
    """Vertex modes are the barycentric coordinates; each edge mode vanishes
    on the two edges it does not belong to (boundary adaptation)."""
    N = 5
    t = np.linspace(0.05, 0.95, 7)
    A_e0 = O.ba_phi(N, t, 0 * t)         # edge eta = 0
    A_e1 = O.ba_phi(N, 0 * t, t)         # edge csi = 0
    A_e2 = O.ba_phi(N, t, 1 - t)         # edge csi + eta = 1
    fa = slice(3, 3 + N - 1)             # family A: on eta = 0
    fb = slice(3 + N - 1, 3 + 2 * (N - 1))   # family B: on csi = 0
    fc = slice(3 + 2 * (N - 1), 3 + 3 * (N - 1))  # family C: on csi + eta = 1
    interior = slice(3 + 3 * (N - 1), None)
    assert np.abs(A_e1[fa]).max() < 1e-14 and np.abs(A_e2[fa]).max() < 1e-14
    assert np.abs(A_e0[fb]).max() < 1e-14 and np.abs(A_e2[fb]).max() < 1e-14
    assert np.abs(A_e0[fc]).max() < 1e-14 and np.abs(A_e1[fc]).max() < 1e-14
    for E in (A_e0, A_e1, A_e2):
        assert np.abs(E[interior]).max() < 1e-14


@pytest.mark.parametrize("N", [2, 4])
def test_seismograms_do_not_depend_on_the_basis(N):
    """Dubiner<N> and BoundaryAdapted<N> span the same space and the SIPG
    forms are integrated exactly, so the discrete solution, sampled at the
    receivers, is the same function; only the rounding differs."""
    from tspeed_b200 import workloads as W
    m = W.jittered_rect(5, 4, 500.0, 400.0, seed=3)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1750.0), np.full(m.ne, 2100.0))
    tri = m.tri.astype(np.int64)
    geo = O.geometry(m.xy, tri)
    nb, ned = O.neighbours(tri)
    rcv = W.surface_receivers(m, 4)
    dt, n = 2e-4, 150
    F = [(0.0, O.ricker(t, 80.0, 0.0125, -1.0)) for t in O.force_times(dt, n)]
    out = {}
    for basis in ("dubiner", "ba"):
        sp = O.make_space(N, basis)
        row_ptr, cols, blocks, minv = O.assemble(sp, geo, nb, ned, lam, mu, rho, 10.0)
        se, sphi = O.locate(N, m.xy, tri, geo, 255.0, 205.0, basis=basis)
        rl = [O.locate(N, m.xy, tri, geo, x, y, basis=basis) for (x, y) in rcv]
        _, seis, _ = O.leapfrog(row_ptr, cols, blocks, minv, m.ne, sp.Np, dt, n, se, sphi, F,
                                [r[0] for r in rl], [r[1] for r in rl],
                                minv_ref=None if basis == "dubiner" else sp.minv_ref)
        out[basis] = seis
    assert (np.abs(out["dubiner"][-1]) > 0).all()
    assert rel(out["ba"], out["dubiner"]) < 1e-12


def test_field_and_points_output_match_reference_bytes(golden):
    """FESpace::field_out / points_out text of the reference (final step),
    byte for byte (FESpace_imp.hpp:70-105)."""
    g = golden
    o = oracle_setup(g)
    ne = g["tri"].shape[0]
    assert O.field_text(O.field_values(o["sp"], g["u_final"], ne)) == bytes(g["field_txt"]).decode()
    assert O.points_text(g["xy"], g["tri"]) == bytes(g["points_txt"]).decode()


def test_projection_and_l2_error_match_reference(golden):
    """FESpace::transform of the generator's field and FESpace::L2error of
    that projection and of the final displacement (FESpace_imp.hpp:107-179)."""
    g = golden
    o = oracle_setup(g)
    ne, tri = g["tri"].shape[0], g["tri"].astype(np.int64)
    fun = golden_field(g)
    proj = O.transform(o["sp"], g["xy"], tri, o["geo"], fun)
    tol = 1e-13 if o["basis"] == "dubiner" else 1e-11  # cond(M_ref) for BoundaryAdapted
    assert np.abs(proj - g["proj"]).max() / np.abs(g["proj"]).max() < tol
    qp = O.quadrature_points(o["sp"], g["xy"], tri)
    fx, fy = fun(qp[..., 0], qp[..., 1])
    l2p = O.l2_error(o["sp"], o["geo"], g["proj"], np.stack([fx, fy], -1))
    assert abs(l2p - float(g["l2_proj"])) <= l2_proj_tol(g)
    nq = o["sp"].B.shape[0]
    l2u = O.l2_error(o["sp"], o["geo"], g["u_final"], np.zeros((ne, nq, 2)))
    assert abs(l2u - float(g["l2_u"])) <= 1e-14 * float(g["l2_u"])
