"""The oracle restatement against the golden vectors of the reference (CPU)."""
import numpy as np
import pytest

import tsp_oracle as O
from helpers import oracle_setup, rel


def test_neighbours_match_reference(golden):
    nb, ned = O.neighbours(golden["tri"].astype(np.int64))
    assert (nb == golden["neigh"]).all() and (ned == golden["nedge"]).all()


def test_geometry_and_minv(golden):
    o = oracle_setup(golden)
    assert np.array_equal(o["geo"].detJ, golden["detJ"])
    assert np.max(np.abs(o["minv"] - golden["minv"]) / np.abs(golden["minv"])) == 0.0


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


def test_leapfrog_matches_reference(golden):
    o = oracle_setup(golden)
    ne, Np = golden["tri"].shape[0], o["sp"].Np
    u, seis, snaps = O.leapfrog(o["row_ptr"], o["cols"], o["blocks"], o["minv"], ne, Np, float(golden["dt"]),
                                int(golden["nsteps"]), o["src_elem"], o["src_phi"], o["F"], o["rcv_elem"],
                                o["rcv_phi"], snap_steps=(1,))
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
