"""CPU oracle for the tspeed leap-frog path (TEST INFRASTRUCTURE ONLY).

A numpy restatement of the reference's algorithm for the explicit time loop:
Dubiner basis and Gauss rule, triangle geometry, neighbour tables, the SIPG
operator blocks B = c*N^2*S + I + A, the inverse mass, point location for
sources and receivers, and the leap-frog recurrence. Every function cites the
reference file:line it restates (paths relative to the reference project).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may import
this module; the product never does. Parity of this restatement is pinned
against the reference's own sources compiled by oracle/Makefile
(oracle/_ref/tsp_ref_run, see tests/test_oracle_vs_ref.py) and against the
committed golden vectors in tests/golden/.

Layouts:
  * reference vector layout ("component-major"): u[c*ne*Np + e*Np + i]
    (FESpace_imp.hpp:152-153, TimeAdvance.cpp:73-74);
  * merged block layout: blocks[b][m*Np+i][n*Np+j] = B^{mn}(row, col_b)_{ij}
    for the block-CSR pattern of MyMat (MyMat.cpp:128-154).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


# --------------------------------------------------------------------------
# Reference element: Jacobi polynomials, Dubiner basis, Gauss rule.
# --------------------------------------------------------------------------
def jacobi(n: int, alpha: int, beta: int, z: np.ndarray) -> np.ndarray:
    """Three-term recurrence of ShapeFunctions.cpp:25-60 (P_n^{alpha,beta});
    a negative degree gives zero there (the loop does not run on a zero
    start, ShapeFunctions.cpp:37-39)."""
    z = np.asarray(z, dtype=np.float64)
    if n < 0:
        return np.zeros_like(z)
    if n == 0:
        return np.ones_like(z)
    if n == 1:
        return 0.5 * (alpha - beta + (alpha + beta + 2.0) * z)
    apb = alpha + beta
    p2 = np.ones_like(z)
    p1 = 0.5 * (alpha - beta + (alpha + beta + 2.0) * z)
    p = p1
    for k in range(2, n + 1):
        a1 = 2.0 * k * (k + apb) * (2.0 * k + apb - 2.0)
        a2 = (2.0 * k + apb - 1.0) * (alpha * alpha - beta * beta)
        a3 = (2.0 * k + apb - 2.0) * (2.0 * k + apb - 1.0) * (2.0 * k + apb)
        a4 = 2.0 * (k + alpha - 1.0) * (k + beta - 1.0) * (2.0 * k + apb)
        a2, a3, a4 = a2 / a1, a3 / a1, a4 / a1
        p = (a2 + a3 * z) * p1 - a4 * p2
        p2, p1 = p1, p
    return p


def dubiner_index(N: int):
    """Basis ordering of ShapeFunctions_imp.hpp:29-31: j outer, i inner."""
    return [(i, j) for j in range(N + 1) for i in range(N + 1 - j)]


def dubiner_phi(N: int, csi, eta) -> np.ndarray:
    """phi_ij(csi, eta), ShapeFunctions_imp.hpp:33-34. Returns [Np, npts]."""
    csi = np.atleast_1d(np.asarray(csi, dtype=np.float64))
    eta = np.atleast_1d(np.asarray(eta, dtype=np.float64))
    out = []
    for (i, j) in dubiner_index(N):
        cij = math.sqrt((2.0 * i + 1) * 2.0 * (i + j + 1) / 4.0 ** i)
        v = cij * (2.0 ** i) * ((1 - eta) ** i) * jacobi(i, 0, 0, 2 * csi / (1 - eta) - 1) \
            * jacobi(j, 2 * i + 1, 0, 2 * eta - 1)
        out.append(v)
    return np.array(out)


def dubiner_grad(N: int, csi, eta) -> np.ndarray:
    """Reference gradients, ShapeFunctions_imp.hpp:35-50. Returns [Np, npts, 2]."""
    csi = np.atleast_1d(np.asarray(csi, dtype=np.float64))
    eta = np.atleast_1d(np.asarray(eta, dtype=np.float64))
    out = []
    for (i, j) in dubiner_index(N):
        cij = math.sqrt((2.0 * i + 1) * 2.0 * (i + j + 1) / 4.0 ** i)
        g = np.zeros((csi.size, 2))
        xx = 2 * csi / (1 - eta) - 1
        if i == 0 and j == 0:
            pass
        elif i == 0:
            g[:, 1] = cij * (j + 2) * jacobi(j - 1, 2, 1, 2 * eta - 1)
        elif j == 0:
            g[:, 0] = cij * 2.0 ** i * (1 - eta) ** (i - 1) * (i + 1) * jacobi(i - 1, 1, 1, xx)
            g[:, 1] = cij * 2.0 ** i * (-i * (1 - eta) ** (i - 1) * jacobi(i, 0, 0, xx)
                                        + csi * (1 - eta) ** (i - 2) * (i + 1) * jacobi(i - 1, 1, 1, xx))
        else:
            pj = jacobi(j, 2 * i + 1, 0, 2 * eta - 1)
            g[:, 0] = cij * 2.0 ** i * (1 - eta) ** (i - 1) * (i + 1) * jacobi(i - 1, 1, 1, xx) * pj
            g[:, 1] = cij * 2.0 ** i * (-i * (1 - eta) ** (i - 1) * jacobi(i, 0, 0, xx) * pj
                                        + csi * (1 - eta) ** (i - 2) * (i + 1) * jacobi(i - 1, 1, 1, xx) * pj
                                        + (1 - eta) ** i * (2 * i + j + 2) * jacobi(i, 0, 0, xx)
                                        * jacobi(j - 1, 2 * i + 2, 1, 2 * eta - 1))
        out.append(g)
    return np.array(out)


def ba_phi(N: int, csi, eta) -> np.ndarray:
    """BoundaryAdapted<N> basis, ShapeFunctions_imp.hpp:55-118 (order: the
    three vertex modes, the edge modes of the three families, then the
    interior modes j outer / i inner with i + j < N). Returns [Np, npts]."""
    csi = np.atleast_1d(np.asarray(csi, dtype=np.float64))
    eta = np.atleast_1d(np.asarray(eta, dtype=np.float64))
    l0 = 1 - csi - eta
    xx = 2 * csi / (1 - eta) - 1
    yy = 2 * eta - 1
    out = [l0, csi.copy(), eta.copy()]
    for i in range(1, N):
        out.append(l0 * csi * (1 - eta) ** (i - 1) * jacobi(i - 1, 1, 1, xx))
    for j in range(1, N):
        out.append(l0 * eta * jacobi(j - 1, 1, 1, yy))
    for j in range(1, N):
        out.append(csi * eta * jacobi(j - 1, 1, 1, yy))
    for j in range(1, N):
        for i in range(1, N):
            if i + j < N:
                out.append(l0 * csi * eta * (1 - eta) ** (i - 1) * jacobi(i - 1, 1, 1, xx)
                           * jacobi(j - 1, 2 * i + 1, 1, yy))
    return np.array(out)


def ba_grad(N: int, csi, eta) -> np.ndarray:
    """Gradients of BoundaryAdapted<N>, ShapeFunctions_imp.hpp:59-116.
    Returns [Np, npts, 2]."""
    csi = np.atleast_1d(np.asarray(csi, dtype=np.float64))
    eta = np.atleast_1d(np.asarray(eta, dtype=np.float64))
    n = csi.size
    l0 = 1 - csi - eta
    xx = 2 * csi / (1 - eta) - 1
    yy = 2 * eta - 1
    out = [np.stack([-np.ones(n), -np.ones(n)], 1), np.stack([np.ones(n), np.zeros(n)], 1),
           np.stack([np.zeros(n), np.ones(n)], 1)]
    for i in range(1, N):
        g0 = (1 - 2 * csi - eta) * (1 - eta) ** (i - 1) * jacobi(i - 1, 1, 1, xx) \
            + l0 * csi * (1 - eta) ** (i - 2) * jacobi(i - 2, 2, 2, xx) * (i + 2)
        g1 = -(1 - eta) ** (i - 2) * csi * (i + csi - i * csi - i * eta) * jacobi(i - 1, 1, 1, xx) \
            + csi * csi * l0 * (1 - eta) ** (i - 3) * (i + 2) * jacobi(i - 2, 2, 2, xx)
        out.append(np.stack([g0, g1], 1))
    for j in range(1, N):
        g0 = -eta * jacobi(j - 1, 1, 1, yy)
        g1 = (1 - csi - 2 * eta) * jacobi(j - 1, 1, 1, yy) + l0 * eta * jacobi(j - 2, 2, 2, yy) * (j + 2)
        out.append(np.stack([g0, g1], 1))
    for j in range(1, N):
        g0 = eta * jacobi(j - 1, 1, 1, yy)
        g1 = csi * jacobi(j - 1, 1, 1, yy) + eta * csi * (j + 2) * jacobi(j - 2, 2, 2, yy)
        out.append(np.stack([g0, g1], 1))
    for j in range(1, N):
        for i in range(1, N):
            if i + j < N:
                pa, pb = jacobi(i - 1, 1, 1, xx), jacobi(j - 1, 2 * i + 1, 1, yy)
                g0 = eta * (1 - eta) ** (i - 2) * pb * ((1 - 2 * csi - eta) * (1 - eta) * pa
                                                       + l0 * csi * (i + 2) * jacobi(i - 2, 2, 2, xx))
                g1 = csi * (1 - eta) ** (i - 3) * (
                    ((1 - eta) ** 2 * (1 - csi - 2 * eta) - (1 - eta) * eta * l0 * (i - 1)) * pa * pb
                    + csi * l0 * eta * (i + 2) * jacobi(i - 2, 2, 2, xx) * pb
                    + l0 * eta * (1 - eta) ** 2 * (j + 2 * i + 2) * pa * jacobi(j - 2, 2 * i + 2, 2, yy))
                out.append(np.stack([g0, g1], 1))
    return np.array(out)


def basis_phi(N: int, basis: str, csi, eta) -> np.ndarray:
    return ba_phi(N, csi, eta) if basis == "ba" else dubiner_phi(N, csi, eta)


def basis_grad(N: int, basis: str, csi, eta) -> np.ndarray:
    return ba_grad(N, csi, eta) if basis == "ba" else dubiner_grad(N, csi, eta)


def gauleg(n: int, a: float, b: float):
    """Gauss-Legendre nodes/weights by Newton iteration, QuadratureRule_imp.hpp:23-61."""
    x = np.zeros(n)
    w = np.zeros(n)
    m = (n + 1.0) / 2.0
    xm = 0.5 * (b + a)
    xl = 0.5 * (b - a)
    eps = np.finfo(np.float64).eps
    i = 1
    while i <= m:
        z = math.cos(math.pi * (i - 0.25) / (n + 0.5))
        while True:
            p1, p2 = 1.0, 0.0
            for j in range(1, n + 1):
                p3 = p2
                p2 = p1
                p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j
            pp = n * (z * p1 - p2) / (z * z - 1.0)
            z1 = z
            z = z1 - p1 / pp
            if not abs(z - z1) > eps:
                break
        x[i - 1] = xm - xl * z
        x[n - i] = xm + xl * z
        w[i - 1] = 2.0 * xl / ((1.0 - z * z) * pp * pp)
        w[n - i] = w[i - 1]
        i += 1
    return x, w


@dataclass
class Rule:
    nodes2d: np.ndarray  # [Q*Q, 2]
    w2d: np.ndarray      # [Q*Q]
    x1d: np.ndarray      # [Q] on [0, 1]
    w1d: np.ndarray      # [Q]

    def edge_nodes(self, e: int) -> np.ndarray:
        """Edge parametrisation of QuadratureRule_imp.hpp:66-91."""
        x = self.x1d
        if e == 2:
            return np.stack([x, np.zeros_like(x)], 1)
        if e == 0:
            return np.stack([1.0 - x, x], 1)
        if e == 1:
            return np.stack([np.zeros_like(x), 1.0 - x], 1)
        raise ValueError("edge must be 0, 1 or 2")


def gauss_rule(Q: int) -> Rule:
    """Collapsed Gauss<Q> rule, QuadratureRule_imp.hpp:92-119 (Q = N + 1)."""
    w1, x1 = None, None
    x1, w1 = gauleg(Q, 0.0, 1.0)
    x, w = gauleg(Q, -1.0, 1.0)
    nodes = np.zeros((Q * Q, 2))
    wts = np.zeros(Q * Q)
    for i in range(Q):
        for j in range(Q):
            wts[i * Q + j] = (1 - x[i]) * w[i] * w[j] / 8.0
            nodes[i * Q + j, 0] = (1 + x[i]) / 2.0
            nodes[i * Q + j, 1] = (1 - x[i]) * (1 + x[j]) / 4.0
    return Rule(nodes, wts, x1, w1)


@dataclass
class Space:
    """Tabulated FESpace<N, Q, S> (FESpace_imp.hpp:25-68): S = Dubiner<N> with
    Q = Gauss<N+1>, or S = BoundaryAdapted<N>. For BoundaryAdapted the
    reference uses Q = Dunavant<2N> (Examples/src/Lamb.cpp:26); on affine
    triangles every integrand is a polynomial of degree <= 2N, which the
    collapsed Gauss<N+1> rule (degree 2N+1) also integrates exactly, so the
    tables agree to rounding."""
    N: int
    Np: int
    rule: Rule
    B: np.ndarray       # [nq, Np]   basis at volume points
    G: np.ndarray       # [Np, nq, 2] reference gradients at volume points
    Bedge: np.ndarray   # [3, Q, Np]
    Gedge: np.ndarray   # [3, Np, Q, 2]
    basis: str = "dubiner"
    minv_ref: np.ndarray = None  # reference inverse mass (FESpace_imp.hpp:48-68)


def make_space(N: int, basis: str = "dubiner") -> Space:
    rule = gauss_rule(N + 1)
    Np = (N + 1) * (N + 2) // 2
    c, e = rule.nodes2d[:, 0], rule.nodes2d[:, 1]
    B = basis_phi(N, basis, c, e).T
    G = basis_grad(N, basis, c, e)
    Bedge = np.zeros((3, N + 1, Np))
    Gedge = np.zeros((3, Np, N + 1, 2))
    for ed in range(3):
        en = rule.edge_nodes(ed)
        Bedge[ed] = basis_phi(N, basis, en[:, 0], en[:, 1]).T
        Gedge[ed] = basis_grad(N, basis, en[:, 0], en[:, 1])
    if basis == "ba":
        minv_ref = np.linalg.inv(B.T @ (rule.w2d[:, None] * B))
    else:
        minv_ref = np.eye(Np)  # orthonormal: M_ref = I (FESpace_imp.hpp:51-54)
    return Space(N, Np, rule, B, G, Bedge, Gedge, basis, minv_ref)


# --------------------------------------------------------------------------
# Geometry and mesh.
# --------------------------------------------------------------------------
@dataclass
class Geom:
    detJ: np.ndarray     # [ne] signed
    invJ: np.ndarray     # [ne, 2, 2]
    elen: np.ndarray     # [ne, 3]
    enrm: np.ndarray     # [ne, 3, 2]


def geometry(xy: np.ndarray, tri: np.ndarray) -> Geom:
    """Triangle::setJac/setdetJ/setinvJac and Edge::length/normal,
    Geometry.cpp:100-105, 125-132, 178-198 (edge i is opposite vertex i)."""
    p = xy[tri]  # [ne, 3, 2]
    J = np.zeros((tri.shape[0], 2, 2))
    J[:, :, 0] = p[:, 1] - p[:, 0]
    J[:, :, 1] = p[:, 2] - p[:, 0]
    det = J[:, 0, 0] * J[:, 1, 1] - J[:, 1, 0] * J[:, 0, 1]
    invdet = 1.0 / det
    inv = np.zeros_like(J)
    inv[:, 0, 0] = J[:, 1, 1] * invdet
    inv[:, 1, 0] = -J[:, 1, 0] * invdet
    inv[:, 0, 1] = -J[:, 0, 1] * invdet
    inv[:, 1, 1] = J[:, 0, 0] * invdet
    ends = [(1, 2), (2, 0), (0, 1)]
    elen = np.zeros((tri.shape[0], 3))
    enrm = np.zeros((tri.shape[0], 3, 2))
    for k, (a, b) in enumerate(ends):
        pa, pb = p[:, a], p[:, b]
        d = pa - pb
        elen[:, k] = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1])
        nx = -pa[:, 1] + pb[:, 1]
        ny = pa[:, 0] - pb[:, 0]
        nn = np.sqrt(nx * nx + ny * ny)
        enrm[:, k, 0] = nx / nn
        enrm[:, k, 1] = ny / nn
    return Geom(det, inv, elen, enrm)


def neighbours(tri: np.ndarray):
    """Neighbour tables of Mesh::M_neighbors (Mesh.cpp:33-128).

    Two triangles are neighbours across edge a of the first and edge b of the
    second when the directed edges are reversed copies of each other (the nine
    cases of Mesh.cpp:49-111). Returns neigh[ne,3] (-1 on the boundary) and
    neighedges[ne,3]. The reference compares all pairs; a dictionary of
    directed edges gives the same tables for conforming meshes.
    """
    ne = tri.shape[0]
    neigh = -np.ones((ne, 3), dtype=np.int64)
    nedg = -np.ones((ne, 3), dtype=np.int64)
    ends = [(1, 2), (2, 0), (0, 1)]
    table = {}
    for e in range(ne):
        for k, (a, b) in enumerate(ends):
            table[(int(tri[e, a]), int(tri[e, b]))] = (e, k)
    for e in range(ne):
        for k, (a, b) in enumerate(ends):
            hit = table.get((int(tri[e, b]), int(tri[e, a])))
            if hit is not None and hit[0] != e:
                neigh[e, k] = hit[0]
                nedg[e, k] = hit[1]
    return neigh, nedg


def bsr_pattern(neigh: np.ndarray):
    """Block-CSR pattern of MyMat(Mesh_ptr, nln), MyMat.cpp:128-154: per row the
    diagonal block first, then the neighbours in edge order 0, 1, 2."""
    ne = neigh.shape[0]
    row_ptr = np.zeros(ne + 1, dtype=np.int64)
    cols = []
    for e in range(ne):
        cols.append(e)
        for k in range(3):
            if neigh[e, k] >= 0:
                cols.append(int(neigh[e, k]))
        row_ptr[e + 1] = len(cols)
    return row_ptr, np.array(cols, dtype=np.int64)


def harmonic(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Parameters::avg_p, Parameters.cpp:37-45."""
    s = a + b
    with np.errstate(divide="ignore", invalid="ignore"):
        out = np.where(s == 0, 0.0, 2 * a * b / np.where(s == 0, 1.0, s))
    return out


# --------------------------------------------------------------------------
# Operator assembly (Matrices_imp.hpp:22-215, TimeAdvance_imp.hpp:32).
# --------------------------------------------------------------------------
def _sigma_n(g0, g1, lam, mu, n0, n1):
    """(sigma(phi e_m) . n)_c for m in {0,1}, c in {0,1} (Matrices_imp.hpp:22-47 with
    CTensorProduct TimeAdvance.cpp:60-64). g0, g1: physical gradients."""
    # m = 0: sigma = [[(l+2m) g0, mu g1], [mu g1, l g0]]
    # m = 1: sigma = [[l g1, mu g0], [mu g0, (l+2m) g1]]
    t00 = (lam + 2 * mu) * g0 * n0 + mu * g1 * n1   # m=0, row 0
    t01 = mu * g1 * n0 + lam * g0 * n1              # m=0, row 1
    t10 = lam * g1 * n0 + mu * g0 * n1              # m=1, row 0
    t11 = mu * g0 * n0 + (lam + 2 * mu) * g1 * n1   # m=1, row 1
    return ((t00, t01), (t10, t11))


def assemble(sp: Space, geo: Geom, neigh, nedg, lam, mu, rho, penalty: float):
    """Returns (row_ptr, cols, blocks[nnzb, 2Np, 2Np], minv[ne]).

    A: stress_loc, Matrices_imp.hpp:73-94 (|detJ| weights);
    I: interelement + symmetrize, Matrices_imp.hpp:95-141, 213 and
       MyMat.cpp:156-187 (I <- I + I^T);
    S: stability, Matrices_imp.hpp:142-182 (harmonic lambda, mu; S^10 = S^01);
    B = penalty*N*N*S + I + A, TimeAdvance_imp.hpp:32;
    invM = 1/rho * 1/detJ * I_Np, Matrices_imp.hpp:183-190.
    """
    N, Np = sp.N, sp.Np
    ne = geo.detJ.shape[0]
    R = 2 * Np
    row_ptr, cols = bsr_pattern(neigh)
    nnzb = cols.shape[0]
    blocks = np.zeros((nnzb, R, R))
    pos = {}
    for e in range(ne):
        for b in range(row_ptr[e], row_ptr[e + 1]):
            pos[(e, int(cols[b]))] = b

    # ---- A (volume) ----
    g = np.einsum("iqa,eak->eqik", sp.G, geo.invJ)           # physical grads [ne,nq,Np,2]
    dx = np.abs(geo.detJ)[:, None] * sp.rule.w2d[None, :]   # [ne, nq]
    Gkl = np.einsum("eqik,eqjl,eq->eklij", g, g, dx)          # [ne,2,2,Np,Np]
    l = lam[:, None, None]
    m_ = mu[:, None, None]
    A00 = (l + 2 * m_) * Gkl[:, 0, 0] + m_ * Gkl[:, 1, 1]
    A11 = (l + 2 * m_) * Gkl[:, 1, 1] + m_ * Gkl[:, 0, 0]
    A01 = l * Gkl[:, 0, 1] + m_ * Gkl[:, 1, 0]
    A10 = m_ * Gkl[:, 0, 1] + l * Gkl[:, 1, 0]
    d = row_ptr[:-1]
    blocks[d, :Np, :Np] += A00
    blocks[d, :Np, Np:] += A01
    blocks[d, Np:, :Np] += A10
    blocks[d, Np:, Np:] += A11

    # ---- I (consistency, before symmetrisation) and S (penalty) ----
    Q = N + 1
    w1 = sp.rule.w1d
    Inon = np.zeros_like(blocks)
    S = np.zeros_like(blocks)
    for e in range(ne):
        for k in range(3):
            nb = int(neigh[e, k])
            if nb < 0:
                continue
            kp = int(nedg[e, k])
            L = geo.elen[e, k]
            n0, n1 = geo.enrm[e, k]
            ds = L * w1                                       # [Q]
            ge = np.einsum("iqa,ak->iqk", sp.Gedge[k], geo.invJ[e])  # [Np,Q,2]
            t = _sigma_n(ge[:, :, 0], ge[:, :, 1], lam[e], mu[e], n0, n1)
            be = sp.Bedge[k]                                  # [Q, Np]
            bn = sp.Bedge[kp][::-1]                           # kk = Q-1-k
            bd, bo = pos[(e, e)], pos[(e, nb)]
            for mm in range(2):
                for nn in range(2):
                    tm = t[mm][nn] * ds[None, :]              # [Np, Q]
                    Inon[bd, mm * Np:(mm + 1) * Np, nn * Np:(nn + 1) * Np] -= 0.5 * tm @ be
                    Inon[bo, mm * Np:(mm + 1) * Np, nn * Np:(nn + 1) * Np] += 0.5 * tm @ bn
            al = harmonic(np.array(lam[e]), np.array(lam[nb]))
            am = harmonic(np.array(mu[e]), np.array(mu[nb]))
            c00 = (al + 2 * am) * n0 * n0 + 2 * am * n1 * n1
            c11 = (al + 2 * am) * n1 * n1 + 2 * am * n0 * n0
            c01 = al * n0 * n1
            h = 1.0 / L
            Mself = (be * ds[:, None]).T @ be                 # [Np, Np]
            Mcross = (be * ds[:, None]).T @ bn
            for (mm, nn, c) in ((0, 0, c00), (1, 1, c11), (0, 1, c01), (1, 0, c01)):
                S[bd, mm * Np:(mm + 1) * Np, nn * Np:(nn + 1) * Np] += c * h * Mself
                S[bo, mm * Np:(mm + 1) * Np, nn * Np:(nn + 1) * Np] -= c * h * Mcross
    # I <- I + I^T (block (e, c) gets block (c, e) transposed).
    Isym = Inon.copy()
    for e in range(ne):
        for b in range(row_ptr[e], row_ptr[e + 1]):
            c = int(cols[b])
            Isym[b] += Inon[pos[(c, e)]].T
    blocks += penalty * N * N * S + Isym
    minv = (1.0 / rho) / geo.detJ
    return row_ptr, cols, blocks, minv


def transform(sp: Space, xy, tri, geo: Geom, fun):
    """FESpace::transform (FESpace_imp.hpp:136-179): per element
    rhs_i = sum_q f(map(x_q)) |detJ| w_q phi_i(x_q), uh = 1/detJ * M^-1 rhs with
    M = I for the orthonormal basis. fun(x, y) -> (fx, fy) on arrays."""
    ne = tri.shape[0]
    p = xy[tri]
    n2 = sp.rule.nodes2d
    X = p[:, 0, 0][:, None] + (p[:, 1, 0] - p[:, 0, 0])[:, None] * n2[None, :, 0] + (p[:, 2, 0] - p[:, 0, 0])[:, None] * n2[None, :, 1]
    Y = p[:, 0, 1][:, None] + (p[:, 1, 1] - p[:, 0, 1])[:, None] * n2[None, :, 0] + (p[:, 2, 1] - p[:, 0, 1])[:, None] * n2[None, :, 1]
    fx, fy = fun(X, Y)
    dx = np.abs(geo.detJ)[:, None] * sp.rule.w2d[None, :]
    rx = np.einsum("eq,qi->ei", fx * dx, sp.B) @ sp.minv_ref.T
    ry = np.einsum("eq,qi->ei", fy * dx, sp.B) @ sp.minv_ref.T
    return np.concatenate([(rx / geo.detJ[:, None]).ravel(), (ry / geo.detJ[:, None]).ravel()])


# Reference points of FESpace::field_out / points_out (FESpace_imp.hpp:31-34,
# 70-84): three near the vertices and the midpoint of the long edge.
FIELD_POINTS = np.array([[0.2, 0.2], [0.8, 0.2], [0.2, 0.8], [0.5, 0.5]])


def field_values(sp: Space, u, ne: int) -> np.ndarray:
    """FESpace::field_out values (FESpace_imp.hpp:85-105): the expansion of
    each component at FIELD_POINTS, [ne, 4, 2]."""
    V = basis_phi(sp.N, sp.basis, FIELD_POINTS[:, 0], FIELD_POINTS[:, 1])  # [Np, 4]
    ux = u[:ne * sp.Np].reshape(ne, sp.Np) @ V
    uy = u[ne * sp.Np:].reshape(ne, sp.Np) @ V
    return np.stack([ux, uy], -1)


def gformat(v: float) -> str:
    """A double as std::ostream prints it by default (precision 6, %g)."""
    return "%g" % v


def field_text(vals) -> str:
    """The lines FESpace::field_out writes: "valx valy" per element and point."""
    return "".join(f"{gformat(x)} {gformat(y)}\n" for x, y in np.asarray(vals).reshape(-1, 2))


def points_text(xy, tri) -> str:
    """FESpace::points_out (FESpace_imp.hpp:70-84): Triangle::map of
    FIELD_POINTS (p0 + J p^, Geometry.cpp:203-207) for every element."""
    lines = []
    for t in tri:
        p0, p1, p2 = xy[t[0]], xy[t[1]], xy[t[2]]
        for a, b in FIELD_POINTS:
            x = p0[0] + ((p1[0] - p0[0]) * a + (p2[0] - p0[0]) * b)
            y = p0[1] + ((p1[1] - p0[1]) * a + (p2[1] - p0[1]) * b)
            lines.append(f"{gformat(x)} {gformat(y)}\n")
    return "".join(lines)


def l2_error(sp: Space, geo: Geom, u, exact) -> float:
    """FESpace::L2error (FESpace_imp.hpp:107-133): sqrt(sum_e detJ_e
    sum_q |u_h(x_q) - u(x_q)|^2 w_q), elements and points in order; exact is
    [ne, nq, 2] at the volume quadrature points."""
    ne, Np = geo.detJ.shape[0], sp.Np
    ax = u[:ne * Np].reshape(ne, Np) @ sp.B.T
    ay = u[ne * Np:].reshape(ne, Np) @ sp.B.T
    err = 0.0
    for e in range(ne):
        loc = 0.0
        for q in range(sp.B.shape[0]):
            dx, dy = ax[e, q] - exact[e, q, 0], ay[e, q] - exact[e, q, 1]
            loc += (dx * dx + dy * dy) * sp.rule.w2d[q]
        err += loc * geo.detJ[e]
    return float(np.sqrt(err))


def quadrature_points(sp: Space, xy, tri) -> np.ndarray:
    """Physical volume quadrature points [ne, nq, 2] (Triangle::map)."""
    p = xy[tri]
    n2 = sp.rule.nodes2d
    X = p[:, 0, 0][:, None] + ((p[:, 1, 0] - p[:, 0, 0])[:, None] * n2[None, :, 0] + (p[:, 2, 0] - p[:, 0, 0])[:, None] * n2[None, :, 1])
    Y = p[:, 0, 1][:, None] + ((p[:, 1, 1] - p[:, 0, 1])[:, None] * n2[None, :, 0] + (p[:, 2, 1] - p[:, 0, 1])[:, None] * n2[None, :, 1])
    return np.stack([X, Y], -1)


# --------------------------------------------------------------------------
# Point location, sources, receivers.
# --------------------------------------------------------------------------
def intriangle(xy: np.ndarray, tri: np.ndarray, e: int, px: float, py: float) -> bool:
    """Triangle::intriangle, Geometry.cpp:112-118 (absolute 1e-6 tolerance)."""
    p0, p1, p2 = xy[tri[e, 0]], xy[tri[e, 1]], xy[tri[e, 2]]
    s = p0[1] * p2[0] - p0[0] * p2[1] + (p2[1] - p0[1]) * px + (p0[0] - p2[0]) * py
    t = p0[0] * p1[1] - p0[1] * p1[0] + (p0[1] - p1[1]) * px + (p1[0] - p0[0]) * py
    A = 1.0 / 2.0 * (-p1[1] * p2[0] + p0[1] * (-p1[0] + p2[0]) + p0[0] * (p1[1] - p2[1]) + p1[0] * p2[1])
    return (s > -1e-6) and (t > -1e-6) and ((s + t) < (2 + 1e-6) * A)


def locate(N: int, xy, tri, geo: Geom, px: float, py: float, basis: str = "dubiner"):
    """PointWiseEntity::M_add, Receivers_imp.hpp:34-51: first element (lowest id)
    that contains the point; reference coordinates by Triangle::invmap
    (Geometry.cpp:199-202); basis values phi_s(x^)."""
    for e in range(tri.shape[0]):
        if intriangle(xy, tri, e, px, py):
            p0 = xy[tri[e, 0]]
            dxp, dyp = px - p0[0], py - p0[1]
            inv = geo.invJ[e]
            r0 = inv[0, 0] * dxp + inv[0, 1] * dyp
            r1 = inv[1, 0] * dxp + inv[1, 1] * dyp
            return e, basis_phi(N, basis, r0, r1)[:, 0]
    raise KeyError(f"point ({px}, {py}) not found")


def ricker(t, f0: float, t0: float, amp: float):
    """Ricker wavelet of Examples/src/Lamb.cpp:37, scaled by amp."""
    return amp * ((1 - 2 * math.pi * math.pi * (f0 * f0) * (t - t0) * (t - t0))
                  * math.exp(-math.pi * math.pi * (f0 * f0) * (t - t0) * (t - t0)))


def force_times(dt: float, nsteps: int):
    """Times at which the force is evaluated: first_step uses f(0)
    (TimeAdvance.cpp:28); step k uses f(M_last_time + dt) with M_last_time
    accumulated in double from dt (TimeAdvance.cpp:31,46,52 and
    TimeAdvance.hpp:230). Entry k is the force time of leap-frog step k
    (k = 0: first_step)."""
    ts = [0.0]
    last = dt
    for _ in range(1, nsteps):
        t = last + dt
        ts.append(t)
        last = t
    return ts


# --------------------------------------------------------------------------
# Leap-frog loop (TimeAdvance.cpp:24-59) in the reference vector layout.
# --------------------------------------------------------------------------
def merged_to_components(blocks: np.ndarray, Np: int):
    return [[blocks[:, m * Np:(m + 1) * Np, n * Np:(n + 1) * Np] for n in range(2)] for m in range(2)]


def apply_B(row_ptr, cols, blocks, u: np.ndarray, ne: int, Np: int) -> np.ndarray:
    """MyMatMultiDim::vecMult (MyMat.hpp:311-319) over BaseMat::vecMult
    (MyMat.cpp:200-218): out_x = B_xx u_x + B_xy u_y, out_y = B_yx u_x + B_yy u_y."""
    ux = u[:ne * Np].reshape(ne, Np)
    uy = u[ne * Np:].reshape(ne, Np)
    rows = np.repeat(np.arange(ne), np.diff(row_ptr))
    out = np.zeros((2, ne, Np))
    comp = merged_to_components(blocks, Np)
    for m in range(2):
        acc = np.zeros((ne, Np))
        for n, v in ((0, ux), (1, uy)):
            prod = np.einsum("bij,bj->bi", comp[m][n], v[cols])
            np.add.at(acc, rows, prod)
        out[m] = acc
    return out.reshape(-1)


def leapfrog(row_ptr, cols, blocks, minv, ne, Np, dt, nsteps, src_elem, src_phi, F,
             rcv_elems, rcv_phi, u0=None, v0=None, snap_steps=(), minv_ref=None):
    """Runs first_step + (nsteps-1) step() calls. F[k] = (Fx, Fy) at the force
    time of step k. Returns (u after nsteps, seismogram [nsteps, nr, 2],
    snapshots {step: u}). Receivers are sampled after every step with the
    arithmetic of TimeAdvance::eval_receivers (TimeAdvance.cpp:68-79).
    minv_ref (non-orthonormal spaces) is the reference-element inverse mass:
    the per-element inverse mass is then minv[e] * minv_ref, a dense Np x Np
    block (Matrices_imp.hpp:187-189)."""
    n = 2 * ne * Np
    u0 = np.zeros(n) if u0 is None else u0
    v0 = np.zeros(n) if v0 is None else v0
    if minv_ref is None:
        minv_diag = np.concatenate([np.repeat(minv, Np), np.repeat(minv, Np)])

        def minv_full(r):
            return minv_diag * r
    else:
        def minv_full(r):
            r = r.reshape(2, ne, Np)
            return ((r @ minv_ref.T) * minv[None, :, None]).ravel()

    def fvec(k):
        f = np.zeros(n)
        f[src_elem * Np:(src_elem + 1) * Np] = F[k][0] * src_phi
        f[ne * Np + src_elem * Np: ne * Np + (src_elem + 1) * Np] = F[k][1] * src_phi
        return f

    def sample(u):
        out = np.zeros((len(rcv_elems), 2))
        for r, (e, ph) in enumerate(zip(rcv_elems, rcv_phi)):
            out[r, 0] = ph @ u[e * Np:(e + 1) * Np]
            out[r, 1] = ph @ u[ne * Np + e * Np: ne * Np + (e + 1) * Np]
        return out

    seis = np.zeros((nsteps, len(rcv_elems), 2))
    snaps = {}
    Bu = apply_B(row_ptr, cols, blocks, u0, ne, Np)
    u1 = u0 + dt * v0 - minv_full(dt * dt / 2 * (Bu - fvec(0)))
    uold, ucur = u0, u1
    seis[0] = sample(ucur)
    if 1 in snap_steps:
        snaps[1] = ucur.copy()
    for k in range(1, nsteps):
        Bu = apply_B(row_ptr, cols, blocks, ucur, ne, Np)
        unew = 2 * ucur - uold + minv_full(-dt * dt * (Bu - fvec(k)))
        uold, ucur = ucur, unew
        seis[k] = sample(ucur)
        if (k + 1) in snap_steps:
            snaps[k + 1] = ucur.copy()
    return ucur, seis, snaps


def energy(row_ptr, cols, blocks, minv, ne, Np, u_prev, u_cur, dt):
    """Discrete leap-frog energy E = 1/2 |u^{n+1}-u^n|_M^2 / dt^2 + 1/2 (u^{n+1})^T B u^n,
    conserved for f = 0 and symmetric B. M = rho*detJ*I = 1/minv per element."""
    mass = np.concatenate([np.repeat(1.0 / minv, Np), np.repeat(1.0 / minv, Np)])
    d = u_cur - u_prev
    Bu = apply_B(row_ptr, cols, blocks, u_prev, ne, Np)
    return 0.5 * np.sum(mass * d * d) / (dt * dt) + 0.5 * float(u_cur @ Bu)
