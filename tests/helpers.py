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


def golden_field(g):
    """The field the golden generator projects (tests/golden/make_golden.py
    runs the reference harness, oracle/ref_harness.cpp, which defines it):
    smooth for Dubiner cases, linear for BoundaryAdapted ones."""
    if "basis" in g and str(g["basis"]) == "ba":
        return lambda x, y: (1e-3 + 2e-6 * x - 3e-6 * y + 0 * x, -2e-3 + 1e-6 * x + 4e-6 * y + 0 * x)
    return lambda x, y: (np.sin(x / 97.0) * np.cos(y / 61.0), 1e-6 * x * y)


def l2_proj_tol(g):
    """Absolute tolerance on the golden projection error: rounding of the
    field's values (|f| <= 1 on a domain of area A) dominates,
    1e-13 * sqrt(A) * max|f|."""
    xy = g["xy"]
    area = float(np.ptp(xy[:, 0]) * np.ptp(xy[:, 1]))
    return 1e-13 * np.sqrt(area) * 1.0 + 1e-12 * float(g["l2_proj"])


# ---- operator storage formats, emulated on the oracle's FP64 blocks ----

def bf16_round(x):
    """float32 values rounded to bfloat16 (round to nearest, ties to even),
    returned as float64."""
    x = np.asarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def pow2_scale(m):
    """Power-of-two scale 2^ceil(log2 m) (1 for m = 0): values / scale lie in [-1, 1]."""
    m = np.asarray(m, np.float64)
    return np.where(m > 0, 2.0 ** np.ceil(np.log2(np.where(m > 0, m, 1.0))), 1.0)


def bf16_block_scaled(blocks):
    """The library's BF16 storage: per block, scale = 2^ceil(log2 max|float(B)|),
    entries bf16(float(B) / scale) (the device's k_assemble)."""
    b32 = np.asarray(blocks).astype(np.float32)
    sc = pow2_scale(np.abs(b32).max(axis=(1, 2)))[:, None, None]
    return bf16_round(b32 / sc) * sc


def fixed_point_rows(blocks, planes):
    """Fixed point with a shared power-of-two exponent per block row and
    8 bits per BF16 plane after a 9-bit leading plane (the tensor-core form's
    slicing with `planes` planes): 8 * planes + 1 significant bits."""
    B = np.asarray(blocks, np.float64)
    m = np.abs(B).max(axis=2, keepdims=True)
    ex = np.ceil(np.log2(np.where(m > 0, m, 1.0)))
    return np.rint(B * 2.0 ** (8 * planes - ex)) * 2.0 ** (ex - 8 * planes)
