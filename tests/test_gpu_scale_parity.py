"""Parity at benchmark size against the reference's own stepping loop (GPU).

The goldens come from the reference's sources compiled unmodified
(oracle/_ref, tests/golden/make_golden.py, SCALE_CASES), run over a
benchmark configuration's full step count, one reference process per shot:

  g_config1_full    configuration 1 in full: 1,600 triangles, N=4,
                    homogeneous, 2,000 steps, 8 receivers;
  g_config3_sample  the 64-shot configuration's shape on its x0.2 sample:
                    1,600 triangles, N=5, log-normal vp, 8 shots, 3,000 steps,
                    128 receivers (stored every 30th step).

Every FP64 form (the plain row kernel, the matrix-free operator, each batched
FP64 kernel on the tensor or CUDA cores) must reproduce the reference within
1e-12 relative over the whole run (receiver traces and final displacement);
the FP32-operator forms within the 1e-4 seismogram budget.
"""
import numpy as np
import pytest

from conftest import load_golden
from helpers import rel
from tspeed_b200 import capi

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-4


def run_golden(g, precision="fp64", op="explicit", shots=None, monkeypatch=None, variant=None):
    """Runs the golden problem; shots: indices into the golden's sources
    (a source may repeat: the batched kernels need several shots). Returns
    (seismograms [S][nsteps][nr][2], {shot index in `shots`: final u})."""
    if monkeypatch is not None:
        if variant is None:
            monkeypatch.delenv("TSP_BATCHED_VARIANT", raising=False)
        else:
            monkeypatch.setenv("TSP_BATCHED_VARIANT", str(variant))
    src = g["src"]
    shots = list(range(len(src))) if shots is None else list(shots)
    n = int(g["nsteps"])
    with capi.Simulation.create(g["xy"], g["tri"], int(g["N"]), g["lam"], g["mu"], g["rho"],
                                [tuple(src[k]) for k in shots], g["rcv"], penalty=float(g["penalty"]),
                                precision=precision, op=op) as s:
        if variant is not None:
            assert s.kernel_variant == variant
        s.set_dt(float(g["dt"]))
        for i, k in enumerate(shots):
            f0, t0, amp, sdir = g["ricker"][k]
            s.set_ricker(i, f0, t0, amp, int(sdir), n)
        s.set_seismogram_capacity(n)
        s.first_step()
        s.run(n - 1)
        seis = s.seismograms(0, n)
        us = {i: s.u(i) for i in range(len(shots))}
        last = s.progress()
    assert last[0] == n
    assert abs(last[1] - float(g["last_time"])) <= 1e-12 * float(g["last_time"])
    return seis, us


def seis_err(g, seis, shots):
    every = int(g["seis_every"])
    ref = g["seis"][list(shots)]
    return rel(seis[:, ::every], ref)


# ---- configuration 1 in full (one shot) ----

@pytest.mark.parametrize("op", ["explicit", "matrix_free"])
def test_config1_full_fp64_single_shot(op):
    g = load_golden("g_config1_full")
    seis, us = run_golden(g, op=op, shots=[0])
    e_s, e_u = seis_err(g, seis, [0]), rel(us[0], g["u_final"][0])
    print(op, "config 1 vs reference: seismograms", e_s, "u", e_u)
    assert e_s < FP64_TOL and e_u < FP64_TOL


@pytest.mark.parametrize("variant", [5, 13, 6, 9, 10, 3, 2])
def test_config1_full_fp64_batched(variant, monkeypatch):
    """The batched FP64 kernels need several shots: the golden's source twice."""
    g = load_golden("g_config1_full")
    seis, us = run_golden(g, shots=[0, 0], monkeypatch=monkeypatch, variant=variant)
    for i in range(2):
        e_s = seis_err(g, seis[i:i + 1], [0])
        e_u = rel(us[i], g["u_final"][0])
        print("variant", variant, "shot", i, "seismograms", e_s, "u", e_u)
        assert e_s < FP64_TOL and e_u < FP64_TOL


@pytest.mark.parametrize("shots,variant", [([0], None), ([0, 0], 0), ([0, 0], 4), ([0, 0], 7), ([0, 0], 8)])
def test_config1_full_fp32_operator(shots, variant, monkeypatch):
    g = load_golden("g_config1_full")
    seis, _ = run_golden(g, precision="fp32", shots=shots, monkeypatch=monkeypatch, variant=variant)
    errs = [seis_err(g, seis[i:i + 1], [0]) for i in range(len(shots))]
    print("fp32 variant", variant, "config 1 seismogram errors vs reference", errs)
    assert max(errs) < MIXED_TOL


# ---- the 64-shot configuration's shape on its x0.2 sample (8 shots) ----

@pytest.mark.parametrize("variant", [5, 13, 6, 9, 10, 3, 2])
def test_config3_sample_fp64_batched(variant, monkeypatch):
    g = load_golden("g_config3_sample")
    seis, us = run_golden(g, monkeypatch=monkeypatch, variant=variant)
    e_s = seis_err(g, seis, range(len(g["src"])))
    e_u = max(rel(us[int(k)], g["u_final"][i]) for i, k in enumerate(g["u_shots"]))
    print("variant", variant, "config 3 sample vs reference: seismograms", e_s, "u", e_u)
    assert e_s < FP64_TOL and e_u < FP64_TOL


def test_config3_sample_fp64_plain_row_kernel():
    """The single-shot drop-in (row kernel), shot by shot: the final
    displacement within 1e-12, and the receiver traces within 1e-12 of the
    gather's scale. A deep source's wavefront has barely reached the surface
    after 3,000 steps (shot 0: its traces are 2e4 times weaker than the
    shallow shots'); rounding differences of summation order are set by the
    field's magnitude, not by those weak traces, so traces are measured
    against the norm of the whole 8-shot gather, as the batched tests do.
    A shot with strong arrivals (3) is also held to 1e-12 of its own traces."""
    g = load_golden("g_config3_sample")
    every = int(g["seis_every"])
    gather = np.linalg.norm(g["seis"])
    for i, k in enumerate(g["u_shots"]):
        seis, us = run_golden(g, shots=[int(k)])
        e_s = float(np.linalg.norm(seis[0, ::every] - g["seis"][int(k)]) / gather)
        e_u = rel(us[0], g["u_final"][i])
        print("shot", int(k), "seismograms (of the gather)", e_s, "u", e_u)
        assert e_s < FP64_TOL and e_u < FP64_TOL
    seis, _ = run_golden(g, shots=[3])
    e3 = seis_err(g, seis, [3])
    print("shot 3 seismograms", e3)
    assert e3 < FP64_TOL


@pytest.mark.parametrize("variant", [7, 8, 0, 4])
def test_config3_sample_fp32_operator(variant, monkeypatch):
    """FP32 operator / FP64 state: the warp-specialised CUDA-core kernel
    (7: 6 FMA warps per SM, 8: 8 FMA warps), the k-split CUDA-core kernel (0) and
    the tensor-core fixed-point kernel (4), against the reference's FP64 run."""
    g = load_golden("g_config3_sample")
    seis, _ = run_golden(g, precision="fp32", monkeypatch=monkeypatch, variant=variant)
    e_s = seis_err(g, seis, range(len(g["src"])))
    print("fp32 variant", variant, "config 3 sample seismogram error vs reference", e_s)
    assert e_s < MIXED_TOL
