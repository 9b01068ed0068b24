"""Engine features beyond parity: graphs, energy, checkpoint/resume, CFL
estimate, watchdog and error codes (GPU)."""
import numpy as np
import pytest

import tsp_oracle as O
from helpers import rel
from tspeed_b200 import capi
from tspeed_b200 import workloads as W

pytestmark = pytest.mark.gpu


def small(N=3, nx=6, ny=4, precision="fp64", nshots=1):
    m = W.jittered_rect(nx, ny, 100.0 * nx, 100.0 * ny, seed=5)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    shots = [(0.4 * m.Lx + 10 * k, 0.5 * m.Ly) for k in range(nshots)]
    s = capi.Simulation.create(m.xy, m.tri, N, lam, mu, rho, shots, W.surface_receivers(m, 3), penalty=10.0,
                               precision=precision)
    return m, (lam, mu, rho), s


def test_graph_run_equals_single_steps():
    _, _, a = small()
    _, _, b = small()
    for s in (a, b):
        s.set_dt(1e-4)
        s.set_ricker(0, 20.0, 0.05, -1.0, 1, 200)
        s.first_step()
    a.run(37)
    a.run(37)
    a.run(1)
    for _ in range(75):
        b.step()
    assert np.array_equal(a.u(), b.u())
    assert np.array_equal(a.seismograms(0, 76), b.seismograms(0, 76))
    assert a.progress() == b.progress()


def test_energy_conserved_without_force():
    m, mat, s = small(N=4)
    rng = np.random.default_rng(3)
    u0 = 1e-3 * rng.standard_normal(2 * m.ne * s.Np)
    lmax = s.estimate_lmax(200)
    dt = 0.5 * 2 / np.sqrt(lmax)
    s.set_dt(dt)
    s.set_initial(0, u0, None)
    s.enable_energy(True)
    s.first_step()
    s.run(299)
    E = s.energy(0, 300)
    assert np.all(np.isfinite(E)) and E[0] > 0
    assert np.max(np.abs(E - E[0])) / E[0] < 1e-10


def test_lmax_matches_dense_eigenvalue():
    m, (lam, mu, rho), s = small(N=2, nx=4, ny=3)
    est = s.estimate_lmax(2000)
    sp = O.make_space(2)
    tri = m.tri.astype(np.int64)
    geo = O.geometry(m.xy, tri)
    nb, ned = O.neighbours(tri)
    row_ptr, cols, blocks, minv = O.assemble(sp, geo, nb, ned, lam, mu, rho, 10.0)
    n = 2 * m.ne * sp.Np
    Bd = np.stack([O.apply_B(row_ptr, cols, blocks, e, m.ne, sp.Np) for e in np.eye(n)], 1)
    mv = np.concatenate([np.repeat(minv, sp.Np)] * 2)
    true = np.max(np.linalg.eigvals(mv[:, None] * Bd).real)
    assert abs(est - true) / true < 1e-6


def test_checkpoint_resume_bit_exact():
    _, _, a = small(nshots=2)
    _, _, b = small(nshots=2)
    for s in (a, b):
        s.set_dt(1e-4)
        for k in range(2):
            s.set_ricker(k, 20.0, 0.05, -1.0, 1, 100)
    a.first_step()
    a.run(20)
    up, uc, k, t = a.get_state()
    b.set_state(up, uc, k, t)
    a.run(30)
    b.run(30)
    assert np.array_equal(a.u(0), b.u(0)) and np.array_equal(a.u(1), b.u(1))
    assert a.progress() == b.progress()


def test_nonfinite_watchdog():
    m, _, s = small()
    s.set_dt(1e-4)
    s.first_step()
    assert s.check_finite()
    up, uc, k, t = s.get_state()
    uc[0, 5] = np.nan
    s.set_state(up, uc, k, t)
    assert not s.check_finite()


def test_error_codes():
    m, (lam, mu, rho), s = small()
    with pytest.raises(capi.TspError) as e:
        s.step()
    assert e.value.code == -4  # step before first_step
    with pytest.raises(capi.TspError) as e:
        s.first_step()
    assert e.value.code == -4  # no dt
    with pytest.raises(capi.TspError) as e:
        capi.Simulation.create(m.xy, m.tri, 3, lam, mu, rho, [(-50.0, 10.0)], [])
    assert e.value.code == -5  # source outside the mesh
    cw = m.tri.copy()
    cw[0] = cw[0][::-1]
    with pytest.raises(capi.TspError) as e:
        capi.Simulation.create(m.xy, cw, 3, lam, mu, rho, [(250.0, 200.0)], [])
    assert e.value.code == -6  # clockwise triangle
    with pytest.raises(capi.TspError):
        s.seismograms(0, 10 ** 9)


def test_autotuner_choice_and_override(monkeypatch):
    """The batched FP32 step is chosen by the autotuner at creation (one of
    the CUDA-core variants 0/1/2 or the tensor-core variant 4); the chosen
    kernel stays within the 1e-4 budget of FP64; TSP_BATCHED_VARIANT forces
    a variant."""
    m = W.jittered_rect(8, 5, 800.0, 500.0, seed=31)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    rng = np.random.default_rng(4)
    shots = [(40 + 720 * rng.random(), 40 + 420 * rng.random()) for _ in range(70)]
    rcv = W.surface_receivers(m, 4)
    n = 80
    seis = {}
    monkeypatch.delenv("TSP_BATCHED_VARIANT", raising=False)
    dt = None
    for prec in ("fp64", "fp32"):
        with capi.Simulation.create(m.xy, m.tri, 5, lam, mu, rho, shots, rcv, penalty=10.0, precision=prec) as s:
            if prec == "fp32":
                assert s.kernel_variant in (7, 8, 0, 1, 2, 4)
            if dt is None:
                dt = 0.4 * 2 / np.sqrt(s.estimate_lmax(60))
            s.set_dt(dt)
            for k in range(70):
                s.set_ricker(k, 25.0, 0.04, -1.0, 1, n)
            s.first_step()
            s.run(n - 1)
            seis[prec] = s.seismograms(0, n)
    err = np.linalg.norm(seis["fp32"] - seis["fp64"]) / np.linalg.norm(seis["fp64"])
    assert err < 1e-4, err
    monkeypatch.setenv("TSP_BATCHED_VARIANT", "2")
    with capi.Simulation.create(m.xy, m.tri, 5, lam, mu, rho, shots, rcv, penalty=10.0, precision="fp32") as s:
        assert s.kernel_variant == 2


def test_fp64_autotuner_choice_and_override(monkeypatch):
    """FP64 with several shots: the autotuner times the FP64 kernels (5, 6
    warp-specialised DMMA; 3 single-role DMMA; 2 CUDA cores) and keeps one;
    TSP_BATCHED_VARIANT forces one; every choice gives the same results to
    rounding."""
    m = W.jittered_rect(8, 5, 800.0, 500.0, seed=33)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    shots = [(100.0 + 9 * k, 120.0 + 3 * (k % 50)) for k in range(40)]
    rcv = W.surface_receivers(m, 4)
    n = 40
    out = {}
    for forced in (None, "5", "13", "6", "9", "10", "3", "2"):
        if forced is None:
            monkeypatch.delenv("TSP_BATCHED_VARIANT", raising=False)
        else:
            monkeypatch.setenv("TSP_BATCHED_VARIANT", forced)
        with capi.Simulation.create(m.xy, m.tri, 4, lam, mu, rho, shots, rcv, penalty=10.0) as s:
            v = s.kernel_variant
            assert v in (5, 13, 6, 9, 10, 3, 2) if forced is None else v == int(forced)
            s.set_dt(2e-4)
            for k in range(len(shots)):
                s.set_ricker(k, 25.0, 0.04, -1.0, 1, n)
            s.first_step()
            s.run(n - 1)
            out[forced] = s.seismograms(0, n)
    for forced in ("5", "6", "9", "10", "3"):
        assert np.linalg.norm(out[forced] - out["2"]) <= 1e-13 * np.linalg.norm(out["2"])
    assert np.linalg.norm(out[None] - out["2"]) <= 1e-13 * np.linalg.norm(out["2"])


@pytest.mark.parametrize("precision,op,nshots,variant", [
    ("fp64", "explicit", 1, None), ("fp64", "matrix_free", 1, None), ("fp64", "explicit", 3, "5"),
    ("fp64", "explicit", 3, "6"), ("fp64", "explicit", 3, "9"), ("fp64", "explicit", 3, "10"),
    ("fp64", "explicit", 3, "3"), ("fp64", "explicit", 3, "2"),
    ("fp32", "explicit", 1, None), ("fp32", "explicit", 3, "0"), ("fp32", "explicit", 3, "4"),
    ("fp32", "explicit", 3, "7"), ("fp32", "explicit", 3, "8")])
def test_unstable_dt_is_reported_as_nonfinite(precision, op, nshots, variant, monkeypatch):
    """A time step of 3x the CFL limit is an ordinary numerical blow-up: the
    state overflows to Inf/NaN within a few hundred steps. Every step kernel
    raises the device's non-finite flag, tsp_run_timed returns
    TSP_ERR_NONFINITE (-7) and the watchdog reports it; new initial values
    clear it and a stable run is clean again."""
    if variant is None:
        monkeypatch.delenv("TSP_BATCHED_VARIANT", raising=False)
    else:
        monkeypatch.setenv("TSP_BATCHED_VARIANT", variant)
    m = W.jittered_rect(5, 4, 500.0, 400.0, seed=12)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    shots = [(120.0 + 100 * k, 150.0 + 50 * k) for k in range(nshots)]
    rng = np.random.default_rng(6)
    with capi.Simulation.create(m.xy, m.tri, 3, lam, mu, rho, shots, W.surface_receivers(m, 2), penalty=10.0,
                                precision=precision, op=op) as s:
        dt_cfl = 2 / np.sqrt(s.estimate_lmax(200))
        u0 = [1e-3 * rng.standard_normal(2 * s.ne * s.Np) for _ in range(nshots)]
        s.set_dt(3 * dt_cfl)
        for k in range(nshots):
            s.set_initial(k, u0[k], None)
        s.first_step()
        with pytest.raises(capi.TspError) as e:
            s.run_timed(600)
        assert e.value.code == -7
        assert not s.check_finite()
        s.set_dt(0.4 * dt_cfl)
        for k in range(nshots):
            s.set_initial(k, u0[k], None)
        s.first_step()
        s.run_timed(100)
        assert s.check_finite()


def test_run_pieces_match_single_steps():
    """tsp_run replays pieces of at most 256 steps (and the powers of two of
    the remainder), so runs of many different lengths share a bounded set of
    graphs: they give exactly the state and receiver samples of single
    steps."""
    m = W.jittered_rect(4, 3, 400.0, 300.0, seed=4)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    mk = lambda: capi.Simulation.create(m.xy, m.tri, 2, lam, mu, rho, [(150.0, 140.0)],  # noqa: E731
                                        W.surface_receivers(m, 2), penalty=10.0)
    with mk() as a, mk() as b:
        for s in (a, b):
            s.set_dt(2e-4)
            s.set_ricker(0, 20.0, 0.05, -1.0, 1, 2000)
            s.set_seismogram_capacity(2000)
            s.first_step()
        total = 1
        for n in (1, 2, 3, 7, 255, 256, 257, 300, 511, 13):
            a.run(n)
            total += n
        for _ in range(total - 1):
            b.step()
        assert a.progress() == b.progress()
        assert np.array_equal(a.u(), b.u())
        assert np.array_equal(a.seismograms(0, total), b.seismograms(0, total))


def test_u_all_matches_per_shot_reads():
    """tsp_get_u_all (device transpose, chunked read-back) returns exactly the
    per-shot tsp_get_u vectors."""
    m = W.jittered_rect(6, 4, 600.0, 400.0, seed=8)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    shots = [(100.0 + 40 * k, 120.0 + 20 * (k % 5)) for k in range(11)]
    with capi.Simulation.create(m.xy, m.tri, 3, lam, mu, rho, shots, W.surface_receivers(m, 2), penalty=10.0,
                                precision="fp64") as s:
        s.set_dt(1e-4)
        for k in range(len(shots)):
            s.set_ricker(k, 20.0, 0.05, -1.0, k % 2, 40)
        s.first_step()
        s.run(20)
        allu = s.u_all()
        for k in range(len(shots)):
            assert np.array_equal(allu[k], s.u(k))


def test_pooled_allocations_are_reused_and_released():
    """Handles created one after the other draw on the library's cached
    device pool; results do not depend on reuse, and the cache can be
    returned to the driver."""
    m = W.jittered_rect(6, 4, 600.0, 400.0, seed=81)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    rcv = W.surface_receivers(m, 3)
    out = []
    for _ in range(3):
        with capi.Simulation.create(m.xy, m.tri, 3, lam, mu, rho, [(300.0, 200.0)], rcv, penalty=10.0) as s:
            s.set_dt(2e-4)
            s.set_ricker(0, 25.0, 0.04, -1.0, 1, 60)
            s.first_step()
            s.run(59)
            out.append(s.seismograms(0, 60))
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])
    capi.release_cached_memory(0)
    with capi.Simulation.create(m.xy, m.tri, 3, lam, mu, rho, [(300.0, 200.0)], rcv, penalty=10.0) as s:
        s.set_dt(2e-4)
        s.set_ricker(0, 25.0, 0.04, -1.0, 1, 60)
        s.first_step()
        s.run(59)
        assert np.array_equal(s.seismograms(0, 60), out[0])


def test_fp64_tensor_peak_probe():
    """The FP64 tensor-core throughput probe behind the benchmark's FP64
    roofline returns a plausible B200 rate (nominal 40 TFLOP/s)."""
    v = capi.fp64_tensor_peak(0)
    print("FP64 tensor peak", v)
    assert 10.0 < v < 60.0


def test_bounded_wait_gives_up_and_device_stays_usable():
    """Failure detection on the device without a fault: a wait on a barrier
    phase that nothing completes gives up after its limit (about a second),
    raises the abort flag, the kernel ends normally, and a simulation runs
    on the same device right after."""
    completed, aborted = capi.selftest_bounded_wait(0)
    assert completed == 0 and aborted == 1
    m = W.jittered_rect(3, 2, 300.0, 200.0, seed=5)
    lam, mu, rho = W.lame(np.full(m.ne, 3000.0), np.full(m.ne, 1732.0), np.full(m.ne, 2200.0))
    with capi.Simulation.create(m.xy, m.tri, 2, lam, mu, rho, [(150.0, 100.0), (80.0, 60.0)], [],
                                penalty=10.0) as s:
        s.set_dt(1e-4)
        s.set_ricker(0, 20.0, 0.05, -1.0, 1, 10)
        s.set_ricker(1, 20.0, 0.05, -1.0, 1, 10)
        s.first_step()
        s.run(9)
        assert s.check_finite()
