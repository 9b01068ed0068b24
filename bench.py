"""Benchmark of the leap-frog path: DOF-steps/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the 64-shot batched configuration -- 200x100 jittered
squares (40,000 triangles), Dubiner N=5 (1.68 M DOFs per shot), per-element
log-normal vp, 64 Ricker shots at seeded interior points, 128 surface
receivers, dt = 0.4 x CFL from a device power iteration -- in the mixed
form: FP32 operator blocks, FP32 products and sums, FP64 state, recurrence,
sources and receivers, the batched kernel chosen by the library's autotuner
(its seismogram error against the reference's own FP64 run is reported;
--precision fp64 selects exact FP64 on the FP64 tensor cores). One bench
"step" is one leap-frog step of all 64 shots. Under torchrun each rank runs its own 64 shots (weak
scaling, no collective in the data path); the timed region is bracketed by a
barrier and a device synchronise, timed with CUDA events on the engine's
stream, max over ranks.

Also reported: the plain FP64 single-shot drop-in on the same mesh, the
other batched form (exact FP64, or the FP32 operator), the seismogram error
of each form against FP64 from the CUDA-core FP64 kernel over the full step
count and against the reference's own run (a committed golden of 8 shots
over 3,000 steps), the energy drift of each form, an end-to-end number
through the public C-ABI with host buffers, the roofline of the step kernel
and the reference's CPU path on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from tspeed_b200 import capi  # noqa: E402
from tspeed_b200 import workloads as W  # noqa: E402
from tspeed_b200.shard import max_over_ranks, shots_for_rank  # noqa: E402

METRIC = "DOF-steps/s on 1 B200: mixed/batched vs plain FP64, at seismogram err <=1e-4"
UNIT = "DOF-steps/s"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "tsp_ref_run")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def captured_traffic(kernel, ne, nshots):
    """DRAM bytes per launch of `kernel` from the committed ncu record
    (profiles/traffic.json), scaled to ne element rows; None if not recorded
    for this shot count."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            rec = json.load(f)[kernel]
    except Exception:
        return None
    if rec["shots"] != nshots:
        return None
    return rec["bytes"] * ne / rec["elements"]


# Batched FP32 step kernels by variant (tsp_get_kernel_variant), for 2Np = 42.
KERNELS = {0: "k_step_batched32k<42>", 1: "k_step_batched32p<42,64,4>", 2: "k_step_batched32<42>",
           4: "k_step_batched_fx<42>", 7: "k_step_batched32w<42,3,3,2,1,6>", 8: "k_step_batched32w<42,4,2,2,1,3>"}


def bytes_per_step(ne, Np, nnzb, nshots, precision):
    """Algorithmic HBM bytes of one step: every block once, the state read
    (u^k, u^{k-1}) and written (u^{k+1}) once per shot, minv once. The
    tensor-core form ("fx") stores each operator entry as three BF16
    fixed-point slices (6 bytes)."""
    R = 2 * Np
    bblk = {"fp64": 8, "fp32": 4, "bf16": 2, "fx": 6}[precision]
    extra = nnzb * 4 if precision == "bf16" else 0
    return nnzb * R * R * bblk + extra + nshots * 2 * ne * Np * 24 + ne * 8


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        self.index = vis.split(",")[local_rank].strip() if vis else str(local_rank)
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.index, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_problem(args, rank, world):
    """One global list of nshots x world shots; this rank takes its slice
    (weak scaling: nshots per GPU)."""
    p = W.config(3, scale=args.scale, nshots=args.nshots * world, shot_seed=1000)
    p.sources = [p.sources[i] for i in shots_for_rank(len(p.sources), rank, world)]
    return p


def estimate_dt(sim, cfl_fraction=0.4, iters=60):
    lmax = sim.estimate_lmax(iters)
    return cfl_fraction * 2.0 / math.sqrt(lmax), lmax


# FP64 batched step kernels at 2Np = 42 by variant (tsp_get_kernel_variant):
# 5 warp-specialised DMMA, two consumer groups of 8 warps with a 3-stage ring
# each; 6 the same kernel with one group of 16 warps and a 6-stage ring; 9 and
# 10 the same kernel with the epilogue in update warps (two groups, 2-stage
# rings / one group, 5-stage ring); 13 as 5 with u^{k-1} requested before
# the products under a warpgroup register split; 3 the single-role DMMA
# kernel; 2 the CUDA-core kernel.
D64_KERNELS = {5: "k_step_batched64w<42,3,2,1,8,1,0,0,0>", 6: "k_step_batched64w<42,6,1,1,8,2,1,0,0>",
               9: "k_step_batched64w<42,2,2,1,8,1,2,1,0>", 10: "k_step_batched64w<42,5,1,1,8,2,2,2,0>",
               13: "k_step_batched64w<42,3,2,1,8,1,3,0,112>",
               3: "k_step_batched64d<42>", 2: "k_step_batched<42,double>"}

# Nominal dense FP64 tensor-core rate of a B200 (DMMA); MEASURED_PEAKS.json
# holds no FP64 figure.
FP64_TENSOR_NOMINAL_TFLOPS = 40.0


_FP64_PEAK = {}


def fp64_tensor_peak(device):
    """FP64 tensor-core rate measured on this GPU (register-only DMMA loop in
    the library, tsp_fp64_tensor_peak); MEASURED_PEAKS.json has no FP64 figure."""
    if device not in _FP64_PEAK:
        try:
            _FP64_PEAK[device] = capi.fp64_tensor_peak(device)
        except Exception:
            _FP64_PEAK[device] = None
    return _FP64_PEAK[device]


def fp64_tensor_roofline(nnzb, Np, nshots, ms_step, kernel, device=0):
    """Roofline of the FP64 batched step against the FP64 tensor cores:
    algorithmic flops 2 * nnzb * (2Np)^2 * shots per step."""
    flops = 2.0 * nnzb * (2 * Np) ** 2 * nshots
    ach = flops / (ms_step / 1e3) / 1e12
    meas = fp64_tensor_peak(device)
    peak = FP64_TENSOR_NOMINAL_TFLOPS
    return {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
            "kernel": kernel,
            "peak_source": "nominal B200 FP64 tensor rate (no driver-measured FP64 figure exists)",
            "peak_measured": meas, "frac_of_measured": (ach / meas) if meas else None,
            "peak_measured_source": "register-only DMMA loop on this GPU (tsp_fp64_tensor_peak)",
            "algorithmic_flops_per_step": flops}


# FP32 CUDA-core peak of a B200: 148 SMs x 128 FP32 lanes x 2 flops x 1.965 GHz.
FP32_SIMT_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def fp32_pipe_roofline(nnzb, Np, nshots, ms_step, kernel):
    """The FP32-operator CUDA-core step against the FP32 pipe: algorithmic
    flops 2 * nnzb * (2Np)^2 * shots per step."""
    flops = 2.0 * nnzb * (2 * Np) ** 2 * nshots
    ach = flops / (ms_step / 1e3) / 1e12
    return {"bound": "fp32 pipe", "achieved": ach, "peak": FP32_SIMT_NOMINAL_TFLOPS, "unit": "TFLOP/s",
            "frac": ach / FP32_SIMT_NOMINAL_TFLOPS, "kernel": kernel,
            "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 flops x 1.965 GHz",
            "algorithmic_flops_per_step": flops}


def graph_pieces(n, chunk=256):
    """Graph replays tsp_run issues for n steps (pieces of `chunk` steps and
    the powers of two of the remainder); each ends with one k_advance."""
    pieces = 0
    while n > 0:
        ln = chunk if n >= chunk else 1 << (n.bit_length() - 1)
        n -= ln
        pieces += 1
    return pieces


def prepare(sim, prob, dt, nsteps):
    sim.set_dt(dt)
    for k, s in enumerate(prob.sources):
        sim.set_ricker(k, s.f0, s.t0, s.amp, s.direction, nsteps)


def cpu_reference_sample(nprocs=1, nsteps=20, scale=0.5, timeout=900):
    """The reference's own CPU path (oracle/_ref, compiled from its sources)
    on a bounded sample of the workload: the same configuration shrunk to
    `scale` per axis (x0.5: 10,000 triangles, whose operator, like the full
    configuration's, is far larger than the host caches: the per-DOF rate
    matches the full 40,000-triangle mesh's, while a x0.2 sample fits in cache
    and runs 1.5x faster), one shot per process, `nprocs` processes in
    parallel (the reference is single-threaded), `nsteps` steps each; the
    reference's set-up (O(ne^2) neighbour search, assembly) is not timed.
    Returns (DOF-steps/s, sample text)."""
    if not os.path.exists(REF_BIN):
        return None, "reference binary missing"
    p = W.config(3, scale=scale, nshots=max(1, nprocs))
    ne, Np = p.mesh.ne, p.Np
    with tempfile.TemporaryDirectory() as tmp:
        msh, rcv, mat = (os.path.join(tmp, n) for n in ("m.msh", "m.rcv", "m.mat"))
        W.write_gmsh(msh, p.mesh)
        W.write_rcv(rcv, p.receivers)
        np.stack([p.lam, p.mu, p.rho], 1).astype(np.float64).tofile(mat)
        procs = []
        for k in range(nprocs):
            s = p.sources[k]
            cmd = [REF_BIN, "--mesh", msh, "--N", str(p.N), "--mat", mat, "--rcv", rcv, "--out",
                   os.path.join(tmp, f"o{k}"), "--dt", "1e-4", "--nsteps", str(nsteps), "--src", repr(s.x),
                   repr(s.y), "--ricker", repr(s.f0), repr(s.t0), repr(s.amp), "--penalty", repr(p.penalty)]
            procs.append(subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
        loops = []
        for pr in procs:
            out, err = pr.communicate(timeout=timeout)
            if pr.returncode != 0:
                return None, "reference run failed: " + err.strip()[-200:]
            loops.append(json.loads(out.strip().splitlines()[-1])["loop_s"])
    dofs = 2 * ne * Np
    value = nprocs * dofs * nsteps / max(loops)
    sample = (f"{p.mesh.ne} triangles (config shrunk x{scale} per axis), N={p.N}, {nsteps} steps, "
              f"{nprocs} single-threaded process(es), one shot each; loop time only")
    return value, sample


GOLDEN_C3 = os.path.join(ROOT, "tests", "golden", "g_config3_sample.npz")


def run_on_golden(g, precision, shots, variant=None):
    """Runs a golden problem (committed fixture) with the given shots
    (indices into its sources); returns the seismograms sampled like the
    golden's, [S][nsteps / every][nr][2]."""
    old = os.environ.get("TSP_BATCHED_VARIANT")
    if variant is None:
        os.environ.pop("TSP_BATCHED_VARIANT", None)
    else:
        os.environ["TSP_BATCHED_VARIANT"] = str(variant)
    try:
        n = int(g["nsteps"])
        with capi.Simulation.create(g["xy"], g["tri"], int(g["N"]), g["lam"], g["mu"], g["rho"],
                                    [tuple(g["src"][k]) for k in shots], g["rcv"], penalty=float(g["penalty"]),
                                    precision=precision) as s:
            v = s.kernel_variant
            s.set_dt(float(g["dt"]))
            for i, k in enumerate(shots):
                f0, t0, amp, sdir = g["ricker"][k]
                s.set_ricker(i, f0, t0, amp, int(sdir), n)
            s.set_seismogram_capacity(n)
            s.first_step()
            s.run(n - 1)
            return s.seismograms(0, n)[:, ::int(g["seis_every"])], v
    finally:
        if old is None:
            os.environ.pop("TSP_BATCHED_VARIANT", None)
        else:
            os.environ["TSP_BATCHED_VARIANT"] = old


def errors_vs_reference():
    """Seismogram relative L2 error of each form against the reference's own
    FP64 run of the 64-shot configuration's shape on its x0.2 sample
    (tests/golden/g_config3_sample.npz: 1,600 triangles, N=5, log-normal vp,
    8 shots, 3,000 steps, 128 receivers; made by the reference's stepping
    loop compiled from its sources)."""
    if not os.path.exists(GOLDEN_C3):
        return None
    g = np.load(GOLDEN_C3)
    ns = len(g["src"])
    ref = g["seis"]
    out = {"golden": "tests/golden/g_config3_sample.npz", "shots": ns, "steps": int(g["nsteps"]),
           "receivers": int(len(g["rcv"])), "forms": {}}

    def err(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    for name, prec, var in (("batched_fp64", "fp64", None), ("batched_fp32_operator", "fp32", None),
                            ("batched_fp32_cuda_core", "fp32", 0)):
        seis, v = run_on_golden(g, prec, list(range(ns)), var)
        out["forms"][name] = {"err": err(seis, ref), "kernel_variant": v}
    # The single-shot drop-in runs shot by shot; a deep source's traces are
    # orders of magnitude weaker than the shallow ones' (its wavefront has
    # barely reached the surface), so each shot's trace error is measured
    # against the whole gather's norm, as the batched forms' errors are.
    errs = []
    gather = float(np.linalg.norm(ref))
    for k in (0, ns - 1):
        seis, _ = run_on_golden(g, "fp64", [k])
        errs.append(float(np.linalg.norm(seis[0] - ref[k])) / gather)
    out["forms"]["plain_fp64_single_shot"] = {"err": max(errs), "shots_checked": [0, ns - 1],
                                              "normalised_by": "norm of the 8-shot gather"}
    return out


def energy_drift(prob, dt, nsteps=500):
    """Discrete-energy drift max_k |E^k - E^0| / E^0 of each timed form, with
    the sources off and a seeded initial field per shot (a Gaussian pulse of
    the vertical displacement, 150 m wide, at the shot's source point,
    projected on the device), over nsteps steps of the configuration's mesh."""
    pts = capi.quadrature_points(prob.N, prob.mesh.xy, prob.mesh.tri)
    out = {"steps": nsteps, "initial_field": "Gaussian pulse of u_y (sigma 150 m) at each source point",
           "forms": {}}
    for name, prec, nsh in (("batched_fp64", "fp64", prob.nshots), ("batched_fp32_operator", "fp32", prob.nshots),
                            ("plain_fp64_single_shot", "fp64", 1), ("plain_fp32_operator_single_shot", "fp32", 1)):
        with capi.Simulation.create(prob.mesh.xy, prob.mesh.tri, prob.N, prob.lam, prob.mu, prob.rho,
                                    [(sr.x, sr.y) for sr in prob.sources[:nsh]], [], penalty=prob.penalty,
                                    precision=prec) as s:
            s.set_dt(dt)
            for k in range(nsh):
                sr = prob.sources[k]
                r2 = (pts[..., 0] - sr.x) ** 2 + (pts[..., 1] - sr.y) ** 2
                vals = np.zeros(pts.shape)
                vals[..., 1] = 1e-3 * np.exp(-r2 / (2 * 150.0 ** 2))
                s.set_initial_values(k, vals, None)
            s.enable_energy(True)
            s.first_step()
            s.run(nsteps - 1)
            E = s.energy(0, nsteps)
            v = s.kernel_variant
        out["forms"][name] = {"drift": float(np.max(np.abs(E - E[0])) / E[0]), "kernel_variant": v}
    return out


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # One single-threaded reference process per host core, capped so that
    # the processes' operators (1.4 GB each at the x0.5 sample) stay well
    # inside host memory.
    ncores = min(os.cpu_count() or 1, 32)
    nsteps = max(10, args.steps)
    v, sample = cpu_reference_sample(nprocs=ncores, nsteps=nsteps, scale=args.ref_scale)
    cfg = config_dict(args, None)
    # What this arm actually ran (a bounded sample of the configuration, per
    # DOF-step), so that its config does not read as the full configuration.
    cfg["reference_sample"] = sample
    if v is None:
        print(json.dumps({"impl": "reference", "unavailable": sample}))
        return 0
    line = {"impl": "reference", "sample": sample, "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ncores, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def mesh_batch_forms(args):
    """Config 4: 256 independent jittered meshes (500..20,000 triangles,
    N in 3..8, own material, own Ricker source, per-mesh dt = 0.4 x CFL),
    advanced together by one graph per step chunk. Forms: FP32 explicit
    blocks vs the FP64 matrix-free operator (explicit FP64 blocks of this
    batch, ~273 GB, do not fit in HBM). Seismogram error of the FP32 form
    against FP64 over --accuracy-steps (default 400)."""
    probs = W.mesh_batch(nmesh=256, scale=args.scale)
    K, Wm = args.steps, max(3, args.warmup)
    nacc = 400 if args.accuracy_steps < 0 else args.accuracy_steps
    total = max(Wm + 2 * K + 1, nacc)
    out = {"metric": "DOF-steps/s, uneven multi-mesh batch", "unit": UNIT, "workload": "config4",
           "meshes": len(probs), "triangles": int(sum(p.mesh.ne for p in probs)),
           "dofs": int(sum(p.dofs_per_shot for p in probs)), "steps": K, "warmup": Wm, "forms": {}}
    dt = None
    seis = {}
    for form in ("matrix_free-fp64", "explicit-fp32"):
        op, prec = form.split("-")
        t0 = time.perf_counter()
        with capi.Batch(probs, precision=prec, op=op) as b:
            setup = time.perf_counter() - t0
            if dt is None:
                dt = 0.4 * 2 / np.sqrt(b.estimate_lmax(60))
            b.set_dt(dt)
            b.set_ricker(total)
            b.set_seismogram_capacity(total)
            b.first_step()
            b.run(Wm)
            b.run_timed(K)
            ms = b.run_timed(K)
            done = 1 + Wm + 2 * K
            if total > done:
                b.run(total - done)
            seis[form] = [b.seismograms(m, 0, total) for m in range(len(probs))]
            dofs = b.total_dofs
        out["forms"][form] = {"ms_per_step": ms / K, "value": dofs * K / (ms / 1e3), "setup_s": setup}
    ref = np.concatenate([x.ravel() for x in seis["matrix_free-fp64"]])
    lo = np.concatenate([x.ravel() for x in seis["explicit-fp32"]])
    out["forms"]["explicit-fp32"]["seismogram_rel_l2_vs_fp64"] = float(np.linalg.norm(lo - ref) / np.linalg.norm(ref))
    out["accuracy_steps"] = total
    print(json.dumps(out))
    return 0


def single_shot_forms(args):
    """Single-shot configurations (2: 160k triangles N=6; 5: 655k triangles
    N=6) with several operator forms on the same inputs: time per step,
    DOF-steps/s, HBM roofline of the explicit forms, and the seismogram error
    of every form against explicit FP64 over the timed steps."""
    k = int(args.workload[-1])
    prob = W.config(k, scale=args.scale)
    K, Wm = args.steps, max(3, args.warmup)
    hbm, peak_kind = peaks()
    out = {"metric": "DOF-steps/s per operator form (single shot)", "unit": UNIT, "workload": args.workload,
           "mesh_triangles": prob.mesh.ne, "N": prob.N, "dofs": prob.dofs_per_shot, "steps": K, "warmup": Wm,
           "forms": {}}
    dt = None
    seis = {}
    for form in args.forms.split(","):
        op, prec = form.split("-")
        with capi.Simulation.from_problem(prob, precision=prec, op=op) as s:
            if dt is None:
                dt, _ = estimate_dt(s)
            total = Wm + 2 * K + 1
            prepare(s, prob, dt, total)
            s.set_seismogram_capacity(total)
            s.first_step()
            s.run(Wm)
            s.run_timed(K)
            ms = s.run_timed(K)
            seis[form] = s.seismograms(0, total)
            nnzb = s.nnzb
        d = {"ms_per_step": ms / K, "value": prob.dofs_per_shot * K / (ms / 1e3)}
        if op == "explicit":
            algo = bytes_per_step(prob.mesh.ne, prob.Np, nnzb, 1, prec)
            d["roofline_frac"] = algo / (ms / K / 1e3) / 1e9 / hbm
            d["algorithmic_bytes_per_step"] = algo
        out["forms"][form] = d
    ref = seis.get("explicit-fp64")
    if ref is not None and np.linalg.norm(ref) > 0:
        for form, sg in seis.items():
            out["forms"][form]["seismogram_rel_l2_vs_explicit_fp64"] = float(np.linalg.norm(sg - ref) / np.linalg.norm(ref))
    out["dt"] = dt
    out["peak_gbs"] = hbm
    out["peak_source"] = peak_kind
    print(json.dumps(out))
    return 0


def config_dict(args, prob):
    form = ("FP64 operator and state on the FP64 tensor cores (exact FP64)" if args.precision == "fp64" else
            "FP32 operator / FP64 state, batched kernel chosen by the autotuner" if args.precision == "fp32" else
            "BF16 operator / FP64 state")
    d = {"workload": "64-shot batched DG leap-frog: 200x100 jittered squares (40,000 triangles), Dubiner N=5, "
                     "log-normal vp, 128 receivers, " + form,
         "mesh_triangles": prob.mesh.ne if prob else 40000, "N": 5, "shots_per_gpu": args.nshots,
         "precision": args.precision, "dofs_per_shot": prob.dofs_per_shot if prob else 1680000,
         "l2": "inputs larger than L2 (state 0.86 GB per level, blocks %s GB)" %
               {"fp64": "2.25", "fp32": "1.1", "bf16": "0.56"}[args.precision],
         "parallelism": f"shots x{args.gpus}"}
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp64", "fp32", "bf16"])
    ap.add_argument("--nshots", type=int, default=64)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--accuracy-steps", type=int, default=-1, help="steps of the FP64 comparison (-1: config's)")
    ap.add_argument("--ref-scale", type=float, default=0.5,
                    help="per-axis scale of the sample the reference's CPU path runs (--impl reference)")
    ap.add_argument("--no-extras", action="store_true", help="skip plain-FP64, accuracy, e2e and CPU legs")
    ap.add_argument("--workload", default="config3", choices=["config3", "config2", "config4", "config5"],
                    help="config3: the 64-shot headline; config2/config5: single-shot forms side by side")
    ap.add_argument("--forms", default="explicit-fp64,explicit-fp32,matrix_free-fp64")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "config4":
        return mesh_batch_forms(args)
    if args.workload != "config3":
        return single_shot_forms(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local_rank))
        dist = tdist

    prob = make_problem(args, rank, world)
    K, Wm = args.steps, max(3, args.warmup)
    sim = capi.Simulation.from_problem(prob, precision=args.precision, device=local_rank)
    variant = sim.kernel_variant if (prob.nshots > 1 and args.precision == "fp32") else None
    variant64 = sim.kernel_variant if (prob.nshots > 1 and args.precision == "fp64") else None
    dt, lmax = estimate_dt(sim)
    prepare(sim, prob, dt, K + Wm + 2)
    sim.set_seismogram_capacity(K + Wm + 2)
    sim.first_step()
    sim.run(Wm)
    sim.run_timed(K)  # instantiate the K-step graph outside the timed region
    sampler = ClockSampler(local_rank)
    if dist:
        import torch
        dist.barrier()
        torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.4)
    ms = sim.run_timed(K)
    clocks = sampler.stop()
    if dist:
        ms = max_over_ranks(ms, dist, device=f"cuda:{local_rank}")
        dist.barrier()
    dofs = prob.dofs_per_shot
    value = world * prob.nshots * dofs * K / (ms / 1e3)
    ms_step = ms / K
    hbm, peak_kind = peaks()
    form = "fx" if variant == 4 else args.precision
    algo = bytes_per_step(prob.mesh.ne, prob.Np, sim.nnzb, prob.nshots, form)
    achieved = algo / (ms_step / 1e3) / 1e9
    kernel = (KERNELS.get(variant, "batched") if variant is not None else
              "k_step_rows<42>" if prob.nshots == 1 else
              D64_KERNELS.get(variant64, "batched") if args.precision == "fp64" else "k_step_batched<42>")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": Wm,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("bf16x3 fixed-point operator, f64 state" if form == "fx" else
                      "f32 operator (FP32 products and sums), f64 state" if args.precision == "fp32" else
                      "bf16 operator, f64 state" if args.precision == "bf16" else "f64"), "data": "synthetic",
            "config": config_dict(args, prob), "dt": dt, "lmax": lmax,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": (captured_traffic(kernel, prob.mesh.ne, prob.nshots)
                                     if variant is not None else
                                     captured_traffic("k_step_rows<42,double>", prob.mesh.ne, prob.nshots)
                                     if prob.nshots == 1 and args.precision == "fp64" else None)
                         if prob.N == 5 else None,
                         "traffic_source": "ncu capture (profiles/traffic.json) scaled by element rows",
                         "kernel": kernel, "kernel_variant": variant,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_step": algo},
            "gpu_launches": K + graph_pieces(K), "clocks": clocks}
    if args.precision == "fp64" and prob.nshots > 1:
        # The FP64 batched step is bound by the FP64 tensor cores (DMMA), not HBM.
        line["roofline_hbm"] = line["roofline"]
        line["roofline"] = fp64_tensor_roofline(sim.nnzb, prob.Np, prob.nshots, ms_step, kernel, local_rank)
        line["roofline"]["kernel_variant"] = variant64
        tr = captured_traffic(kernel, prob.mesh.ne, prob.nshots) if prob.N == 5 else None
        line["roofline"]["traffic"] = tr
        line["roofline"]["traffic_unit"] = "bytes per launch (ncu, profiles/traffic.json, scaled by element rows)"
        line["roofline_hbm"]["traffic"] = tr
    if args.precision == "fp32" and prob.nshots > 1 and variant in (7, 8, 0, 1, 2):
        line["roofline_fp32_pipe"] = fp32_pipe_roofline(sim.nnzb, prob.Np, prob.nshots, ms_step, kernel)
    sim.close()

    if rank == 0 and world == 1 and not args.no_extras:
        # Plain FP64 single-shot drop-in on the same mesh.
        p1 = W.config(3, scale=args.scale, nshots=1, shot_seed=1000)
        with capi.Simulation.from_problem(p1, precision="fp64") as s1:
            prepare(s1, p1, dt, K + Wm + 2)
            s1.first_step()
            s1.run(Wm)
            s1.run_timed(K)
            ms1 = s1.run_timed(K)
            nnzb1 = s1.nnzb
        v1 = p1.dofs_per_shot * K / (ms1 / 1e3)
        a1 = bytes_per_step(p1.mesh.ne, p1.Np, nnzb1, 1, "fp64") / (ms1 / K / 1e3) / 1e9
        line["plain_fp64_single_shot"] = {"value": v1, "unit": UNIT, "ms_per_step": ms1 / K,
                                          "roofline_frac": a1 / hbm, "achieved_gbs": a1}
        line["speedup_vs_plain_fp64"] = value / v1
        # The FP32-operator single-shot drop-in on the same mesh and shot.
        with capi.Simulation.from_problem(p1, precision="fp32") as s1f:
            prepare(s1f, p1, dt, K + Wm + 2)
            s1f.first_step()
            s1f.run(Wm)
            s1f.run_timed(K)
            ms1f = s1f.run_timed(K)
        a1f = bytes_per_step(p1.mesh.ne, p1.Np, nnzb1, 1, "fp32") / (ms1f / K / 1e3) / 1e9
        line["plain_fp32_operator_single_shot"] = {"value": p1.dofs_per_shot * K / (ms1f / 1e3), "unit": UNIT,
                                                   "ms_per_step": ms1f / K, "roofline_frac": a1f / hbm,
                                                   "achieved_gbs": a1f, "speedup_vs_plain_fp64": ms1 / ms1f}
        # Mixed precision for all shots: FP32 operator, autotuned batched kernel.
        if prob.nshots > 1 and args.precision == "fp64":
            with capi.Simulation.from_problem(prob, precision="fp32") as s32:
                v32var = s32.kernel_variant
                prepare(s32, prob, dt, K + Wm + 2)
                s32.first_step()
                s32.run(Wm)
                s32.run_timed(K)
                ms32 = s32.run_timed(K)
            v32 = prob.nshots * dofs * K / (ms32 / 1e3)
            line["batched_fp32_operator"] = {"value": v32, "unit": UNIT, "ms_per_step": ms32 / K,
                                             "speedup_vs_plain_fp64": v32 / v1,
                                             "kernel": KERNELS.get(v32var, "batched"), "kernel_variant": v32var}
        # Exact FP64 for all shots: the FP64 tensor-core batched step.
        if prob.nshots > 1 and args.precision != "fp64":
            with capi.Simulation.from_problem(prob, precision="fp64") as s64:
                v64var = s64.kernel_variant
                prepare(s64, prob, dt, K + Wm + 2)
                s64.first_step()
                s64.run(Wm)
                s64.run_timed(K)
                ms64 = s64.run_timed(K)
                nnzb64 = s64.nnzb
            v64 = prob.nshots * dofs * K / (ms64 / 1e3)
            line["batched_fp64"] = {"value": v64, "unit": UNIT, "ms_per_step": ms64 / K,
                                    "speedup_vs_plain_fp64": v64 / v1, "seismogram_err": "exact FP64",
                                    "roofline": fp64_tensor_roofline(nnzb64, prob.Np, prob.nshots, ms64 / K,
                                                                     D64_KERNELS.get(v64var, "batched"))}
        # Accuracy of the measured form over the full step count against FP64
        # computed by the CUDA-core FP64 kernel (TSP_BATCHED_VARIANT=2): for the
        # FP64 tensor-core form this is the difference of two FP64 summation
        # orders; for the mixed forms the precision error. With several shots
        # the mixed FP32 form is reported too.
        nacc = prob.nsteps if args.accuracy_steps < 0 else args.accuracy_steps
        if nacc > 0:
            forms = [args.precision] + (["fp32"] if args.precision == "fp64" and prob.nshots > 1 else [])
            seis = {}
            for key, prec in [("ref", "fp64")] + [(f, f) for f in forms]:
                old = os.environ.get("TSP_BATCHED_VARIANT")
                if key == "ref":
                    os.environ["TSP_BATCHED_VARIANT"] = "2"
                try:
                    with capi.Simulation.from_problem(prob, precision=prec) as s:
                        prepare(s, prob, dt, nacc)
                        s.set_seismogram_capacity(nacc)
                        s.first_step()
                        s.run(nacc - 1)
                        seis[key] = s.seismograms(0, nacc)
                finally:
                    if key == "ref":
                        if old is None:
                            os.environ.pop("TSP_BATCHED_VARIANT", None)
                        else:
                            os.environ["TSP_BATCHED_VARIANT"] = old
            ref = seis["ref"]
            errs = {f: float(np.linalg.norm(seis[f] - ref) / np.linalg.norm(ref)) for f in forms}
            line["seismogram_rel_l2_err_vs_fp64"] = errs[args.precision]
            line["accuracy_reference"] = "FP64, CUDA-core batched kernel (TSP_BATCHED_VARIANT=2)"
            line["accuracy_steps"] = nacc
            if "batched_fp32_operator" in line:
                line["batched_fp32_operator"]["seismogram_rel_l2_err_vs_fp64"] = errs["fp32"]
        # The forms against the reference itself (committed golden of the
        # reference's own run), and their discrete-energy drift.
        vs_ref = errors_vs_reference()
        if vs_ref is not None:
            line["seismogram_rel_l2_err_vs_reference"] = vs_ref
        if prob.nshots > 1:
            line["energy_drift"] = energy_drift(prob, dt)
        # End to end through the public C-ABI with host buffers.
        ne_steps = K
        t0 = time.perf_counter()
        with capi.Simulation.from_problem(prob, precision=args.precision) as s:
            prepare(s, prob, dt, ne_steps)
            s.set_seismogram_capacity(ne_steps)
            s.first_step()
            s.run(ne_steps - 1)
            sg = s.seismograms(0, ne_steps)
        t_e2e = time.perf_counter() - t0
        h2d = (prob.mesh.xy.nbytes + prob.mesh.tri.nbytes + 3 * prob.mesh.ne * 8 + prob.nshots * 16 +
               len(prob.receivers) * 16 + prob.nshots * ne_steps * 16)
        d2h = sg.nbytes
        line["e2e"] = {"value": prob.nshots * dofs * ne_steps / t_e2e, "unit": UNIT,
                       "h2d_bytes_per_step": h2d / ne_steps, "d2h_bytes_per_step": d2h / ne_steps,
                       "wall_s": t_e2e, "steps": ne_steps,
                       "includes": "tsp_create (mesh upload, device assembly, point location, kernel choice), "
                                   "force tables, first_step + run, read-back of every step's receiver samples "
                                   "(the shot gathers)"}
        v_cpu, sample = cpu_reference_sample(nprocs=1, nsteps=10)
        line["cpu_baseline"] = {"value": v_cpu, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
