"""ctypes binding of the tspeed_b200 C-ABI (include/tspeed_b200.h).

`Simulation` is a thin Python face of one handle; the C++ face for users of
the reference's classes is include/tspeed_gpu.hpp. Nothing here computes:
every operation is a call into libtspeed_b200.so, and importing fails loudly
when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# TSP_CHECKED=1 selects the build whose kernels range-check every gather
# index on the device (tsp_checked_build; TSP_ERR_INDEX on a failure).
LIB_PATH = os.path.join(_HERE, "libtspeed_b200_checked.so" if os.environ.get("TSP_CHECKED") == "1"
                        else "libtspeed_b200.so")

TSP_PREC = {"fp64": 0, "fp32": 1, "bf16": 2}
TSP_OP = {"explicit": 0, "matrix_free": 1}
# Modal basis: Dubiner<N> (orthonormal) or BoundaryAdapted<N> (ShapeFunctions.hpp).
TSP_BASIS = {"dubiner": 0, "ba": 1, "boundary_adapted": 1}
STATUS = {0: "TSP_OK", -1: "TSP_ERR_ARG", -2: "TSP_ERR_CUDA", -3: "TSP_ERR_NOMEM", -4: "TSP_ERR_STATE",
          -5: "TSP_ERR_NOT_FOUND", -6: "TSP_ERR_MESH", -7: "TSP_ERR_NONFINITE", -8: "TSP_ERR_TIMEOUT",
          -9: "TSP_ERR_UNSUPPORTED", -10: "TSP_ERR_INDEX"}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class TspProblem(C.Structure):
    _fields_ = [("nverts", C.c_int32), ("xy", _dp), ("ne", C.c_int32), ("tri", _ip), ("N", C.c_int32),
                ("lambda_", _dp), ("mu", _dp), ("rho", _dp), ("penalty", C.c_double), ("precision", C.c_int32),
                ("op_kind", C.c_int32), ("nshots", C.c_int32), ("src_xy", _dp), ("nrcv", C.c_int32),
                ("rcv_xy", _dp), ("device", C.c_int32), ("basis", C.c_int32)]


class TspBlockProblem(C.Structure):
    _fields_ = [("ne", C.c_int32), ("Np", C.c_int32), ("nnzb", C.c_int32), ("row_ptr", _ip), ("col", _ip),
                ("blocks", _dp), ("minv", _dp), ("precision", C.c_int32), ("nshots", C.c_int32),
                ("src_elem", _ip), ("src_phi", _dp), ("nrcv", C.c_int32), ("rcv_elem", _ip), ("rcv_phi", _dp),
                ("device", C.c_int32), ("ref_invmass", _dp)]


# Every symbol the header declares, with its ctypes signature.
SIGNATURES = {
    "tsp_version": (C.c_char_p, []),
    "tsp_create": (C.c_int, [C.POINTER(TspProblem), C.POINTER(C.c_void_p)]),
    "tsp_create_from_blocks": (C.c_int, [C.POINTER(TspBlockProblem), C.POINTER(C.c_void_p)]),
    "tsp_destroy": (C.c_int, [C.c_void_p]),
    "tsp_last_error": (C.c_char_p, [C.c_void_p]),
    "tsp_get_sizes": (C.c_int, [C.c_void_p, _ip, _ip, _ip, _ip, _lp]),
    "tsp_set_dt": (C.c_int, [C.c_void_p, C.c_double]),
    "tsp_set_force_table": (C.c_int, [C.c_void_p, C.c_int32, _dp, C.c_int64]),
    "tsp_set_ricker": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int64]),
    "tsp_force_times": (C.c_int, [C.c_double, C.c_int64, _dp]),
    "tsp_set_initial": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp]),
    "tsp_first_step": (C.c_int, [C.c_void_p]),
    "tsp_step": (C.c_int, [C.c_void_p]),
    "tsp_run": (C.c_int, [C.c_void_p, C.c_int64]),
    "tsp_run_timed": (C.c_int, [C.c_void_p, C.c_int64, _dp]),
    "tsp_get_progress": (C.c_int, [C.c_void_p, _lp, _dp]),
    "tsp_get_kernel_variant": (C.c_int, [C.c_void_p, _ip]),
    "tsp_checked_build": (C.c_int, []),
    "tsp_get_u": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "tsp_get_u_all": (C.c_int, [C.c_void_p, _dp]),
    "tsp_get_seismograms": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, _dp]),
    "tsp_set_seismogram_capacity": (C.c_int, [C.c_void_p, C.c_int64]),
    "tsp_enable_energy": (C.c_int, [C.c_void_p, C.c_int32]),
    "tsp_get_energy": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, _dp]),
    "tsp_get_state": (C.c_int, [C.c_void_p, _dp, _dp, _lp, _dp]),
    "tsp_set_state": (C.c_int, [C.c_void_p, _dp, _dp, C.c_int64, C.c_double]),
    "tsp_check_finite": (C.c_int, [C.c_void_p, _ip]),
    "tsp_apply": (C.c_int, [C.c_void_p, _dp, _dp]),
    "tsp_estimate_lmax": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "tsp_estimate_lmax_noalloc": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "tsp_export_operator": (C.c_int, [C.c_void_p, _ip, _ip, _dp, _dp]),
    "tsp_export_points": (C.c_int, [C.c_void_p, _ip, _dp, _ip, _dp]),
    "tsp_batch_create": (C.c_int, [C.POINTER(TspProblem), C.c_int32, C.POINTER(C.c_void_p)]),
    "tsp_batch_destroy": (C.c_int, [C.c_void_p]),
    "tsp_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "tsp_batch_info": (C.c_int, [C.c_void_p, _ip, _lp]),
    "tsp_batch_estimate_lmax": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "tsp_batch_set_dt": (C.c_int, [C.c_void_p, _dp]),
    "tsp_batch_set_ricker": (C.c_int, [C.c_void_p, _dp, _dp, _dp, _dp, _ip, C.c_int64]),
    "tsp_batch_set_seismogram_capacity": (C.c_int, [C.c_void_p, C.c_int64]),
    "tsp_batch_first_step": (C.c_int, [C.c_void_p]),
    "tsp_batch_run": (C.c_int, [C.c_void_p, C.c_int64]),
    "tsp_batch_run_timed": (C.c_int, [C.c_void_p, C.c_int64, _dp]),
    "tsp_batch_get_u": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "tsp_batch_get_seismograms": (C.c_int, [C.c_void_p, C.c_int32, C.c_int64, C.c_int64, _dp]),
    "tsp_quadrature_points": (C.c_int, [C.c_int32, C.c_int32, _dp, C.c_int32, _ip, _dp]),
    "tsp_project": (C.c_int, [C.c_int32, C.c_int32, _dp, C.c_int32, _ip, _dp, _dp]),
    "tsp_project_basis": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _dp, C.c_int32, _ip, _dp, _dp]),
    "tsp_get_ref_invmass": (C.c_int, [C.c_void_p, _ip, _dp]),
    "tsp_field_values": (C.c_int, [C.c_void_p, C.c_int32, _dp]),
    "tsp_write_field": (C.c_int, [C.c_void_p, C.c_int32, C.c_char_p, C.c_int64]),
    "tsp_l2_error": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp]),
    "tsp_points_out": (C.c_int, [C.c_int32, _dp, C.c_int32, _ip, C.c_char_p]),
    "tsp_set_initial_values": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp]),
    "tsp_release_cached_memory": (C.c_int, [C.c_int32]),
    "tsp_fp64_tensor_peak": (C.c_int, [C.c_int32, _dp]),
    "tsp_selftest_bounded_wait": (C.c_int, [C.c_int32, _ip, _ip]),
    "tsp_locate_points": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _dp, C.c_int32, _ip, C.c_int32, _dp, _ip, _dp]),
    "tsp_eval_basis": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _dp, _dp]),
    "tsp_quadrature_rule": (C.c_int, [C.c_int32, _dp, _dp]),
    "tsp_gmsh_read": (C.c_int, [C.c_char_p, _ip, _dp, _ip, _ip, _ip]),
    "tsp_mesh_neighbours": (C.c_int, [C.c_int32, _ip, _ip, _ip]),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m tspeed_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class TspError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def _check(rc: int, h=None):
    if rc != 0:
        raise TspError(rc, lib().tsp_last_error(h).decode())


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def gmsh_read(path: str):
    L = lib()
    nv, ne = C.c_int32(0), C.c_int32(0)
    _check(L.tsp_gmsh_read(path.encode(), C.byref(nv), None, C.byref(ne), None, None))
    xy = np.zeros((nv.value, 2))
    tri = np.zeros((ne.value, 3), dtype=np.int32)
    reg = np.zeros(ne.value, dtype=np.int32)
    _check(L.tsp_gmsh_read(path.encode(), C.byref(nv), _d(xy), C.byref(ne), _i(tri), _i(reg)))
    return xy, tri, reg


def mesh_neighbours(tri):
    tri = _i32(tri)
    ne = tri.shape[0]
    nb = np.zeros((ne, 3), dtype=np.int32)
    ned = np.zeros((ne, 3), dtype=np.int32)
    _check(lib().tsp_mesh_neighbours(ne, _i(tri), _i(nb), _i(ned)))
    return nb, ned


def quadrature_points(N: int, xy, tri):
    xy, tri = _f64(xy), _i32(tri)
    pts = np.zeros((tri.shape[0], (N + 1) ** 2, 2))
    _check(lib().tsp_quadrature_points(N, xy.shape[0], _d(xy), tri.shape[0], _i(tri), _d(pts)))
    return pts


def project(N: int, xy, tri, fvals, basis: str = "dubiner"):
    """FESpace::transform of a field sampled at quadrature_points()."""
    xy, tri, fvals = _f64(xy), _i32(tri), _f64(fvals)
    Np = (N + 1) * (N + 2) // 2
    out = np.zeros(2 * tri.shape[0] * Np)
    _check(lib().tsp_project_basis(N, TSP_BASIS[basis], xy.shape[0], _d(xy), tri.shape[0], _i(tri), _d(fvals),
                                   _d(out)))
    return out


def points_out(xy, tri, fname: str):
    """FESpace::points_out: the physical field_out points of every element."""
    xy, tri = _f64(xy), _i32(tri)
    _check(lib().tsp_points_out(xy.shape[0], _d(xy), tri.shape[0], _i(tri), os.fsencode(fname)))


def locate_points(N: int, xy, tri, pts, basis: str = "dubiner"):
    """PointWiseEntity::M_add for many points: (elem[npts], phi[npts][Np])."""
    xy, tri = _f64(xy), _i32(tri)
    pts = _f64(np.asarray(pts, dtype=np.float64).reshape(-1, 2))
    elem = np.zeros(pts.shape[0], dtype=np.int32)
    phi = np.zeros((pts.shape[0], (N + 1) * (N + 2) // 2))
    _check(lib().tsp_locate_points(N, TSP_BASIS[basis], xy.shape[0], _d(xy), tri.shape[0], _i(tri), pts.shape[0],
                                   _d(pts), _i(elem), _d(phi)))
    return elem, phi


def eval_basis(N: int, rpts, basis: str = "dubiner"):
    """Basis values phi[npts][Np] at reference points rpts[npts][2]."""
    rpts = _f64(np.asarray(rpts, dtype=np.float64).reshape(-1, 2))
    out = np.zeros((rpts.shape[0], (N + 1) * (N + 2) // 2))
    _check(lib().tsp_eval_basis(N, TSP_BASIS[basis], rpts.shape[0], _d(rpts), _d(out)))
    return out


def quadrature_rule(N: int):
    """Collapsed Gauss<N+1> volume rule: reference nodes [(N+1)^2, 2], weights."""
    r, w = np.zeros(((N + 1) ** 2, 2)), np.zeros((N + 1) ** 2)
    _check(lib().tsp_quadrature_rule(N, _d(r), _d(w)))
    return r, w


def selftest_bounded_wait(device: int = 0):
    """(completed, abort_raised) of a kernel whose bounded wait must time out."""
    c, a = C.c_int32(), C.c_int32()
    _check(lib().tsp_selftest_bounded_wait(device, C.byref(c), C.byref(a)))
    return c.value, a.value


def fp64_tensor_peak(device: int = 0) -> float:
    """Measured FP64 tensor-core (DMMA) throughput, TFLOP/s."""
    v = C.c_double()
    _check(lib().tsp_fp64_tensor_peak(device, C.byref(v)))
    return v.value


def release_cached_memory(device: int = 0):
    """Returns the device memory cached by the library's allocator pool."""
    _check(lib().tsp_release_cached_memory(device))


def force_times(dt: float, n: int):
    out = np.zeros(n)
    _check(lib().tsp_force_times(dt, n, _d(out)))
    return out


class Simulation:
    """One engine handle. Host vectors use the reference layout
    u[c*ne*Np + e*Np + i]."""

    def __init__(self, handle, keep=()):
        self._h = handle
        self._keep = keep
        ne, Np, S, nr = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        nnzb = C.c_int64()
        _check(lib().tsp_get_sizes(self._h, C.byref(ne), C.byref(Np), C.byref(S), C.byref(nr), C.byref(nnzb)), self._h)
        self.ne, self.Np, self.nshots, self.nrcv, self.nnzb = ne.value, Np.value, S.value, nr.value, nnzb.value
        self.R = 2 * self.Np

    # ---- construction ----
    @classmethod
    def create(cls, xy, tri, N, lam, mu, rho, src_xy, rcv_xy, penalty=2.0, precision="fp64", op="explicit",
               device=0, basis="dubiner"):
        xy, tri = _f64(xy), _i32(tri)
        lam, mu, rho = _f64(lam), _f64(mu), _f64(rho)
        src = _f64(np.asarray(src_xy, dtype=np.float64).reshape(-1, 2))
        rcv = _f64(np.asarray(rcv_xy, dtype=np.float64).reshape(-1, 2))
        p = TspProblem(xy.shape[0], _d(xy), tri.shape[0], _i(tri), N, _d(lam), _d(mu), _d(rho), penalty,
                       TSP_PREC[precision], TSP_OP[op], src.shape[0], _d(src), rcv.shape[0],
                       _d(rcv) if rcv.shape[0] else None, device, TSP_BASIS[basis])
        h = C.c_void_p()
        _check(lib().tsp_create(C.byref(p), C.byref(h)))
        return cls(h)

    @classmethod
    def from_problem(cls, prob, precision="fp64", op="explicit", device=0):
        return cls.create(prob.mesh.xy, prob.mesh.tri, prob.N, prob.lam, prob.mu, prob.rho,
                          [(s.x, s.y) for s in prob.sources], prob.receivers, penalty=prob.penalty,
                          precision=precision, op=op, device=device, basis=getattr(prob, "basis", "dubiner"))

    @classmethod
    def from_blocks(cls, row_ptr, col, blocks, minv, src_elem, src_phi, rcv_elem, rcv_phi, precision="fp64",
                    device=0, ref_invmass=None):
        """ref_invmass: the reference inverse mass [Np][Np] of a
        non-orthonormal basis (None for Dubiner)."""
        ref_invmass = None if ref_invmass is None else _f64(ref_invmass)
        row_ptr, col = _i32(row_ptr), _i32(col)
        blocks, minv = _f64(blocks), _f64(minv)
        src_elem, src_phi = _i32(np.atleast_1d(src_elem)), _f64(np.atleast_2d(src_phi))
        rcv_elem, rcv_phi = _i32(np.atleast_1d(rcv_elem)), _f64(np.asarray(rcv_phi).reshape(len(rcv_elem), -1))
        ne = row_ptr.shape[0] - 1
        Np = blocks.shape[1] // 2
        p = TspBlockProblem(ne, Np, col.shape[0], _i(row_ptr), _i(col), _d(blocks), _d(minv), TSP_PREC[precision],
                            src_elem.shape[0], _i(src_elem), _d(src_phi), rcv_elem.shape[0],
                            _i(rcv_elem) if len(rcv_elem) else None, _d(rcv_phi) if len(rcv_elem) else None, device,
                            _d(ref_invmass))
        h = C.c_void_p()
        _check(lib().tsp_create_from_blocks(C.byref(p), C.byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            lib().tsp_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- setters ----
    def set_dt(self, dt: float):
        _check(lib().tsp_set_dt(self._h, dt), self._h)

    def set_force_table(self, shot: int, F):
        F = _f64(np.asarray(F).reshape(-1, 2))
        _check(lib().tsp_set_force_table(self._h, shot, _d(F), F.shape[0]), self._h)

    def set_ricker(self, shot: int, f0: float, t0: float, amp: float, direction: int, n: int):
        _check(lib().tsp_set_ricker(self._h, shot, f0, t0, amp, direction, n), self._h)

    def set_initial(self, shot: int, u0=None, v0=None):
        u0 = None if u0 is None else _f64(u0)
        v0 = None if v0 is None else _f64(v0)
        _check(lib().tsp_set_initial(self._h, shot, _d(u0), _d(v0)), self._h)

    def set_initial_values(self, shot: int, u_vals=None, v_vals=None):
        """Initial u / v from field values at quadrature_points(), projected on
        the device (FESpace::transform)."""
        u_vals = None if u_vals is None else _f64(u_vals)
        v_vals = None if v_vals is None else _f64(v_vals)
        _check(lib().tsp_set_initial_values(self._h, shot, _d(u_vals), _d(v_vals)), self._h)

    def set_seismogram_capacity(self, n: int):
        _check(lib().tsp_set_seismogram_capacity(self._h, n), self._h)

    def enable_energy(self, on: bool = True):
        _check(lib().tsp_enable_energy(self._h, int(on)), self._h)

    # ---- stepping ----
    def first_step(self):
        _check(lib().tsp_first_step(self._h), self._h)

    def step(self):
        _check(lib().tsp_step(self._h), self._h)

    def run(self, n: int):
        _check(lib().tsp_run(self._h, n), self._h)

    def run_timed(self, n: int) -> float:
        ms = C.c_double()
        _check(lib().tsp_run_timed(self._h, n, C.byref(ms)), self._h)
        return ms.value

    def progress(self):
        k, t = C.c_int64(), C.c_double()
        _check(lib().tsp_get_progress(self._h, C.byref(k), C.byref(t)), self._h)
        return k.value, t.value

    @property
    def kernel_variant(self) -> int:
        """Batched-step kernel chosen by the autotuner (or TSP_BATCHED_VARIANT):
        FP32: 7/8 warp-specialised CUDA-core kernels with bulk-copy rings,
        0/1/2 other CUDA-core kernels, 4 tensor-core fixed-point kernel; FP64
        with several shots: 5 and 6 warp-specialised FP64 tensor-core kernels
        (two groups of 8 consumer warps / one group of 16), 3 single-role
        one, 2 CUDA-core kernel."""
        v = C.c_int32()
        _check(lib().tsp_get_kernel_variant(self._h, C.byref(v)), self._h)
        return v.value

    @property
    def basis(self) -> str:
        b = C.c_int32()
        _check(lib().tsp_get_ref_invmass(self._h, C.byref(b), None), self._h)
        return "dubiner" if b.value == 0 else "ba"

    def ref_invmass(self):
        """M_ref^-1 of the handle's basis, [Np][Np] (identity for Dubiner)."""
        out = np.zeros((self.Np, self.Np))
        _check(lib().tsp_get_ref_invmass(self._h, None, _d(out)), self._h)
        return out

    # ---- outputs ----
    def field_values(self, shot: int = 0):
        """FESpace::field_out values of the current displacement, [ne, 4, 2]."""
        out = np.zeros((self.ne, 4, 2))
        _check(lib().tsp_field_values(self._h, shot, _d(out)), self._h)
        return out

    def write_field(self, fname: str, step: int, shot: int = 0):
        """FESpace::field_out(fname, u, step): writes fname + "u_<step>.field"."""
        _check(lib().tsp_write_field(self._h, shot, os.fsencode(fname), step), self._h)

    def l2_error(self, exact, shot: int = 0) -> float:
        """FESpace::L2error against exact values at quadrature_points()."""
        exact = _f64(exact)
        err = C.c_double()
        _check(lib().tsp_l2_error(self._h, shot, _d(exact), C.byref(err)), self._h)
        return err.value

    def u(self, shot: int = 0):
        out = np.zeros(2 * self.ne * self.Np)
        _check(lib().tsp_get_u(self._h, shot, _d(out)), self._h)
        return out

    def u_all(self):
        """u() of every shot: [nshots][2*ne*Np], reference layout."""
        out = np.zeros((self.nshots, 2 * self.ne * self.Np))
        _check(lib().tsp_get_u_all(self._h, _d(out)), self._h)
        return out

    def seismograms(self, k0: int, nk: int):
        out = np.zeros((self.nshots, nk, self.nrcv, 2))
        _check(lib().tsp_get_seismograms(self._h, k0, nk, _d(out)), self._h)
        return out

    def energy(self, k0: int, nk: int):
        out = np.zeros(nk)
        _check(lib().tsp_get_energy(self._h, k0, nk, _d(out)), self._h)
        return out

    def get_state(self):
        n = 2 * self.ne * self.Np
        a, b = np.zeros((self.nshots, n)), np.zeros((self.nshots, n))
        k, t = C.c_int64(), C.c_double()
        _check(lib().tsp_get_state(self._h, _d(a), _d(b), C.byref(k), C.byref(t)), self._h)
        return a, b, k.value, t.value

    def set_state(self, u_prev, u_cur, steps_done: int, last_time: float):
        _check(lib().tsp_set_state(self._h, _d(_f64(u_prev)), _d(_f64(u_cur)), steps_done, last_time), self._h)

    def check_finite(self) -> bool:
        bad = C.c_int32()
        _check(lib().tsp_check_finite(self._h, C.byref(bad)), self._h)
        return bad.value == 0

    def apply(self, x):
        x = _f64(x)
        y = np.zeros_like(x)
        _check(lib().tsp_apply(self._h, _d(x), _d(y)), self._h)
        return y

    def estimate_lmax(self, iters: int = 100) -> float:
        out = C.c_double()
        _check(lib().tsp_estimate_lmax(self._h, iters, C.byref(out)), self._h)
        return out.value

    def export_operator(self):
        row_ptr = np.zeros(self.ne + 1, dtype=np.int32)
        col = np.zeros(self.nnzb, dtype=np.int32)
        blocks = np.zeros((self.nnzb, self.R, self.R))
        minv = np.zeros(self.ne)
        _check(lib().tsp_export_operator(self._h, _i(row_ptr), _i(col), _d(blocks), _d(minv)), self._h)
        return row_ptr, col, blocks, minv

    def export_points(self):
        se = np.zeros(self.nshots, dtype=np.int32)
        sp = np.zeros((self.nshots, self.Np))
        re = np.zeros(self.nrcv, dtype=np.int32)
        rp = np.zeros((self.nrcv, self.Np))
        _check(lib().tsp_export_points(self._h, _i(se), _d(sp), _i(re) if self.nrcv else None,
                                       _d(rp) if self.nrcv else None), self._h)
        return se, sp, re, rp


def _bcheck(rc: int, b=None):
    if rc != 0:
        raise TspError(rc, lib().tsp_batch_last_error(b).decode())


class Batch:
    """Many independent meshes of uneven size and degree, one source each,
    advanced together (tsp_batch_*). Problems are workloads.Problem objects
    with one source."""

    def __init__(self, problems, precision="fp64", op="explicit", device=0):
        self._keep = []
        arr = (TspProblem * len(problems))()
        for i, pr in enumerate(problems):
            xy, tri = _f64(pr.mesh.xy), _i32(pr.mesh.tri)
            lam, mu, rho = _f64(pr.lam), _f64(pr.mu), _f64(pr.rho)
            src = _f64(np.array([[pr.sources[0].x, pr.sources[0].y]]))
            rcv = _f64(np.asarray(pr.receivers, dtype=np.float64).reshape(-1, 2))
            self._keep += [xy, tri, lam, mu, rho, src, rcv]
            arr[i] = TspProblem(xy.shape[0], _d(xy), tri.shape[0], _i(tri), pr.N, _d(lam), _d(mu), _d(rho),
                                pr.penalty, TSP_PREC[precision], TSP_OP[op], 1, _d(src), rcv.shape[0],
                                _d(rcv) if rcv.shape[0] else None, device)
        h = C.c_void_p()
        _bcheck(lib().tsp_batch_create(arr, len(problems), C.byref(h)))
        self._b = h
        self.problems = problems
        self._keep = []
        ng, td = C.c_int32(), C.c_int64()
        _bcheck(lib().tsp_batch_info(self._b, C.byref(ng), C.byref(td)), self._b)
        self.ngroups, self.total_dofs = ng.value, td.value

    def close(self):
        if getattr(self, "_b", None):
            lib().tsp_batch_destroy(self._b)
            self._b = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def estimate_lmax(self, iters=100):
        out = np.zeros(len(self.problems))
        _bcheck(lib().tsp_batch_estimate_lmax(self._b, iters, _d(out)), self._b)
        return out

    def set_dt(self, dt):
        self.dt = _f64(dt)
        _bcheck(lib().tsp_batch_set_dt(self._b, _d(self.dt)), self._b)

    def set_ricker(self, n):
        ps = self.problems
        f0 = _f64([p.sources[0].f0 for p in ps])
        t0 = _f64([p.sources[0].t0 for p in ps])
        amp = _f64([p.sources[0].amp for p in ps])
        di = _i32([p.sources[0].direction for p in ps])
        _bcheck(lib().tsp_batch_set_ricker(self._b, _d(self.dt), _d(f0), _d(t0), _d(amp), _i(di), n), self._b)

    def set_seismogram_capacity(self, n):
        _bcheck(lib().tsp_batch_set_seismogram_capacity(self._b, n), self._b)

    def first_step(self):
        _bcheck(lib().tsp_batch_first_step(self._b), self._b)

    def run(self, n):
        _bcheck(lib().tsp_batch_run(self._b, n), self._b)

    def run_timed(self, n):
        ms = C.c_double()
        _bcheck(lib().tsp_batch_run_timed(self._b, n, C.byref(ms)), self._b)
        return ms.value

    def u(self, m):
        p = self.problems[m]
        out = np.zeros(2 * p.mesh.ne * p.Np)
        _bcheck(lib().tsp_batch_get_u(self._b, m, _d(out)), self._b)
        return out

    def seismograms(self, m, k0, nk):
        out = np.zeros((nk, len(self.problems[m].receivers), 2))
        _bcheck(lib().tsp_batch_get_seismograms(self._b, m, k0, nk, _d(out)), self._b)
        return out
