"""Python host mirror of the reference's solver interface, over libqesb200.so.

The reference drives the lambda solve through C++ objects:

    qes::Domain domain(Nx, Ny, Nz, dx, dy, dz);            src/qes/Domain.cpp:7-31
    WINDSGeneralData *WGD = ...;  // e..n, icellflag, u0..w  src/winds/WINDSGeneralData.h:231-274
    Solver *solver = SolverFactory::create(type, domain, tol); src/winds/SolverFactory.cpp:35-60
    solver->resetLambda();                                  src/winds/Solver.h:115-120
    solver->solve(WGD, itermax);                            src/winds/Solver_CPU.cpp:42-238

This module offers the same names with the same argument meaning, backed by
the C ABI of include/qesb.h (ctypes; numpy arrays in the reference layouts).
The C++ adaptor with the identical interface is qes-public_b200/host/Solver_B200.h.

There is no CPU fallback: if the shared library or a CUDA device is missing,
the calls raise.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libqesb200.so")

QESB_OK = 0
_STATUS = {
    1: "QESB_ERR_ARG",
    2: "QESB_ERR_CUDA",
    3: "QESB_ERR_NOMEM",
    4: "QESB_ERR_STATE",
    5: "QESB_ERR_NUMERIC",
    6: "QESB_ERR_NODEV",
}

# SolverFactory solve types (src/winds/SolverFactory.h:48-51) plus this build's.
CPU_Type, DYNAMIC_P, Global_M, Shared_M = 1, 2, 3, 4
B200_Type = 5


class QesbError(RuntimeError):
    """A non-OK status from the C ABI (the reference would have exited)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, status)}: {message}")
        self.status = status


class Grid(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("dx", C.c_float),
                ("dy", C.c_float), ("dz_array", C.POINTER(C.c_float))]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("residual", C.c_double),
                ("ms_total", C.c_double), ("ms_sor", C.c_double), ("path", C.c_int),
                ("sweeps_per_launch", C.c_int), ("launches", C.c_int), ("pre_iterations", C.c_int),
                ("max_divergence", C.c_double), ("window_drift", C.c_double),
                ("ms_sweeps", C.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Fp64Report(C.Structure):
    _fields_ = [("lambda_max_abs_err", C.c_double), ("lambda_max_abs", C.c_double),
                ("wind_max_err", C.c_double), ("ms", C.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Building(C.Structure):
    _fields_ = [("x_start", C.c_float), ("y_start", C.c_float), ("length", C.c_float),
                ("width", C.c_float), ("height", C.c_float), ("base_height", C.c_float)]


class Inflow(C.Structure):
    _fields_ = [("u_ref", C.c_float), ("z_ref", C.c_float), ("p", C.c_float),
                ("dir_deg", C.c_float)]


_lib_handle = None

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)


def lib() -> C.CDLL:
    """Load libqesb200.so (built by qes-public_b200/Makefile)."""
    global _lib_handle
    if _lib_handle is None:
        if not os.path.exists(LIB_PATH):
            raise QesbError(4, f"{LIB_PATH} is not built (run __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        V = C.c_void_p
        sig = {
            "qesb_version": ([], C.c_char_p),
            "qesb_last_error": ([], C.c_char_p),
            "qesb_create": ([C.POINTER(Grid), C.c_float, C.c_int, C.POINTER(V)], C.c_int),
            "qesb_destroy": ([V], C.c_int),
            "qesb_reset_lambda": ([V], C.c_int),
            "qesb_set_inputs": ([V] + [V] * 10, C.c_int),
            "qesb_set_inputs_device": ([V] + [V] * 10, C.c_int),
            "qesb_solve": ([V, C.c_int, V, V, V, C.POINTER(Stats)], C.c_int),
            "qesb_solve_device": ([V, C.c_int, V, V, V, C.POINTER(Stats)], C.c_int),
            "qesb_set_lambda": ([V, V], C.c_int),
            "qesb_get_lambda": ([V, V], C.c_int),
            "qesb_get_divergence": ([V, V], C.c_int),
            "qesb_get_residual_history": ([V, V, C.c_int], C.c_int),
            "qesb_set_tolerance": ([V, C.c_float], C.c_int),
            "qesb_set_prephase": ([V, C.c_float, C.c_float, C.c_int], C.c_int),
            "qesb_set_prephase_start": ([V, C.c_float, C.c_int], C.c_int),
            "qesb_set_inputs_flags": ([V, V, V, V, V], C.c_int),
            "qesb_set_window_rule": ([V, C.c_int, C.c_double], C.c_int),
            "qesb_fp64_same_sor": ([V, V, C.c_float, C.c_int, C.c_int, V, V, V, V, C.POINTER(Fp64Report)],
                                   C.c_int),
            "qesb_time_sweeps": ([V, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_int)], C.c_int),
            "qesb_autotune": ([V, C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int], C.c_int),
            "qesb_solve_batch": ([C.POINTER(V), C.c_int, C.c_int, C.POINTER(V), C.POINTER(V), C.POINTER(V),
                                  C.POINTER(Stats)], C.c_int),
            "qesb_autotune_batch": ([C.POINTER(V), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_float), C.c_int],
                                    C.c_int),
            "qesb_wall_log_law": ([V, C.c_float, C.c_float, V, V, V], C.c_int),
            "qesb_workspace_write": ([C.c_char_p, C.POINTER(Grid), C.c_double] + [V] * 13, C.c_int),
            "qesb_workspace_dims": ([C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                     C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
            "qesb_workspace_read": ([C.c_char_p, C.c_int, C.c_int, C.c_int] + [V] * 14, C.c_int),
            "qesb_num_variants": ([], C.c_int),
            "qesb_set_option": ([V, C.c_char_p, C.c_int], C.c_int),
            "qesb_set_stream": ([V, V], C.c_int),
            "qesb_get_stream": ([V, C.POINTER(V)], C.c_int),
            "qesb_solve_noalloc": ([C.POINTER(Grid), C.c_float, C.c_int] + [V] * 14
                                   + [V, C.POINTER(Stats)], C.c_int),
            "qesb_umma_selftest": ([V, V, V, C.c_int, C.c_int, C.c_int, C.c_int], C.c_int),
            "qesb_warmnet_load": ([C.c_char_p, C.c_int, C.POINTER(V)], C.c_int),
            "qesb_warmnet_destroy": ([V], C.c_int),
            "qesb_warm_start": ([V, V], C.c_int),
            "qesb_warm_start_batch": ([C.POINTER(V), C.c_int, V], C.c_int),
            "qesb_conv3d": ([V, C.c_int, C.c_int, V, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, V,
                             C.c_int, C.c_int, V, V, V, C.c_int, V, V, V], C.c_int),
            "qesb_conv3d_items": ([V, C.c_int, C.c_int, V, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   V, C.c_int, C.c_int, V, V, V, C.c_int, V, V, V], C.c_int),
            "qesb_net_set_conv_path": ([C.c_int], C.c_int),
            "qesb_conv3d_wgrad": ([V, C.c_int, C.c_int, V, C.c_int, C.c_int, C.c_int, C.c_int, V, C.c_int,
                                   C.c_long, V, V, V], C.c_int),
            "qesb_compute_divergence": ([V], C.c_int),
            "qesb_warm_input": ([V, V, C.c_int, V], C.c_int),
            "qesb_warm_input_half": ([V, V, C.c_int, V], C.c_int),
            "qesb_warm_target": ([V, V, V, V], C.c_int),
            "qesb_warm_apply": ([V, V, C.c_int, V], C.c_int),
            "qesb_warm_apply_up2": ([V, V, C.c_int, V], C.c_int),
            "qesb_net_pool2": ([V, V, C.c_int, C.c_int, C.c_int, C.c_int, V], C.c_int),
            "qesb_net_pool2_f32": ([V, V, C.c_int, C.c_int, C.c_int, V], C.c_int),
            "qesb_net_skip_grad": ([V, C.c_int, C.c_int, V, V, V, C.c_int, C.c_int, C.c_int, C.c_int, V],
                                   C.c_int),
            "qesb_net_up_grad": ([V, C.c_int, V, V, C.c_int, C.c_int, C.c_int, C.c_int, V], C.c_int),
            "qesb_net_to_bf16": ([V, V, V, C.c_long, V], C.c_int),
            "qesb_net_colsum": ([V, C.c_long, C.c_int, V, V], C.c_int),
            "qesb_net_mse": ([V, C.c_int, V, V, C.c_long, C.c_float, V, V, V], C.c_int),
            "qesb_net_mse_coarse": ([V, C.c_int, V, V, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, V, V, V],
                                    C.c_int),
            "qesb_net_adam_conv": ([V, V, V, V, C.c_int, C.c_int, C.c_int, V, C.c_int, V, C.c_int, C.c_float,
                                    C.c_float, C.c_float, C.c_float, C.c_int, C.c_float, V], C.c_int),
            "qesb_net_adam_vec": ([V, V, V, V, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
                                   C.c_float, V], C.c_int),
            "qesb_city_dz": ([C.c_int, C.c_float, C.c_float, _FP], C.c_int),
            "qesb_city_build": ([C.POINTER(Grid), C.c_int, C.POINTER(Building), C.POINTER(Inflow)]
                                + [V] * 10, C.c_int),
            "qesb_city_build_device": ([C.POINTER(Grid), C.c_int, C.POINTER(Building), C.POINTER(Inflow)]
                                       + [V] * 10 + [V], C.c_int),
            "qesb_city_inflow": ([C.POINTER(Grid), V, C.POINTER(Inflow), V, V, V], C.c_int),
            "qesb_city_random": ([C.POINTER(Grid), C.c_uint64, C.c_int, C.c_float, C.c_float,
                                  C.c_float, C.c_float, C.POINTER(Building), _IP,
                                  C.POINTER(Inflow)], C.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib_handle = L
    return _lib_handle


def check(status: int) -> None:
    if status != QESB_OK:
        raise QesbError(status, lib().qesb_last_error().decode())


def _ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return a.ctypes.data_as(C.c_void_p)


# ---------------------------------------------------------------------------
# qes::Domain mirror (src/qes/Domain.h:94-196, Domain.cpp:7-151)
# ---------------------------------------------------------------------------
class Domain:
    """Staggered grid: nx = Nx+1, ny = Ny+1, nz = Nz+2 (Domain.cpp:11-13).

    dz_array: None for a uniform grid of spacing dz (defineVerticalStretching(float)),
    or the nz-1 values including the ghost layer at index 0 (the layout of
    Domain::dz_array after defineVerticalStretching(vector), Domain.cpp:121-133).
    """

    def __init__(self, Nx: int, Ny: int, Nz: int, dx: float, dy: float, dz: float,
                 dz_array: np.ndarray | None = None):
        self._nx, self._ny, self._nz = Nx + 1, Ny + 1, Nz + 2
        self._dx, self._dy = np.float32(dx), np.float32(dy)
        if dz_array is None:
            self.dz_array = np.full(self._nz - 1, dz, dtype=np.float32)
        else:
            self.dz_array = np.ascontiguousarray(dz_array, dtype=np.float32)
            assert self.dz_array.shape == (self._nz - 1,)
        self._dz = np.float32(self.dz_array.min())
        zf = np.zeros(self._nz, dtype=np.float32)
        zf[0] = -self.dz_array[0]
        for k in range(2, self._nz):
            zf[k] = np.float32(zf[k - 1] + self.dz_array[k - 1])
        z = np.zeros(self._nz - 1, dtype=np.float32)
        z[0] = np.float32(-0.5) * self.dz_array[0]
        for k in range(1, self._nz - 1):
            z[k] = np.float32(0.5) * np.float32(zf[k] + zf[k + 1])
        self.z_face, self.z = zf, z

    def nx(self): return self._nx
    def ny(self): return self._ny
    def nz(self): return self._nz
    def dx(self): return float(self._dx)
    def dy(self): return float(self._dy)
    def dz(self): return float(self._dz)

    @property
    def base(self):
        return self._nx - 1, self._ny - 1, self._nz - 2

    def numCellCentered(self): return (self._nx - 1) * (self._ny - 1) * (self._nz - 1)
    def numFaceCentered(self): return self._nx * self._ny * self._nz
    def cell(self, i, j, k): return i + j * (self._nx - 1) + k * (self._nx - 1) * (self._ny - 1)
    def face(self, i, j, k): return i + j * self._nx + k * self._nx * self._ny

    def cell_shape(self):  # numpy (k, j, i) view shape of a cell array
        return (self._nz - 1, self._ny - 1, self._nx - 1)

    def face_shape(self):
        return (self._nz, self._ny, self._nx)

    def grid_struct(self) -> Grid:
        Nx, Ny, Nz = self.base
        g = Grid(Nx, Ny, Nz, float(self._dx), float(self._dy),
                 self.dz_array.ctypes.data_as(_FP))
        g._keep = self.dz_array
        return g


# ---------------------------------------------------------------------------
# WINDSGeneralData mirror: only the fields the solve reads and writes
# (src/winds/WINDSGeneralData.h:231-274).
# ---------------------------------------------------------------------------
class WINDSGeneralData:
    FIELDS_CELL = ("e", "f", "g", "h", "m", "n")
    FIELDS_FACE = ("u0", "v0", "w0", "u", "v", "w")

    def __init__(self, domain: Domain):
        self.domain = domain
        nc, nf = domain.numCellCentered(), domain.numFaceCentered()
        for name in self.FIELDS_CELL:
            setattr(self, name, np.ones(nc, dtype=np.float32))
        self.icellflag = np.ones(nc, dtype=np.int32)
        for name in self.FIELDS_FACE:
            setattr(self, name, np.zeros(nf, dtype=np.float32))

    def inputs(self):
        return (self.e, self.f, self.g, self.h, self.m, self.n, self.icellflag,
                self.u0, self.v0, self.w0)


# ---------------------------------------------------------------------------
# Solver mirror
# ---------------------------------------------------------------------------
class Solver_B200:
    """Solver(qes::Domain, const float &tol) backed by the B200 kernels.

    solve(WGD, itermax) has Solver::solve's semantics: it reads e..n,
    icellflag, u0, v0, w0 from WGD and writes WGD.u, WGD.v, WGD.w. lambda
    persists between calls until resetLambda(), as in the reference CPU solvers.
    """

    omega = 1.78  # src/winds/Solver.h:83
    alpha1 = alpha2 = 1

    def __init__(self, domain: Domain, tol: float, device: int = 0):
        self.domain = domain
        self.tol = np.float32(tol)
        self._h = C.c_void_p()
        g = domain.grid_struct()
        check(lib().qesb_create(C.byref(g), float(self.tol), device, C.byref(self._h)))
        self._inputs_id = None
        self.last_stats: dict | None = None

    def close(self):
        if self._h:
            lib().qesb_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # Solver::resetLambda
    def resetLambda(self):
        check(lib().qesb_reset_lambda(self._h))

    def set_option(self, key: str, value: int):
        check(lib().qesb_set_option(self._h, key.encode(), int(value)))

    def set_prephase(self, omega: float, tol: float = 1e-3, max_iterations: int = 10000):
        """Over-relaxed SOR pre-phase before the reference loop (omega 0: off)."""
        check(lib().qesb_set_prephase(self._h, float(omega), float(tol), int(max_iterations)))

    def set_prephase_start(self, omega: float, iterations: int):
        """Start stage of the pre-phase: its first `iterations` sweeps at this
        omega (iterations 0: none)."""
        check(lib().qesb_set_prephase_start(self._h, float(omega), int(iterations)))

    def set_window_rule(self, window: int, tol: float = 0.0):
        """Window stopping rule: the reference loop also stops after every
        window-th iteration n when FP64 max|lambda_n - lambda_(n-window)| <= tol
        (window 0: off, the reference's rule alone)."""
        check(lib().qesb_set_window_rule(self._h, int(window), float(tol)))

    def fp64_same_sor(self, pre_omega: float, pre_iterations: int, iterations: int, u_ptr=None, v_ptr=None,
                      w_ptr=None, want_lambda: bool = False, lambda0: np.ndarray | None = None) -> dict:
        """qesb_fp64_same_sor: the same red-black SOR replayed in FP64 on the
        device from lambda0 (None: zero) with a solve's pre-phase and
        reference-loop iteration counts, and the errors of the handle's FP32
        lambda and of the given FP32 winds (device pointers) against it."""
        rep = Fp64Report()
        lam = np.empty(self.domain.numCellCentered(), np.float64) if want_lambda else None
        l0 = None if lambda0 is None else np.ascontiguousarray(lambda0, np.float32)
        check(lib().qesb_fp64_same_sor(self._h, _ptr(l0), float(pre_omega), int(pre_iterations), int(iterations),
                                       u_ptr, v_ptr, w_ptr, _ptr(lam), C.byref(rep)))
        out = rep.as_dict()
        out["lambda_max_rel_err"] = out["lambda_max_abs_err"] / max(out["lambda_max_abs"], 1e-30)
        if want_lambda:
            out["lambda64"] = lam
        return out

    def set_tolerance(self, tol: float):
        self.tol = np.float32(tol)
        check(lib().qesb_set_tolerance(self._h, float(self.tol)))

    def set_inputs(self, WGD: WINDSGeneralData):
        arrs = [np.ascontiguousarray(a) for a in WGD.inputs()]
        check(lib().qesb_set_inputs(self._h, *[_ptr(a) for a in arrs]))

    def set_inputs_flags(self, WGD: WINDSGeneralData):
        """qesb_set_inputs_flags: icellflag and u0, v0, w0 only; the stair-step
        wall coefficients computed from the flags on the device."""
        arrs = [np.ascontiguousarray(a) for a in (WGD.icellflag, WGD.u0, WGD.v0, WGD.w0)]
        check(lib().qesb_set_inputs_flags(self._h, *[_ptr(a) for a in arrs]))

    def set_inputs_device(self, e, f, g, h, m, n, icellflag, u0, v0, w0):
        """Device pointers (ints) in the reference layouts."""
        check(lib().qesb_set_inputs_device(self._h, e, f, g, h, m, n, icellflag, u0, v0, w0))

    # Solver::solve
    def solve(self, WGD: WINDSGeneralData, itermax: int, set_inputs: bool = True) -> dict:
        if set_inputs:
            self.set_inputs(WGD)
        st = Stats()
        check(lib().qesb_solve(self._h, int(itermax), _ptr(WGD.u), _ptr(WGD.v), _ptr(WGD.w),
                               C.byref(st)))
        self.last_stats = st.as_dict()
        return self.last_stats

    def solve_device(self, itermax: int, u_ptr, v_ptr, w_ptr) -> dict:
        st = Stats()
        check(lib().qesb_solve_device(self._h, int(itermax), u_ptr, v_ptr, w_ptr, C.byref(st)))
        self.last_stats = st.as_dict()
        return self.last_stats

    def wall_log_law(self, z0: float, dz: float, u_ptr, v_ptr, w_ptr) -> None:
        """qesb_wall_log_law: the log-law wall treatment (Wall::wallLogBC's
        stair-step part) in place on device wind arrays (pointers as ints)."""
        check(lib().qesb_wall_log_law(self._h, float(z0), float(dz), u_ptr, v_ptr, w_ptr))

    @property
    def lambda_(self) -> np.ndarray:
        out = np.empty(self.domain.numCellCentered(), dtype=np.float32)
        check(lib().qesb_get_lambda(self._h, _ptr(out)))
        return out

    @lambda_.setter
    def lambda_(self, value: np.ndarray):
        a = np.ascontiguousarray(value, dtype=np.float32)
        assert a.size == self.domain.numCellCentered()
        check(lib().qesb_set_lambda(self._h, _ptr(a)))

    def time_sweeps(self, n: int) -> tuple[float, int]:
        """Device ms of n back-to-back fused-sweep launches, and iterations per launch."""
        ms, k = C.c_float(), C.c_int()
        check(lib().qesb_time_sweeps(self._h, int(n), C.byref(ms), C.byref(k)))
        return ms.value, k.value

    def autotune(self) -> tuple[int, list[float]]:
        """Times every sweep variant on the current inputs; returns the chosen
        index and the microseconds per iteration of each."""
        n = lib().qesb_num_variants()
        us = (C.c_float * n)()
        best = C.c_int()
        check(lib().qesb_autotune(self._h, C.byref(best), us, n))
        return best.value, list(us)

    def set_stream(self, stream_ptr: int | None):
        check(lib().qesb_set_stream(self._h, stream_ptr))

    def stream_ptr(self) -> int:
        """The cudaStream_t the handle's work runs on."""
        out = C.c_void_p()
        check(lib().qesb_get_stream(self._h, C.byref(out)))
        return out.value or 0

    def residual_history(self, n: int) -> np.ndarray:
        out = np.empty(n, dtype=np.float64)
        check(lib().qesb_get_residual_history(self._h, _ptr(out), int(n)))
        return out

    @property
    def R(self) -> np.ndarray:
        out = np.empty(self.domain.numCellCentered(), dtype=np.float32)
        check(lib().qesb_get_divergence(self._h, _ptr(out)))
        return out


def workspace_write(path: str, wgd: "WINDSGeneralData", t: float = 0.0) -> None:
    """qesb_workspace_write: wgd's winds, inputs and grid as a workspace file
    (NetCDF classic) with the reference's variable names and layouts."""
    g = wgd.domain.grid_struct()
    arrs = [np.ascontiguousarray(a) for a in (wgd.u, wgd.v, wgd.w, wgd.u0, wgd.v0, wgd.w0, wgd.icellflag,
                                              wgd.e, wgd.f, wgd.g, wgd.h, wgd.m, wgd.n)]
    check(lib().qesb_workspace_write(os.fsencode(path), C.byref(g), float(t), *[_ptr(a) for a in arrs]))


def workspace_read(path: str) -> "WINDSGeneralData":
    """qesb_workspace_read: a workspace file (NetCDF classic) as a
    WINDSGeneralData on its own grid (dz_array from the file)."""
    Nx, Ny, Nz, dx, dy = C.c_int(), C.c_int(), C.c_int(), C.c_float(), C.c_float()
    check(lib().qesb_workspace_dims(os.fsencode(path), C.byref(Nx), C.byref(Ny), C.byref(Nz), C.byref(dx),
                                    C.byref(dy)))
    dz = np.empty(Nz.value + 1, dtype=np.float32)
    check(lib().qesb_workspace_read(os.fsencode(path), Nx.value, Ny.value, Nz.value, _ptr(dz),
                                    *[None] * 13))
    d = Domain(Nx.value, Ny.value, Nz.value, dx.value, dy.value, float(dz.min()), dz)
    w = WINDSGeneralData(d)
    check(lib().qesb_workspace_read(os.fsencode(path), Nx.value, Ny.value, Nz.value, None,
                                    *[_ptr(a) for a in (w.icellflag, w.e, w.f, w.g, w.h, w.m, w.n, w.u0, w.v0,
                                                        w.w0, w.u, w.v, w.w)]))
    return w


def autotune_batch(solvers) -> tuple[int, list[float]]:
    """qesb_autotune_batch: times every sweep launch shape on the domain list
    qesb_solve_batch would run for these solvers (inputs set), keeps the
    fastest as solvers[0]'s "batch_variant" option, and returns it with each
    shape's microseconds per iteration over the list (0 for the fused tile
    shapes, which batches do not use)."""
    n = len(solvers)
    V = C.c_void_p
    hs = (V * n)(*[s._h for s in solvers])
    nv = lib().qesb_num_variants()
    us = (C.c_float * nv)()
    best = C.c_int()
    check(lib().qesb_autotune_batch(hs, n, C.byref(best), us, nv))
    return best.value, list(us)


def solve_batch(solvers, itermax: int, u_ptrs=None, v_ptrs=None, w_ptrs=None) -> list[dict]:
    """qesb_solve_batch: the solvers' domains (inputs already set, lambda as the
    start) solved together; u/v/w_ptrs are lists of device pointers (ints) or
    None. Returns each domain's stats."""
    n = len(solvers)
    V = C.c_void_p
    hs = (V * n)(*[s._h for s in solvers])

    def ptrs(p):
        return None if p is None else (V * n)(*p)

    st = (Stats * n)()
    check(lib().qesb_solve_batch(hs, n, int(itermax), ptrs(u_ptrs), ptrs(v_ptrs), ptrs(w_ptrs), st))
    out = [st[i].as_dict() for i in range(n)]
    for s, d in zip(solvers, out):
        s.last_stats = d
    return out


def solve_noalloc(domain: Domain, tol: float, itermax: int, e, f, g, h, m, n, icellflag, u0, v0, w0,
                  lam, u, v, w, stream=None) -> dict:
    """qesb_solve_noalloc: device pointers (ints) in the reference layouts;
    lam is read and updated in place. Allocates nothing on the device."""
    st = Stats()
    gs = domain.grid_struct()
    check(lib().qesb_solve_noalloc(C.byref(gs), float(np.float32(tol)), int(itermax), e, f, g, h, m, n,
                                   icellflag, u0, v0, w0, lam, u, v, w, stream, C.byref(st)))
    return st.as_dict()


class SolverFactory:
    """SolverFactory::create (src/winds/SolverFactory.cpp:35-60) with the B200 type.

    This package builds only the B200 solver; asking it for another type is
    the reference's "Invalid solver type" error."""

    @staticmethod
    def create(solveType: int, domain: Domain, tolerance: float) -> Solver_B200:
        if solveType == B200_Type:
            return Solver_B200(domain, tolerance)
        raise QesbError(1, "Invalid solver type")


# ---------------------------------------------------------------------------
# synthetic cities
# ---------------------------------------------------------------------------
def city_dz(Nz: int, dz0: float, ratio: float) -> np.ndarray:
    dz = np.empty(Nz + 1, dtype=np.float32)
    check(lib().qesb_city_dz(Nz, dz0, ratio, dz.ctypes.data_as(_FP)))
    return dz


def city_build(domain: Domain, buildings, inflow: Inflow) -> WINDSGeneralData:
    """WINDSGeneralData with flags, wall coefficients and power-law inflow set."""
    wgd = WINDSGeneralData(domain)
    nb = len(buildings)
    arr = (Building * max(nb, 1))(*buildings)
    g = domain.grid_struct()
    check(lib().qesb_city_build(C.byref(g), nb, arr, C.byref(inflow),
                                *[_ptr(a) for a in (wgd.icellflag, wgd.e, wgd.f, wgd.g, wgd.h,
                                                    wgd.m, wgd.n, wgd.u0, wgd.v0, wgd.w0)]))
    return wgd


def city_build_device(domain: Domain, buildings, inflow: Inflow, arrays: dict, stream=None):
    """qesb_city_build_device into device arrays: `arrays` maps icellflag, e,
    f, g, h, m, n, u0, v0, w0 to device pointers (ints) in the reference
    layouts."""
    nb = len(buildings)
    arr = (Building * max(nb, 1))(*buildings)
    g = domain.grid_struct()
    names = ("icellflag", "e", "f", "g", "h", "m", "n", "u0", "v0", "w0")
    check(lib().qesb_city_build_device(C.byref(g), nb, arr, C.byref(inflow), *[arrays[k] for k in names], stream))


def city_inflow(wgd: WINDSGeneralData, inflow: Inflow) -> WINDSGeneralData:
    """A copy of wgd sharing its flags and coefficients, with u0, v0, w0 of
    another inflow over the same buildings."""
    out = WINDSGeneralData(wgd.domain)
    out.icellflag, out.e, out.f, out.g, out.h, out.m, out.n = (wgd.icellflag, wgd.e, wgd.f, wgd.g, wgd.h,
                                                                wgd.m, wgd.n)
    g = wgd.domain.grid_struct()
    check(lib().qesb_city_inflow(C.byref(g), _ptr(wgd.icellflag), C.byref(inflow), _ptr(out.u0), _ptr(out.v0),
                                 _ptr(out.w0)))
    return out


def prephase_omega(Nx: int, Ny: int) -> float:
    """Over-relaxation factor for the warm-start pre-phase on an Nx x Ny
    stretched-z city grid: 2 - 7.5 / max(Nx, Ny), within [1.85, 1.97]
    (measured best: 1.95 at 128, 1.97 at 256; 1.98 stalls at 256)."""
    return float(min(1.97, max(1.85, 2.0 - 7.5 / max(Nx, Ny))))


@dataclass
class City:
    domain: Domain
    buildings: list
    inflow: Inflow
    seed: int


def city_random(domain: Domain, seed: int, max_buildings: int, fp=(10.0, 40.0),
                h=(10.0, 60.0)) -> City:
    buf = (Building * max(max_buildings, 1))()
    n = C.c_int()
    inf = Inflow()
    g = domain.grid_struct()
    check(lib().qesb_city_random(C.byref(g), seed, max_buildings, fp[0], fp[1], h[0], h[1], buf,
                                 C.byref(n), C.byref(inf)))
    return City(domain, [buf[i] for i in range(n.value)], inf, seed)


# ---------------------------------------------------------------------------
# the benchmark configurations (grid + generator parameters)
# ---------------------------------------------------------------------------
def config_domain(name: str) -> Domain:
    """Grids of the named workloads (sizes Nx x Ny x Nz)."""
    if name == "cuboid100":      # 100x100x50, dx=dy=dz=1 m
        return Domain(100, 100, 50, 1.0, 1.0, 1.0)
    if name == "city400":        # 400x400x100, dx=dy=2 m, dz 1 m x 1.03^k
        return Domain(400, 400, 100, 2.0, 2.0, 1.0, city_dz(100, 1.0, 1.03))
    if name == "city800":        # 800x800x128, same generator
        return Domain(800, 800, 128, 2.0, 2.0, 1.0, city_dz(128, 1.0, 1.03))
    if name == "city128":        # 128x128x64 training domains
        return Domain(128, 128, 64, 2.0, 2.0, 1.0, city_dz(64, 1.0, 1.03))
    if name == "city256":        # 256x256x64 evaluation domains
        return Domain(256, 256, 64, 2.0, 2.0, 1.0, city_dz(64, 1.0, 1.03))
    raise KeyError(name)


def cuboid100() -> WINDSGeneralData:
    """One 20x20x20 m cuboid centred in a 100x100x50 m domain; inflow
    u = 5 m/s (z/10 m)^0.15 from 270 deg."""
    d = config_domain("cuboid100")
    return city_build(d, [Building(40.0, 40.0, 20.0, 20.0, 20.0, 0.0)], Inflow(5.0, 10.0, 0.15, 270.0))


def random_city(name: str, seed: int) -> tuple[WINDSGeneralData, City]:
    counts = {"city400": (60, 60), "city800": (150, 150), "city128": (20, 40), "city256": (40, 80)}
    d = config_domain(name)
    lo, hi = counts[name]
    nb = lo if lo == hi else lo + (seed * 2654435761 % (hi - lo + 1))
    c = city_random(d, seed, nb)
    return city_build(d, c.buildings, c.inflow), c
