"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke(), and
bench.py's CPU-baseline / reference legs). The product never imports it.

Two checkers, loaded with ctypes:
  port  — oracle/_build/libqesoracle.so, the plain-C restatement in
          oracle/qes_oracle.c (always available once oracle/Makefile ran);
  ref   — oracle/_ref/libqesref.so, the reference's own Solver_CPU,
          Solver_CPU_RB and Wall code compiled from its sources with the shim
          headers in oracle/shim (built only where the reference tree exists;
          the built library travels with the repository copy).
Arrays are numpy, in the reference layouts (see include/qesb.h).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(HERE, "_build", "libqesoracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libqesref.so")
REF_GPU_PATH = os.path.join(HERE, "_ref", "libqesref_gpu.so")

_V = C.c_void_p
_port = None
_ref = None
_ref_gpu = None


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_V)


def port() -> C.CDLL:
    global _port
    if _port is None:
        L = C.CDLL(PORT_PATH)
        i, f, d = C.c_int, C.c_float, C.c_double
        L.qo_divergence.argtypes = [i, i, i, f, f] + [_V] * 11
        L.qo_divergence.restype = None
        L.qo_sor.argtypes = [i, i, i, i, i] + [_V] * 8 + [f, i, _V, _V]
        L.qo_sor.restype = i
        L.qo_sor_omega.argtypes = [i, i, i, i, i] + [_V] * 8 + [f, i, _V, _V, f]
        L.qo_sor_omega.restype = i
        L.qo_sor_window.argtypes = [i, i, i, i, i] + [_V] * 8 + [f, i, _V, _V, f, i, d, _V, _V]
        L.qo_sor_window.restype = i
        L.qo_sor_rb_f64_omega.argtypes = [i, i, i] + [_V] * 8 + [d, i, _V, d]
        L.qo_sor_rb_f64_omega.restype = i
        L.qo_correct.argtypes = [i, i, i, f, f] + [_V] * 11
        L.qo_correct.restype = None
        L.qo_divergence_f64.argtypes = [i, i, i, f, f] + [_V] * 11
        L.qo_divergence_f64.restype = None
        L.qo_sor_rb_f64.argtypes = [i, i, i] + [_V] * 8 + [d, i, _V]
        L.qo_sor_rb_f64.restype = i
        L.qo_correct_f64.argtypes = [i, i, i, f, f] + [_V] * 11
        L.qo_correct_f64.restype = None
        L.qo_max_divergence.argtypes = [i, i, i, f, f] + [_V] * 5 + [i]
        L.qo_max_divergence.restype = d
        L.qo_wall_log.argtypes = [i, i, i, f, f, f] + [_V] * 4
        L.qo_wall_log.restype = i
        _port = L
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(REF_PATH)
        i, f = C.c_int, C.c_float
        L.qesref_walls.argtypes = [i, i, i, f, f] + [_V] * 8
        L.qesref_walls.restype = i
        L.qesref_set_velocity_zero.argtypes = [i, i, i, f, f] + [_V] * 5
        L.qesref_set_velocity_zero.restype = i
        L.qesref_solve.argtypes = [i, i, i, i, f, f] + [_V] * 11 + [f, i] + [_V] * 5
        L.qesref_solve.restype = C.c_double
        L.qesref_wall_log_bc.argtypes = [i, i, i, f, f, _V, _V, f, _V, _V, _V]
        L.qesref_wall_log_bc.restype = i
        L.qesref_set_threads.argtypes = [i]
        L.qesref_set_threads.restype = None
        L.qr_rect_building_flags.argtypes = [i, i, i, f, f, _V, i, _V, _V, _V]
        L.qr_rect_building_flags.restype = i
        L.qesref_set_threads(1)
        _ref = L
    return _ref


def _dims(dom):
    Nx, Ny, Nz = dom.base
    return Nx, Ny, Nz, dom.dx(), dom.dy()


# ----------------------------------------------------------------------------- port
def divergence(dom, w):
    R = np.zeros(dom.numCellCentered(), np.float32)
    port().qo_divergence(*_dims(dom), _p(dom.dz_array), _p(w.e), _p(w.f), _p(w.g), _p(w.h),
                         _p(w.m), _p(w.n), _p(w.u0), _p(w.v0), _p(w.w0), _p(R))
    return R


def sor(dom, w, R, tol, itermax, ordering=1, err_fp64=True, lam=None, hist=False, omega=None):
    """Returns (lambda, iterations, final_error, history-or-None). omega:
    None for the reference's 1.78f, else the float omega of an over-relaxed
    pre-phase."""
    Nx, Ny, Nz = dom.base
    L = np.zeros(dom.numCellCentered(), np.float32) if lam is None else lam.astype(np.float32).copy()
    H = np.zeros(max(itermax, 1), np.float64) if hist else None
    fe = C.c_double()
    args = (ordering, int(err_fp64), Nx, Ny, Nz, _p(w.e), _p(w.f), _p(w.g), _p(w.h), _p(w.m), _p(w.n), _p(R),
            _p(L), float(np.float32(tol)), int(itermax), C.byref(fe), _p(H))
    if omega is None:
        it = port().qo_sor(*args)
    else:
        it = port().qo_sor_omega(*args, float(np.float32(omega)))
    return L, it, fe.value, (H[:it] if hist else None)


def sor_window(dom, w, R, tol, itermax, window, wtol, lam=None, omega=None, ordering=1):
    """SOR with the solver's window rule (qo_sor_window): returns (lambda,
    iterations, stop kind 0/1/2 for itermax/tol/window, last window drift)."""
    Nx, Ny, Nz = dom.base
    L = np.zeros(dom.numCellCentered(), np.float32) if lam is None else lam.astype(np.float32).copy()
    fe, stop, drift = C.c_double(), C.c_int(), C.c_double()
    it = port().qo_sor_window(ordering, 1, Nx, Ny, Nz, _p(w.e), _p(w.f), _p(w.g), _p(w.h), _p(w.m), _p(w.n),
                              _p(R), _p(L), float(np.float32(tol)), int(itermax), C.byref(fe), None,
                              float(np.float32(1.78 if omega is None else omega)), int(window), float(wtol),
                              C.byref(stop), C.byref(drift))
    return L, it, stop.value, drift.value


def correct(dom, w, L):
    nf = dom.numFaceCentered()
    u, v, ww = (np.zeros(nf, np.float32) for _ in range(3))
    port().qo_correct(*_dims(dom), _p(dom.dz_array), _p(w.f), _p(w.h), _p(w.n), _p(w.icellflag),
                      _p(L), _p(w.u0), _p(w.v0), _p(w.w0), _p(u), _p(v), _p(ww))
    return u, v, ww


def solve(dom, w, tol, itermax, ordering=1, err_fp64=True, lam=None):
    """Full reference-semantics solve on the port: (u, v, w, lambda, iters, err)."""
    R = divergence(dom, w)
    L, it, fe, _ = sor(dom, w, R, tol, itermax, ordering, err_fp64, lam)
    u, v, ww = correct(dom, w, L)
    return u, v, ww, L, it, fe


def solve_f64(dom, w, tol, itermax, phases=None):
    """FP64 run of the same red-black SOR: (u, v, w, lambda, iters, err) in double.
    phases: optional [(omega, tol, itermax), ...] run in order before the
    reference loop (the solver's over-relaxed pre-phase); omega is taken as
    the float the GPU uses, widened to double."""
    Nx, Ny, Nz = dom.base
    nc, nf = dom.numCellCentered(), dom.numFaceCentered()
    R = np.zeros(nc, np.float64)
    port().qo_divergence_f64(*_dims(dom), _p(dom.dz_array), _p(w.e), _p(w.f), _p(w.g), _p(w.h),
                             _p(w.m), _p(w.n), _p(w.u0), _p(w.v0), _p(w.w0), _p(R))
    L = np.zeros(nc, np.float64)
    fe = C.c_double()
    for om, ptol, pit in (phases or ()):
        port().qo_sor_rb_f64_omega(Nx, Ny, Nz, _p(w.e), _p(w.f), _p(w.g), _p(w.h), _p(w.m), _p(w.n), _p(R),
                                   _p(L), float(ptol), int(pit), C.byref(fe), float(np.float32(om)))
    it = port().qo_sor_rb_f64(Nx, Ny, Nz, _p(w.e), _p(w.f), _p(w.g), _p(w.h), _p(w.m), _p(w.n),
                              _p(R), _p(L), float(tol), int(itermax), C.byref(fe))
    u, v, ww = (np.zeros(nf, np.float64) for _ in range(3))
    port().qo_correct_f64(*_dims(dom), _p(dom.dz_array), _p(w.f), _p(w.h), _p(w.n),
                          _p(w.icellflag), _p(L), _p(w.u0), _p(w.v0), _p(w.w0), _p(u), _p(v),
                          _p(ww))
    return u, v, ww, L, it, fe.value


def max_divergence(dom, flag, u, v, w, kmax=None):
    Nx, Ny, Nz = dom.base
    if kmax is None:
        kmax = dom.nz() - 4
    u, v, w = (np.ascontiguousarray(a, np.float32) for a in (u, v, w))
    return port().qo_max_divergence(*_dims(dom), _p(dom.dz_array), _p(flag), _p(u), _p(v), _p(w),
                                    int(kmax))


# ----------------------------------------------------------------------------- reference
def ref_set_threads(n: int) -> None:
    """OpenMP threads for Solver_CPU_RB (1 by default: see qesref_set_threads)."""
    ref().qesref_set_threads(int(n))


def ref_walls(dom, icellflag):
    """Reference Wall::defineWalls + solverCoefficients: (icellflag, e, f, g, h, m, n)."""
    nc = dom.numCellCentered()
    flag = icellflag.astype(np.int32).copy()
    outs = [np.zeros(nc, np.float32) for _ in range(6)]
    ref().qesref_walls(*_dims(dom), _p(dom.dz_array), _p(flag), *[_p(a) for a in outs])
    return (flag, *outs)


def ref_rect_building_flags(dom, buildings, icellflag):
    """The reference's own building rasterisation (RectangularBuilding::parseValues,
    PolyBuilding::setPolyBuilding and setCellFlags, stair-step): buildings as rows of
    (x_start, y_start, length, width, height, base height), rotation 0, applied in order
    to a copy of icellflag; returns (icellflag, ibuilding_flag)."""
    b = np.ascontiguousarray(np.asarray(buildings, np.float32).reshape(-1, 6))
    flag = icellflag.astype(np.int32).copy()
    ib = np.zeros_like(flag)
    ref().qr_rect_building_flags(*_dims(dom), _p(dom.dz_array), len(b), _p(b), _p(flag), _p(ib))
    return flag, ib


def ref_set_velocity_zero(dom, icellflag, u0, v0, w0):
    u0, v0, w0 = (a.astype(np.float32).copy() for a in (u0, v0, w0))
    ref().qesref_set_velocity_zero(*_dims(dom), _p(dom.dz_array), _p(icellflag), _p(u0), _p(v0),
                                   _p(w0))
    return u0, v0, w0


def wall_log(dom, icellflag, z0, u, v, w, dz=None):
    """The stair-step log-law wall treatment (qo_wall_log) on copies of u, v,
    w; dz defaults to min(dz_array), the nominal dz of the reference domain
    the tests build. Returns (u, v, w), or None for cut-cell flags."""
    u, v, w = (np.ascontiguousarray(a, dtype=np.float32).copy() for a in (u, v, w))
    dz = float(np.min(dom.dz_array)) if dz is None else dz
    r = port().qo_wall_log(*dom.base, float(dom.dx()), dz, float(z0),
                           _p(np.ascontiguousarray(icellflag, dtype=np.int32)), _p(u), _p(v), _p(w))
    return None if r != 0 else (u, v, w)


def ref_wall_log_bc(dom, icellflag, z0, u, v, w):
    """The reference's Wall::defineWalls + Wall::wallLogBC(WGD, true) on copies
    of u, v, w (the reference build). Returns (u, v, w, flags after defineWalls)."""
    u, v, w = (np.ascontiguousarray(a, dtype=np.float32).copy() for a in (u, v, w))
    flag = np.ascontiguousarray(icellflag, dtype=np.int32).copy()
    ref().qesref_wall_log_bc(*_dims(dom), _p(dom.dz_array), _p(flag), float(z0), _p(u), _p(v), _p(w))
    return u, v, w, flag


def ref_solve(dom, w, tol, itermax, kind=0, lam=None, want_lambda=True):
    """Reference Solver::solve. kind 0 = Solver_CPU, 1 = Solver_CPU_RB.
    Returns (u, v, w, lambda-or-None, seconds)."""
    nc, nf = dom.numCellCentered(), dom.numFaceCentered()
    u, v, ww = (np.zeros(nf, np.float32) for _ in range(3))
    L = np.zeros(nc, np.float32) if want_lambda else None
    lam = None if lam is None else np.ascontiguousarray(lam, np.float32)
    t = ref().qesref_solve(kind, *_dims(dom), _p(dom.dz_array), _p(w.e), _p(w.f), _p(w.g),
                           _p(w.h), _p(w.m), _p(w.n), _p(w.icellflag), _p(w.u0), _p(w.v0),
                           _p(w.w0), float(tol), int(itermax), _p(lam), _p(u), _p(v), _p(ww),
                           _p(L))
    return u, v, ww, L, t


# ----------------------------------------------------------------------------- reference GPU solver
def ref_gpu_available() -> bool:
    return os.path.exists(REF_GPU_PATH)


def ref_gpu() -> C.CDLL:
    global _ref_gpu
    if _ref_gpu is None:
        L = C.CDLL(REF_GPU_PATH)
        i, f = C.c_int, C.c_float
        L.qesref_solve_gpu.argtypes = [i, i, i, f, f] + [_V] * 11 + [f, i] + [_V] * 3
        L.qesref_solve_gpu.restype = C.c_double
        _ref_gpu = L
    return _ref_gpu


def capture_stdout(fn):
    """Runs fn with file descriptor 1 redirected; returns (result, text)."""
    import sys
    import tempfile

    fd = sys.stdout.fileno()
    sys.stdout.flush()
    saved = os.dup(fd)
    with tempfile.TemporaryFile(mode="w+") as tmp:
        os.dup2(tmp.fileno(), fd)
        try:
            res = fn()
        finally:
            sys.stdout.flush()
            os.dup2(saved, fd)
            os.close(saved)
        tmp.seek(0)
        return res, tmp.read()


def ref_solve_gpu(dom, w, tol, itermax):
    """The reference's Solver_GPU_GlobalMemory::solve (timing comparator).
    Returns (u, v, w, seconds, iterations)."""
    import re

    nf = dom.numFaceCentered()
    u, v, ww = (np.zeros(nf, np.float32) for _ in range(3))
    t, text = capture_stdout(lambda: ref_gpu().qesref_solve_gpu(
        *_dims(dom), _p(dom.dz_array), _p(w.e), _p(w.f), _p(w.g), _p(w.h), _p(w.m), _p(w.n),
        _p(w.icellflag), _p(w.u0), _p(w.v0), _p(w.w0), float(tol), int(itermax), _p(u), _p(v), _p(ww)))
    if t < 0:
        raise ValueError("reference GPU solver not run on this grid: its dz over-read could cross a page")
    m = re.findall(r"Residual after (\d+) itertations", text)
    return u, v, ww, t, int(m[-1]) if m else -1
