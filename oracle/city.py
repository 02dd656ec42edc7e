"""ORACLE — test infrastructure only (tests/ and bench.py's reference leg).

The benchmark's synthetic cities built without the product library: the
seeded layout, building flags and power-law inflow from the oracle's C
restatement (qo_city_random, qo_city_flags, qo_city_inflow in
oracle/qes_oracle.c), the wall coefficients and solid-face zeroing from the
reference's own Wall.cpp (oracle/_ref: Wall::defineWalls +
Wall::solverCoefficients, Wall::setVelocityZero). tests/test_generator.py
checks these inputs against the product generator's bit for bit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import oracle as O

_V = C.c_void_p
_sig_done = False


def _lib():
    global _sig_done
    L = O.port()
    if not _sig_done:
        i, f = C.c_int, C.c_float
        L.qo_city_random.argtypes = [i, i, f, f, C.c_uint64, i, f, f, f, f, _V, _V]
        L.qo_city_random.restype = i
        L.qo_city_flags.argtypes = [i, i, i, f, f, _V, i, _V, _V]
        L.qo_city_flags.restype = None
        L.qo_city_inflow.argtypes = [i, i, i, _V, _V, _V, _V, _V]
        L.qo_city_inflow.restype = None
        _sig_done = True
    return L


def _p(a):
    return a.ctypes.data_as(_V)


class Domain:
    """The grid quantities the oracle and the reference build need (the
    layout of qes::Domain, src/qes/Domain.cpp:7-31): base counts, dx, dy and
    dz_array (nz-1 values, ghost layer at 0)."""

    def __init__(self, Nx, Ny, Nz, dx, dy, dz_array):
        self.base = (Nx, Ny, Nz)
        self._dx, self._dy = float(np.float32(dx)), float(np.float32(dy))
        self.dz_array = np.ascontiguousarray(dz_array, np.float32)

    def dx(self):
        return self._dx

    def dy(self):
        return self._dy

    def nx(self):
        return self.base[0] + 1

    def ny(self):
        return self.base[1] + 1

    def nz(self):
        return self.base[2] + 2

    def numCellCentered(self):
        Nx, Ny, Nz = self.base
        return Nx * Ny * (Nz + 1)

    def numFaceCentered(self):
        Nx, Ny, Nz = self.base
        return (Nx + 1) * (Ny + 1) * (Nz + 2)


class Inputs:
    """The WINDSGeneralData fields the solve reads."""

    def __init__(self, domain):
        self.domain = domain


def stretched_dz(Nz, dz0, ratio):
    """dz[k] = dz0 ratio^(k-1) for k >= 1 (dz0 and ratio as floats, the
    product formed in double and rounded per entry), dz[0] = dz[1]."""
    dz = np.empty(Nz + 1, np.float32)
    d = float(np.float32(dz0))
    r = float(np.float32(ratio))
    for k in range(1, Nz + 1):
        dz[k] = np.float32(d)
        d *= r
    dz[0] = dz[1]
    return dz


# grids and building counts of the benchmark workloads (Nx, Ny, Nz, dx, dy, dz0, ratio)
GRIDS = {"city128": (128, 128, 64, 2.0, 2.0, 1.0, 1.03), "city256": (256, 256, 64, 2.0, 2.0, 1.0, 1.03),
         "city400": (400, 400, 100, 2.0, 2.0, 1.0, 1.03), "city800": (800, 800, 128, 2.0, 2.0, 1.0, 1.03)}
COUNTS = {"city128": (20, 40), "city256": (40, 80), "city400": (60, 60), "city800": (150, 150)}


def domain(name):
    Nx, Ny, Nz, dx, dy, dz0, ratio = GRIDS[name]
    return Domain(Nx, Ny, Nz, dx, dy, stretched_dz(Nz, dz0, ratio))


def city_layout(dom, seed, max_buildings, fp=(10.0, 40.0), h=(10.0, 60.0)):
    """(buildings [n][6], inflow [4]) of the seed's city."""
    Nx, Ny, _ = dom.base
    b = np.zeros((max(max_buildings, 1), 6), np.float32)
    inflow = np.zeros(4, np.float32)
    n = _lib().qo_city_random(Nx, Ny, dom.dx(), dom.dy(), int(seed), int(max_buildings), fp[0], fp[1], h[0], h[1],
                              _p(b), _p(inflow))
    return b[:n].copy(), inflow


def city_flags(dom, buildings):
    """The restatement's cell flags of a city (qo_city_flags): fluid 1, ground
    plane 2, then each building's stair-step cells 0, in order."""
    Nx, Ny, Nz = dom.base
    flag = np.empty(dom.numCellCentered(), np.int32)
    b = np.ascontiguousarray(buildings, np.float32)
    _lib().qo_city_flags(Nx, Ny, Nz, dom.dx(), dom.dy(), _p(dom.dz_array), len(b), _p(b) if len(b) else None,
                         _p(flag))
    return flag


def city_inputs(dom, buildings, inflow):
    """Inputs of a city: flags and inflow from the restatement, wall
    coefficients and solid faces from the reference build."""
    Nx, Ny, Nz = dom.base
    flag = np.empty(dom.numCellCentered(), np.int32)
    b = np.ascontiguousarray(buildings, np.float32)
    _lib().qo_city_flags(Nx, Ny, Nz, dom.dx(), dom.dy(), _p(dom.dz_array), len(b), _p(b) if len(b) else None,
                         _p(flag))
    nf = dom.numFaceCentered()
    u0, v0, w0 = (np.empty(nf, np.float32) for _ in range(3))
    _lib().qo_city_inflow(Nx, Ny, Nz, _p(dom.dz_array), _p(np.ascontiguousarray(inflow, np.float32)), _p(u0),
                          _p(v0), _p(w0))
    w = Inputs(dom)
    w.icellflag, w.e, w.f, w.g, w.h, w.m, w.n = O.ref_walls(dom, flag)
    w.u0, w.v0, w.w0 = O.ref_set_velocity_zero(dom, w.icellflag, u0, v0, w0)
    return w


def random_city(name, seed):
    """The benchmark city `name` for `seed` (as the product's random_city)."""
    dom = domain(name)
    lo, hi = COUNTS[name]
    nb = lo if lo == hi else lo + (seed * 2654435761 % (hi - lo + 1))
    b, inflow = city_layout(dom, seed, nb)
    return city_inputs(dom, b, inflow)
