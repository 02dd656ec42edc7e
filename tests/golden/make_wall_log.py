"""Generate tests/golden/wall_log_city.npz from the reference's own
Wall::defineWalls + Wall::wallLogBC (oracle/_ref, built from the reference
sources by oracle/Makefile):

    python tests/golden/make_wall_log.py

The case: a 30x26x12 stretched grid with random buildings, one building
against the +x and +y domain edges (the front and left lists reach across the
row and plane ends by flat index, as Domain::cellAdd does) and one raised
building (base 3 m, so cells below it have a wall above). The winds are those
of 150 red-black iterations (the oracle's Solver_CPU_RB restatement), as the
log law is applied after a solve (qesWindsMain.cpp:157-166). Stored: inputs,
the reference's flags after defineWalls, and the faces whose u0, v0 or w0
wallLogBC changed (flat face index and the three values after it).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "qes-public_b200"))
sys.path.insert(0, ROOT)

import qesb  # noqa: E402
from oracle import oracle as O  # noqa: E402

Z0 = 0.1


def case():
    d = qesb.Domain(30, 26, 12, 2.0, 2.0, 1.0, qesb.city_dz(12, 1.0, 1.04))
    c = qesb.city_random(d, 77, 4, fp=(6, 12), h=(4, 10))
    bl = list(c.buildings) + [qesb.Building(48.0, 42.0, 12.0, 10.0, 7.0, 0.0),
                              qesb.Building(14.0, 22.0, 10.0, 8.0, 7.0, 3.0)]
    w = qesb.city_build(d, bl, c.inflow)
    u, v, ww, _, _, _ = O.solve(d, w, 1e-9, 150, ordering=1, err_fp64=False)
    return d, w, u, v, ww


def main():
    d, w, u, v, ww = case()
    ur, vr, wr, flag = O.ref_wall_log_bc(d, w.icellflag, Z0, u, v, ww)
    idx = np.flatnonzero((ur != u) | (vr != v) | (wr != ww)).astype(np.int32)
    np.savez_compressed(os.path.join(HERE, "wall_log_city.npz"), Nx=30, Ny=26, Nz=12, dx=2.0, dy=2.0,
                        dz_array=d.dz_array, z0=Z0, icellflag=flag, u=u, v=v, w=ww, changed=idx,
                        ref_u=ur[idx], ref_v=vr[idx], ref_w=wr[idx])
    print("faces changed:", idx.size)


if __name__ == "__main__":
    main()
