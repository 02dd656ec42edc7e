"""Pins the log-law wall treatment of the oracle (qo_wall_log, the C
restatement of the stair-step part of Wall::wallLogBC, src/winds/Wall.cpp:
656-803, with the lists of Wall::defineWalls, :287-340) before the GPU kernel
is checked against it: bit for bit against the fixture made by the reference's
own compiled code (tests/golden/make_wall_log.py) and, where the reference
build is present, against it directly."""
import numpy as np
import pytest

import qesb
from oracle import oracle as O


def _fixture():
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "wall_log_city.npz"))
    d = qesb.Domain(int(z["Nx"]), int(z["Ny"]), int(z["Nz"]), float(z["dx"]), float(z["dy"]), 1.0, z["dz_array"])
    return d, z


def wall_sides(d, flag):
    """Per side (below, above, back, front, right, left), the number of cells
    Wall::defineWalls lists (fluid cells, k in [1, nz-3], neighbours by flat
    cell index, the back and right sides guarded by i > 0 and j > 0)."""
    Nx, Ny, Nz = d.base
    X, XY = Nx, Nx * Ny
    fl = flag.astype(np.int64)
    solid = (fl == 0) | (fl == 2)
    c = np.arange(XY, (Nz) * XY)  # k in [1, nz-3] = [1, Nz-1]
    i, j = c % X, (c // X) % Ny
    fluid = ~solid[c]
    out = [fluid & solid[c - XY], fluid & solid[c + XY], fluid & solid[c - 1] & (i > 0), fluid & solid[c + 1],
           fluid & solid[c - X] & (j > 0), fluid & solid[c + X]]
    return [int(m.sum()) for m in out]


def test_restatement_matches_reference_fixture():
    d, z = _fixture()
    u, v, w = z["u"], z["v"], z["w"]
    out = O.wall_log(d, z["icellflag"], float(z["z0"]), u, v, w)
    assert out is not None
    idx = z["changed"]
    for a, a0, ref in zip(out, (u, v, w), (z["ref_u"], z["ref_v"], z["ref_w"])):
        np.testing.assert_array_equal(a[idx], ref)
        keep = np.ones(a.size, bool)
        keep[idx] = False
        np.testing.assert_array_equal(a[keep], a0[keep])
    # every side's list is exercised, including the wall-above cells under the
    # raised building
    assert all(n > 0 for n in wall_sides(d, z["icellflag"]))


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("seed,z0", [(3, 0.1), (11, 0.05), (29, 0.2)])
def test_restatement_matches_reference_build(seed, z0):
    d = qesb.Domain(36, 30, 14, 2.0, 2.0, 1.0, qesb.city_dz(14, 1.0, 1.05))
    c = qesb.city_random(d, seed, 5, fp=(6, 14), h=(4, 12))
    bl = list(c.buildings) + [qesb.Building(58.0, 50.0, 14.0, 10.0, 8.0, 0.0),
                              qesb.Building(10.0, 12.0, 10.0, 10.0, 9.0, 2.5)]
    w = qesb.city_build(d, bl, c.inflow)
    u, v, ww, _, _, _ = O.solve(d, w, 1e-9, 80, ordering=1, err_fp64=False)
    ur, vr, wr, flag = O.ref_wall_log_bc(d, w.icellflag, z0, u, v, ww)
    np.testing.assert_array_equal(flag, w.icellflag)
    got = O.wall_log(d, flag, z0, u, v, ww)
    for a, b in zip(got, (ur, vr, wr)):
        np.testing.assert_array_equal(a, b)


def test_cut_cell_flags_are_rejected():
    d, z = _fixture()
    flag = z["icellflag"].copy()
    Nx, Ny, _ = d.base
    flag[2 * Nx * Ny + Nx + 3] = 7
    assert O.wall_log(d, flag, 0.1, z["u"], z["v"], z["w"]) is None
