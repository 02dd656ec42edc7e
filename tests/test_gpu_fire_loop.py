"""QES-Fire's solve pattern (qesFireMain.cpp:232-259): u0 changes at every fire
step and Solver::solve runs again without resetLambda, so each solve starts
from the previous step's lambda. The handle keeps lambda between solves, so a
sequence of solves on the GPU must equal the oracle's chain of solves, each
from the lambda the one before left, bit for bit: iterations, lambda and winds,
with and without the over-relaxed pre-phase."""
import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1.1e-3


def _steps(n):
    d = qesb.Domain(70, 45, 21, 2.0, 2.0, 1.0, qesb.city_dz(21, 1.0, 1.03))
    c = qesb.city_random(d, 9, 8, fp=(6, 18), h=(4, 30))
    base = qesb.city_build(d, c.buildings, c.inflow)
    nz, ny, nx = d.face_shape()
    i = np.arange(nx)[None, None, :]
    j = np.arange(ny)[None, :, None]
    k = np.arange(nz)[:, None, None]
    out = []
    for t in range(n):
        # a moving updraft over a fire centre, faces of solid cells zeroed as
        # Wall::setVelocityZero does (the reference's own routine, oracle/_ref)
        g = np.exp(-((i * 2.0 - 30.0 - 6.0 * t) ** 2 + (j * 2.0 - 44.0) ** 2) / 200.0) * np.minimum(1.0, k / 8.0)
        w = qesb.WINDSGeneralData(d)
        w.icellflag, w.e, w.f, w.g, w.h, w.m, w.n = (base.icellflag, base.e, base.f, base.g, base.h, base.m,
                                                      base.n)
        u0 = base.u0.copy()
        v0 = base.v0.copy()
        w0 = (base.w0.reshape(nz, ny, nx) + 2.5 * g).astype(np.float32).ravel()
        w.u0, w.v0, w.w0 = O.ref_set_velocity_zero(d, base.icellflag, u0, v0, w0) if O.ref_available() else (
            u0, v0, w0)
        out.append(w)
    return d, out


@pytest.mark.parametrize("pre", [False, True])
def test_fire_steps_warm_start_from_previous_lambda(pre):
    d, seq = _steps(4)
    got = []
    with qesb.Solver_B200(d, TOL) as s:
        if pre:
            s.set_prephase(1.95, 3e-3, 5000)
        for w in seq:
            st = s.solve(w, 5000)
            got.append((st["iterations"], st["pre_iterations"], s.lambda_, w.u.copy(), w.w.copy()))
    L = np.zeros(d.numCellCentered(), np.float32)
    for w, (it, pit, Lg, ug, wg) in zip(seq, got):
        R = O.divergence(d, w)
        if pre:
            L, ip, *_ = O.sor(d, w, R, 3e-3, 5000, lam=L, omega=1.95)
            assert pit == ip
        L, io, *_ = O.sor(d, w, R, TOL, 5000, lam=L)
        assert it == io
        np.testing.assert_array_equal(Lg, L)
        uo, _, wo = O.correct(d, w, L)
        np.testing.assert_array_equal(ug, uo)
        np.testing.assert_array_equal(wg, wo)
    # the later steps start close to their answer
    assert max(g[0] + g[1] for g in got[1:]) < got[0][0] + got[0][1]
