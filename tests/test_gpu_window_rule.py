"""The window stopping rule (qesb_set_window_rule) on the GPU: single,
batched and full-coefficient solves stop on the oracle's iteration with the
oracle's bits, and report the oracle's last window drift."""
import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _city(nx=72, ny=56, nz=24, seed=31, nb=7):
    d = qesb.Domain(nx, ny, nz, 2.0, 2.0, 1.0, qesb.city_dz(nz, 1.0, 1.03))
    c = qesb.city_random(d, seed, nb, fp=(6, 20), h=(4, 30))
    return qesb.city_build(d, c.buildings, c.inflow)


@pytest.mark.parametrize("path,variant", [(1, -1), (1, 48), (1, 18), (1, 0), (0, -1)])
def test_single_solve_window_stop_matches_oracle(path, variant):
    w = _city()
    d = w.domain
    K, wtol = 16, 1e-2
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_option("path", path)
        if variant >= 0:
            s.set_option("variant", variant)  # 0: a fused tile shape, which the rule replaces by a sweep shape
        s.set_window_rule(K, wtol)
        st = s.solve(w, 5000)
        lam = s.lambda_
    L, it, stop, drift = O.sor_window(d, w, O.divergence(d, w), 1e-9, 5000, K, wtol)
    assert stop == 2 and st["converged"] == 2
    assert st["iterations"] == it and st["window_drift"] == drift
    np.testing.assert_array_equal(lam, L)
    u, v, ww = O.correct(d, w, L)
    np.testing.assert_array_equal(w.u, u)
    np.testing.assert_array_equal(w.v, v)
    np.testing.assert_array_equal(w.w, ww)


def test_batch_window_stop_with_prephase_matches_oracle_chain():
    import torch

    ws = [_city(70, 45, 21, 9, 8), _city(131, 40, 15, 3, 6), _city(40, 33, 9, 2, 3)]
    K, wtol, pre = 32, 5e-3, (1.9, 3e-3, 4000)
    solvers = [qesb.Solver_B200(w.domain, 1e-9) for w in ws]
    try:
        for s, w in zip(solvers, ws):
            s.set_inputs(w)
            s.set_prephase(*pre)
            s.set_window_rule(K, wtol)
        outs = [[torch.zeros(w.domain.numFaceCentered(), dtype=torch.float32, device="cuda") for _ in range(3)]
                for w in ws]
        st = qesb.solve_batch(solvers, 8000, *[[o[q].data_ptr() for o in outs] for q in range(3)])
        lams = [s.lambda_ for s in solvers]
    finally:
        for s in solvers:
            s.close()
    for w, x, L in zip(ws, st, lams):
        d = w.domain
        R = O.divergence(d, w)
        Lp, itp, *_ = O.sor(d, w, R, pre[1], pre[2], omega=pre[0])
        Lo, it, stop, drift = O.sor_window(d, w, R, 1e-9, 8000, K, wtol, lam=Lp)
        assert (x["pre_iterations"], x["iterations"], x["converged"]) == (itp, it, stop) and stop == 2
        assert x["window_drift"] == drift
        np.testing.assert_array_equal(L, Lo)
    u, v, ww = O.correct(ws[0].domain, ws[0], lams[0])
    np.testing.assert_array_equal(outs[0][0].cpu().numpy(), u)
    np.testing.assert_array_equal(outs[0][2].cpu().numpy(), ww)


def test_batch_refuses_mixed_window_lengths():
    ws = [_city(40, 33, 9, 2, 3), _city(36, 30, 9, 4, 3)]
    solvers = [qesb.Solver_B200(w.domain, 1e-3) for w in ws]
    try:
        for s, w in zip(solvers, ws):
            s.set_inputs(w)
        solvers[0].set_window_rule(16, 1e-2)
        with pytest.raises(qesb.QesbError, match="different window lengths"):
            qesb.solve_batch(solvers, 100)
    finally:
        for s in solvers:
            s.close()
