"""Batched solves (qesb_solve_batch): domains of different sizes solved in
one persistent bulk-staged loop give, domain by domain, the bits of separate
solves and of the oracle, each stopping on its own iteration."""
import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _cities():
    out = []
    for (nx, ny, nz, seed, nb) in [(70, 45, 21, 9, 8), (131, 40, 15, 3, 6), (300, 19, 11, 5, 6), (40, 33, 9, 2, 3)]:
        d = qesb.Domain(nx, ny, nz, 2.0, 2.0, 1.0, qesb.city_dz(nz, 1.0, 1.03))
        c = qesb.city_random(d, seed, nb, fp=(6, 18), h=(4, 16))
        out.append(qesb.city_build(d, c.buildings, c.inflow))
    return out


def _batch(ws, tol, itermax, lam0s, variant=-1, pdl=1):
    import torch

    solvers = [qesb.Solver_B200(w.domain, tol) for w in ws]
    try:
        if variant >= 0:
            solvers[0].set_option("variant", variant)
        solvers[0].set_option("pdl", pdl)
        for s, w, l0 in zip(solvers, ws, lam0s):
            s.set_inputs(w)
            if l0 is not None:
                s.lambda_ = l0
        outs = [[torch.zeros(w.domain.numFaceCentered(), dtype=torch.float32, device="cuda") for _ in range(3)]
                for w in ws]
        st = qesb.solve_batch(solvers, itermax, *[[o[q].data_ptr() for o in outs] for q in range(3)])
        lams = [s.lambda_ for s in solvers]
        winds = [[t.cpu().numpy() for t in o] for o in outs]
        return st, lams, winds
    finally:
        for s in solvers:
            s.close()


@pytest.mark.parametrize("variant,pdl", [(-1, 1), (18, 1), (21, 1), (23, 1), (26, 1), (40, 1), (41, 1), (42, 1),
                                         (44, 1), (46, 1), (48, 1), (50, 1), (57, 1), (59, 1), (59, 0)])
def test_batch_matches_oracle_per_domain(variant, pdl):
    """Per domain the oracle's bits; z-march list shapes with and without
    programmatic dependent launches between the list kernels."""
    ws = _cities()
    rng = np.random.default_rng(11)
    lam0s = [None, rng.standard_normal(ws[1].domain.numCellCentered()).astype(np.float32), None, None]
    tol = 1.1e-3
    st, lams, winds = _batch(ws, tol, 3000, lam0s, variant, pdl)
    for w, l0, s, L, (u, v, ww) in zip(ws, lam0s, st, lams, winds):
        d = w.domain
        Lo, it, fe, _ = O.sor(d, w, O.divergence(d, w), tol, 3000, ordering=1, err_fp64=True, lam=l0)
        assert s["iterations"] == it and s["converged"] == 1, (s, it)
        np.testing.assert_array_equal(L, Lo)
        uo, vo, wo = O.correct(d, w, Lo)
        np.testing.assert_array_equal(u, uo)
        np.testing.assert_array_equal(v, vo)
        np.testing.assert_array_equal(ww, wo)
        assert 0 < s["ms_sor"] <= s["ms_total"]
        assert s["max_divergence"] == O.max_divergence(d, w.icellflag, u, v, ww)
    # the domains stop on different iterations
    assert len({s["iterations"] for s in st}) > 1


def test_batch_equals_single_solves_at_itermax():
    ws = _cities()
    st, lams, winds = _batch(ws, 1e-9, 57, [None] * len(ws))
    for w, s, L in zip(ws, st, lams):
        with qesb.Solver_B200(w.domain, 1e-9) as one:
            one.set_option("variant", 19)
            s1 = one.solve(w, 57)
            assert s1["iterations"] == s["iterations"] == 57 and not s["converged"]
            np.testing.assert_array_equal(one.lambda_, L)


def test_batch_rejects_repeated_and_non_stair_step_handles():
    w = _cities()[0]
    with qesb.Solver_B200(w.domain, 1e-3) as s:
        s.set_inputs(w)
        with pytest.raises(qesb.QesbError):
            qesb.solve_batch([s, s], 10)
        s.set_option("path", 0)
        with pytest.raises(qesb.QesbError):
            qesb.solve_batch([s], 10)


def test_batch_prephase_per_domain():
    """Domains of one batch with and without an over-relaxed pre-phase: each
    matches the oracle's two-phase (or one-phase) solve."""
    import torch

    ws = _cities()
    tol = 1.1e-3
    pre = [(1.9, 1e-3, 4000), None, (1.95, 1e-3, 80), None]
    solvers = [qesb.Solver_B200(w.domain, tol) for w in ws]
    try:
        for s, w, p in zip(solvers, ws, pre):
            s.set_inputs(w)
            if p:
                s.set_prephase(*p)
        st = qesb.solve_batch(solvers, 4000)
        lams = [s.lambda_ for s in solvers]
    finally:
        for s in solvers:
            s.close()
    for w, p, sti, L in zip(ws, pre, st, lams):
        d = w.domain
        R = O.divergence(d, w)
        lam0 = None
        if p:
            lam0, itp, *_ = O.sor(d, w, R, p[1], p[2], omega=p[0])
            assert sti["pre_iterations"] == itp
        else:
            assert sti["pre_iterations"] == 0
        Lo, it, *_ = O.sor(d, w, R, tol, 4000, lam=lam0)
        assert sti["iterations"] == it
        np.testing.assert_array_equal(L, Lo)
    torch.cuda.synchronize()


@pytest.mark.parametrize("variant", [-1, 51])
def test_prephase_start_stage_single_and_batch(variant):
    """A pre-phase start stage (its first sweeps at another omega): per
    domain of a batch, with and without one, and in a single solve, the
    oracle's three-phase solve bit for bit; pre_iterations counts the stage."""
    ws = _cities()
    tol = 1.1e-3
    cfg = [((1.7, 12), (1.95, 1e-3, 4000)), (None, (1.9, 1e-3, 4000)), ((1.5, 5), (1.9, 2e-3, 60)), (None, None)]

    def setup(s, w, c):
        s.set_inputs(w)
        if variant >= 0:
            s.set_option("variant", variant)
        if c[1]:
            s.set_prephase(*c[1])
        if c[0]:
            s.set_prephase_start(*c[0])

    def oracle(w, c):
        d = w.domain
        R = O.divergence(d, w)
        lam, npre = None, 0
        if c[1]:
            if c[0]:
                lam, n0, *_ = O.sor(d, w, R, -1.0, c[0][1], omega=c[0][0])
                npre += n0
            lam, n1, *_ = O.sor(d, w, R, c[1][1], c[1][2], omega=c[1][0], lam=lam)
            npre += n1
        Lo, it, *_ = O.sor(d, w, R, tol, 4000, lam=lam)
        return npre, it, Lo

    solvers = [qesb.Solver_B200(w.domain, tol) for w in ws]
    try:
        for s, w, c in zip(solvers, ws, cfg):
            setup(s, w, c)
        st = qesb.solve_batch(solvers, 4000)
        lams = [s.lambda_ for s in solvers]
    finally:
        for s in solvers:
            s.close()
    for w, c, sti, L in zip(ws, cfg, st, lams):
        npre, it, Lo = oracle(w, c)
        assert sti["pre_iterations"] == npre and sti["iterations"] == it
        np.testing.assert_array_equal(L, Lo)
    with qesb.Solver_B200(ws[0].domain, tol) as s:
        setup(s, ws[0], cfg[0])
        st0 = s.solve(ws[0], 4000, set_inputs=False)
        npre, it, Lo = oracle(ws[0], cfg[0])
        assert st0["pre_iterations"] == npre and st0["iterations"] == it
        np.testing.assert_array_equal(s.lambda_, Lo)


def test_batch_autotune_keeps_lambda_and_results_exact():
    """qesb_autotune_batch times the sweep shapes on the batch's own domain
    list, leaves every lambda as it was, and the batch it tunes still gives
    the oracle's bits."""
    import torch

    ws = _cities()
    rng = np.random.default_rng(5)
    lam0s = [rng.standard_normal(w.domain.numCellCentered()).astype(np.float32) for w in ws]
    solvers = [qesb.Solver_B200(w.domain, 1.1e-3) for w in ws]
    try:
        for s, w, l0 in zip(solvers, ws, lam0s):
            s.set_inputs(w)
            s.lambda_ = l0
        best, us = qesb.autotune_batch(solvers)
        nv = qesb.lib().qesb_num_variants()
        assert 5 <= best < nv and len(us) == nv
        assert all(u > 0 for u in us[5:]) and us[best] == min(us[5:])
        for s, l0 in zip(solvers, lam0s):
            np.testing.assert_array_equal(s.lambda_, l0)
        outs = [[torch.zeros(w.domain.numFaceCentered(), dtype=torch.float32, device="cuda") for _ in range(3)]
                for w in ws]
        st = qesb.solve_batch(solvers, 3000, *[[o[q].data_ptr() for o in outs] for q in range(3)])
        for w, l0, s, x, o in zip(ws, lam0s, st, solvers, outs):
            d = w.domain
            Lo, it, _, _ = O.sor(d, w, O.divergence(d, w), 1.1e-3, 3000, ordering=1, err_fp64=True, lam=l0)
            assert s["iterations"] == it
            np.testing.assert_array_equal(x.lambda_, Lo)
            np.testing.assert_array_equal(o[0].cpu().numpy(), O.correct(d, w, Lo)[0])
        with pytest.raises(qesb.QesbError):
            solvers[0].set_option("batch_variant", 2)  # a fused tile shape: not a batch shape
    finally:
        for s in solvers:
            s.close()


def test_flags_only_inputs_give_the_same_solve():
    """qesb_set_inputs_flags (icellflag and the initial winds; the stair-step
    wall coefficients computed on the device) gives the solve that
    qesb_set_inputs gives from the reference's full arrays, bit for bit."""
    for (nx, ny, nz, seed, nb) in [(70, 45, 21, 9, 8), (131, 40, 15, 3, 6)]:
        d = qesb.Domain(nx, ny, nz, 2.0, 2.0, 1.0, qesb.city_dz(nz, 1.0, 1.03))
        c = qesb.city_random(d, seed, nb, fp=(6, 18), h=(4, 16))
        w = qesb.city_build(d, c.buildings, c.inflow)
        out = []
        for flags_only in (False, True):
            with qesb.Solver_B200(d, 1.1e-3) as s:
                if flags_only:
                    s.set_inputs_flags(w)
                else:
                    s.set_inputs(w)
                st = s.solve(w, 3000, set_inputs=False)
                out.append((st["iterations"], st["max_divergence"], s.lambda_, w.u.copy(), w.w.copy()))
        a, b = out
        assert a[0] == b[0] and a[1] == b[1]
        for x, y in zip(a[2:], b[2:]):
            np.testing.assert_array_equal(x, y)
