"""Pins the oracle (the plain-C restatement in oracle/qes_oracle.c) before it
is trusted as the checker: bit-exact against the golden vectors made by the
reference's own compiled Solver_CPU / Solver_CPU_RB (tests/golden/make_golden.py)
and, where the reference build is present, against it directly."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("name", ["small_cuboid.npz", "small_city.npz"])
@pytest.mark.parametrize("kind,tag", [(0, "cpu"), (1, "rb")])
def test_port_matches_reference_golden(golden, name, kind, tag):
    d, w, z = golden(name)
    it = int(z["itermax"])
    u, v, ww, L, iters, _ = O.solve(d, w, 1e-9, it, ordering=kind, err_fp64=False)
    assert iters == it  # tol = 1e-9 is never reached in FP32
    np.testing.assert_array_equal(L, z[f"{tag}_lambda"])
    np.testing.assert_array_equal(u, z[f"{tag}_u"])
    np.testing.assert_array_equal(v, z[f"{tag}_v"])
    np.testing.assert_array_equal(ww, z[f"{tag}_w"])


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref absent")
@pytest.mark.parametrize("kind", [0, 1])
def test_port_matches_reference_build_random_city(kind):
    import qesb

    d = qesb.Domain(30, 26, 14, 2.0, 2.0, 1.0, qesb.city_dz(14, 1.0, 1.05))
    c = qesb.city_random(d, 123, 4, fp=(6, 14), h=(4, 14))
    w = qesb.city_build(d, c.buildings, c.inflow)
    lam0 = np.random.default_rng(1).standard_normal(d.numCellCentered()).astype(np.float32)
    ur, vr, wr, Lr, _ = O.ref_solve(d, w, 1e-9, 60, kind=kind, lam=lam0)
    u, v, ww, L, it, _ = O.solve(d, w, 1e-9, 60, ordering=kind, err_fp64=False, lam=lam0)
    np.testing.assert_array_equal(L, Lr)
    np.testing.assert_array_equal(u, ur)
    np.testing.assert_array_equal(v, vr)
    np.testing.assert_array_equal(ww, wr)


def test_cuboid100_golden_is_converged_field():
    """The 10 000-iteration Solver_CPU field is mass-consistent in the solved
    layers below the top (the fixture's stored max divergence)."""
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "cuboid100.npz"))
    assert float(z["max_div"]) < 1e-3
    assert np.isfinite(z["u"]).all()


def test_ordering_agrees_after_convergence(golden):
    """Lexicographic (Solver_CPU) and red-black (Solver_CPU_RB) orderings agree
    once converged; they differ while converging (iteration counts differ)."""
    d, w, z = golden("small_cuboid.npz")
    u0, v0, w0, *_ = O.solve(d, w, 1e-9, 3000, ordering=0, err_fp64=False)
    u1, v1, w1, *_ = O.solve(d, w, 1e-9, 3000, ordering=1, err_fp64=False)
    assert max(np.abs(u0 - u1).max(), np.abs(v0 - v1).max(), np.abs(w0 - w1).max()) < 1e-4


def test_fp64_same_sor_close_to_fp32(golden):
    d, w, z = golden("small_city.npz")
    u, v, ww, L, it, _ = O.solve(d, w, 1e-9, 2000, ordering=1)
    u8, v8, w8, L8, it8, _ = O.solve_f64(d, w, 1e-13, 2000)
    assert it == 2000 and it8 < 2000  # FP64 converges; FP32 plateaus at its ulp
    assert np.abs(u - u8).max() < 1e-3
    assert np.abs(L - L8).max() / np.abs(L8).max() < 1e-4


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref absent")
def test_window_rule_stop_matches_chained_reference_solves():
    """The window rule (stop after iteration n, a multiple of K, when
    max|lambda_n - lambda_(n-K)| <= wtol in double) restated in the oracle
    stops where the reference's own red-black solver, run K iterations per
    Solver::solve call with lambda carried over and the drift taken here in
    numpy, first meets it; and with the same lambda."""
    import qesb

    d = qesb.Domain(40, 34, 14, 2.0, 2.0, 1.0, qesb.city_dz(14, 1.0, 1.03))
    c = qesb.city_random(d, 77, 5, fp=(6, 14), h=(4, 16))
    w = qesb.city_build(d, c.buildings, c.inflow)
    K, wtol = 16, 2e-3
    L, it, stop, drift = O.sor_window(d, w, O.divergence(d, w), 1e-9, 4000, K, wtol)
    assert stop == 2 and it % K == 0 and drift <= wtol
    lam = np.zeros(d.numCellCentered(), np.float32)
    n = 0
    while True:
        _, _, _, nxt, _ = O.ref_solve(d, w, -1.0, K, kind=1, lam=lam)
        n += K
        dr = float(np.abs(nxt.astype(np.float64) - lam.astype(np.float64)).max())
        lam = nxt
        if dr <= wtol:
            break
        assert n < 4000
    assert n == it and dr == drift
    np.testing.assert_array_equal(lam, L)
