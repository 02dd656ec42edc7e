"""GPU parity: the sm_100a solver through the C ABI against the oracle.

The red-black sweep, R and the correction use the reference's per-operation
rounding, so against the red-black reference (Solver_CPU_RB, via the golden
vectors or the oracle port) lambda, u, v, w must agree BIT FOR BIT after any
number of iterations. Against the lexicographic Solver_CPU the two orderings
only meet at convergence; there the bar is max|du|, |dv|, |dw| <= 1e-3 m/s.
"""
import os

import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

WIND_TOL = 1e-3  # m/s, max|du| against Solver_CPU at convergence


def gpu_solve(d, w, itermax, tol=1e-9, path=1, lam=None, k=0, variant=-1):
    with qesb.Solver_B200(d, tol) as s:
        s.set_option("path", path)
        if k:
            s.set_option("sweeps_per_launch", k)
        s.set_option("variant", variant)
        s.set_inputs(w)
        if lam is not None:
            s.lambda_ = lam
        st = s.solve(w, itermax, set_inputs=False)
        return w.u.copy(), w.v.copy(), w.w.copy(), s.lambda_, st, s.R


@pytest.mark.parametrize("name", ["small_cuboid.npz", "small_city.npz"])
@pytest.mark.parametrize("path", [0, 1])
def test_bit_exact_against_reference_red_black(golden, name, path):
    d, w, z = golden(name)
    it = int(z["itermax"])
    u, v, ww, L, st, _ = gpu_solve(d, w, it, path=path)
    assert st["iterations"] == it and st["path"] == path
    np.testing.assert_array_equal(L, z["rb_lambda"])
    np.testing.assert_array_equal(u, z["rb_u"])
    np.testing.assert_array_equal(v, z["rb_v"])
    np.testing.assert_array_equal(ww, z["rb_w"])


def test_divergence_R_bit_exact(golden):
    d, w, z = golden("small_city.npz")
    *_, R = gpu_solve(d, w, 1)
    np.testing.assert_array_equal(R, O.divergence(d, w))


# fused tile shapes (0-4), scalar split (5-10), float4 split (11-13),
# window-order split (14-17), bulk-copy staged (18-22), cp.async staged (23-27),
# register-capped split (28-35), window-order split with prefetch (36-39),
# z-march (40-50), z-march staged by tensor-map copies (51-57; 58-60 with equal plane-step shares per CTA)
N_VARIANTS = 61
ZM = 40  # first z-march variant
BULK = 18


@pytest.mark.parametrize("variant", range(N_VARIANTS))
def test_fused_sweeps_bit_exact(variant):
    """Every sweep variant (the fused kernel's tile shapes with K = 1 and 2
    iterations per launch, and the streaming split path), an odd iteration
    count (a partial last fused launch), ragged tiles at the domain edges and a
    random warm start."""
    d = qesb.Domain(70, 45, 21, 2.0, 2.0, 1.0, qesb.city_dz(21, 1.0, 1.03))
    c = qesb.city_random(d, 9, 8, fp=(6, 18), h=(4, 30))
    w = qesb.city_build(d, c.buildings, c.inflow)
    lam0 = np.random.default_rng(3).standard_normal(d.numCellCentered()).astype(np.float32)
    u, v, ww, L, st, _ = gpu_solve(d, w, 37, lam=lam0, variant=variant)
    uo, vo, wo, Lo, it, _ = O.solve(d, w, 1e-9, 37, ordering=1, lam=lam0)
    assert st["path"] == 1
    assert st["iterations"] == it == 37
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(v, vo)
    np.testing.assert_array_equal(ww, wo)


def test_variant_count_matches_library():
    assert qesb.lib().qesb_num_variants() == N_VARIANTS


@pytest.mark.parametrize("variant", range(BULK, N_VARIANTS))
@pytest.mark.parametrize("nx", [300, 515])
def test_bulk_sweeps_multi_chunk_rows_bit_exact(variant, nx):
    """Bulk-staged sweeps on rows longer than one 128-cell span (two and three
    spans per colour row, the last one partial), against the oracle."""
    d = qesb.Domain(nx, 19, 11, 2.0, 2.0, 1.0, qesb.city_dz(11, 1.0, 1.03))
    c = qesb.city_random(d, 5, 6, fp=(6, 18), h=(4, 16))
    w = qesb.city_build(d, c.buildings, c.inflow)
    lam0 = np.random.default_rng(4).standard_normal(d.numCellCentered()).astype(np.float32)
    u, v, ww, L, st, _ = gpu_solve(d, w, 23, lam=lam0, variant=variant)
    uo, vo, wo, Lo, it, _ = O.solve(d, w, 1e-9, 23, ordering=1, lam=lam0)
    assert st["path"] == 1 and st["iterations"] == it == 23
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(ww, wo)


@pytest.mark.parametrize("path,variant", [(0, -1), (1, 0), (1, 1), (1, 5), (1, BULK), (1, BULK + 3), (1, BULK + 5), (1, BULK + 8)])
@pytest.mark.parametrize("tol", [2e-3, 1.1e-3, 7e-4])
def test_stopping_rule_matches_oracle(golden, path, variant, tol):
    """A reachable tolerance: the loop stops on the same iteration as the
    reference loop `while (iter < itermax && max_error > tol)` with the error
    taken in FP64, and lambda is the same bits."""
    d, w, z = golden("small_city.npz")
    u, v, ww, L, st, _ = gpu_solve(d, w, 5000, tol=tol, path=path, variant=variant)
    Lo, it, fe, hist = O.sor(d, w, O.divergence(d, w), tol, 5000, ordering=1, err_fp64=True,
                             hist=True)
    assert st["converged"] == 1 and st["path"] == path
    assert st["iterations"] == it < 5000
    assert st["residual"] == fe <= np.float32(tol)
    np.testing.assert_array_equal(L, Lo)


def test_warm_start_and_persistence(golden):
    """lambda persists between solves (Solver_CPU semantics) and a caller's
    lambda acts as the starting point."""
    d, w, z = golden("small_cuboid.npz")
    lam0 = np.linspace(-3, 3, d.numCellCentered()).astype(np.float32)
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.lambda_ = lam0
        s.solve(w, 40, set_inputs=False)
        s.solve(w, 25, set_inputs=False)
        L = s.lambda_
        u = w.u.copy()
        s.resetLambda()
        assert not s.lambda_.any()
    L1, *_ = O.sor(d, w, O.divergence(d, w), 1e-9, 40, lam=lam0)
    L2, *_ = O.sor(d, w, O.divergence(d, w), 1e-9, 25, lam=L1)
    np.testing.assert_array_equal(L, L2)
    np.testing.assert_array_equal(u, O.correct(d, w, L2)[0])


def test_converged_winds_match_solver_cpu_cuboid100():
    """100x100x50 single cuboid, reference settings (tol 1e-9, itermax 10000):
    max|du| against the reference Solver_CPU's own 10 000-iteration field."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "cuboid100.npz"))
    w = qesb.cuboid100()
    d = w.domain
    u, v, ww, L, st, _ = gpu_solve(d, w, 10000)
    assert st["iterations"] == 10000
    s = int(z["stride"])
    err = max(np.abs(u[::s] - z["u"]).max(), np.abs(v[::s] - z["v"]).max(),
              np.abs(ww[::s] - z["w"]).max())
    assert err <= WIND_TOL, err
    for comp, key in ((u, "u_sum"), (v, "v_sum"), (ww, "w_sum")):
        assert abs(comp.astype(np.float64).sum() - float(z[key])) <= WIND_TOL * comp.size
    div = O.max_divergence(d, w.icellflag, u, v, ww)
    assert div <= float(z["max_div"]) * 1.05 + 1e-6, (div, float(z["max_div"]))
    # the solver's own FP64 final check is the same number
    assert st["max_divergence"] == div


@pytest.mark.parametrize("variant", [5, 17, BULK + 1, ZM + 2])
def test_final_divergence_check_matches_oracle_metric(golden, variant):
    """qesb_stats.max_divergence (computed on the device in FP64 after the
    correction) equals the oracle's metric on the same winds, for single and
    batched solves."""
    d, w, z = golden("small_city.npz")
    u, v, ww, L, st, _ = gpu_solve(d, w, 300, tol=1.1e-3, variant=variant)
    assert st["max_divergence"] == O.max_divergence(d, w.icellflag, u, v, ww) > 0


def test_nan_input_is_reported():
    d = qesb.Domain(20, 16, 10, 1.0, 1.0, 1.0)
    w = qesb.city_build(d, [qesb.Building(6.0, 5.0, 4.0, 4.0, 4.0, 0.0)],
                        qesb.Inflow(5.0, 10.0, 0.15, 270.0))
    w.e[d.cell(10, 8, 4)] = np.nan
    with qesb.Solver_B200(d, 1e-9) as s:
        with pytest.raises(qesb.QesbError) as ei:
            s.solve(w, 100)
        assert ei.value.status == 5


def test_general_coefficients_take_full_path():
    """Coefficients that are not stair-step (a cut-cell-like fraction) are
    solved on the full-coefficient path and still match the oracle bit for bit."""
    d = qesb.Domain(24, 20, 12, 1.0, 1.0, 1.0)
    w = qesb.city_build(d, [qesb.Building(8.0, 6.0, 6.0, 7.0, 6.0, 0.0)],
                        qesb.Inflow(4.0, 10.0, 0.2, 250.0))
    w.e[d.cell(5, 5, 3)] *= np.float32(0.37)
    u, v, ww, L, st, _ = gpu_solve(d, w, 90)
    assert st["path"] == 0
    Lo, *_ = O.sor(d, w, O.divergence(d, w), 1e-9, 90)
    np.testing.assert_array_equal(L, Lo)


def test_fp64_same_sor_error_is_stated(golden):
    """The FP32 sweep's error against an FP64 run of the same SOR, per result."""
    d, w, z = golden("small_city.npz")
    u, v, ww, L, st, _ = gpu_solve(d, w, 3000)
    u8, v8, w8, L8, it8, _ = O.solve_f64(d, w, 1e-30, 3000)
    werr = max(np.abs(u - u8).max(), np.abs(v - v8).max(), np.abs(ww - w8).max())
    lerr = np.abs(L - L8).max() / np.abs(L8).max()
    assert werr < 1e-3 and lerr < 1e-4


@pytest.mark.parametrize("graph", [0, 1])
def test_graph_and_plain_launches_agree(golden, graph):
    d, w, z = golden("small_city.npz")
    with qesb.Solver_B200(d, 1.1e-3) as s:
        s.set_option("graph", graph)
        st = s.solve(w, 5000)
        L = s.lambda_
    Lo, it, *_ = O.sor(d, w, O.divergence(d, w), 1.1e-3, 5000)
    assert st["iterations"] == it
    np.testing.assert_array_equal(L, Lo)


@pytest.mark.parametrize("variant", [1, 5, BULK + 1, BULK + 6, ZM, ZM + 1])
def test_full_size_city400_packed_equals_full_path(variant):
    """400x400x100 stretched city: after 24 iterations the packed paths (fused
    and split) and the full-coefficient path hold the same lambda bits and the
    same residual history."""
    w, c = qesb.random_city("city400", 0)
    d = w.domain
    out = {}
    for path in (0, 1):
        with qesb.Solver_B200(d, 1e-9) as s:
            s.set_option("path", path)
            s.set_option("variant", variant)
            st = s.solve(w, 24)
            out[path] = (s.lambda_, s.residual_history(24), st, w.u.copy())
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    np.testing.assert_array_equal(out[0][3], out[1][3])
    assert out[1][2]["path"] == 1 and out[0][2]["path"] == 0


def test_full_size_city800_bit_exact_against_oracle():
    """The largest configuration, 800x800x128 with 150 buildings: the default
    (autotuned) sweep holds the oracle's lambda bits, residual history and
    corrected winds after 6 iterations."""
    w, _ = qesb.random_city("city800", 0)
    d = w.domain
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.autotune()
        st = s.solve(w, 6, set_inputs=False)
        L, H = s.lambda_, s.residual_history(6)
    assert st["path"] == 1 and st["iterations"] == 6
    R = O.divergence(d, w)
    Lo, it, _, Ho = O.sor(d, w, R, 1e-9, 6, hist=True)
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(H, Ho)
    uo, vo, wo = O.correct(d, w, Lo)
    np.testing.assert_array_equal(w.u, uo)
    np.testing.assert_array_equal(w.v, vo)
    np.testing.assert_array_equal(w.w, wo)


def test_autotune_restores_lambda_and_results_stay_exact(golden):
    d, w, z = golden("small_city.npz")
    lam0 = np.random.default_rng(7).standard_normal(d.numCellCentered()).astype(np.float32)
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.lambda_ = lam0
        best, us = s.autotune()
        assert 0 <= best < len(us) and all(u > 0 for u in us)
        np.testing.assert_array_equal(s.lambda_, lam0)
        st = s.solve(w, 150, set_inputs=False)
        L = s.lambda_
    Lo, it, *_ = O.sor(d, w, O.divergence(d, w), 1e-9, 150, lam=lam0)
    assert st["iterations"] == it == 150
    np.testing.assert_array_equal(L, Lo)


@pytest.mark.parametrize("variant", [5, 16, BULK + 1, ZM])
@pytest.mark.parametrize("omega,pre_tol,pre_max", [(1.9, 1e-3, 5000), (1.95, 5e-4, 150)])
def test_overrelaxed_prephase_then_reference_loop(variant, omega, pre_tol, pre_max):
    """qesb_set_prephase: red-black SOR with another omega until its own rule
    (or cap), then the reference loop (omega 1.78, the handle's tolerance)
    from that lambda; both phases bit-exact against the oracle."""
    d = qesb.Domain(70, 45, 21, 2.0, 2.0, 1.0, qesb.city_dz(21, 1.0, 1.03))
    c = qesb.city_random(d, 9, 8, fp=(6, 18), h=(4, 30))
    w = qesb.city_build(d, c.buildings, c.inflow)
    tol = 1.1e-3
    with qesb.Solver_B200(d, tol) as s:
        s.set_option("variant", variant)
        s.set_prephase(omega, pre_tol, pre_max)
        st = s.solve(w, 5000)
        L = s.lambda_
        u = w.u.copy()
    R = O.divergence(d, w)
    Lp, itp, *_ = O.sor(d, w, R, pre_tol, pre_max, omega=omega)
    Lo, it, *_ = O.sor(d, w, R, tol, 5000, lam=Lp)
    assert st["pre_iterations"] == itp
    assert st["iterations"] == it and st["converged"] == 1
    np.testing.assert_array_equal(L, Lo)
    np.testing.assert_array_equal(u, O.correct(d, w, Lo)[0])
