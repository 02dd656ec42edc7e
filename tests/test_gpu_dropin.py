"""The C++ drop-in: Solver_B200 derived from the reference's own Solver
class and registered in the reference's own SolverFactory as type 5 (the
registration of INTEGRATION.md applied to src/winds/SolverFactory.{h,cpp} by
oracle/Makefile), driven through Solver* exactly as qesWinds drives its
solver. Type 5's u, v, w and lambda must equal the oracle's red-black result
and those of the reference's type 1 (Solver_CPU_RB in this OpenMP build)
through the same factory."""
import os
import subprocess

import numpy as np
import pytest

import qesb
from oracle import oracle as O

DEMO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                    "solver_b200_demo")
needs_demo = pytest.mark.skipif(not os.path.exists(DEMO), reason="drop-in demo not built (needs the reference tree)")
Nx, Ny, Nz, SEED, NB, ITERMAX = 40, 32, 16, 2024, 5, 150


def _run(tmp_path, calls, solver_type):
    """One demo run. The reference's Solver_CPU_RB (type 1) runs on one OpenMP
    thread: with more, the unsynchronised max_error reset inside its parallel
    region (Solver_CPU_RB.cpp:166) can end a solve early, at random."""
    out = tmp_path / f"out_{solver_type}_{calls}.bin"
    r = subprocess.run([DEMO, str(out), str(Nx), str(Ny), str(Nz), str(SEED), str(NB), str(ITERMAX), "1e-9",
                        str(calls), str(solver_type)], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, OMP_NUM_THREADS="1"))
    return r, out


def _read(out):
    d = qesb.Domain(Nx, Ny, Nz, 2.0, 2.0, 1.0, qesb.city_dz(Nz, 1.0, 1.03))
    nf, nc = d.numFaceCentered(), d.numCellCentered()
    raw = np.fromfile(out, dtype=np.float32)
    assert raw.size == 3 * nf + nc
    return d, raw[:nf], raw[nf:2 * nf], raw[2 * nf:3 * nf], raw[3 * nf:]


def _oracle(d, calls):
    c = qesb.city_random(d, SEED, NB, fp=(6, 16), h=(4, 20))
    w = qesb.city_build(d, c.buildings, c.inflow)
    L = None
    for _ in range(calls):
        uo, vo, wo, L, it, _ = O.solve(d, w, 1e-9, ITERMAX, ordering=1, lam=L)
    return uo, vo, wo, L


@needs_demo
def test_factory_type_1_is_the_reference_red_black_solver(tmp_path):
    """Type 1 through the patched factory is the reference's own Solver_CPU_RB
    (this build has OpenMP): its result is the oracle's red-black result."""
    r, out = _run(tmp_path, 1, 1)
    assert r.returncode == 0, r.stderr
    assert "Red/Black CPU Solver" in r.stdout
    d, u, v, ww, lam = _read(out)
    uo, vo, wo, L = _oracle(d, 1)
    np.testing.assert_array_equal(lam, L)
    np.testing.assert_array_equal(u, uo)


@needs_demo
def test_factory_rejects_unknown_types_as_the_reference_does(tmp_path):
    r, _ = _run(tmp_path, 1, 9)
    assert r.returncode != 0
    assert "Invalid solver type" in r.stderr


@needs_demo
@pytest.mark.gpu
@pytest.mark.parametrize("calls", [1, 2])
def test_dropin_type_5_through_the_reference_factory(tmp_path, calls):
    r, out = _run(tmp_path, calls, 5)
    assert r.returncode == 0, r.stderr
    assert "B200 Solver" in r.stdout and f"Residual after {ITERMAX} itertations" in r.stdout
    d, u, v, ww, lam = _read(out)
    uo, vo, wo, L = _oracle(d, calls)
    np.testing.assert_array_equal(lam, L)
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(v, vo)
    np.testing.assert_array_equal(ww, wo)
    r1, out1 = _run(tmp_path, calls, 1)
    assert r1.returncode == 0, r1.stderr
    _, u1, v1, w1, lam1 = _read(out1)
    np.testing.assert_array_equal(lam, lam1)
    np.testing.assert_array_equal(u, u1)
    np.testing.assert_array_equal(ww, w1)


@needs_demo
@pytest.mark.gpu
def test_dropin_stair_step_inputs_from_cpp(tmp_path):
    """Solver_B200::useStairStepInputs: the adaptor uploads only icellflag and the
    initial winds (qesb_set_inputs_flags) and the library rebuilds e..n from the
    flags; the result is the oracle's red-black result, as with the full arrays."""
    out = tmp_path / "stair.bin"
    r = subprocess.run([DEMO, str(out), str(Nx), str(Ny), str(Nz), str(SEED), str(NB), str(ITERMAX), "1e-9", "2",
                        "5", "-", "stair"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d, u, v, ww, lam = _read(out)
    uo, vo, wo, L = _oracle(d, 2)
    np.testing.assert_array_equal(lam, L)
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(v, vo)
    np.testing.assert_array_equal(ww, wo)


@needs_demo
@pytest.mark.gpu
def test_dropin_learned_warm_start_from_cpp(tmp_path):
    """Solver_B200::useLearnedStart through the reference factory: the C++
    caller's solves from lambda = 0 start from the network (qesb_warm_start).
    The result is the same warm-started solve run from Python, bit for bit."""
    from qesb import warmstart as ws

    nx, ny, nz, itermax = 64, 48, 32, 120
    out = tmp_path / "warm.bin"
    r = subprocess.run([DEMO, str(out), str(nx), str(ny), str(nz), str(SEED), str(NB), str(itermax), "1e-9", "1",
                        "5", ws.DEFAULT_WEIGHTS], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Learned warm start" in r.stdout
    d = qesb.Domain(nx, ny, nz, 2.0, 2.0, 1.0, qesb.city_dz(nz, 1.0, 1.03))
    nf, nc = d.numFaceCentered(), d.numCellCentered()
    raw = np.fromfile(out, dtype=np.float32)
    lam = raw[3 * nf:]
    c = qesb.city_random(d, SEED, NB, fp=(6, 16), h=(4, 20))
    w = qesb.city_build(d, c.buildings, c.inflow)
    net = ws.WarmStartNet.from_file(ws.DEFAULT_WEIGHTS, device=0)
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        net.warm_start(s)
        s.solve(w, itermax, set_inputs=False)
        lam_py = s.lambda_
    np.testing.assert_array_equal(lam, lam_py)
    cold, *_ = O.sor(d, w, O.divergence(d, w), 1e-9, itermax)
    assert np.abs(lam - cold).max() > 0  # the start was the network's
