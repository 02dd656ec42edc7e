"""The C++ drop-in: Solver_B200 derived from the reference's own Solver
class (built by oracle/Makefile against src/winds/Solver.h with the shim
WINDSGeneralData), driven through Solver* exactly as qesWinds drives its
solver. Its u, v, w and lambda must equal the oracle's red-black result."""
import os
import subprocess

import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEMO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                    "solver_b200_demo")


@pytest.mark.skipif(not os.path.exists(DEMO), reason="drop-in demo not built (needs the reference tree)")
@pytest.mark.parametrize("calls", [1, 2])
def test_dropin_through_reference_solver_base(tmp_path, calls):
    Nx, Ny, Nz, seed, nb, itermax = 40, 32, 16, 2024, 5, 150
    out = tmp_path / "out.bin"
    r = subprocess.run([DEMO, str(out), str(Nx), str(Ny), str(Nz), str(seed), str(nb), str(itermax),
                        "1e-9", str(calls)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert f"Residual after {itermax} itertations" in r.stdout
    d = qesb.Domain(Nx, Ny, Nz, 2.0, 2.0, 1.0, qesb.city_dz(Nz, 1.0, 1.03))
    c = qesb.city_random(d, seed, nb, fp=(6, 16), h=(4, 20))
    w = qesb.city_build(d, c.buildings, c.inflow)
    nf, nc = d.numFaceCentered(), d.numCellCentered()
    raw = np.fromfile(out, dtype=np.float32)
    assert raw.size == 3 * nf + nc
    u, v, ww, lam = raw[:nf], raw[nf:2 * nf], raw[2 * nf:3 * nf], raw[3 * nf:]
    L = None
    for _ in range(calls):
        uo, vo, wo, L, it, _ = O.solve(d, w, 1e-9, itermax, ordering=1, lam=L)
    np.testing.assert_array_equal(lam, L)
    np.testing.assert_array_equal(u, uo)
    np.testing.assert_array_equal(v, vo)
    np.testing.assert_array_equal(ww, wo)
