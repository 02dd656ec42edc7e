"""The FP64 run of the same SOR on the device (qesb_fp64_same_sor), the
precision check of an FP32 solve: bit for bit the oracle's double-precision
restatement on a small city (R, pre-phase, reference loop, correction), and
at 800 x 800 x 128 the FP32 pipeline's winds within 1e-3 m/s of it."""
import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

WIND_TOL = 1e-3


@pytest.mark.parametrize("start", [None, (1.6, 10)])
def test_fp64_replay_matches_the_oracle_bit_for_bit(start):
    """With a pre-phase start stage set, the replay runs it too: its first
    sweeps at the stage's omega, as the FP32 solve did."""
    import torch

    d = qesb.Domain(72, 56, 24, 2.0, 2.0, 1.0, qesb.city_dz(24, 1.0, 1.03))
    c = qesb.city_random(d, 31, 7, fp=(6, 20), h=(4, 30))
    w = qesb.city_build(d, c.buildings, c.inflow)
    nf = d.numFaceCentered()
    uvw = [torch.empty(nf, dtype=torch.float32, device="cuda") for _ in range(3)]
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.set_prephase(1.9, 3e-3, 2000)
        if start:
            s.set_prephase_start(*start)
        s.set_window_rule(16, 1e-2)
        st = s.solve_device(3000, *[t.data_ptr() for t in uvw])
        rep = s.fp64_same_sor(1.9, st["pre_iterations"], st["iterations"], *[t.data_ptr() for t in uvw],
                              want_lambda=True)
        lam32 = s.lambda_
    assert st["pre_iterations"] > 0 and st["converged"] == 2
    npre = st["pre_iterations"]
    phases = [(start[0], -1.0, start[1]), (1.9, -1.0, npre - start[1])] if start else [(1.9, -1.0, npre)]
    u64, v64, w64, L64, _, _ = O.solve_f64(d, w, -1.0, st["iterations"], phases=phases)
    np.testing.assert_array_equal(rep["lambda64"], L64)
    assert rep["lambda_max_abs"] == np.abs(L64).max()
    assert rep["lambda_max_abs_err"] == np.abs(lam32.astype(np.float64) - L64).max()
    winds = [t.cpu().numpy().astype(np.float64) for t in uvw]
    assert rep["wind_max_err"] == max(np.abs(a - b).max() for a, b in zip(winds, (u64, v64, w64)))
    assert 0 < rep["wind_max_err"] < WIND_TOL


def test_city800_winds_within_tolerance_of_the_fp64_run():
    """800 x 800 x 128, 150 buildings: the pre-phase pipeline to the
    benchmark's rule in FP32, then the same SOR in FP64 with its iteration
    counts; the FP32 winds stay within 1e-3 m/s of the FP64 ones."""
    import torch

    w, _ = qesb.random_city("city800", 0)
    d = w.domain
    nf = d.numFaceCentered()
    uvw = [torch.empty(nf, dtype=torch.float32, device="cuda") for _ in range(3)]
    om = qesb.prephase_omega(800, 800)
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.set_prephase(om, 3e-3, 10000)
        s.set_window_rule(32, 4e-3)
        st = s.solve_device(10000, *[t.data_ptr() for t in uvw])
        rep = s.fp64_same_sor(om, st["pre_iterations"], st["iterations"], *[t.data_ptr() for t in uvw])
    assert rep["wind_max_err"] < WIND_TOL, rep
    assert rep["lambda_max_abs_err"] / rep["lambda_max_abs"] < 1e-4, rep
