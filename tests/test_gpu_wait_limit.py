"""Bounded device waits end in an error status, not a hang.

The bulk-copy sweep kernels, and the z-march shapes staged by tensor-map
copies, wait on a shared-memory barrier for each stage's copies. With the handle option "wait_limit" at 1 poll, a correct solve on
correct data meets stages whose copies have not landed yet: the kernel gives
up, lets its copies in flight land, flags the fault and returns, and the solve
reports QESB_ERR_CUDA. With the limit back at its default, the same handle
solves again and matches the oracle bit for bit.
"""
import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# option "variant" index of bulk_w4_s3, the first bulk-copy sweep shape
# (after the 5 fused tile shapes and the 13 streaming split shapes), and of
# zmt_y4x2_b5, the first z-march shape staged by tensor-map copies, and of zmtb_y4x2_b5
BULK_W4_S3 = 18
ZMT_Y4X2_B5 = 51
ZMTB_Y4X2_B5 = 59  # the same with equal plane-step shares per CTA


def _city():
    d = qesb.Domain(96, 80, 24, 2.0, 2.0, 1.0, qesb.city_dz(24, 1.0, 1.03))
    c = qesb.city_random(d, 11, 8, fp=(6, 20), h=(4, 30))
    return d, qesb.city_build(d, c.buildings, c.inflow)


@pytest.mark.parametrize("variant", [BULK_W4_S3, ZMT_Y4X2_B5, ZMTB_Y4X2_B5])
def test_stage_wait_timeout_is_an_error_status_and_the_handle_recovers(variant):
    d, w = _city()
    itermax = 60
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.set_option("variant", variant)
        s.set_option("wait_limit", 1)
        with pytest.raises(qesb.QesbError) as ei:
            s.solve(w, itermax, set_inputs=False)
        assert ei.value.status == 2
        assert "stage wait gave up" in str(ei.value)
        s.set_option("wait_limit", 0)
        s.resetLambda()
        st = s.solve(w, itermax, set_inputs=False)
        lam = s.lambda_
    assert st["iterations"] == itermax
    u, v, ww, L, it, _ = O.solve(d, w, 1e-9, itermax, ordering=1)
    assert it == itermax
    np.testing.assert_array_equal(lam, L)
    np.testing.assert_array_equal(w.u, u)
    np.testing.assert_array_equal(w.w, ww)


def test_wait_limit_rejects_negative_values():
    d, _ = _city()
    with qesb.Solver_B200(d, 1e-9) as s:
        with pytest.raises(qesb.QesbError):
            s.set_option("wait_limit", -1)
