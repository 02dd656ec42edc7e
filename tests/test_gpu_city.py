"""Device-side input set-up (qesb_city_build_device): flags, wall
coefficients and initial winds equal the host generator's bit for bit, and a
solve from them equals the solve from the host-built inputs."""
import numpy as np
import pytest

import qesb

pytestmark = pytest.mark.gpu

NAMES = ("icellflag", "e", "f", "g", "h", "m", "n", "u0", "v0", "w0")


def _device_build(d, buildings, inflow):
    import torch

    nc, nf = d.numCellCentered(), d.numFaceCentered()
    t = {k: torch.full((nc,), -7, dtype=torch.int32, device="cuda") for k in ("icellflag",)}
    for k in ("e", "f", "g", "h", "m", "n"):
        t[k] = torch.full((nc,), float("nan"), dtype=torch.float32, device="cuda")
    for k in ("u0", "v0", "w0"):
        t[k] = torch.full((nf,), float("nan"), dtype=torch.float32, device="cuda")
    qesb.city_build_device(d, buildings, inflow, {k: v.data_ptr() for k, v in t.items()})
    return t


def _cases():
    out = []
    for name, seed in (("city128", 1000), ("city256", 500003)):
        w, c = qesb.random_city(name, seed)
        out.append((w.domain, c.buildings, c.inflow))
    # uneven grid, buildings touching the edges, raised bases, overlaps
    d = qesb.Domain(53, 37, 19, 2.0, 2.0, 1.0, qesb.city_dz(19, 1.0, 1.05))
    b = [qesb.Building(1.0, 1.0, 20.0, 12.0, 9.0, 0.0), qesb.Building(90.0, 60.0, 30.0, 30.0, 14.0, 3.5),
         qesb.Building(40.0, 20.0, 15.0, 15.0, 6.0, 0.0), qesb.Building(45.0, 25.0, 12.0, 8.0, 20.0, 2.0),
         qesb.Building(0.0, 70.0, 105.0, 4.0, 3.0, 0.0)]
    out.append((d, b, qesb.Inflow(6.5, 10.0, 0.2, 33.0)))
    w = qesb.cuboid100()
    out.append((w.domain, [qesb.Building(40.0, 40.0, 20.0, 20.0, 20.0, 0.0)], qesb.Inflow(5.0, 10.0, 0.15, 270.0)))
    return out


@pytest.mark.parametrize("case", range(4))
def test_device_build_equals_host_build(case):
    d, b, inflow = _cases()[case]
    host = qesb.city_build(d, b, inflow)
    dev = _device_build(d, b, inflow)
    for k in NAMES:
        np.testing.assert_array_equal(dev[k].cpu().numpy(), getattr(host, k), err_msg=k)


def test_solve_from_device_inputs_equals_host_inputs():
    import torch

    d, b, inflow = _cases()[2]
    host = qesb.city_build(d, b, inflow)
    dev = _device_build(d, b, inflow)
    with qesb.Solver_B200(d, 1.1e-3) as s:
        s.set_inputs_device(*[dev[k].data_ptr() for k in ("e", "f", "g", "h", "m", "n", "icellflag", "u0", "v0",
                                                          "w0")])
        outs = [torch.zeros(d.numFaceCentered(), dtype=torch.float32, device="cuda") for _ in range(3)]
        st_dev = s.solve_device(3000, *[o.data_ptr() for o in outs])
        L_dev = s.lambda_
    with qesb.Solver_B200(d, 1.1e-3) as s:
        st_host = s.solve(host, 3000)
        L_host = s.lambda_
    assert st_dev["iterations"] == st_host["iterations"]
    np.testing.assert_array_equal(L_dev, L_host)
    np.testing.assert_array_equal(outs[0].cpu().numpy(), host.u)
