"""The log-law wall treatment on the GPU (qesb_wall_log_law) against the
oracle's restatement of Wall::wallLogBC (pinned to the reference build in
tests/test_wall_log_oracle.py) and the reference's own fixture.

Tolerance: the reference evaluates atan2, cos and sin of floats with the C
library's float functions (its atan2f is not correctly rounded); the kernel
evaluates them in double and rounds to float, so a treated face may differ by a
float ulp or two of its speed. A later side reads faces an earlier side wrote,
so such a difference also reaches faces of smaller speed (an ulp of a 0.5 m/s
neighbour, 6e-8 m/s, lands on a 0.014 m/s face). The bound is therefore
absolute: |diff| <= REL x the largest speed among the reference's treated faces
(about four float ulps of it; measured: at most 1.2e-6 m/s at ~8 m/s, 81-98 %
of treated faces bit-identical). Everything else (the distances' logarithms,
|U| in double, the 20-step u* iteration in float) is the reference's
arithmetic, so a wrong formula or side order would show as errors of the order
of the speed. At least MATCH of the treated faces must be bit-identical, and
every other face must be untouched."""
import os

import numpy as np
import pytest

import qesb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

REL = 1e-6
MATCH = 0.5


def _log_law_gpu(d, flag, z0, u, v, w, dz):
    import torch

    wgd = qesb.WINDSGeneralData(d)
    wgd.icellflag = np.ascontiguousarray(flag, dtype=np.int32)
    t = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda() for a in (u, v, w)]
    with qesb.Solver_B200(d, 1e-3) as s:
        s.set_inputs(wgd)
        s.wall_log_law(z0, dz, *[x.data_ptr() for x in t])
    torch.cuda.synchronize()
    return [x.cpu().numpy() for x in t]


def _compare(got, ref, before):
    changed = np.zeros(got[0].size, bool)
    for g, r, b in zip(got, ref, before):
        changed |= r != b
    bound = REL * float(np.max(np.sqrt(sum(r[changed].astype(np.float64) ** 2 for r in ref))))
    stats = []
    for g, r, b in zip(got, ref, before):
        np.testing.assert_array_equal(g[~changed], b[~changed])  # untreated faces untouched
        err = np.abs(g[changed].astype(np.float64) - r[changed])
        assert np.all(err <= bound), float(np.max(err / bound))
        stats.append((float(err.max()) if err.size else 0.0, float(np.mean(g[changed] == r[changed]))))
    assert min(m for _, m in stats) >= MATCH, stats
    return int(changed.sum()), stats


def test_matches_reference_fixture():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "wall_log_city.npz"))
    d = qesb.Domain(int(z["Nx"]), int(z["Ny"]), int(z["Nz"]), float(z["dx"]), float(z["dy"]), 1.0, z["dz_array"])
    u, v, w = z["u"], z["v"], z["w"]
    ref = [a.copy() for a in (u, v, w)]
    for a, r in zip(ref, (z["ref_u"], z["ref_v"], z["ref_w"])):
        a[z["changed"]] = r
    got = _log_law_gpu(d, z["icellflag"], float(z["z0"]), u, v, w, float(np.min(z["dz_array"])))
    n, stats = _compare(got, ref, (u, v, w))
    print("fixture: faces treated", n, "max |diff| and identical fraction per component", stats)


@pytest.mark.parametrize("seed,z0", [(5, 0.1), (17, 0.03)])
def test_solve_then_log_law_matches_oracle(seed, z0):
    """A solve on the GPU, then the log law on its device winds, against the
    oracle's solve (bit-identical winds) and its wallLogBC restatement."""
    import torch

    d = qesb.Domain(96, 80, 24, 2.0, 2.0, 1.0, qesb.city_dz(24, 1.0, 1.04))
    c = qesb.city_random(d, seed, 12, fp=(8, 20), h=(6, 30))
    bl = list(c.buildings) + [qesb.Building(20.0, 24.0, 16.0, 12.0, 14.0, 4.0)]  # raised: walls above
    w = qesb.city_build(d, bl, c.inflow)
    nf = d.numFaceCentered()
    t = [torch.zeros(nf, dtype=torch.float32, device="cuda") for _ in range(3)]
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.solve_device(120, *[x.data_ptr() for x in t])
        before = [x.cpu().numpy() for x in t]
        dz = float(np.min(d.dz_array))
        s.wall_log_law(z0, dz, *[x.data_ptr() for x in t])
        got = [x.cpu().numpy() for x in t]
    uo, vo, wo, _, _, _ = O.solve(d, w, 1e-9, 120, ordering=1, err_fp64=True)
    for a, b in zip(before, (uo, vo, wo)):
        np.testing.assert_array_equal(a, b)
    ref = O.wall_log(d, w.icellflag, z0, uo, vo, wo, dz=dz)
    n, stats = _compare(got, ref, before)
    assert n > 1000
    print("seed", seed, "faces treated", n, stats)


def test_full_size_city256():
    """The benchmark's 256x256x64 city: log law on the GPU after 40 iterations,
    against the restatement applied to the same winds."""
    import torch

    w, _ = qesb.random_city("city256", 500003)
    d = w.domain
    t = [torch.zeros(d.numFaceCentered(), dtype=torch.float32, device="cuda") for _ in range(3)]
    with qesb.Solver_B200(d, 1e-9) as s:
        s.set_inputs(w)
        s.solve_device(40, *[x.data_ptr() for x in t])
        before = [x.cpu().numpy() for x in t]
        dz = float(np.min(d.dz_array))
        s.wall_log_law(0.1, dz, *[x.data_ptr() for x in t])
        got = [x.cpu().numpy() for x in t]
    ref = O.wall_log(d, w.icellflag, 0.1, *before, dz=dz)
    n, stats = _compare(got, ref, before)
    print("city256 faces treated", n, stats)


def test_cut_cell_flags_are_rejected_unchanged():
    import torch

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "wall_log_city.npz"))
    d = qesb.Domain(int(z["Nx"]), int(z["Ny"]), int(z["Nz"]), float(z["dx"]), float(z["dy"]), 1.0, z["dz_array"])
    flag = z["icellflag"].copy()
    Nx, Ny, _ = d.base
    flag[3 * Nx * Ny + 2 * Nx + 5] = 8
    wgd = qesb.WINDSGeneralData(d)
    wgd.icellflag = flag
    t = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (z["u"], z["v"], z["w"])]
    with qesb.Solver_B200(d, 1e-3) as s:
        s.set_inputs(wgd)
        with pytest.raises(qesb.QesbError):
            s.wall_log_law(0.1, 1.0, *[x.data_ptr() for x in t])
        with pytest.raises(qesb.QesbError):
            s.wall_log_law(0.0, 1.0, *[x.data_ptr() for x in t])
    for x, a in zip(t, (z["u"], z["v"], z["w"])):
        np.testing.assert_array_equal(x.cpu().numpy(), a)
