"""qesb_solve_noalloc: the solve for callers that cannot allocate device memory.

Callers whose GPU memory is owned by another allocator, or long-running loops
that must not allocate after start-up, get a solve whose scratch lives in a
fixed device array inside the library. Here it is checked, through the C ABI,
against the handle-based entry point (qesb_solve_device) on two calls in a
row: lambda carried over between calls must give the same bits on both
paths, since both round every operation as the reference does. This file is
collected last so that a failing run that stops at the first failure has
already run every other test; it needs nothing from them and passes alone.
"""
import numpy as np
import pytest

import qesb

pytestmark = pytest.mark.gpu


def _city():
    d = qesb.Domain(72, 56, 24, 2.0, 2.0, 1.0, qesb.city_dz(24, 1.0, 1.03))
    c = qesb.city_random(d, 31, 7, fp=(6, 20), h=(4, 30))
    return d, qesb.city_build(d, c.buildings, c.inflow)


def test_noalloc_matches_handle_solve_on_two_calls():
    import torch

    d, w = _city()
    dev = torch.device("cuda:0")
    ins = [torch.from_numpy(a).to(dev) for a in w.inputs()]
    ptrs = [t.data_ptr() for t in ins]
    nf, nc = d.numFaceCentered(), d.numCellCentered()
    lam0 = np.random.default_rng(5).standard_normal(nc).astype(np.float32)
    itermax, tol = 90, 1e-9

    # existing entry point: handle, device inputs, lambda kept on the handle
    ref_out = []
    with qesb.Solver_B200(d, tol) as s:
        s.set_inputs_device(*ptrs)
        s.lambda_ = lam0
        for _ in range(2):
            uvw = [torch.empty(nf, dtype=torch.float32, device=dev) for _ in range(3)]
            st = s.solve_device(itermax, *[t.data_ptr() for t in uvw])
            torch.cuda.synchronize()
            ref_out.append(([t.cpu().numpy() for t in uvw], s.lambda_, st["iterations"]))

    # no-allocation entry point: the caller's lambda buffer carries over
    lam = torch.from_numpy(lam0.copy()).to(dev)
    for call in range(2):
        uvw = [torch.full((nf,), float("nan"), dtype=torch.float32, device=dev) for _ in range(3)]
        st = qesb.solve_noalloc(d, tol, itermax, *ptrs, lam.data_ptr(), *[t.data_ptr() for t in uvw])
        torch.cuda.synchronize()
        (ru, rv, rw), rl, rit = ref_out[call]
        assert st["iterations"] == rit == itermax
        np.testing.assert_array_equal(lam.cpu().numpy(), rl)
        np.testing.assert_array_equal(uvw[0].cpu().numpy(), ru)
        np.testing.assert_array_equal(uvw[1].cpu().numpy(), rv)
        np.testing.assert_array_equal(uvw[2].cpu().numpy(), rw)


def _handle_solve(d, ptrs, lam0, itermax, tol):
    import torch

    dev = torch.device("cuda:0")
    nf = d.numFaceCentered()
    with qesb.Solver_B200(d, tol) as s:
        s.set_inputs_device(*ptrs)
        s.lambda_ = lam0
        uvw = [torch.empty(nf, dtype=torch.float32, device=dev) for _ in range(3)]
        st = s.solve_device(itermax, *[t.data_ptr() for t in uvw])
        torch.cuda.synchronize()
        return st, s.lambda_, [t.cpu().numpy() for t in uvw]


def test_noalloc_stops_inside_a_chunk_like_the_handle_solve():
    """tol 1e-3 on this city stops at iteration 186 (the oracle's count),
    inside the entry point's third 64-iteration chunk: the kernels after the
    stop must leave lambda alone and the host loop must end there."""
    import torch

    from oracle import oracle as O

    d, w = _city()
    dev = torch.device("cuda:0")
    ins = [torch.from_numpy(a).to(dev) for a in w.inputs()]
    ptrs = [t.data_ptr() for t in ins]
    nc, nf = d.numCellCentered(), d.numFaceCentered()
    tol, itermax = 1e-3, 300
    _, it_oracle, _, _ = O.sor(d, w, O.divergence(d, w), tol, itermax)
    assert it_oracle % 64 != 0 and it_oracle < itermax
    rst, rlam, (ru, rv, rw) = _handle_solve(d, ptrs, np.zeros(nc, np.float32), itermax, tol)
    lam = torch.zeros(nc, dtype=torch.float32, device=dev)
    uvw = [torch.empty(nf, dtype=torch.float32, device=dev) for _ in range(3)]
    st = qesb.solve_noalloc(d, tol, itermax, *ptrs, lam.data_ptr(), *[t.data_ptr() for t in uvw])
    torch.cuda.synchronize()
    assert st["iterations"] == rst["iterations"] == it_oracle
    assert st["converged"] == rst["converged"] == 1
    assert st["residual"] == rst["residual"] <= tol
    np.testing.assert_array_equal(lam.cpu().numpy(), rlam)
    for a, b in zip(uvw, (ru, rv, rw)):
        np.testing.assert_array_equal(a.cpu().numpy(), b)


def test_noalloc_zero_iterations_corrects_the_given_lambda():
    import torch

    d, w = _city()
    dev = torch.device("cuda:0")
    ins = [torch.from_numpy(a).to(dev) for a in w.inputs()]
    ptrs = [t.data_ptr() for t in ins]
    nc, nf = d.numCellCentered(), d.numFaceCentered()
    lam0 = np.random.default_rng(9).standard_normal(nc).astype(np.float32)
    rst, rlam, (ru, rv, rw) = _handle_solve(d, ptrs, lam0, 0, 1e-9)
    lam = torch.from_numpy(lam0.copy()).to(dev)
    uvw = [torch.empty(nf, dtype=torch.float32, device=dev) for _ in range(3)]
    st = qesb.solve_noalloc(d, 1e-9, 0, *ptrs, lam.data_ptr(), *[t.data_ptr() for t in uvw])
    torch.cuda.synchronize()
    assert st["iterations"] == rst["iterations"] == 0
    np.testing.assert_array_equal(lam.cpu().numpy(), lam0)
    for a, b in zip(uvw, (ru, rv, rw)):
        np.testing.assert_array_equal(a.cpu().numpy(), b)


def test_noalloc_reports_nan_in_lambda():
    """A NaN initial wind reaches R and then lambda: the solve stops and
    returns QESB_ERR_NUMERIC (the array keeps no state that a later call
    could trip over: the next call on good inputs matches the handle path)."""
    import torch

    d, w = _city()
    dev = torch.device("cuda:0")
    nc, nf = d.numCellCentered(), d.numFaceCentered()
    bad_u0 = w.u0.copy()
    bad_u0[d.face(30, 20, 5)] = np.nan
    bad = [torch.from_numpy(a).to(dev) for a in w.inputs()[:7] + (bad_u0,) + w.inputs()[8:]]
    lam = torch.zeros(nc, dtype=torch.float32, device=dev)
    uvw = [torch.empty(nf, dtype=torch.float32, device=dev) for _ in range(3)]
    with pytest.raises(qesb.QesbError) as ei:
        qesb.solve_noalloc(d, 1e-9, 50, *[t.data_ptr() for t in bad], lam.data_ptr(),
                           *[t.data_ptr() for t in uvw])
    assert ei.value.status == 5
    good = [torch.from_numpy(a).to(dev) for a in w.inputs()]
    ptrs = [t.data_ptr() for t in good]
    rst, rlam, _ = _handle_solve(d, ptrs, np.zeros(nc, np.float32), 40, 1e-9)
    lam.zero_()
    st = qesb.solve_noalloc(d, 1e-9, 40, *ptrs, lam.data_ptr(), *[t.data_ptr() for t in uvw])
    torch.cuda.synchronize()
    assert st["iterations"] == rst["iterations"] == 40
    np.testing.assert_array_equal(lam.cpu().numpy(), rlam)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    big = qesb.Domain(400, 400, 100, 2.0, 2.0, 1.0)  # 16.2 M cells > the built-in maximum
    one = torch.zeros(1, dtype=torch.float32, device="cuda:0").data_ptr()
    with pytest.raises(qesb.QesbError) as ei:
        qesb.solve_noalloc(big, 1e-3, 10, *([one] * 14))
    assert ei.value.status == 1
    assert "exceeds the built-in scratch" in str(ei.value)
