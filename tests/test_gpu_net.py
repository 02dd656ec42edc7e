"""Warm-start network kernels: the tcgen05 tensor-core core against numpy."""
import numpy as np
import pytest

import qesb

pytestmark = pytest.mark.gpu


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bfloat16 bit patterns."""
    b = np.ascontiguousarray(x, np.float32).view(np.uint32)
    return ((b + 0x7FFF + ((b >> 16) & 1)) >> 16).astype(np.uint16)


def bf16_value(bits: np.ndarray) -> np.ndarray:
    return (bits.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("N,K,a_mn,b_mn", [(16, 64, 0, 0), (32, 128, 0, 0), (64, 448, 0, 0), (128, 192, 0, 0),
                                           (256, 64, 0, 0), (64, 128, 1, 0), (64, 128, 0, 1), (128, 256, 1, 1),
                                           (16, 64, 1, 1)])
def test_umma_gemm_core(N, K, a_mn, b_mn):
    import ctypes as C

    rng = np.random.default_rng(N * 1000 + K + 7 * a_mn + 13 * b_mn)
    A = bf16_bits(rng.standard_normal((128, K)).astype(np.float32))
    B = bf16_bits(rng.standard_normal((N, K)).astype(np.float32))
    Af, Bf = bf16_value(A).astype(np.float64), bf16_value(B).astype(np.float64)
    ref = Af @ Bf.T
    Ain = np.ascontiguousarray(A.T) if a_mn else A
    Bin = np.ascontiguousarray(B.T) if b_mn else B
    out = np.zeros((128, N), np.float32)
    qesb.check(qesb.lib().qesb_umma_selftest(Ain.ctypes.data_as(C.c_void_p), Bin.ctypes.data_as(C.c_void_p),
                                             out.ctypes.data_as(C.c_void_p), N, K, a_mn, b_mn))
    np.testing.assert_allclose(out, ref, rtol=1e-5, atol=1e-4 * np.sqrt(K))


# ---------------------------------------------------------------------------
# implicit-GEMM conv3d kernels against torch (CPU, float64)
# ---------------------------------------------------------------------------
def _bf16(t):
    import torch
    return t.to(torch.bfloat16)


def _bm_forward(w):
    """torch weight [Cout][Cin][3][3][3] -> Bm [Cout][Kp], k = tap*Cin + c."""
    import torch
    co, ci = w.shape[:2]
    k = 27 * ci
    kp = (k + 63) // 64 * 64
    bm = torch.zeros(co, kp, dtype=w.dtype)
    bm[:, :k] = w.permute(0, 2, 3, 4, 1).reshape(co, k)
    return bm, kp


def _bm_dgrad(w):
    """Bd [Cin][Kp'], k = tap*Cout + co, tap of the forward kernel."""
    import torch
    co, ci = w.shape[:2]
    k = 27 * co
    kp = (k + 63) // 64 * 64
    bd = torch.zeros(ci, kp, dtype=w.dtype)
    bd[:, :k] = w.permute(1, 2, 3, 4, 0).reshape(ci, k)
    return bd, kp


def _cl(t):
    """[1][C][D][H][W] -> channels-last [D][H][W][C] contiguous."""
    return t[0].permute(1, 2, 3, 0).contiguous()


def _run_conv(x1, c1, up1, x2, c2, D, H, W, sign, bm, kp, n, bias=None, relu=0, mask=None):
    import torch
    dev = "cuda:0"
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    yf = torch.zeros(D * H * W * n, dtype=torch.float32, device=dev)
    g = lambda t: t.data_ptr() if t is not None else None
    qesb.check(qesb.lib().qesb_conv3d(g(x1), c1, up1, g(x2), c2, D, H, W, sign, g(bm), kp, n, None, g(yf),
                                      g(bias), relu, g(mask), g(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return yf.view(D, H, W, n).cpu().double()


@pytest.mark.parametrize("D,H,W,ci,co", [(8, 12, 20, 16, 32), (6, 8, 8, 32, 16), (4, 6, 10, 64, 128),
                                         (8, 8, 16, 128, 64)])
def test_conv3d_forward(D, H, W, ci, co):
    import torch
    torch.manual_seed(D * H + ci)
    x = _bf16(torch.randn(1, ci, D, H, W))
    w = _bf16(torch.randn(co, ci, 3, 3, 3) / (27 * ci) ** 0.5)
    b = torch.randn(co)
    ref = torch.nn.functional.conv3d(x.double(), w.double(), b.double(), padding=1)
    ref = torch.relu(ref)
    bm, kp = _bm_forward(w)
    dev = "cuda:0"
    xd, bmd, bd = _cl(x).to(dev), bm.to(dev), b.float().to(dev)
    out = _run_conv(xd, ci, 0, None, 0, D, H, W, 1, bmd, kp, co, bias=bd, relu=1)
    np.testing.assert_allclose(out.numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)


def test_conv3d_concat_upsampled_input():
    import torch
    torch.manual_seed(3)
    D, H, W, c1, c2, co = 8, 12, 20, 32, 16, 16
    x1 = _bf16(torch.randn(1, c1, D // 2, H // 2, W // 2))
    x2 = _bf16(torch.randn(1, c2, D, H, W))
    w = _bf16(torch.randn(co, c1 + c2, 3, 3, 3) / (27 * 48) ** 0.5)
    up = torch.nn.functional.interpolate(x1.double(), scale_factor=2, mode="nearest")
    ref = torch.nn.functional.conv3d(torch.cat([up, x2.double()], 1), w.double(), padding=1)
    bm, kp = _bm_forward(w)
    dev = "cuda:0"
    x1d, x2d, bmd = _cl(x1).to(dev), _cl(x2).to(dev), bm.to(dev)
    out = _run_conv(x1d, c1, 1, x2d, c2, D, H, W, 1, bmd, kp, co)
    np.testing.assert_allclose(out.numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("D,H,W,ci,co", [(8, 12, 20, 16, 32), (4, 6, 10, 64, 128)])
def test_conv3d_input_gradient_with_relu_mask(D, H, W, ci, co):
    import torch
    torch.manual_seed(11 + ci)
    x = torch.relu(_bf16(torch.randn(1, ci, D, H, W)).double())  # a ReLU output, as layer inputs are
    w = _bf16(torch.randn(co, ci, 3, 3, 3) / (27 * ci) ** 0.5)
    dy = _bf16(torch.randn(1, co, D, H, W))
    xr = x.clone().requires_grad_(True)
    y = torch.nn.functional.conv3d(xr, w.double(), padding=1)
    (y * dy.double()).sum().backward()
    ref = xr.grad * (x > 0)
    bd, kp = _bm_dgrad(w)
    dev = "cuda:0"
    dyd, bdd, md = _cl(dy).to(dev), bd.to(dev), _cl(_bf16(x)).to(dev)
    out = _run_conv(dyd, co, 0, None, 0, D, H, W, -1, bdd, kp, ci, mask=md)
    np.testing.assert_allclose(out.numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("D,H,W,ci,co,up", [(8, 12, 20, 16, 32, 0), (4, 6, 10, 64, 16, 0), (8, 8, 16, 32, 64, 1)])
def test_conv3d_weight_gradient(D, H, W, ci, co, up):
    import torch
    torch.manual_seed(5 + ci + up)
    dev = "cuda:0"
    if up:
        c1, c2 = ci, 16
        x1 = _bf16(torch.randn(1, c1, D // 2, H // 2, W // 2))
        x2 = _bf16(torch.randn(1, c2, D, H, W))
        xin = torch.cat([torch.nn.functional.interpolate(x1.double(), scale_factor=2, mode="nearest"),
                         x2.double()], 1)
    else:
        c1, c2 = ci, 0
        x1 = _bf16(torch.randn(1, ci, D, H, W))
        x2 = None
        xin = x1.double()
    cin = c1 + c2
    w = torch.zeros(co, cin, 3, 3, 3, dtype=torch.float64, requires_grad=True)
    dy = _bf16(torch.randn(1, co, D, H, W))
    y = torch.nn.functional.conv3d(xin, w, padding=1)
    (y * dy.double()).sum().backward()
    ref = w.grad.permute(2, 3, 4, 1, 0).reshape(27 * cin, co)  # [tap*cin + c][co]
    dW = torch.zeros(27 * cin * co, dtype=torch.float32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    # keep every device tensor referenced until the kernel has run
    x1d = _cl(x1).to(dev)
    x2d = _cl(x2).to(dev) if x2 is not None else None
    dyd = _cl(dy).to(dev)
    qesb.check(qesb.lib().qesb_conv3d_wgrad(x1d.data_ptr(), c1, up, x2d.data_ptr() if x2d is not None else None,
                                            c2, D, H, W, dyd.data_ptr(), co, 256, dW.data_ptr(), err.data_ptr(),
                                            None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    np.testing.assert_allclose(dW.view(27 * cin, co).cpu().double().numpy(), ref.numpy(), rtol=1e-4, atol=1e-3)


# ---------------------------------------------------------------------------
# direct conv3d kernel (rows of 128 voxels): same contract as the implicit GEMM
# ---------------------------------------------------------------------------
@pytest.fixture
def conv_path():
    yield lambda p: qesb.check(qesb.lib().qesb_net_set_conv_path(p))
    qesb.check(qesb.lib().qesb_net_set_conv_path(0))


@pytest.mark.parametrize("D,H,W,ci,co", [(4, 6, 128, 16, 16), (3, 5, 256, 16, 32), (4, 4, 128, 48, 16),
                                         (2, 3, 128, 32, 32)])
def test_conv3d_direct_forward_matches_torch_and_gemm(conv_path, D, H, W, ci, co):
    import torch
    torch.manual_seed(D * H + ci + co)
    x = _bf16(torch.randn(1, ci, D, H, W))
    w = _bf16(torch.randn(co, ci, 3, 3, 3) / (27 * ci) ** 0.5)
    b = torch.randn(co)
    ref = torch.relu(torch.nn.functional.conv3d(x.double(), w.double(), b.double(), padding=1))
    bm, kp = _bm_forward(w)
    dev = "cuda:0"
    xd, bmd, bd = _cl(x).to(dev), bm.to(dev), b.float().to(dev)
    out = _run_conv(xd, ci, 0, None, 0, D, H, W, 1, bmd, kp, co, bias=bd, relu=1)
    np.testing.assert_allclose(out.numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)
    conv_path(1)
    out_gemm = _run_conv(xd, ci, 0, None, 0, D, H, W, 1, bmd, kp, co, bias=bd, relu=1)
    np.testing.assert_allclose(out.numpy(), out_gemm.numpy(), rtol=1e-5, atol=1e-5)


def test_conv3d_direct_concat_upsampled_input():
    import torch
    torch.manual_seed(5)
    D, H, W, c1, c2, co = 4, 6, 128, 32, 16, 16
    x1 = _bf16(torch.randn(1, c1, D // 2, H // 2, W // 2))
    x2 = _bf16(torch.randn(1, c2, D, H, W))
    w = _bf16(torch.randn(co, c1 + c2, 3, 3, 3) / (27 * 48) ** 0.5)
    up = torch.nn.functional.interpolate(x1.double(), scale_factor=2, mode="nearest")
    ref = torch.nn.functional.conv3d(torch.cat([up, x2.double()], 1), w.double(), padding=1)
    bm, kp = _bm_forward(w)
    dev = "cuda:0"
    out = _run_conv(_cl(x1).to(dev), c1, 1, _cl(x2).to(dev), c2, D, H, W, 1, bm.to(dev), kp, co)
    np.testing.assert_allclose(out.numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("ci,co", [(16, 16), (32, 16), (16, 32)])
def test_conv3d_direct_input_gradient_with_relu_mask(ci, co):
    import torch
    D, H, W = 3, 4, 128
    torch.manual_seed(17 + ci + co)
    x = torch.relu(_bf16(torch.randn(1, ci, D, H, W)).double())
    w = _bf16(torch.randn(co, ci, 3, 3, 3) / (27 * ci) ** 0.5)
    dy = _bf16(torch.randn(1, co, D, H, W))
    xr = x.clone().requires_grad_(True)
    y = torch.nn.functional.conv3d(xr, w.double(), padding=1)
    (y * dy.double()).sum().backward()
    ref = xr.grad * (x > 0)
    bd, kp = _bm_dgrad(w)
    dev = "cuda:0"
    out = _run_conv(_cl(dy).to(dev), co, 0, None, 0, D, H, W, -1, bd.to(dev), kp, ci, mask=_cl(_bf16(x)).to(dev))
    np.testing.assert_allclose(out.numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("D,H,W,c1,c2,co,up", [(4, 6, 128, 16, 0, 16, 0), (4, 6, 64, 32, 0, 32, 0),
                                               (4, 6, 128, 32, 16, 16, 1), (2, 4, 32, 64, 64, 64, 1)])
def test_conv3d_items_stack_along_z_without_crosstalk(D, H, W, c1, c2, co, up):
    """qesb_conv3d_items: three grids stacked along z in one launch give, item
    by item, the convolution of each grid alone (zero padding at every item's
    z faces), against torch per item; direct and implicit-GEMM paths, with and
    without an upsampled concatenated input."""
    import torch
    torch.manual_seed(D + H + W + c1 + co)
    items, ci = 3, c1 + c2
    x1 = [_bf16(torch.randn(1, c1, D // 2, H // 2, W // 2) if up else torch.randn(1, c1, D, H, W))
          for _ in range(items)]
    x2 = [_bf16(torch.randn(1, c2, D, H, W)) for _ in range(items)] if c2 else None
    w = _bf16(torch.randn(co, ci, 3, 3, 3) / (27 * ci) ** 0.5)
    b = torch.randn(co)
    bm, kp = _bm_forward(w)
    dev = "cuda:0"
    x1d = torch.cat([_cl(t) for t in x1], 0).to(dev)
    x2d = torch.cat([_cl(t) for t in x2], 0).to(dev) if c2 else None
    bmd, bd = bm.to(dev), b.float().to(dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    yf = torch.zeros(items * D * H * W * co, dtype=torch.float32, device=dev)
    g = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
    qesb.check(qesb.lib().qesb_conv3d_items(g(x1d), c1, up, g(x2d), c2, items, D, H, W, 1, g(bmd), kp, co, None,
                                            g(yf), g(bd), 1, None, g(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    out = yf.view(items, D, H, W, co).cpu().double()
    for i in range(items):
        xin = torch.nn.functional.interpolate(x1[i].double(), scale_factor=2, mode="nearest") if up else x1[i].double()
        if c2:
            xin = torch.cat([xin, x2[i].double()], 1)
        ref = torch.relu(torch.nn.functional.conv3d(xin, w.double(), b.double(), padding=1))
        np.testing.assert_allclose(out[i].numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)


@pytest.mark.parametrize("path", [0, 2, 3, 4, 6])
@pytest.mark.parametrize("items,D,H,W,co", [(1, 1, 5, 128, 16), (1, 3, 6, 256, 32), (3, 4, 7, 128, 16),
                                            (2, 6, 4, 128, 32), (1, 17, 9, 128, 16), (2, 10, 6, 64, 32)])
def test_conv3d_zmarch_and_direct_paths_match_torch(conv_path, path, items, D, H, W, co):
    """The z-marching convolutions (tensor-map staging, planes through a ring,
    copies, MMAs and read-out of different planes overlapping): three output
    planes per MMA (path 0) and one (path 6), 2 and 4 rows per CTA (paths 3,
    4), and the direct kernel, for 16-channel forward convolutions: odd heights
    (partial row tiles), one-plane and many-plane items cut into z chunks,
    stacked items, rows of 256, 128 and 64; against torch per item."""
    import torch
    torch.manual_seed(items + D + H + W + co + path)
    ci = 16
    xs = [_bf16(torch.randn(1, ci, D, H, W)) for _ in range(items)]
    w = _bf16(torch.randn(co, ci, 3, 3, 3) / (27 * ci) ** 0.5)
    b = torch.randn(co)
    bm, kp = _bm_forward(w)
    dev = "cuda:0"
    xd = torch.cat([_cl(t) for t in xs], 0).to(dev)
    bmd, bd = bm.to(dev), b.float().to(dev)
    conv_path(path)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    for relu, fp32 in ((1, True), (0, False)):
        yf = torch.zeros(items * D * H * W * co, dtype=torch.float32, device=dev) if fp32 else None
        y = None if fp32 else torch.zeros(items * D * H * W * co, dtype=torch.bfloat16, device=dev)
        g = lambda t: t.data_ptr() if t is not None else None  # noqa: E731
        qesb.check(qesb.lib().qesb_conv3d_items(g(xd), ci, 0, None, 0, items, D, H, W, 1, g(bmd), kp, co, g(y),
                                                g(yf), g(bd), relu, None, g(err), None))
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        out = (yf if fp32 else y.float()).view(items, D, H, W, co).cpu().double()
        for i in range(items):
            ref = torch.nn.functional.conv3d(xs[i].double(), w.double(), b.double(), padding=1)
            if relu:
                ref = torch.relu(ref)
            tol = 1e-4 if fp32 else 1e-2
            np.testing.assert_allclose(out[i].numpy(), _cl(ref).numpy(), rtol=tol, atol=tol)


@pytest.mark.parametrize("items,D,H,W,c1,c2,up,co", [
    (2, 4, 6, 64, 16, 0, 0, 32),     # rows of 64, a partial row tile
    (1, 5, 9, 64, 32, 0, 0, 32),
    (2, 4, 8, 64, 64, 32, 1, 32),    # upsampled + concatenated input, split over its channels
    (2, 4, 8, 32, 32, 0, 0, 64),     # rows of 32
    (1, 4, 10, 32, 64, 0, 0, 64),    # rows of 32 that would need a split: the implicit GEMM instead
    (1, 4, 6, 128, 32, 16, 1, 16),   # rows of 128, one output row per CTA (48 channels unsplit)
    (2, 2, 3, 128, 16, 0, 0, 32),
    (1, 4, 4, 256, 16, 16, 0, 16),   # two row tiles, a concatenation without upsampling
    (1, 2, 4, 64, 128, 64, 1, 64),   # twelve channel splits
])
def test_conv3d_zmarch_flat_windows_match_torch(conv_path, items, D, H, W, c1, c2, up, co):
    """The default forward path: the z-marching kernel with flattened 128-row
    windows (rows of 64 and 32 voxels), concatenated and upsampled inputs
    (the upsampling done on the output grid first), and channel splits whose
    FP32 partial sums are added in launch order; stacked items, partial row
    tiles; against torch per item and against the implicit GEMM."""
    import torch
    torch.manual_seed(items + D + H + W + c1 + c2 + co)
    ci = c1 + c2
    x1 = [_bf16(torch.randn(1, c1, D // 2, H // 2, W // 2) if up else torch.randn(1, c1, D, H, W))
          for _ in range(items)]
    x2 = [_bf16(torch.randn(1, c2, D, H, W)) for _ in range(items)] if c2 else None
    w = _bf16(torch.randn(co, ci, 3, 3, 3) / (27 * ci) ** 0.5)
    b = torch.randn(co)
    bm, kp = _bm_forward(w)
    dev = "cuda:0"
    x1d = torch.cat([_cl(t) for t in x1], 0).to(dev)
    x2d = torch.cat([_cl(t) for t in x2], 0).to(dev) if c2 else None
    bmd, bd = bm.to(dev), b.float().to(dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    g = lambda t: t.data_ptr() if t is not None else None  # noqa: E731

    def run():
        yf = torch.zeros(items * D * H * W * co, dtype=torch.float32, device=dev)
        qesb.check(qesb.lib().qesb_conv3d_items(g(x1d), c1, up, g(x2d), c2, items, D, H, W, 1, g(bmd), kp, co,
                                                None, g(yf), g(bd), 1, None, g(err), None))
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        return yf.view(items, D, H, W, co).cpu().double()

    conv_path(0)
    out = run()
    for i in range(items):
        xin = torch.nn.functional.interpolate(x1[i].double(), scale_factor=2, mode="nearest") if up else x1[i].double()
        if c2:
            xin = torch.cat([xin, x2[i].double()], 1)
        ref = torch.relu(torch.nn.functional.conv3d(xin, w.double(), b.double(), padding=1))
        np.testing.assert_allclose(out[i].numpy(), _cl(ref).numpy(), rtol=1e-4, atol=1e-4)
    conv_path(1)
    np.testing.assert_allclose(out.numpy(), run().numpy(), rtol=1e-5, atol=1e-5)
