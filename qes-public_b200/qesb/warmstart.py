"""Learned warm start for the lambda solve.

A 4-level 3D convolutional encoder-decoder (channels 16 -> 32 -> 64 -> 128,
2x2x2 average pooling down, nearest upsampling and skip concatenation up)
maps per-cell features of a domain (R / max|R|, solid flag, dz profile,
boundary flag, height) to lambda / max|R|. Every convolution (forward, input
gradient, weight gradient) runs in the library's tcgen05 kernels with BF16
operands and FP32 accumulation (qesb_conv3d, qesb_conv3d_wgrad); pooling,
gradient routing, the loss and Adam are the library's kernels too. torch only
provides device buffers and the stream.

The prediction is written into a solver handle as its starting lambda; SOR
then runs to the same stopping rule as from lambda = 0, so the network can
only change how many sweeps are needed, never the answer's tolerance.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from . import Solver_B200, check, lib

IN_CH = 16           # input channels (5 used, zero-padded to a tensor-core multiple)
HEAD_N = 16          # head GEMM width (channel 0 is the prediction)


def _p(t):
    return None if t is None else t.data_ptr()


def _kpad(k):
    return (k + 63) // 64 * 64


class Conv:
    """One 3x3x3 convolution: FP32 master weights W[27*cin][cout] (row
    tap*cin + c), Adam moments, and the two BF16 GEMM layouts the kernels
    read: Bm[cout][Kp] (forward) and Bd[cin][Kd] (input gradient)."""

    def __init__(self, torch, dev, c1, c2, cout, relu, up1, cin_real=None, cout_real=None, init_std=None,
                 gen=None):
        self.c1, self.c2, self.cout, self.relu, self.up1 = c1, c2, cout, relu, up1
        self.cin = c1 + c2
        self.cout_real = cout if cout_real is None else cout_real
        self.Kp, self.Kd = _kpad(27 * self.cin), _kpad(27 * cout)
        n = 27 * self.cin * cout
        cr = self.cin if cin_real is None else cin_real
        std = math.sqrt(2.0 / (27 * cr)) if init_std is None else init_std
        w = torch.randn(27, self.cin, cout, generator=gen) * std
        if cin_real is not None:
            w[:, cin_real:, :] = 0.0
        w[:, :, self.cout_real:] = 0.0
        f32 = dict(dtype=torch.float32, device=dev)
        self.W = w.reshape(n).to(dev)
        self.b = torch.zeros(cout, **f32)
        self.mW, self.vW = torch.zeros(n, **f32), torch.zeros(n, **f32)
        self.mb, self.vb = torch.zeros(cout, **f32), torch.zeros(cout, **f32)
        self.dW, self.db = torch.zeros(n, **f32), torch.zeros(cout, **f32)
        self.Bm = torch.zeros(cout * self.Kp, dtype=torch.bfloat16, device=dev)
        self.Bd = torch.zeros(self.cin * self.Kd, dtype=torch.bfloat16, device=dev)
        self.sync()

    def sync(self, stream=None):
        """BF16 layouts from the FP32 masters (an Adam call with lr = 0, g = 0)."""
        z = self.dW.zero_()
        check(lib().qesb_net_adam_conv(_p(self.W), _p(self.mW), _p(self.vW), _p(z), self.cin, self.cout,
                                       self.cout_real, _p(self.Bm), self.Kp, _p(self.Bd), self.Kd, 0.0, 0.9,
                                       0.999, 1e-8, 1, 1.0, stream))

    def params(self):
        return {"W": self.W, "b": self.b}


@dataclass
class Shapes:
    D: int
    H: int
    W: int

    def level(self, l):
        return self.D >> l, self.H >> l, self.W >> l

    def V(self, l):
        d, h, w = self.level(l)
        return d * h * w


class WarmStartNet:
    """The encoder-decoder and its training step, on one CUDA device."""

    CH = (16, 32, 64, 128)

    def __init__(self, device=0, seed=0):
        import torch

        self.torch = torch
        self.dev = torch.device(f"cuda:{device}")
        g = torch.Generator().manual_seed(seed)
        c1, c2, c3, c4 = self.CH
        T, d = torch, self.dev
        mk = lambda *a, **k: Conv(T, d, *a, gen=g, **k)  # noqa: E731
        self.layers = {
            "e1a": mk(IN_CH, 0, c1, 1, 0, cin_real=5), "e1": mk(c1, 0, c1, 1, 0),
            "e2a": mk(c1, 0, c2, 1, 0), "e2": mk(c2, 0, c2, 1, 0),
            "e3a": mk(c2, 0, c3, 1, 0), "e3": mk(c3, 0, c3, 1, 0),
            "e4a": mk(c3, 0, c4, 1, 0), "e4": mk(c4, 0, c4, 1, 0),
            "d3a": mk(c4, c3, c3, 1, 1), "d3": mk(c3, 0, c3, 1, 0),
            "d2a": mk(c3, c2, c2, 1, 1), "d2": mk(c2, 0, c2, 1, 0),
            "d1a": mk(c2, c1, c1, 1, 1), "d1": mk(c1, 0, c1, 1, 0),
            "head": mk(c1, 0, HEAD_N, 0, 0, cout_real=1, init_std=1e-3),
        }
        self.err = torch.zeros(1, dtype=torch.int32, device=d)
        self.loss = torch.zeros(1, dtype=torch.float64, device=d)
        self.step_count = 0
        self._buf = {}
        self._shape = None

    # ------------------------------------------------------------------ buffers
    def _bufs(self, s: Shapes):
        key = (s.D, s.H, s.W)
        if key in self._buf:
            return self._buf[key]
        T, d = self.torch, self.dev
        bf = lambda l, c: T.zeros(s.V(l) * c, dtype=T.bfloat16, device=d)  # noqa: E731
        f32 = lambda l, c: T.zeros(s.V(l) * c, dtype=T.float32, device=d)  # noqa: E731
        c1, c2, c3, c4 = self.CH
        b = {
            "x": bf(0, IN_CH),
            "e1a": bf(0, c1), "e1": bf(0, c1), "p1": bf(1, c1),
            "e2a": bf(1, c2), "e2": bf(1, c2), "p2": bf(2, c2),
            "e3a": bf(2, c3), "e3": bf(2, c3), "p3": bf(3, c3),
            "e4a": bf(3, c4), "e4": bf(3, c4),
            "d3a": bf(2, c3), "d3": bf(2, c3),
            "d2a": bf(1, c2), "d2": bf(1, c2),
            "d1a": bf(0, c1), "d1": bf(0, c1),
            "y": f32(0, HEAD_N),
            # gradients
            "g0": bf(0, HEAD_N), "gA0": bf(0, c1), "gB0": bf(0, c1),
            "gA1": bf(1, c2), "gB1": bf(1, c2), "gA2": bf(2, c3), "gB2": bf(2, c3),
            "gA3": bf(3, c4), "gB3": bf(3, c4),
            "gup1": f32(0, c2), "gsk1": f32(0, c1), "gup2": f32(1, c3), "gsk2": f32(1, c2),
            "gup3": f32(2, c4), "gsk3": f32(2, c3),
            "gp1": f32(1, c1), "gp2": f32(2, c2), "gp3": f32(3, c3),
        }
        self._buf[key] = b
        return b

    # ------------------------------------------------------------------ kernels
    def _conv(self, L: Conv, x1, x2, lvl, s: Shapes, y=None, yf=None, stream=None):
        D, H, W = s.level(lvl)
        check(lib().qesb_conv3d(_p(x1), L.c1, L.up1, _p(x2), L.c2, D, H, W, 1, _p(L.Bm), L.Kp, L.cout, _p(y),
                                _p(yf), _p(L.b), L.relu, None, _p(self.err), stream))

    def _dgrad(self, L: Conv, gy, lvl, s: Shapes, rows, n, y=None, yf=None, mask=None, stream=None):
        """Input gradient for input channels [rows, rows + n) of layer L."""
        D, H, W = s.level(lvl)
        B = self.torch.narrow(L.Bd, 0, rows * L.Kd, n * L.Kd)
        check(lib().qesb_conv3d(_p(gy), L.cout, 0, None, 0, D, H, W, -1, _p(B), L.Kd, n, _p(y), _p(yf), None, 0,
                                _p(mask), _p(self.err), stream))

    def _wgrad(self, L: Conv, x1, x2, gy, lvl, s: Shapes, stream=None):
        D, H, W = s.level(lvl)
        V = D * H * W
        vchunk = max(64, min(8192, (V // (4 * 148) + 63) // 64 * 64))
        check(lib().qesb_conv3d_wgrad(_p(x1), L.c1, L.up1, _p(x2), L.c2, D, H, W, _p(gy), L.cout, vchunk, _p(L.dW),
                                      _p(self.err), stream))
        check(lib().qesb_net_colsum(_p(gy), V, L.cout, _p(L.db), stream))

    def _pool(self, x, y, lvl, s, c, stream=None):
        D, H, W = s.level(lvl)
        check(lib().qesb_net_pool2(_p(x), _p(y), D, H, W, c, stream))

    # ------------------------------------------------------------------ passes
    def forward(self, s: Shapes, stream=None):
        """Runs the network on buffer 'x' of shape s; returns the FP32 head
        output [V][16] (channel 0 = lambda / max|R|)."""
        b, Ls = self._bufs(s), self.layers
        c1, c2, c3, _ = self.CH
        self._conv(Ls["e1a"], b["x"], None, 0, s, y=b["e1a"], stream=stream)
        self._conv(Ls["e1"], b["e1a"], None, 0, s, y=b["e1"], stream=stream)
        self._pool(b["e1"], b["p1"], 0, s, c1, stream)
        self._conv(Ls["e2a"], b["p1"], None, 1, s, y=b["e2a"], stream=stream)
        self._conv(Ls["e2"], b["e2a"], None, 1, s, y=b["e2"], stream=stream)
        self._pool(b["e2"], b["p2"], 1, s, c2, stream)
        self._conv(Ls["e3a"], b["p2"], None, 2, s, y=b["e3a"], stream=stream)
        self._conv(Ls["e3"], b["e3a"], None, 2, s, y=b["e3"], stream=stream)
        self._pool(b["e3"], b["p3"], 2, s, c3, stream)
        self._conv(Ls["e4a"], b["p3"], None, 3, s, y=b["e4a"], stream=stream)
        self._conv(Ls["e4"], b["e4a"], None, 3, s, y=b["e4"], stream=stream)
        self._conv(Ls["d3a"], b["e4"], b["e3"], 2, s, y=b["d3a"], stream=stream)
        self._conv(Ls["d3"], b["d3a"], None, 2, s, y=b["d3"], stream=stream)
        self._conv(Ls["d2a"], b["d3"], b["e2"], 1, s, y=b["d2a"], stream=stream)
        self._conv(Ls["d2"], b["d2a"], None, 1, s, y=b["d2"], stream=stream)
        self._conv(Ls["d1a"], b["d2"], b["e1"], 0, s, y=b["d1a"], stream=stream)
        self._conv(Ls["d1"], b["d1a"], None, 0, s, y=b["d1"], stream=stream)
        self._conv(Ls["head"], b["d1"], None, 0, s, yf=b["y"], stream=stream)
        return b["y"]

    def backward(self, s: Shapes, tgt, w, inv_count, stream=None):
        """Loss (weighted MSE on channel 0) and all parameter gradients into
        each layer's dW / db (zeroed here first)."""
        b, Ls, T = self._bufs(s), self.layers, self.torch
        c1, c2, c3, c4 = self.CH
        for L in Ls.values():
            L.dW.zero_()
            L.db.zero_()
        self.loss.zero_()
        check(lib().qesb_net_mse(_p(b["y"]), HEAD_N, _p(tgt), _p(w), s.V(0), float(inv_count), _p(b["g0"]),
                                 _p(self.loss), stream))
        # head and the level-1 decoder
        self._wgrad(Ls["head"], b["d1"], None, b["g0"], 0, s, stream)
        self._dgrad(Ls["head"], b["g0"], 0, s, 0, c1, y=b["gA0"], mask=b["d1"], stream=stream)
        self._wgrad(Ls["d1"], b["d1a"], None, b["gA0"], 0, s, stream)
        self._dgrad(Ls["d1"], b["gA0"], 0, s, 0, c1, y=b["gB0"], mask=b["d1a"], stream=stream)
        self._wgrad(Ls["d1a"], b["d2"], b["e1"], b["gB0"], 0, s, stream)
        self._dgrad(Ls["d1a"], b["gB0"], 0, s, 0, c2, yf=b["gup1"], stream=stream)
        self._dgrad(Ls["d1a"], b["gB0"], 0, s, c2, c1, yf=b["gsk1"], stream=stream)
        D, H, W = s.level(0)
        check(lib().qesb_net_up_grad(_p(b["gup1"]), c2, _p(b["d2"]), _p(b["gA1"]), D, H, W, c2, stream))
        # level 2 decoder
        self._wgrad(Ls["d2"], b["d2a"], None, b["gA1"], 1, s, stream)
        self._dgrad(Ls["d2"], b["gA1"], 1, s, 0, c2, y=b["gB1"], mask=b["d2a"], stream=stream)
        self._wgrad(Ls["d2a"], b["d3"], b["e2"], b["gB1"], 1, s, stream)
        self._dgrad(Ls["d2a"], b["gB1"], 1, s, 0, c3, yf=b["gup2"], stream=stream)
        self._dgrad(Ls["d2a"], b["gB1"], 1, s, c3, c2, yf=b["gsk2"], stream=stream)
        D, H, W = s.level(1)
        check(lib().qesb_net_up_grad(_p(b["gup2"]), c3, _p(b["d3"]), _p(b["gA2"]), D, H, W, c3, stream))
        # level 3 decoder
        self._wgrad(Ls["d3"], b["d3a"], None, b["gA2"], 2, s, stream)
        self._dgrad(Ls["d3"], b["gA2"], 2, s, 0, c3, y=b["gB2"], mask=b["d3a"], stream=stream)
        self._wgrad(Ls["d3a"], b["e4"], b["e3"], b["gB2"], 2, s, stream)
        self._dgrad(Ls["d3a"], b["gB2"], 2, s, 0, c4, yf=b["gup3"], stream=stream)
        self._dgrad(Ls["d3a"], b["gB2"], 2, s, c4, c3, yf=b["gsk3"], stream=stream)
        D, H, W = s.level(2)
        check(lib().qesb_net_up_grad(_p(b["gup3"]), c4, _p(b["e4"]), _p(b["gA3"]), D, H, W, c4, stream))
        # bottom
        self._wgrad(Ls["e4"], b["e4a"], None, b["gA3"], 3, s, stream)
        self._dgrad(Ls["e4"], b["gA3"], 3, s, 0, c4, y=b["gB3"], mask=b["e4a"], stream=stream)
        self._wgrad(Ls["e4a"], b["p3"], None, b["gB3"], 3, s, stream)
        self._dgrad(Ls["e4a"], b["gB3"], 3, s, 0, c3, yf=b["gp3"], stream=stream)
        # encoder level 3
        D, H, W = s.level(2)
        check(lib().qesb_net_skip_grad(_p(b["gsk3"]), c3, 0, _p(b["gp3"]), _p(b["e3"]), _p(b["gA2"]), D, H, W, c3,
                                       stream))
        self._wgrad(Ls["e3"], b["e3a"], None, b["gA2"], 2, s, stream)
        self._dgrad(Ls["e3"], b["gA2"], 2, s, 0, c3, y=b["gB2"], mask=b["e3a"], stream=stream)
        self._wgrad(Ls["e3a"], b["p2"], None, b["gB2"], 2, s, stream)
        self._dgrad(Ls["e3a"], b["gB2"], 2, s, 0, c2, yf=b["gp2"], stream=stream)
        # encoder level 2
        D, H, W = s.level(1)
        check(lib().qesb_net_skip_grad(_p(b["gsk2"]), c2, 0, _p(b["gp2"]), _p(b["e2"]), _p(b["gA1"]), D, H, W, c2,
                                       stream))
        self._wgrad(Ls["e2"], b["e2a"], None, b["gA1"], 1, s, stream)
        self._dgrad(Ls["e2"], b["gA1"], 1, s, 0, c2, y=b["gB1"], mask=b["e2a"], stream=stream)
        self._wgrad(Ls["e2a"], b["p1"], None, b["gB1"], 1, s, stream)
        self._dgrad(Ls["e2a"], b["gB1"], 1, s, 0, c1, yf=b["gp1"], stream=stream)
        # encoder level 1
        D, H, W = s.level(0)
        check(lib().qesb_net_skip_grad(_p(b["gsk1"]), c1, 0, _p(b["gp1"]), _p(b["e1"]), _p(b["gA0"]), D, H, W, c1,
                                       stream))
        self._wgrad(Ls["e1"], b["e1a"], None, b["gA0"], 0, s, stream)
        self._dgrad(Ls["e1"], b["gA0"], 0, s, 0, c1, y=b["gB0"], mask=b["e1a"], stream=stream)
        self._wgrad(Ls["e1a"], b["x"], None, b["gB0"], 0, s, stream)

    def adam(self, lr, stream=None, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        for L in self.layers.values():
            check(lib().qesb_net_adam_conv(_p(L.W), _p(L.mW), _p(L.vW), _p(L.dW), L.cin, L.cout, L.cout_real,
                                           _p(L.Bm), L.Kp, _p(L.Bd), L.Kd, lr, b1, b2, eps, self.step_count, 1.0,
                                           stream))
            n = L.cout_real
            check(lib().qesb_net_adam_vec(_p(L.b), _p(L.mb), _p(L.vb), _p(L.db), n, lr, b1, b2, eps,
                                          self.step_count, 1.0, stream))

    def check_err(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core kernel's completion wait gave up")

    # ------------------------------------------------------------------ solver glue
    def input_from(self, solver: Solver_B200, s: Shapes, scale):
        """Network input of the solver's current inputs into buffer 'x'."""
        check(lib().qesb_compute_divergence(solver._h))
        check(lib().qesb_warm_input(solver._h, _p(self._bufs(s)["x"]), IN_CH, _p(scale)))

    def warm_start(self, solver: Solver_B200, stream=None):
        """Predicts lambda for the solver's inputs and sets it as the start."""
        s = shapes_of(solver)
        scale = self.torch.zeros(1, dtype=self.torch.int32, device=self.dev)
        self.input_from(solver, s, scale)
        y = self.forward(s, stream)
        check(lib().qesb_warm_apply(solver._h, _p(y), HEAD_N, _p(scale)))
        return s

    # ------------------------------------------------------------------ persistence
    def state(self) -> dict:
        out = {}
        for name, L in self.layers.items():
            out[f"{name}.W"] = L.W.cpu().numpy()
            out[f"{name}.b"] = L.b.cpu().numpy()
        out["step"] = np.array(self.step_count)
        return out

    def save(self, path):
        np.savez_compressed(path, **self.state())

    def load(self, path):
        z = np.load(path)
        for name, L in self.layers.items():
            L.W.copy_(self.torch.from_numpy(z[f"{name}.W"]).to(self.dev))
            L.b.copy_(self.torch.from_numpy(z[f"{name}.b"]).to(self.dev))
            L.sync()
        self.step_count = int(z["step"])


def shapes_of(solver: Solver_B200) -> Shapes:
    Nx, Ny, Nz = solver.domain.base
    if Nx % 8 or Ny % 8 or Nz % 8:
        raise ValueError("the warm-start network needs Nx, Ny, Nz divisible by 8")
    return Shapes(Nz, Ny, Nx)


DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "weights",
                               "warmstart_city.npz")
