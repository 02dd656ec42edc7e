"""Learned warm start for the lambda solve.

A 3D convolutional encoder-decoder (channels 16 -> 32 -> 64 -> 128 by
default, 2x2x2 average pooling down, nearest upsampling and skip
concatenation up) maps per-cell features of a domain (R / max|R|, solid flag,
dz profile, boundary flag, height) to lambda / max|R|, at the cell grid
(res = 1) or at the grid halved in every direction (res = 2: features
2x2x2-averaged, prediction interpolated trilinearly back to the cells). Every convolution (forward, input
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
    """The encoder-decoder and its training step, on one CUDA device.

    Levels l = 0..L-1 with channels CH[l]; level l runs on the grid divided
    by 2^l. Encoder: two convolutions per level, 2x2x2 average pooling down.
    Decoder: from level L-2 up to 0, a convolution of [upsample(level l+1),
    skip e_l] then a second convolution; a linear head gives lambda / max|R|.
    Four levels (16-128 channels) by default; deeper stacks train worse here.
    """

    CH = (16, 32, 64, 128)

    def __init__(self, device=0, seed=0, channels=None, res=1):
        """res = 2: the network runs on the grid halved in every direction
        (input 2x2x2-averaged, prediction interpolated trilinearly back)."""
        import torch

        if res not in (1, 2):
            raise ValueError("res must be 1 or 2")
        self.res = res
        self.torch = torch
        self.dev = torch.device(f"cuda:{device}")
        self.CH = tuple(channels) if channels else self.CH
        g = torch.Generator().manual_seed(seed)
        T, d, C = torch, self.dev, self.CH
        mk = lambda *a, **k: Conv(T, d, *a, gen=g, **k)  # noqa: E731
        L = len(C)
        self.nlev = L
        self.layers = {}
        for l in range(L):
            cin = IN_CH if l == 0 else C[l - 1]
            self.layers[f"e{l}a"] = mk(cin, 0, C[l], 1, 0, **({"cin_real": 5} if l == 0 else {}))
            self.layers[f"e{l}"] = mk(C[l], 0, C[l], 1, 0)
        for l in range(L - 2, -1, -1):
            self.layers[f"d{l}a"] = mk(C[l + 1], C[l], C[l], 1, 1)
            self.layers[f"d{l}"] = mk(C[l], 0, C[l], 1, 0)
        self.layers["head"] = mk(C[0], 0, HEAD_N, 0, 0, cout_real=1, init_std=1e-3)
        self.err = torch.zeros(1, dtype=torch.int32, device=d)
        self.loss = torch.zeros(1, dtype=torch.float64, device=d)
        self.step_count = 0
        self._buf = {}

    # ------------------------------------------------------------------ buffers
    def _bufs(self, s: Shapes):
        key = (s.D, s.H, s.W)
        if key in self._buf:
            return self._buf[key]
        if any(x % (1 << (self.nlev - 1)) for x in (s.D, s.H, s.W)):
            raise ValueError(f"grid {key} not divisible by {1 << (self.nlev - 1)}")
        T, d, C, L = self.torch, self.dev, self.CH, self.nlev
        bf = lambda l, c: T.zeros(s.V(l) * c, dtype=T.bfloat16, device=d)  # noqa: E731
        f32 = lambda l, c: T.zeros(s.V(l) * c, dtype=T.float32, device=d)  # noqa: E731
        b = {"x": bf(0, IN_CH), "y": f32(0, HEAD_N), "g0": bf(0, HEAD_N)}
        for l in range(L):
            b[f"e{l}a"], b[f"e{l}"] = bf(l, C[l]), bf(l, C[l])
            b[f"gA{l}"], b[f"gB{l}"] = bf(l, C[l]), bf(l, C[l])
            if l > 0:
                b[f"p{l}"] = bf(l, C[l - 1])      # pool of e_{l-1}
                b[f"gp{l}"] = f32(l, C[l - 1])    # its gradient
        for l in range(L - 1):
            b[f"d{l}a"], b[f"d{l}"] = bf(l, C[l]), bf(l, C[l])
            b[f"gup{l}"] = f32(l, C[l + 1])       # gradient of upsample(level l+1) at level l
            b[f"gsk{l}"] = f32(l, C[l])           # gradient of the skip e_l from the decoder
        # the zero fills ran on torch's stream; the kernels may run on another
        T.cuda.synchronize(d)
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

    # ------------------------------------------------------------------ passes
    def forward(self, s: Shapes, stream=None):
        """Runs the network on buffer 'x' of shape s; returns the FP32 head
        output [V][16] (channel 0 = lambda / max|R|)."""
        b, Ls, C, L = self._bufs(s), self.layers, self.CH, self.nlev
        for l in range(L):
            xin = b["x"] if l == 0 else b[f"p{l}"]
            if l > 0:
                D, H, W = s.level(l - 1)
                check(lib().qesb_net_pool2(_p(b[f"e{l - 1}"]), _p(b[f"p{l}"]), D, H, W, C[l - 1], stream))
            self._conv(Ls[f"e{l}a"], xin, None, l, s, y=b[f"e{l}a"], stream=stream)
            self._conv(Ls[f"e{l}"], b[f"e{l}a"], None, l, s, y=b[f"e{l}"], stream=stream)
        for l in range(L - 2, -1, -1):
            below = b[f"e{l + 1}"] if l == L - 2 else b[f"d{l + 1}"]
            self._conv(Ls[f"d{l}a"], below, b[f"e{l}"], l, s, y=b[f"d{l}a"], stream=stream)
            self._conv(Ls[f"d{l}"], b[f"d{l}a"], None, l, s, y=b[f"d{l}"], stream=stream)
        self._conv(Ls["head"], b["d0"], None, 0, s, yf=b["y"], stream=stream)
        return b["y"]

    def backward(self, s: Shapes, tgt, w, inv_count, stream=None, coarse=((8, 0.0),)):
        """Loss (weighted MSE on channel 0, plus beta * MSE of the F^3-block
        means of the error for each (F, beta) in `coarse`) and all parameter
        gradients into each layer's dW / db (zeroed here first)."""
        b, Ls, C, L = self._bufs(s), self.layers, self.CH, self.nlev
        for layer in Ls.values():
            layer.dW.zero_()
            layer.db.zero_()
        self.loss.zero_()
        check(lib().qesb_net_mse(_p(b["y"]), HEAD_N, _p(tgt), _p(w), s.V(0), float(inv_count), _p(b["g0"]),
                                 _p(self.loss), stream))
        for F, beta in coarse:
            if beta > 0:
                check(lib().qesb_net_mse_coarse(_p(b["y"]), HEAD_N, _p(tgt), _p(w), s.D, s.H, s.W, F, float(beta),
                                                _p(b["g0"]), _p(self.loss), stream))
        # head: gradient into d0 (through d0's ReLU)
        self._wgrad(Ls["head"], b["d0"], None, b["g0"], 0, s, stream)
        self._dgrad(Ls["head"], b["g0"], 0, s, 0, C[0], y=b["gA0"], mask=b["d0"], stream=stream)
        # decoder, top to bottom: gA{l} holds the pre-activation gradient of d{l}
        for l in range(L - 1):
            self._wgrad(Ls[f"d{l}"], b[f"d{l}a"], None, b[f"gA{l}"], l, s, stream)
            self._dgrad(Ls[f"d{l}"], b[f"gA{l}"], l, s, 0, C[l], y=b[f"gB{l}"], mask=b[f"d{l}a"], stream=stream)
            below = b[f"e{l + 1}"] if l == L - 2 else b[f"d{l + 1}"]
            self._wgrad(Ls[f"d{l}a"], below, b[f"e{l}"], b[f"gB{l}"], l, s, stream)
            self._dgrad(Ls[f"d{l}a"], b[f"gB{l}"], l, s, 0, C[l + 1], yf=b[f"gup{l}"], stream=stream)
            self._dgrad(Ls[f"d{l}a"], b[f"gB{l}"], l, s, C[l + 1], C[l], yf=b[f"gsk{l}"], stream=stream)
            D, H, W = s.level(l)
            check(lib().qesb_net_up_grad(_p(b[f"gup{l}"]), C[l + 1], _p(below), _p(b[f"gA{l + 1}"]), D, H, W,
                                         C[l + 1], stream))
        # encoder, bottom to top: gA{l} holds the pre-activation gradient of e{l}
        for l in range(L - 1, -1, -1):
            if l < L - 1:
                D, H, W = s.level(l)
                check(lib().qesb_net_skip_grad(_p(b[f"gsk{l}"]), C[l], 0, _p(b[f"gp{l + 1}"]), _p(b[f"e{l}"]),
                                               _p(b[f"gA{l}"]), D, H, W, C[l], stream))
            self._wgrad(Ls[f"e{l}"], b[f"e{l}a"], None, b[f"gA{l}"], l, s, stream)
            self._dgrad(Ls[f"e{l}"], b[f"gA{l}"], l, s, 0, C[l], y=b[f"gB{l}"], mask=b[f"e{l}a"], stream=stream)
            xin = b["x"] if l == 0 else b[f"p{l}"]
            self._wgrad(Ls[f"e{l}a"], xin, None, b[f"gB{l}"], l, s, stream)
            if l > 0:
                self._dgrad(Ls[f"e{l}a"], b[f"gB{l}"], l, s, 0, C[l - 1], yf=b[f"gp{l}"], stream=stream)

    def adam(self, lr, stream=None, b1=0.9, b2=0.999, eps=1e-8):
        self.step_count += 1
        for L in self.layers.values():
            check(lib().qesb_net_adam_conv(_p(L.W), _p(L.mW), _p(L.vW), _p(L.dW), L.cin, L.cout, L.cout_real,
                                           _p(L.Bm), L.Kp, _p(L.Bd), L.Kd, lr, b1, b2, eps, self.step_count, 1.0,
                                           stream))
            check(lib().qesb_net_adam_vec(_p(L.b), _p(L.mb), _p(L.vb), _p(L.db), L.cout_real, lr, b1, b2, eps,
                                          self.step_count, 1.0, stream))

    def check_err(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core kernel's completion wait gave up")

    # ------------------------------------------------------------------ solver glue
    def net_shapes(self, solver: Solver_B200) -> Shapes:
        """The grid the network runs on for this solver's domain."""
        f = shapes_of(solver)
        return Shapes(f.D // self.res, f.H // self.res, f.W // self.res)

    def input_from(self, solver: Solver_B200, s: Shapes, scale):
        """Network input of the solver's current inputs into buffer 'x' of the
        network grid s (2x2x2 averages of the cell features when res = 2), on
        the solver's stream."""
        check(lib().qesb_compute_divergence(solver._h))
        if self.res == 1:
            check(lib().qesb_warm_input(solver._h, _p(self._bufs(s)["x"]), IN_CH, _p(scale)))
            return
        check(lib().qesb_warm_input_half(solver._h, _p(self._bufs(s)["x"]), IN_CH, _p(scale)))

    def warm_start(self, solver: Solver_B200, stream=None):
        """Predicts lambda for the solver's inputs and sets it as the start.
        Everything runs on the solver's stream (the input and apply kernels
        are the handle's work, ordered there); `stream`, when given, must be
        that stream."""
        s = self.net_shapes(solver)
        hs = solver.stream_ptr()
        if stream is not None and int(stream) != hs:
            raise ValueError("warm_start: stream differs from the solver's stream")
        if getattr(self, "_scale", None) is None:
            self._scale = self.torch.zeros(1, dtype=self.torch.int32, device=self.dev)
            self.torch.cuda.synchronize(self.dev)
        self.input_from(solver, s, self._scale)
        y = self.forward(s, hs)
        apply = lib().qesb_warm_apply if self.res == 1 else lib().qesb_warm_apply_up2
        check(apply(solver._h, _p(y), HEAD_N, _p(self._scale)))
        return s

    # ------------------------------------------------------------------ persistence
    def state(self) -> dict:
        out = {"channels": np.array(self.CH), "res": np.array(self.res)}
        for name, L in self.layers.items():
            out[f"{name}.W"] = L.W.cpu().numpy()
            out[f"{name}.b"] = L.b.cpu().numpy()
        out["step"] = np.array(self.step_count)
        return out

    def layer_order(self):
        """Layer names in the order of the library's weights file."""
        L = self.nlev
        return ([n for l in range(L) for n in (f"e{l}a", f"e{l}")] +
                [n for l in range(L - 2, -1, -1) for n in (f"d{l}a", f"d{l}")] + ["head"])

    def save(self, path):
        """Weights file: the library's "QESBWNT1" format when path ends in
        .qwn (what qesb_warmnet_load reads), else a numpy .npz (with the
        training step count)."""
        if not str(path).endswith(".qwn"):
            np.savez_compressed(path, **self.state())
            return
        with open(path, "wb") as f:
            f.write(b"QESBWNT1")
            f.write(np.array([self.nlev, self.res, IN_CH, HEAD_N], np.int32).tobytes())
            f.write(np.array(self.CH, np.int32).tobytes())
            for name in self.layer_order():
                L = self.layers[name]
                f.write(np.array([L.c1, L.c2, L.cout, L.cout_real, L.relu, L.up1], np.int32).tobytes())
                f.write(L.W.cpu().numpy().astype(np.float32).tobytes())
                f.write(L.b.cpu().numpy().astype(np.float32).tobytes())

    @staticmethod
    def read_qwn(path) -> dict:
        """The arrays of a "QESBWNT1" weights file, as state() names them."""
        raw = open(path, "rb").read()
        if raw[:8] != b"QESBWNT1":
            raise ValueError(f"{path} is not a warm-start network file")
        nlev, res, _, _ = np.frombuffer(raw, np.int32, 4, 8)
        ch = np.frombuffer(raw, np.int32, int(nlev), 24)
        out = {"channels": ch.copy(), "res": np.array(res), "step": np.array(0)}
        pos = 24 + 4 * int(nlev)
        names = ([n for l in range(nlev) for n in (f"e{l}a", f"e{l}")] +
                 [n for l in range(nlev - 2, -1, -1) for n in (f"d{l}a", f"d{l}")] + ["head"])
        for name in names:
            c1, c2, cout, _, _, _ = (int(x) for x in np.frombuffer(raw, np.int32, 6, pos))
            pos += 24
            n = 27 * (c1 + c2) * cout
            out[f"{name}.W"] = np.frombuffer(raw, np.float32, n, pos).copy()
            pos += 4 * n
            out[f"{name}.b"] = np.frombuffer(raw, np.float32, cout, pos).copy()
            pos += 4 * cout
        return out

    @classmethod
    def from_file(cls, path, device=0):
        z = cls.read_qwn(path) if str(path).endswith(".qwn") else dict(np.load(path))
        net = cls(device=device, channels=tuple(int(c) for c in z["channels"]),
                  res=int(z["res"]) if "res" in z else 1)
        for name, L in net.layers.items():
            L.W.copy_(net.torch.from_numpy(z[f"{name}.W"]).to(net.dev))
            L.b.copy_(net.torch.from_numpy(z[f"{name}.b"]).to(net.dev))
            L.sync()
        net.step_count = int(z["step"])
        return net


def shapes_of(solver: Solver_B200) -> Shapes:
    Nx, Ny, Nz = solver.domain.base
    return Shapes(Nz, Ny, Nx)


DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "weights",
                               "warmstart_city.qwn")


class WarmNet:
    """The learned warm start through the C ABI (qesb_warmnet_load,
    qesb_warm_start): inference only, the layer loop in the library."""

    def __init__(self, path=DEFAULT_WEIGHTS, device=0):
        self._p = C.c_void_p()
        check(lib().qesb_warmnet_load(os.fsencode(path), int(device), C.byref(self._p)))

    def warm_start(self, solver: Solver_B200):
        check(lib().qesb_warm_start(solver._h, self._p))

    def warm_start_batch(self, solvers):
        """qesb_warm_start_batch: the starts of several solvers of one grid
        shape in one forward pass (their inputs stacked along z)."""
        arr = (C.c_void_p * len(solvers))(*[s._h for s in solvers])
        check(lib().qesb_warm_start_batch(arr, len(solvers), self._p))

    def close(self):
        if self._p:
            lib().qesb_warmnet_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
