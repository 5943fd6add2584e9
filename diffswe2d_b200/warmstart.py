"""Learned warm start for the boundary-inflow inversion.

A 1D-conv encoder plus MLP maps the gauge waveforms of a run (6 gauges x
1125 samples, eta every 0.02 s over 22.5 s) to the 16 spline controls of the
west-edge inflow.  Its prediction seeds the adjoint inversion
(``inversion.invert``); the plain inversion from the reference's cold start
stays the fallback and the measure of the error (the reference has no learned
part; its inversion is
``Examples/inverse/Monai_Valley/Monai_Velley_BC_inversion_spline_lr002/
bc_inversion_train.py:648-768``).

Every training and inference kernel is this project's (``csrc/nn_b200.cu``):
bf16 matrix products with fp32 accumulation on the tcgen05 tensor cores,
im2col / col2im, activation adjoints, Adam.  The network:

=======  ==============================================  ===========
layer    shape                                           parameters
=======  ==============================================  ===========
conv1    6 -> 32 channels, kernel 9, stride 4, pad 4     1,760
conv2    32 -> 64, kernel 8, stride 4, pad 2             16,448
conv3    64 -> 128, kernel 6, stride 2, pad 2            49,280
fc1      128 x 35 -> 96                                  430,176
fc2      96 -> 96                                        9,312
fc3      96 -> 16 (normalised controls)                  1,552
=======  ==============================================  ===========

GELU after every layer but the last; 508,528 parameters (fp32 master copy,
bf16 copies for the products).  Activations are kept channel-last (NLC), so
a convolution's output matrix [N*L, C] is the next im2col's input and the
last one flattens to fc1's input without a copy.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import torch

from . import _native as nat

ACT_NONE, ACT_GELU = 0, 1
SAMPLES, GAUGES, CONTROLS = 1125, 6, 16
INPUT_SCALE = 100.0                   # eta [m] -> input units (1 cm -> 1)
CONTROL_MEAN, CONTROL_SCALE = 0.0015, 0.0078   # controls ~ U[-0.012, 0.015] m


@dataclass(frozen=True)
class Conv:
    cin: int
    cout: int
    k: int
    stride: int
    pad: int
    lin: int

    @property
    def lout(self) -> int:
        return (self.lin + 2 * self.pad - self.k) // self.stride + 1

    @property
    def kdim(self) -> int:
        return self.k * self.cin

    @property
    def kpad(self) -> int:
        return -(-self.kdim // 16) * 16


@dataclass(frozen=True)
class Dense:
    cin: int
    cout: int

    @property
    def kpad(self) -> int:
        return self.cin


def architecture(samples: int = SAMPLES, gauges: int = GAUGES, controls: int = CONTROLS):
    c1 = Conv(gauges, 32, 9, 4, 4, samples)
    c2 = Conv(32, 64, 8, 4, 2, c1.lout)
    c3 = Conv(64, 128, 6, 2, 2, c2.lout)
    return [c1, c2, c3, Dense(c3.cout * c3.lout, 96), Dense(96, 96), Dense(96, controls)]


def _round_up(x: int, m: int) -> int:
    return -(-x // m) * m


def param_layout(layers) -> List[Tuple[int, int, int, int]]:
    """(weight offset, rows, padded cols, bias offset) per layer in the flat
    parameter vector."""
    out, off = [], 0
    for L in layers:
        w = off
        off += L.cout * L.kpad
        b = off
        off += L.cout
        out.append((w, L.cout, L.kpad, b))
    return out, off


class WarmStartNet:
    """The network, its training state and the buffers of one batch size."""

    def __init__(self, device="cuda", seed: int = 0, samples: int = SAMPLES, gauges: int = GAUGES,
                 controls: int = CONTROLS):
        self.dev = torch.device(device)
        self.layers = architecture(samples, gauges, controls)
        self.layout, self.nparams = param_layout(self.layers)
        self.samples, self.gauges, self.controls = samples, gauges, controls
        self.params = torch.zeros(self.nparams, device=self.dev)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step_count = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        #: limit of each tensor-core wait of the GEMM kernel (nn_gemm_bf16)
        self.wait_ns = nat.NN_GEMM_WAIT_NS
        g = torch.Generator().manual_seed(seed)
        host = torch.zeros(self.nparams)
        for L, (w, rows, kp, b) in zip(self.layers, self.layout):
            fan_in = L.kdim if isinstance(L, Conv) else L.cin
            bound = 1.0 / math.sqrt(fan_in)
            W = (torch.rand((rows, fan_in), generator=g) * 2 - 1) * bound
            Wp = torch.zeros((rows, kp))
            Wp[:, :fan_in] = W
            host[w:w + rows * kp] = Wp.reshape(-1)
            host[b:b + rows] = (torch.rand(rows, generator=g) * 2 - 1) * bound
        self.params.copy_(host)
        self.W_bf16 = [torch.empty((L.cout, L.kpad), dtype=torch.int16, device=self.dev)
                       for L in self.layers]
        self.Wt_bf16 = [torch.empty((L.kpad, L.cout), dtype=torch.int16, device=self.dev)
                        for L in self.layers]
        self._refresh_bf16()
        self._nb = None

    # ----------------------------------------------------------- helpers
    def weight(self, i):
        w, rows, kp, _ = self.layout[i]
        return self.params[w:w + rows * kp].view(rows, kp)

    def bias(self, i):
        _, rows, _, b = self.layout[i]
        return self.params[b:b + rows]

    def weight_grad(self, i):
        w, rows, kp, _ = self.layout[i]
        return self.grads[w:w + rows * kp].view(rows, kp)

    def bias_grad(self, i):
        _, rows, _, b = self.layout[i]
        return self.grads[b:b + rows]

    def _st(self):
        return nat.stream_handle(self.dev)

    def _refresh_bf16(self):
        lib = nat.lib()
        for i, L in enumerate(self.layers):
            W = self.weight(i)
            nat.check(lib.nn_cast_bf16(nat.ptr(W), L.cout, L.kpad, L.kpad, nat.ptr(self.W_bf16[i]),
                                       L.kpad, nat.ptr(self.Wt_bf16[i]), L.cout, self._st()),
                      "nn cast")

    def _gemm(self, A, lda, B, ldb, M, N, K, bias=None, act=ACT_NONE, out_f32=None, out_bf16=None,
              pre=None, ldc=None, ksplit=1):
        ws = None
        if ksplit > 1:
            need = ksplit * M * N
            if self._ws is None or self._ws.numel() < need:
                self._ws = torch.empty(need, device=self.dev)
            ws = self._ws
        rc = nat.lib().nn_gemm_bf16(nat.ptr(A), lda, nat.ptr(B), ldb, M, N, K, nat.ptr(bias), act,
                                    nat.ptr(out_f32), nat.ptr(out_bf16), nat.ptr(pre),
                                    N if ldc is None else ldc, ksplit, nat.ptr(ws), self.wait_ns,
                                    nat.ptr(self.err), self._st())
        nat.check(rc, "nn gemm")

    @staticmethod
    def _ksplit(K: int) -> int:
        return max(1, min(128, K // 2048))

    def _buffers(self, nb: int):
        if self._nb == nb:
            return
        dev, L = self.dev, self.layers
        bf = dict(dtype=torch.int16, device=dev)
        self._ws = None
        self.cols = [torch.empty((nb * c.lout, c.kpad), **bf) for c in L[:3]]
        self.pre = [torch.empty((nb * c.lout, c.cout), device=dev) for c in L[:3]]
        self.act = [torch.empty((nb * c.lout, c.cout), **bf) for c in L[:3]]
        self.pre += [torch.empty((nb, d.cout), device=dev) for d in L[3:]]
        self.act += [torch.empty((nb, d.cout), **bf) for d in L[3:5]]
        self.out = torch.empty((nb, L[5].cout), device=dev)
        self.dpred = torch.empty_like(self.out)
        self.loss = torch.zeros(1, device=dev)
        # backward scratch
        rows = [nb * c.lout for c in L[:3]] + [nb] * 3
        self.rows = rows
        self.rows_pad = [_round_up(r, 64) for r in rows]
        self.dact = [torch.empty((r, l.cout), device=dev) for r, l in zip(rows, L)]
        self.d_bf16 = [torch.empty((r, l.cout), **bf) for r, l in zip(rows, L)]
        self.dT_bf16 = [torch.empty((l.cout, rp), **bf) for rp, l in zip(self.rows_pad, L)]
        ins = [c.kpad for c in L[:3]] + [d.cin for d in L[3:]]
        self.xT_bf16 = [torch.empty((k, rp), **bf) for k, rp in zip(ins, self.rows_pad)]
        self.dcols = [None] + [torch.empty((nb * c.lout, c.kpad), device=dev) for c in L[1:3]]
        self._nb = nb

    # ----------------------------------------------------------- forward
    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: gauge eta [Nb, gauges, samples] fp32 (metres) -> normalised
        controls [Nb, controls] fp32 (a view of an internal buffer)."""
        x = nat.require_cuda_f32("x", x)
        nb, G, T = x.shape
        if G != self.gauges or T != self.samples:
            raise ValueError(f"expected [N, {self.gauges}, {self.samples}] gauge series, got {tuple(x.shape)}")
        self._buffers(nb)
        lib, L = nat.lib(), self.layers
        src_f32, src_bf16 = x, None
        strides = (G * T, 1, T)  # NCL input
        for i in range(3):
            c = L[i]
            scale = INPUT_SCALE if i == 0 else 1.0
            rc = lib.nn_im2col(nat.ptr(src_f32), nat.ptr(src_bf16), nb, c.lin, c.cin, strides[0],
                               strides[1], strides[2], c.k, c.stride, c.pad, c.lout, scale, 0.0,
                               nat.ptr(self.cols[i]), c.kpad, self._st())
            nat.check(rc, "nn im2col")
            self._gemm(self.cols[i], c.kpad, self.W_bf16[i], c.kpad, nb * c.lout, c.cout, c.kpad,
                       bias=self.bias(i), act=ACT_GELU, out_bf16=self.act[i], pre=self.pre[i])
            src_f32, src_bf16 = None, self.act[i]
            strides = (c.lout * c.cout, c.cout, 1)  # NLC
        h = self.act[2]  # [nb * L3, 128] == [nb, 4480]
        for j, i in enumerate(range(3, 6)):
            d = L[i]
            last = i == 5
            self._gemm(h, d.cin, self.W_bf16[i], d.kpad, nb, d.cout, d.kpad, bias=self.bias(i),
                       act=ACT_NONE if last else ACT_GELU, out_f32=self.out if last else None,
                       out_bf16=None if last else self.act[i], pre=self.pre[i])
            if not last:
                h = self.act[i]
        return self.out

    # ---------------------------------------------------------- backward
    def backward(self, dout: torch.Tensor) -> None:
        """Gradients of all parameters into self.grads for the cotangent of
        the last forward's output [Nb, controls]."""
        lib, L, nb = nat.lib(), self.layers, self._nb
        st = self._st()
        self.grads.zero_()
        dact = dout  # [rows, cout] fp32
        for i in range(5, -1, -1):
            lay = L[i]
            M, N = self.rows[i], lay.cout
            Mp = self.rows_pad[i]
            act = ACT_NONE if i == 5 else ACT_GELU
            rc = lib.nn_act_backward(nat.ptr(dact), nat.ptr(self.pre[i]), M, N, N, act,
                                     nat.ptr(self.d_bf16[i]), N, nat.ptr(self.dT_bf16[i]), Mp,
                                     nat.ptr(self.dact[i]), st)
            nat.check(rc, "nn act backward")
            nat.check(lib.nn_colsum(nat.ptr(self.dact[i]), M, N, N, nat.ptr(self.bias_grad(i)), st),
                      "nn colsum")
            # layer input X [M, Kin] (bf16) and its transpose [Kin, Mp]
            if i < 3:
                X, kin = self.cols[i], lay.kpad
            elif i == 3:
                X, kin = self.act[2], lay.cin
            else:
                X, kin = self.act[i - 1], lay.cin
            nat.check(lib.nn_transpose_bf16(nat.ptr(X), M, kin, kin, nat.ptr(self.xT_bf16[i]), Mp, st),
                      "nn transpose")
            # dW [N, Kin] = d^T X
            self._gemm(self.dT_bf16[i], Mp, self.xT_bf16[i], Mp, N, kin, Mp,
                       out_f32=self.weight_grad(i), ldc=lay.kpad, ksplit=self._ksplit(Mp))
            if i == 0:
                break
            # dX [M, Kin] = d W
            if i > 3:
                dst = self.dact_in(i)
                self._gemm(self.d_bf16[i], N, self.Wt_bf16[i], N, M, kin, N, out_f32=dst)
                dact = dst
            elif i == 3:
                dst = self.dact_in(3)  # [nb, 4480] == conv3 output [nb * L3, 128]
                self._gemm(self.d_bf16[i], N, self.Wt_bf16[i], N, M, kin, N, out_f32=dst)
                dact = dst
            else:
                self._gemm(self.d_bf16[i], N, self.Wt_bf16[i], N, M, kin, N, out_f32=self.dcols[i])
                prev = L[i - 1]
                dst = self.dact_in(i)
                rc = lib.nn_col2im(nat.ptr(self.dcols[i]), lay.kpad, nb, lay.lin, lay.cin, lay.k,
                                   lay.stride, lay.pad, lay.lout, nat.ptr(dst), st)
                nat.check(rc, "nn col2im")
                dact = dst

    def dact_in(self, i):
        """Buffer for the adjoint of layer i's input (= layer i-1's output)."""
        if not hasattr(self, "_din") or self._din_nb != self._nb:
            L, nb = self.layers, self._nb
            self._din = {}
            for j in range(1, 6):
                prev_rows = self.rows[j - 1]
                self._din[j] = torch.empty((prev_rows, L[j - 1].cout), device=self.dev)
            self._din_nb = nb
        return self._din[i]

    # ---------------------------------------------------------- training
    def loss_and_grad(self, x, y_norm) -> torch.Tensor:
        pred = self.forward(x)
        nb = pred.shape[0]
        rc = nat.lib().nn_mse(nat.ptr(pred), nat.ptr(y_norm), nb, self.controls, nat.ptr(self.loss),
                              nat.ptr(self.dpred), self._st())
        nat.check(rc, "nn mse")
        self.backward(self.dpred)
        return self.loss

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step_count += 1
        rc = nat.lib().nn_adam(nat.ptr(self.params), nat.ptr(self.grads), nat.ptr(self.m),
                               nat.ptr(self.v), self.nparams, lr, beta1, beta2, eps, self.step_count,
                               self._st())
        nat.check(rc, "nn adam")
        self._refresh_bf16()

    def train_step(self, x, y_norm, lr=1e-3):
        loss = self.loss_and_grad(x, y_norm)
        self.adam_step(lr)
        return loss

    def check_errors(self):
        code = int(self.err.item())
        if code & 2:
            raise RuntimeError(f"nn_gemm_bf16: tensor-core work had not finished when its tensor "
                               f"memory was freed (code {code:#x}); the CUDA context is suspect")
        if code != 0:
            raise RuntimeError(f"a bounded wait in nn_gemm_bf16 ran past its time limit (code {code:#x})")

    def predict_controls(self, gauges_eta: torch.Tensor, batch: int = 256) -> torch.Tensor:
        """Spline control values [N, controls] (metres) for gauge series
        [N, gauges, samples]."""
        outs = []
        for s in range(0, gauges_eta.shape[0], batch):
            y = self.forward(gauges_eta[s:s + batch].contiguous())
            outs.append(y * CONTROL_SCALE + CONTROL_MEAN)
        return torch.cat(outs)

    def state_dict(self):
        return {"params": self.params.detach().cpu(), "step": self.step_count}

    def load_state_dict(self, sd):
        self.params.copy_(sd["params"].to(self.dev))
        self.step_count = int(sd.get("step", 0))
        self._refresh_bf16()


def normalise_controls(values: torch.Tensor) -> torch.Tensor:
    return (values - CONTROL_MEAN) / CONTROL_SCALE


__all__ = ["WarmStartNet", "architecture", "param_layout", "normalise_controls", "Conv", "Dense",
           "SAMPLES", "GAUGES", "CONTROLS", "INPUT_SCALE", "CONTROL_MEAN", "CONTROL_SCALE"]
