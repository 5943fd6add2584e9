"""CPU oracle for the warm-start network's forward and backward passes.

TEST INFRASTRUCTURE ONLY.  Only ``tests/`` import this module; the product
package never imports or calls it.

The network has no counterpart in the reference (DiffSWE2d has no learned
part).  This file restates, in numpy, the network that
``diffswe2d_b200/warmstart.py`` trains with its own CUDA kernels, with the
same bf16 rounding points (im2col columns, weights, stored activations and
activation adjoints are bf16; products accumulate in float64 here, fp32 on
the GPU; bias, pre-activations and bias gradients stay fp32), so that the
GPU gradients can be checked against it layer by layer.  Layer shapes come
from ``diffswe2d_b200.warmstart.architecture`` (plain data).
"""
from __future__ import annotations

import math

import numpy as np

try:
    from scipy.special import erf as _erf
except ImportError:  # pragma: no cover
    _erf = np.vectorize(math.erf)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest, ties to even), returned as
    float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def im2col(x_nlc: np.ndarray, k: int, stride: int, pad: int, lout: int, kpad: int, scale: float = 1.0,
           rnd=bf16):
    """cols[(n*lout + lo), kk*cin + ci] = rnd(scale * x[n, lo*stride - pad + kk, ci])."""
    nb, lin, cin = x_nlc.shape
    cols = np.zeros((nb, lout, kpad), x_nlc.dtype)
    for kk in range(k):
        l = np.arange(lout) * stride - pad + kk
        ok = (l >= 0) & (l < lin)
        cols[:, ok, kk * cin:(kk + 1) * cin] = x_nlc[:, l[ok], :] * x_nlc.dtype.type(scale)
    return rnd(cols.reshape(nb * lout, kpad))


def col2im(dcols: np.ndarray, nb: int, lin: int, cin: int, k: int, stride: int, pad: int, lout: int):
    d = dcols.reshape(nb, lout, -1)
    dx = np.zeros((nb, lin, cin), np.float64)
    for kk in range(k):
        l = np.arange(lout) * stride - pad + kk
        ok = (l >= 0) & (l < lin)
        np.add.at(dx, (slice(None), l[ok]), d[:, ok, kk * cin:(kk + 1) * cin])
    return dx


class WarmStartOracle:
    """params: the flat parameter vector; layers/layout: the network's
    architecture and parameter layout.  exact=True drops the bf16 rounding
    and computes in float64 (the exact gradient of the float64 network, for
    finite-difference checks of this oracle itself)."""

    def __init__(self, params: np.ndarray, layers, layout, input_scale: float, exact: bool = False):
        self.layers, self.layout, self.input_scale = layers, layout, input_scale
        self.ft = np.float64 if exact else np.float32
        self.params = np.asarray(params, self.ft)
        self.r = (lambda a: np.asarray(a, np.float64)) if exact else bf16

    def W(self, i):
        w, rows, kp, _ = self.layout[i]
        return self.params[w:w + rows * kp].reshape(rows, kp)

    def b(self, i):
        _, rows, _, b = self.layout[i]
        return self.params[b:b + rows]

    def _mm(self, a, bT):
        return (np.asarray(a, np.float64) @ np.asarray(bT, np.float64)).astype(self.ft)

    def forward(self, x: np.ndarray):
        """x [nb, gauges, samples] -> (output [nb, controls], cache)."""
        L, r, ft = self.layers, self.r, self.ft
        nb = x.shape[0]
        cache = {"X": [], "pre": []}
        h = np.transpose(x, (0, 2, 1)).astype(ft)  # NLC
        for i in range(3):
            c = L[i]
            cols = im2col(h, c.k, c.stride, c.pad, c.lout, c.kpad,
                          self.input_scale if i == 0 else 1.0, rnd=r).astype(ft)
            pre = self._mm(cols, r(self.W(i)).T) + self.b(i)
            cache["X"].append(cols)
            cache["pre"].append(pre)
            h = r(gelu(pre.astype(np.float64)).astype(ft)).astype(ft).reshape(nb, c.lout, c.cout)
        h = h.reshape(nb, -1)
        for i in range(3, 6):
            pre = self._mm(h, r(self.W(i)).T) + self.b(i)
            cache["X"].append(h)
            cache["pre"].append(pre)
            h = r(gelu(pre.astype(np.float64)).astype(ft)).astype(ft) if i < 5 else pre
        return h, cache

    def backward(self, dout: np.ndarray, cache):
        """Gradients [(dW_i, db_i)] for the output cotangent dout."""
        L, r, ft = self.layers, self.r, self.ft
        nb = dout.shape[0]
        grads = [None] * 6
        dact = dout.astype(ft)
        for i in range(5, -1, -1):
            pre = cache["pre"][i]
            d = dact if i == 5 else (dact.astype(np.float64) * gelu_grad(pre.astype(np.float64))).astype(ft)
            X = cache["X"][i]
            dW = r(d).astype(np.float64).T @ np.asarray(X, np.float64)
            db = d.astype(np.float64).sum(0)
            grads[i] = (dW, db)
            if i == 0:
                break
            dX = r(d).astype(np.float64) @ r(self.W(i)).astype(np.float64)
            if i >= 3:
                dact = dX.astype(ft)
                if i == 3:
                    dact = dact.reshape(nb * L[2].lout, L[2].cout)
            else:
                c = L[i]
                dact = col2im(dX, nb, c.lin, c.cin, c.k, c.stride, c.pad, c.lout).astype(ft)
                dact = dact.reshape(nb * c.lin, c.cin)
        return grads


def mse_grad(pred: np.ndarray, target: np.ndarray):
    """Mean squared error and its gradient (2 (pred - target) / size)."""
    d = pred.astype(np.float64) - target
    return float((d * d).mean()), 2.0 * d / d.size
