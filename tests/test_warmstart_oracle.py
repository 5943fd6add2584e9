"""The warm-start network's CPU oracle (the checker of the GPU gradients)
pinned by central finite differences of its own float64 forward pass."""
import numpy as np

from warmstart_oracle import WarmStartOracle, bf16, col2im, im2col, mse_grad

from diffswe2d_b200.warmstart import architecture, param_layout


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.01171875, 1.0 + 2 ** -9, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3],
                 np.float32)
    got = bf16(x)
    assert got[0] == 1.0
    assert got[1] == 1.0             # halfway, ties to even (1.0)
    assert got[2] == 1.015625        # halfway, ties to even (1.015625)
    assert got[3] == 1.0 and got[4] == 1.0078125
    assert got[5] == -2.5
    assert abs(got[6] - 3.0e-3) <= 3.0e-3 * 2 ** -8


def test_im2col_col2im_are_adjoint():
    rng = np.random.default_rng(0)
    nb, lin, cin, k, stride, pad = 2, 37, 3, 5, 3, 2
    lout = (lin + 2 * pad - k) // stride + 1
    x = rng.normal(size=(nb, lin, cin))
    y = rng.normal(size=(nb * lout, k * cin + 4))
    cols = im2col(x, k, stride, pad, lout, k * cin + 4, rnd=lambda a: a)
    back = col2im(y, nb, lin, cin, k, stride, pad, lout)
    assert np.isclose((cols * y).sum(), (x * back).sum(), rtol=1e-12)


def test_oracle_gradients_match_finite_differences():
    layers = architecture(samples=64, gauges=2, controls=3)
    layout, n = param_layout(layers)
    rng = np.random.default_rng(1)
    params = np.zeros(n)
    for L, (w, rows, kp, b) in zip(layers, layout):
        fan = L.kdim if hasattr(L, "kdim") else L.cin
        W = np.zeros((rows, kp))
        W[:, :fan] = rng.uniform(-1, 1, (rows, fan)) / np.sqrt(fan)
        params[w:w + rows * kp] = W.ravel()
        params[b:b + rows] = rng.uniform(-0.1, 0.1, rows)
    x = rng.normal(scale=0.01, size=(3, 2, 64))
    y = rng.normal(size=(3, 3))

    def loss(p):
        o = WarmStartOracle(p, layers, layout, 100.0, exact=True)
        out, _ = o.forward(x)
        return mse_grad(out, y)[0]

    o = WarmStartOracle(params, layers, layout, 100.0, exact=True)
    out, cache = o.forward(x)
    grads = o.backward(mse_grad(out, y)[1], cache)
    for i, (w, rows, kp, b) in enumerate(layout):
        dW, db = grads[i]
        fan = layers[i].kdim if hasattr(layers[i], "kdim") else layers[i].cin
        for (r, c) in ((0, 0), (rows - 1, fan - 1), (rows // 2, fan // 2)):
            e = 1e-6
            p1, p2 = params.copy(), params.copy()
            p1[w + r * kp + c] += e
            p2[w + r * kp + c] -= e
            fd = (loss(p1) - loss(p2)) / (2 * e)
            assert abs(dW[r, c] - fd) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, r, c, dW[r, c], fd)
        p1, p2 = params.copy(), params.copy()
        p1[b] += 1e-6
        p2[b] -= 1e-6
        fd = (loss(p1) - loss(p2)) / 2e-6
        assert abs(db[0] - fd) <= 1e-6 * max(1.0, abs(fd)) + 1e-9
