"""The warm-start network's CUDA kernels (csrc/nn_b200.cu): the tcgen05 bf16
GEMM against float64 products of the same bf16 operands, the memory-bound
kernels against numpy, and the whole network's gradients against the CPU
oracle (oracle/warmstart_oracle.py)."""
import ctypes

import numpy as np
import pytest
import torch

from warmstart_oracle import WarmStartOracle, bf16, col2im, gelu, gelu_grad, im2col, mse_grad

from diffswe2d_b200 import _native as nat
from diffswe2d_b200.warmstart import INPUT_SCALE, WarmStartNet, architecture

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _bf16_dev(a: np.ndarray) -> torch.Tensor:
    """float32 numpy -> bf16 bit patterns (int16) on the device, rounded as bf16()."""
    b = bf16(np.asarray(a, np.float32)).view(np.uint32) >> 16
    return torch.from_numpy(b.astype(np.uint16).view(np.int16)).to(DEV)


def _as_f32(t: torch.Tensor) -> np.ndarray:
    u = t.cpu().numpy().view(np.uint16).astype(np.uint32) << 16
    return u.view(np.float32)


def _gemm(A, B, M, N, K, lda, ldb, bias=None, act=0, ksplit=1, ldc=None):
    ldc = N if ldc is None else ldc
    out = torch.full((M, ldc), -7.0, device=DEV)
    pre = torch.full((M, ldc), -7.0, device=DEV)
    ob = torch.zeros((M, ldc), dtype=torch.int16, device=DEV)
    ws = torch.empty(max(1, ksplit * M * N), device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    rc = nat.lib().nn_gemm_bf16(nat.ptr(A), lda, nat.ptr(B), ldb, M, N, K, nat.ptr(bias), act,
                                nat.ptr(out), nat.ptr(ob), nat.ptr(pre), ldc, ksplit, nat.ptr(ws),
                                nat.NN_GEMM_WAIT_NS, nat.ptr(err), nat.stream_handle(torch.device(DEV)))
    nat.check(rc, "gemm")
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return out.cpu().numpy(), pre.cpu().numpy(), _as_f32(ob)


@pytest.mark.parametrize("M,N,K,ksplit", [(1, 16, 16, 1), (130, 32, 64, 1), (128, 96, 4480, 1),
                                          (300, 96, 4480, 4), (32, 64, 4096, 16), (1000, 128, 384, 1),
                                          (257, 160, 96, 1), (77, 48, 208, 3), (129, 16, 48, 1)])
def test_gemm_matches_float64_products_of_bf16_operands(M, N, K, ksplit):
    rng = np.random.default_rng(M * 7 + N + K)
    a = rng.normal(size=(M, K)).astype(np.float32)
    b = rng.normal(size=(N, K)).astype(np.float32)
    ref = bf16(a).astype(np.float64) @ bf16(b).astype(np.float64).T
    bound = np.abs(bf16(a)).astype(np.float64) @ np.abs(bf16(b)).astype(np.float64).T
    out, pre, _ = _gemm(_bf16_dev(a), _bf16_dev(b), M, N, K, K, K, ksplit=ksplit)
    err = np.abs(out - ref)
    assert np.all(err <= 2e-6 * bound + 1e-30), float((err / bound).max())
    assert np.array_equal(out, pre)


def test_gemm_epilogue_bias_gelu_and_strides():
    rng = np.random.default_rng(5)
    M, N, K, lda, ldb, ldc = 200, 48, 96, 104, 112, 56
    a = rng.normal(size=(M, lda)).astype(np.float32)
    b = rng.normal(size=(N, ldb)).astype(np.float32)
    bias = rng.normal(size=N).astype(np.float32)
    out, pre, ob = _gemm(_bf16_dev(a), _bf16_dev(b), M, N, K, lda, ldb,
                         bias=torch.from_numpy(bias).to(DEV), act=1, ldc=ldc)
    ref = (bf16(a[:, :K]).astype(np.float64) @ bf16(b[:, :K]).astype(np.float64).T) + bias
    assert np.allclose(pre[:, :N], ref, rtol=1e-5, atol=1e-4)
    assert np.allclose(out[:, :N], gelu(pre[:, :N].astype(np.float64)), rtol=1e-5, atol=1e-6)
    assert np.array_equal(ob[:, :N], bf16(out[:, :N]))
    assert np.all(out[:, N:] == -7.0)  # columns past N untouched


def test_gemm_rejects_bad_shapes():
    lib, z = nat.lib(), ctypes.c_void_p(0)
    A = torch.zeros((16, 16), dtype=torch.int16, device=DEV)
    out = torch.zeros((16, 16), device=DEV)
    s = nat.stream_handle(torch.device(DEV))
    assert lib.nn_gemm_bf16(nat.ptr(A), 16, nat.ptr(A), 16, 16, 16, 12, z, 0, nat.ptr(out), z, z, 16,
                            1, z, nat.NN_GEMM_WAIT_NS, z, s) == nat.SWE_EARG  # K not a multiple of 16
    assert lib.nn_gemm_bf16(nat.ptr(A), 12, nat.ptr(A), 16, 16, 16, 16, z, 0, nat.ptr(out), z, z, 16,
                            1, z, nat.NN_GEMM_WAIT_NS, z, s) == nat.SWE_EARG  # lda < K
    assert lib.nn_gemm_bf16(nat.ptr(A), 16, nat.ptr(A), 16, 16, 16, 16, z, 0, nat.ptr(out), z, z, 16,
                            1, z, -1, z, s) == nat.SWE_EARG  # negative wait limit


def test_gemm_wait_limit_surfaces_as_error():
    """With a wait limit of 0 every wait inside the K loop gives up at once:
    each CTA stops issuing, lets its MMAs drain, frees its tensor memory and
    returns without writing its tile; the error word holds bit 1 (not bit 2,
    the drain completed).  The next call with the normal limit is correct
    (the context is still usable)."""
    rng = np.random.default_rng(5)
    M, N, K = 256, 128, 512  # eight K blocks: waits inside the loop happen
    A = _bf16_dev(rng.normal(size=(M, K)))
    B = _bf16_dev(rng.normal(size=(N, K)))
    out = torch.full((M, N), -7.0, device=DEV)
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    s = nat.stream_handle(torch.device(DEV))
    z = ctypes.c_void_p(0)
    rc = nat.lib().nn_gemm_bf16(nat.ptr(A), K, nat.ptr(B), K, M, N, K, z, 0, nat.ptr(out), z, z, N, 1,
                                z, 0, nat.ptr(err), s)
    nat.check(rc, "gemm")
    torch.cuda.synchronize()
    assert int(err.item()) == 1
    assert bool((out == -7.0).all())
    out2, _, _ = _gemm(A, B, M, N, K, K, K)
    ref = _as_f32(A).astype(np.float64) @ _as_f32(B).astype(np.float64).T
    assert np.abs(out2 - ref).max() <= 1e-3 * np.abs(ref).max()


def test_network_raises_on_gemm_wait_error():
    net = WarmStartNet(DEV, seed=0)
    net.wait_ns = 0
    x = torch.zeros((4, 6, 1125), device=DEV)
    net.predict_controls(x)
    torch.cuda.synchronize()
    with pytest.raises(RuntimeError, match="time limit"):
        net.check_errors()


def test_im2col_col2im_match_oracle():
    rng = np.random.default_rng(2)
    nb, lin, cin, k, stride, pad = 3, 70, 32, 8, 4, 2
    lout = (lin + 2 * pad - k) // stride + 1
    kpad = k * cin
    x = bf16(rng.normal(size=(nb, lin, cin)).astype(np.float32))
    cols = torch.empty((nb * lout, kpad), dtype=torch.int16, device=DEV)
    lib, s = nat.lib(), nat.stream_handle(torch.device(DEV))
    xd = torch.from_numpy(x).to(DEV)
    nat.check(lib.nn_im2col(nat.ptr(xd), None, nb, lin, cin, lin * cin, cin, 1, k, stride, pad, lout,
                            1.0, 0.0, nat.ptr(cols), kpad, s), "im2col")
    assert np.array_equal(_as_f32(cols), im2col(x, k, stride, pad, lout, kpad))
    # NCL input with a scale (the first layer)
    xn = rng.normal(scale=0.01, size=(nb, 6, 1125)).astype(np.float32)
    c1 = architecture()[0]
    cols1 = torch.empty((nb * c1.lout, c1.kpad), dtype=torch.int16, device=DEV)
    xn_d = torch.from_numpy(xn).to(DEV)
    nat.check(lib.nn_im2col(nat.ptr(xn_d), None, nb, 1125, 6, 6 * 1125, 1, 1125,
                            c1.k, c1.stride, c1.pad, c1.lout, INPUT_SCALE, 0.0, nat.ptr(cols1), c1.kpad,
                            s), "im2col")
    ref = im2col(np.transpose(xn, (0, 2, 1)).copy(), c1.k, c1.stride, c1.pad, c1.lout, c1.kpad,
                 INPUT_SCALE)
    assert np.array_equal(_as_f32(cols1), ref)
    dcols = rng.normal(size=(nb * lout, kpad)).astype(np.float32)
    dx = torch.empty((nb, lin, cin), device=DEV)
    dcols_d = torch.from_numpy(dcols).to(DEV)
    nat.check(lib.nn_col2im(nat.ptr(dcols_d), kpad, nb, lin, cin, k, stride, pad, lout, nat.ptr(dx), s),
              "col2im")
    assert np.allclose(dx.cpu().numpy(), col2im(dcols, nb, lin, cin, k, stride, pad, lout),
                       rtol=1e-6, atol=1e-6)


def test_small_kernels_match_numpy():
    rng = np.random.default_rng(3)
    lib, s = nat.lib(), nat.stream_handle(torch.device(DEV))
    M, N, Mp = 150, 40, 192
    dact = rng.normal(size=(M, N)).astype(np.float32)
    pre = rng.normal(size=(M, N)).astype(np.float32)
    d_bf = torch.empty((M, N), dtype=torch.int16, device=DEV)
    dT = torch.full((N, Mp), 123, dtype=torch.int16, device=DEV)
    d32 = torch.empty((M, N), device=DEV)
    # device copies held in names: a temporary freed before the launch could
    # share its memory with the next one
    dact_d, pre_d = torch.from_numpy(dact).to(DEV), torch.from_numpy(pre).to(DEV)
    nat.check(lib.nn_act_backward(nat.ptr(dact_d), nat.ptr(pre_d), M, N, N, 1, nat.ptr(d_bf), N,
                                  nat.ptr(dT), Mp, nat.ptr(d32), s), "act backward")
    ref = (dact.astype(np.float64) * gelu_grad(pre.astype(np.float64)))
    assert np.allclose(d32.cpu().numpy(), ref, rtol=1e-5, atol=1e-6)
    assert np.array_equal(_as_f32(d_bf), bf16(d32.cpu().numpy()))
    T = _as_f32(dT)
    assert np.array_equal(T[:, :M], _as_f32(d_bf).T) and np.all(T[:, M:] == 0)
    cs = torch.empty(N, device=DEV)
    nat.check(lib.nn_colsum(nat.ptr(d32), M, N, N, nat.ptr(cs), s), "colsum")
    assert np.allclose(cs.cpu().numpy(), d32.cpu().numpy().astype(np.float64).sum(0), rtol=1e-5,
                       atol=1e-5)
    W = rng.normal(size=(24, 40)).astype(np.float32)
    Wb = torch.empty((24, 48), dtype=torch.int16, device=DEV)
    WT = torch.empty((40, 32), dtype=torch.int16, device=DEV)
    W_d = torch.from_numpy(W).to(DEV)
    nat.check(lib.nn_cast_bf16(nat.ptr(W_d), 24, 40, 40, nat.ptr(Wb), 48, nat.ptr(WT), 32, s), "cast")
    assert np.array_equal(_as_f32(Wb)[:, :40], bf16(W)) and np.all(_as_f32(Wb)[:, 40:] == 0)
    assert np.array_equal(_as_f32(WT)[:, :24], bf16(W).T) and np.all(_as_f32(WT)[:, 24:] == 0)
    pred = rng.normal(size=(7, 16)).astype(np.float32)
    tgt = rng.normal(size=(7, 16)).astype(np.float32)
    loss = torch.empty(1, device=DEV)
    grad = torch.empty((7, 16), device=DEV)
    pred_d, tgt_d = torch.from_numpy(pred).to(DEV), torch.from_numpy(tgt).to(DEV)
    nat.check(lib.nn_mse(nat.ptr(pred_d), nat.ptr(tgt_d), 7, 16, nat.ptr(loss), nat.ptr(grad), s), "mse")
    l_ref, g_ref = mse_grad(pred, tgt)
    assert abs(float(loss) - l_ref) <= 1e-6 * l_ref
    assert np.allclose(grad.cpu().numpy(), g_ref, rtol=1e-6, atol=1e-9)
    p = rng.normal(size=1000).astype(np.float32)
    g = rng.normal(size=1000).astype(np.float32)
    m = np.zeros(1000, np.float32)
    v = np.zeros(1000, np.float32)
    pd, gd, md, vd = (torch.from_numpy(a.copy()).to(DEV) for a in (p, g, m, v))
    for step in (1, 2):
        nat.check(lib.nn_adam(nat.ptr(pd), nat.ptr(gd), nat.ptr(md), nat.ptr(vd), 1000, 1e-3, 0.9,
                              0.999, 1e-8, step, s), "adam")
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        p = p - 1e-3 * (m / (1 - 0.9 ** step)) / (np.sqrt(v / (1 - 0.999 ** step)) + 1e-8)
    assert np.allclose(pd.cpu().numpy(), p, rtol=1e-5, atol=1e-7)


def test_network_gradients_match_cpu_oracle():
    net = WarmStartNet(DEV, seed=4)
    rng = np.random.default_rng(4)
    nb = 5
    x = (rng.normal(scale=0.008, size=(nb, 6, 1125))).astype(np.float32)
    y = rng.normal(size=(nb, 16)).astype(np.float32)
    xd, yd = torch.from_numpy(x).to(DEV), torch.from_numpy(y).to(DEV)
    loss = float(net.loss_and_grad(xd, yd))
    torch.cuda.synchronize()
    net.check_errors()
    pred = net.out.cpu().numpy()
    o = WarmStartOracle(net.params.cpu().numpy(), net.layers, net.layout, INPUT_SCALE)
    out, cache = o.forward(x)
    l_ref, dout = mse_grad(out, y)
    grads = o.backward(dout, cache)
    print("loss", loss, l_ref)
    assert np.allclose(pred, out, rtol=1e-3, atol=1e-4)
    assert abs(loss - l_ref) <= 1e-3 * l_ref
    for i in range(6):
        gW = net.weight_grad(i).cpu().numpy()
        gb = net.bias_grad(i).cpu().numpy()
        dW, db = grads[i]
        eW = np.abs(gW - dW).max() / np.abs(dW).max()
        eb = np.abs(gb - db).max() / np.abs(db).max()
        print("layer", i, "dW", eW, "db", eb)
        assert eW <= 1e-3 and eb <= 1e-3


def test_training_reduces_loss():
    net = WarmStartNet(DEV, seed=0)
    g = torch.Generator(device=DEV).manual_seed(0)
    x = torch.randn((64, 6, 1125), device=DEV, generator=g) * 0.01
    W = torch.randn((6 * 1125, 16), device=DEV, generator=g) / 80.0
    y = (x.reshape(64, -1) * 100.0) @ W  # a learnable linear target
    first = float(net.train_step(x, y, lr=1e-3))
    for _ in range(60):
        last = float(net.train_step(x, y, lr=1e-3))
    net.check_errors()
    print("loss", first, last)
    assert last < 0.3 * first
