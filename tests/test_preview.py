"""Learned SVF preview: the U-Net kernels against the float64 checker
(oracle/nn.py), the whole network's gradients, training and the preview's
gain over keeping the stale SVF."""
import ctypes as C

import numpy as np
import pytest

from oracle import nn as onn


def test_checker_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((1, 6, 7, 4))
    w = rng.standard_normal((9, 5, 4))
    b = rng.standard_normal(5)
    dy = rng.standard_normal((1, 6, 7, 5))
    dw, db = onn.conv3x3_wgrad(x, dy)
    dx = onn.conv3x3_dgrad(dy, w)
    f = lambda x_, w_, b_: float((onn.conv3x3(x_, w_, b_) * dy).sum())  # noqa: E731
    eps = 1e-6
    for idx in [(0, 2, 3, 1), (0, 0, 0, 0), (0, 5, 6, 3)]:
        xp = x.copy(); xp[idx] += eps  # noqa: E702
        assert abs((f(xp, w, b) - f(x, w, b)) / eps - dx[idx]) < 1e-4
    for idx in [(0, 1, 2), (8, 4, 3), (4, 0, 0)]:
        wp = w.copy(); wp[idx] += eps  # noqa: E702
        assert abs((f(x, wp, b) - f(x, w, b)) / eps - dw[idx]) < 1e-4
    bp = b.copy(); bp[2] += eps  # noqa: E702
    assert abs((f(x, w, bp) - f(x, w, b)) / eps - db[2]) < 1e-4
    # pooling / upsampling are adjoint pairs
    a = rng.standard_normal((1, 4, 6, 3))
    c = rng.standard_normal((1, 2, 3, 3))
    assert abs((onn.pool2(a) * c).sum() - (a * onn.pool2_bwd(c)).sum()) < 1e-9
    assert abs((onn.up2(c) * a).sum() - (c * onn.up2_bwd(a)).sum()) < 1e-9


def test_network_size():
    from solweig_project_b200.preview import UNET
    n = sum(9 * ci * co + co for _, ci, co, _ in UNET)
    assert 250_000 < n < 400_000


# ------------------------------------------------------------------- GPU
def _bf(x):
    import torch
    return torch.as_tensor(np.asarray(x, np.float32)).to(torch.bfloat16)


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(1e-30, np.linalg.norm(b)))


@pytest.mark.gpu
def test_conv_kernels_match_the_checker(cuda):
    import torch
    from solweig_project_b200 import _native as N
    from solweig_project_b200 import engine as E
    rng = np.random.default_rng(1)
    n, h, w, cin, cout = 2, 20, 71, 32, 48
    x = _bf(rng.standard_normal((n, h, w, cin))).cuda()
    wm = torch.tensor(rng.standard_normal((9, cout, cin)).astype(np.float32) * 0.2, device="cuda")
    bias = torch.tensor(rng.standard_normal(cout).astype(np.float32), device="cuda")
    wf = torch.empty(9 * cout * cin, dtype=torch.bfloat16, device="cuda")
    wd = torch.empty_like(wf)
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)  # noqa: E731
    N.call("sw100_nn_weights", p(wm), cin, cout, p(wf), p(wd), E._stream())
    wq = _np(wf).reshape(9, cout, cin)                       # the bf16 weights the kernel uses
    # data gradient: a forward conv with the flipped layout
    dy = _bf(rng.standard_normal((n, h, w, cout))).cuda()
    dx = torch.zeros((n, h, w, cin), dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_conv3x3_tc", p(dy), n, h, w, cout, cout, 0, p(wd), None, cin, p(dx), cin, 0, 0, 0, None,
           E._stream())
    assert _rel(_np(dx), onn.conv3x3_dgrad(_np(dy), wq)) < 1e-2
    # weight and bias gradients
    dw = torch.zeros(9 * cout * cin, dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    N.call("sw100_nn_conv3x3_wgrad", p(x), n, h, w, cin, cin, 0, p(dy), cout, cout, 0, p(dw), p(db), E._stream())
    dw_want, db_want = onn.conv3x3_wgrad(_np(x), _np(dy))
    assert _rel(_np(dw).reshape(9, cout, cin), dw_want) < 1e-5
    assert _rel(_np(db), db_want) < 1e-5


@pytest.mark.gpu
def test_conv_wait_timeout_reports_and_leaves_the_context_usable(cuda):
    """With a wait limit of 0 every pipeline wait of the tensor-core
    convolution runs out at once: the kernel issues nothing more, drains
    the MMAs it issued, frees its tensor memory, writes no output and sets
    err = 1; the context stays usable and the next call (default limit) is
    correct."""
    import torch
    from solweig_project_b200 import _native as N
    from solweig_project_b200 import engine as E
    lib = N.load()
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)  # noqa: E731
    rng = np.random.default_rng(5)
    n, h, w, cin, cout = 1, 16, 40, 64, 32       # 36 K steps: 9 pipeline stages
    x = _bf(rng.standard_normal((n, h, w, cin))).cuda()
    wm = torch.tensor(rng.standard_normal((9, cout, cin)).astype(np.float32) * 0.2, device="cuda")
    wf = torch.empty(9 * cout * cin, dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_weights", p(wm), cin, cout, p(wf), None, E._stream())
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    y = torch.full((n, h, w, cout), 7.0, dtype=torch.float32, device="cuda")
    prev = lib.sw100_set_wait_limit(0)
    try:
        N.call("sw100_nn_conv3x3_tc", p(x), n, h, w, cin, cin, 0, p(wf), None, cout, p(y), cout, 0, 0, 1, p(err),
               E._stream())
        torch.cuda.synchronize()
    finally:
        lib.sw100_set_wait_limit(-1)
    assert prev == 1 << 22
    assert int(err.item()) == 1
    assert bool((y == 7.0).all())                    # no output written
    err.zero_()
    N.call("sw100_nn_conv3x3_tc", p(x), n, h, w, cin, cin, 0, p(wf), None, cout, p(y), cout, 0, 0, 1, p(err),
           E._stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    wq = _np(wf).reshape(9, cout, cin)
    assert _rel(_np(y), onn.conv3x3(_np(x), wq, np.zeros(cout))) < 1e-4


@pytest.mark.gpu
def test_pool_up_and_loss_kernels_match_the_checker(cuda):
    import torch
    from solweig_project_b200 import _native as N
    from solweig_project_b200 import engine as E
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)  # noqa: E731
    rng = np.random.default_rng(2)
    x = _bf(rng.standard_normal((2, 8, 12, 16))).cuda()
    y = torch.zeros((2, 4, 6, 32), dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_pool2", p(x), 2, 8, 12, 16, 16, 0, p(y), 32, 16, 0, 0, E._stream())
    assert _rel(_np(y)[..., 16:], onn.pool2(_np(x))) < 1e-2
    g = torch.zeros((2, 8, 12, 16), dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_pool2", p(y), 2, 8, 12, 16, 32, 16, p(g), 16, 0, 1, 0, E._stream())
    assert _rel(_np(g), onn.pool2_bwd(_np(y)[..., 16:])) < 1e-2
    u = torch.zeros((2, 16, 24, 16), dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_up2", p(x), 2, 8, 12, 16, 16, 0, p(u), 16, 0, 0, E._stream())
    assert np.array_equal(_np(u), onn.up2(_np(x)))
    back = torch.zeros((2, 8, 12, 16), dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_up2", p(u), 2, 8, 12, 16, 16, 0, p(back), 16, 0, 1, E._stream())
    assert _rel(_np(back), onn.up2_bwd(_np(u))) < 1e-2
    pred = torch.tensor(rng.standard_normal((2, 10, 10, 16)).astype(np.float32), device="cuda")
    tgt = torch.tensor(rng.standard_normal((2, 10, 10, 16)).astype(np.float32), device="cuda")
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    dp = torch.zeros((2, 10, 10, 16), dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_mse", p(pred), p(tgt), 2, 10, 10, 16, 15, 3, p(dp), p(loss), E._stream())
    lw, gw = onn.mse(_np(pred), _np(tgt), 15, 3)
    assert abs(float(loss.item()) - lw) / lw < 1e-5
    assert _rel(_np(dp), gw) < 1e-2


@pytest.mark.gpu
def test_network_gradients_match_the_checker(cuda):
    import torch
    from solweig_project_b200.preview import UNET, UNet
    net = UNet(seed=3)
    S = 32
    b = net.buffers(1, S)
    rng = np.random.default_rng(4)
    x = np.zeros((1, S, S, 16), np.float32)
    x[..., :3] = rng.random((1, S, S, 3)) * 0.8
    b["x"].copy_(_bf(x).cuda())
    target = torch.tensor(rng.random((1, S, S, 16)).astype(np.float32), device="cuda")
    net.forward(b)
    net.loss_and_grad(b, target, 4)
    net.grad.zero_()
    net.backward(b)
    torch.cuda.synchronize()
    params = {}
    for name, cin, cout, _ in UNET:
        wf = _np(net.wf[name]).reshape(9, cout, cin)
        params[name] = (wf, net.weight(name)[1].cpu().numpy().astype(np.float64))
    out, cache = onn.unet_forward(None, params, _np(b["x"]))
    loss, dout = onn.mse(out, target.cpu().numpy(), 15, 4)
    assert abs(float(b["loss"].item()) - loss) / loss < 2e-2
    grads = onn.unet_backward(params, cache, dout)
    for name, cin, cout, _ in UNET:
        dw, db = net._slices(net.grad, name)
        e = _rel(dw.cpu().numpy().astype(np.float64).reshape(9, cout, cin), grads[name][0])
        assert e < 0.08, (name, e)
        assert _rel(db.cpu().numpy().astype(np.float64), grads[name][1]) < 0.08, name


@pytest.mark.gpu
@pytest.mark.parametrize("cin,cout,n,h,w", [(16, 16, 2, 20, 71), (32, 48, 1, 17, 33), (128, 64, 2, 8, 8),
                                            (48, 128, 1, 40, 40)])
def test_tensor_core_conv_matches_the_checker(cuda, cin, cout, n, h, w):
    import torch
    from solweig_project_b200 import _native as N
    from solweig_project_b200 import engine as E
    p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)  # noqa: E731
    rng = np.random.default_rng(cin * 7 + cout)
    x = _bf(rng.standard_normal((n, h, w, cin))).cuda()
    wm = torch.tensor(rng.standard_normal((9, cout, cin)).astype(np.float32) * 0.2, device="cuda")
    bias = torch.tensor(rng.standard_normal(cout).astype(np.float32), device="cuda")
    wf = torch.empty(9 * cout * cin, dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_weights", p(wm), cin, cout, p(wf), None, E._stream())
    wq = _np(wf).reshape(9, cout, cin)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    y = torch.zeros((n, h, w, cout), dtype=torch.float32, device="cuda")
    N.call("sw100_nn_conv3x3_tc", p(x), n, h, w, cin, cin, 0, p(wf), p(bias), cout, p(y), cout, 0, 0, 1, p(err),
           E._stream())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert _rel(_np(y), onn.conv3x3(_np(x), wq, _np(bias))) < 1e-5
    # relu + bf16 into a channel slice, as the network writes concatenations
    yb = torch.zeros((n, h, w, cout + 16), dtype=torch.bfloat16, device="cuda")
    N.call("sw100_nn_conv3x3_tc", p(x), n, h, w, cin, cin, 0, p(wf), p(bias), cout, p(yb), cout + 16, 16, 1, 0,
           p(err), E._stream())
    want = np.maximum(onn.conv3x3(_np(x), wq, _np(bias)), 0)
    assert _rel(_np(yb)[..., 16:], want) < 1e-2 and not _np(yb)[..., :16].any()
