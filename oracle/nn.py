"""CPU checker of the learned SVF preview's kernels -- TEST INFRASTRUCTURE.

float64 numpy restatements of the operations the CUDA kernels
(solweig_project_b200/csrc/nn.cu) implement: 3 x 3 same-padding
convolution (forward, data gradient, weight and bias gradient), 2 x 2
average pooling, nearest 2x upsampling, ReLU and the masked mean squared
error, plus the whole U-Net's forward and backward
(solweig_project_b200.preview.UNET) for the end-to-end gradient check.
Tensors are NHWC; 3 x 3 weights are [tap][cout][cin], tap = 3 (dy + 1) +
(dx + 1).  The preview has no counterpart in the reference: these are the
mathematical definitions the kernels must match.
"""
from __future__ import annotations

import numpy as np

F64 = np.float64


def _shift(x, dy, dx):
    """x[n, h + dy, w + dx, :] with zeros outside."""
    out = np.zeros_like(x)
    n, h, w, c = x.shape
    hs0, hs1 = max(0, -dy), min(h, h - dy)
    ws0, ws1 = max(0, -dx), min(w, w - dx)
    if hs0 < hs1 and ws0 < ws1:
        out[:, hs0:hs1, ws0:ws1] = x[:, hs0 + dy:hs1 + dy, ws0 + dx:ws1 + dx]
    return out


def conv3x3(x, w, b=None):
    x = np.asarray(x, F64)
    y = np.zeros(x.shape[:3] + (w.shape[1],), F64)
    for t in range(9):
        y += _shift(x, t // 3 - 1, t % 3 - 1) @ np.asarray(w[t], F64).T
    if b is not None:
        y += np.asarray(b, F64)
    return y


def conv3x3_dgrad(dy, w):
    dy = np.asarray(dy, F64)
    dx = np.zeros(dy.shape[:3] + (w.shape[2],), F64)
    for t in range(9):
        dx += _shift(dy, -(t // 3 - 1), -(t % 3 - 1)) @ np.asarray(w[t], F64)
    return dx


def conv3x3_wgrad(x, dy):
    x, dy = np.asarray(x, F64), np.asarray(dy, F64)
    cin, cout = x.shape[3], dy.shape[3]
    dw = np.zeros((9, cout, cin), F64)
    for t in range(9):
        xs = _shift(x, t // 3 - 1, t % 3 - 1)
        dw[t] = dy.reshape(-1, cout).T @ xs.reshape(-1, cin)
    return dw, dy.reshape(-1, cout).sum(axis=0)


def pool2(x):
    x = np.asarray(x, F64)
    n, h, w, c = x.shape
    return x.reshape(n, h // 2, 2, w // 2, 2, c).mean(axis=(2, 4))


def pool2_bwd(dy):
    return np.repeat(np.repeat(np.asarray(dy, F64), 2, axis=1), 2, axis=2) * 0.25


def up2(x):
    return np.repeat(np.repeat(np.asarray(x, F64), 2, axis=1), 2, axis=2)


def up2_bwd(dy):
    dy = np.asarray(dy, F64)
    n, h, w, c = dy.shape
    return dy.reshape(n, h // 2, 2, w // 2, 2, c).sum(axis=(2, 4))


def mse(pred, target, nc, margin):
    """Mean over the central box and the first nc channels; and its gradient."""
    pred, target = np.asarray(pred, F64), np.asarray(target, F64)
    n, h, w, c = pred.shape
    mask = np.zeros(pred.shape, bool)
    mask[:, margin:h - margin, margin:w - margin, :nc] = True
    d = np.where(mask, pred - target, 0.0)
    count = mask.sum()
    return float((d * d).sum() / count), 2 * d / count


def unet_forward(layers, params, x):
    """Forward of the U-Net described by ``layers`` (preview.UNET) with
    float64 weights {name: (w [9][cout][cin], b)}; returns (out, cache)."""
    a = {"x": np.asarray(x, F64)}

    def conv(name, inp, relu=True):
        y = conv3x3(inp, *params[name])
        return np.maximum(y, 0.0) if relu else y
    a["e1a"] = conv("e1a", a["x"])
    a["e1b"] = conv("e1b", a["e1a"])
    a["e2a"] = conv("e2a", pool2(a["e1b"]))
    a["e2b"] = conv("e2b", a["e2a"])
    a["e3a"] = conv("e3a", pool2(a["e2b"]))
    a["e3b"] = conv("e3b", a["e3a"])
    a["e4a"] = conv("e4a", pool2(a["e3b"]))
    a["e4b"] = conv("e4b", a["e4a"])
    a["e5a"] = conv("e5a", pool2(a["e4b"]))
    a["e5b"] = conv("e5b", a["e5a"])
    a["cat4"] = np.concatenate([up2(a["e5b"]), a["e4b"]], axis=3)
    a["d4"] = conv("d4", a["cat4"])
    a["cat3"] = np.concatenate([up2(a["d4"]), a["e3b"]], axis=3)
    a["d3"] = conv("d3", a["cat3"])
    a["cat2"] = np.concatenate([up2(a["d3"]), a["e2b"]], axis=3)
    a["d2"] = conv("d2", a["cat2"])
    a["cat1"] = np.concatenate([up2(a["d2"]), a["e1b"]], axis=3)
    a["d1"] = conv("d1", a["cat1"])
    a["out"] = conv("head", a["d1"], relu=False)
    return a["out"], a


def unet_backward(params, a, dout):
    """Gradients {name: (dw, db)} of the U-Net given the forward cache."""
    g = {}

    def back(name, inp, out, dy, relu=True):
        if relu:
            dy = dy * (out > 0)
        g[name] = conv3x3_wgrad(inp, dy)
        return conv3x3_dgrad(dy, params[name][0])

    dd1 = back("head", a["d1"], a["out"], dout, relu=False)
    dcat1 = back("d1", a["cat1"], a["d1"], dd1)
    c = a["d2"].shape[3]
    dd2, de1b = up2_bwd(dcat1[..., :c]), dcat1[..., c:]
    dcat2 = back("d2", a["cat2"], a["d2"], dd2)
    c = a["d3"].shape[3]
    dd3, de2b = up2_bwd(dcat2[..., :c]), dcat2[..., c:]
    dcat3 = back("d3", a["cat3"], a["d3"], dd3)
    c = a["d4"].shape[3]
    dd4, de3b = up2_bwd(dcat3[..., :c]), dcat3[..., c:]
    dcat4 = back("d4", a["cat4"], a["d4"], dd4)
    c = a["e5b"].shape[3]
    de5b, de4b = up2_bwd(dcat4[..., :c]), dcat4[..., c:]
    de5a = back("e5b", a["e5a"], a["e5b"], de5b)
    dp4 = back("e5a", pool2(a["e4b"]), a["e5a"], de5a)
    de4a = back("e4b", a["e4a"], a["e4b"], de4b + pool2_bwd(dp4))
    dp3 = back("e4a", pool2(a["e3b"]), a["e4a"], de4a)
    de3a = back("e3b", a["e3a"], a["e3b"], de3b + pool2_bwd(dp3))
    dp2 = back("e3a", pool2(a["e2b"]), a["e3a"], de3a)
    de2a = back("e2b", a["e2a"], a["e2b"], de2b + pool2_bwd(dp2))
    dp1 = back("e2a", pool2(a["e1b"]), a["e2a"], de2a)
    de1a = back("e1b", a["e1a"], a["e1b"], de1b + pool2_bwd(dp1))
    back("e1a", a["x"], a["e1a"], de1a)
    return g
