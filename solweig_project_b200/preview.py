"""Learned SVF preview for edits.

A small U-Net (5 levels, ~340k parameters, BF16 weights and activations,
FP32 accumulation on the 5th-generation tensor cores: tcgen05.mma with
TMEM accumulators for the convolutions' forward and data-gradient passes)
maps a window of the march rasters
(building DSM, canopy top, trunk zone as heights above ground) to the 15
SVF components.  It runs entirely on the library's own kernels
(``sw100_nn_*``: implicit-GEMM 3 x 3 convolutions forward / data-gradient /
weight-gradient, pooling, upsampling, loss, Adam), is trained on the GPU on
SVF fields that the exact sweep computes for seeded synthetic cities, and
previews an edit as

    SVF_post ~ SVF_pre(exact) + net(post window) - net(pre window)

over the window's central block (the context ring only informs the net).
The exact windowed recompute (``DeviceSite.edit_svf_block``) stays the
fallback and the reference point: when the net's error on the pre-edit window, where
the exact answer is already known, exceeds a threshold, the exact path runs
instead.  The reference has no learned path; it recomputes SVF exactly
(shadow.py:409-625).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from . import engine as E

BF16 = torch.bfloat16
F32T = torch.float32
N_OUT = 15           # svf, svfaveg, svfE, ... (library plane order 0..14)
IN_CH = 16           # 3 used

# (name, cin, cout, relu); the wiring is fixed in UNet.forward / backward
UNET = (("e1a", 16, 16, True), ("e1b", 16, 16, True), ("e2a", 16, 32, True), ("e2b", 32, 32, True),
        ("e3a", 32, 48, True), ("e3b", 48, 48, True), ("e4a", 48, 64, True), ("e4b", 64, 64, True),
        ("e5a", 64, 64, True), ("e5b", 64, 64, True), ("d4", 128, 64, True), ("d3", 112, 48, True),
        ("d2", 80, 32, True), ("d1", 48, 16, True), ("head", 16, 16, False))


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


@dataclass
class Act:
    """A view of channels [coff, coff + c) of an NHWC buffer."""
    buf: torch.Tensor
    coff: int
    c: int

    @property
    def stride(self):
        return self.buf.shape[-1]

    @property
    def hw(self):
        return self.buf.shape[1], self.buf.shape[2]


class UNet:
    """Parameters, buffers and the forward / backward passes."""

    def __init__(self, seed: int = 0, device="cuda"):
        E.require_cuda()
        self.device = torch.device(device)
        self.layers = {name: (cin, cout, relu) for name, cin, cout, relu in UNET}
        sizes = [9 * cout * cin + cout for _, cin, cout, _ in UNET]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.n_params = int(self.offsets[-1])
        rng = np.random.default_rng(seed)
        master = np.zeros(self.n_params, np.float32)
        for k, (name, cin, cout, _) in enumerate(UNET):
            fan_in = 9 * (3 if name == "e1a" else cin)
            std = math.sqrt(2.0 / fan_in) * (0.1 if name == "head" else 1.0)
            w = rng.standard_normal((9, cout, cin)).astype(np.float32) * np.float32(std)
            if name == "e1a":
                w[:, :, 3:] = 0.0
            master[self.offsets[k]:self.offsets[k] + 9 * cout * cin] = w.reshape(-1)
        d = self.device
        self.master = torch.from_numpy(master).to(d)
        self.grad = torch.zeros_like(self.master)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.step = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=d)   # set by a tensor-core kernel whose wait expired
        self.wf = {n: torch.empty(9 * co * ci, dtype=BF16, device=d) for n, ci, co, _ in UNET}
        self.wd = {n: torch.empty(9 * co * ci, dtype=BF16, device=d) for n, ci, co, _ in UNET}
        self._bufs = {}
        self.refresh_weights()

    # ------------------------------------------------------------ params
    def _slices(self, t, name):
        k = [n for n, *_ in UNET].index(name)
        cin, cout, _ = self.layers[name]
        o = int(self.offsets[k])
        return t[o:o + 9 * cout * cin], t[o + 9 * cout * cin:o + 9 * cout * cin + cout]

    def weight(self, name):
        return self._slices(self.master, name)

    def refresh_weights(self):
        for name, (cin, cout, _) in self.layers.items():
            w, _ = self._slices(self.master, name)
            N.call("sw100_nn_weights", _p(w), cin, cout, _p(self.wf[name]), _p(self.wd[name]), E._stream())

    def state_dict(self):
        return {"master": self.master.detach().cpu().numpy().copy(), "step": self.step}

    def load_state_dict(self, st):
        self.master.copy_(torch.from_numpy(np.asarray(st["master"], np.float32)))
        self.step = int(st.get("step", 0))
        self.refresh_weights()

    # ----------------------------------------------------------- buffers
    def buffers(self, n, s):
        key = (n, s)
        if key not in self._bufs:
            d = self.device

            def z(h, c, dt=BF16):
                return torch.zeros((n, h, h, c), dtype=dt, device=d)
            b = {"x": z(s, 16), "e1a": z(s, 16), "cat1": z(s, 48), "p1": z(s // 2, 16), "e2a": z(s // 2, 32),
                 "cat2": z(s // 2, 80), "p2": z(s // 4, 32), "e3a": z(s // 4, 48), "cat3": z(s // 4, 112),
                 "p3": z(s // 8, 48), "e4a": z(s // 8, 64), "cat4": z(s // 8, 128), "p4": z(s // 16, 64),
                 "e5a": z(s // 16, 64), "e5b": z(s // 16, 64), "d4": z(s // 8, 64), "d3": z(s // 4, 48),
                 "d2": z(s // 2, 32), "d1": z(s, 16), "out": z(s, 16, F32T)}
            # gradients of the same shapes (bf16), the output gradient included
            for k in list(b):
                if k != "x":
                    b["g_" + k] = torch.zeros_like(b[k], dtype=BF16)
            b["loss"] = torch.zeros(1, dtype=F32T, device=d)
            self._bufs[key] = b
        return self._bufs[key]

    # ----------------------------------------------------------- kernels
    def _conv(self, name, x: Act, y: Act, out_f32=False):
        cin, cout, relu = self.layers[name]
        assert x.c == cin and y.c == cout
        n = x.buf.shape[0]
        h, w = x.hw
        _, b = self._slices(self.master, name)
        N.call("sw100_nn_conv3x3_tc", _p(x.buf), n, h, w, cin, x.stride, x.coff, _p(self.wf[name]), _p(b), cout,
               _p(y.buf), y.stride, y.coff, int(relu), int(out_f32), _p(self.err), E._stream())

    def _dgrad(self, name, dy: Act, dx: Act):
        cin, cout, _ = self.layers[name]
        n = dy.buf.shape[0]
        h, w = dy.hw
        N.call("sw100_nn_conv3x3_tc", _p(dy.buf), n, h, w, cout, dy.stride, dy.coff, _p(self.wd[name]), None, cin,
               _p(dx.buf), dx.stride, dx.coff, 0, 0, _p(self.err), E._stream())

    def _wgrad(self, name, x: Act, dy: Act):
        cin, cout, _ = self.layers[name]
        n = x.buf.shape[0]
        h, w = x.hw
        dw, db = self._slices(self.grad, name)
        N.call("sw100_nn_conv3x3_wgrad", _p(x.buf), n, h, w, cin, x.stride, x.coff, _p(dy.buf), cout, dy.stride,
               dy.coff, _p(dw), _p(db), E._stream())

    def _relu_bwd(self, dy: Act, y: Act):
        n, h, w, _ = y.buf.shape
        N.call("sw100_nn_relu_bwd", _p(dy.buf), _p(y.buf), n * h * w, y.c, dy.stride, dy.coff, y.stride, y.coff,
               E._stream())

    def _pool(self, x: Act, y: Act):
        n = x.buf.shape[0]
        h, w = x.hw
        N.call("sw100_nn_pool2", _p(x.buf), n, h, w, x.c, x.stride, x.coff, _p(y.buf), y.stride, y.coff, 0, 0,
               E._stream())

    def _pool_bwd_acc(self, dy: Act, dx: Act):
        n = dx.buf.shape[0]
        h, w = dx.hw
        N.call("sw100_nn_pool2", _p(dy.buf), n, h, w, dx.c, dy.stride, dy.coff, _p(dx.buf), dx.stride, dx.coff, 1, 1,
               E._stream())

    def _up(self, x: Act, y: Act):
        n = x.buf.shape[0]
        h, w = x.hw
        N.call("sw100_nn_up2", _p(x.buf), n, h, w, x.c, x.stride, x.coff, _p(y.buf), y.stride, y.coff, 0,
               E._stream())

    def _up_bwd(self, dy: Act, dx: Act):
        n = dx.buf.shape[0]
        h, w = dx.hw
        N.call("sw100_nn_up2", _p(dy.buf), n, h, w, dx.c, dy.stride, dy.coff, _p(dx.buf), dx.stride, dx.coff, 1,
               E._stream())

    # ------------------------------------------------------- passes
    def forward(self, b):
        A = lambda k, off=0, c=None: Act(b[k], off, b[k].shape[-1] if c is None else c)  # noqa: E731
        self._conv("e1a", A("x"), A("e1a"))
        self._conv("e1b", A("e1a"), A("cat1", 32, 16))
        self._pool(A("cat1", 32, 16), A("p1"))
        self._conv("e2a", A("p1"), A("e2a"))
        self._conv("e2b", A("e2a"), A("cat2", 48, 32))
        self._pool(A("cat2", 48, 32), A("p2"))
        self._conv("e3a", A("p2"), A("e3a"))
        self._conv("e3b", A("e3a"), A("cat3", 64, 48))
        self._pool(A("cat3", 64, 48), A("p3"))
        self._conv("e4a", A("p3"), A("e4a"))
        self._conv("e4b", A("e4a"), A("cat4", 64, 64))
        self._pool(A("cat4", 64, 64), A("p4"))
        self._conv("e5a", A("p4"), A("e5a"))
        self._conv("e5b", A("e5a"), A("e5b"))
        self._up(A("e5b"), A("cat4", 0, 64))
        self._conv("d4", A("cat4"), A("d4"))
        self._up(A("d4"), A("cat3", 0, 64))
        self._conv("d3", A("cat3"), A("d3"))
        self._up(A("d3"), A("cat2", 0, 48))
        self._conv("d2", A("cat2"), A("d2"))
        self._up(A("d2"), A("cat1", 0, 32))
        self._conv("d1", A("cat1"), A("d1"))
        self._conv("head", A("d1"), Act(b["out"], 0, 16), out_f32=True)
        return b["out"]

    def backward(self, b):
        """Parameter gradients into self.grad (added) from b["g_out"]."""
        A = lambda k, off=0, c=None: Act(b[k], off, b[k].shape[-1] if c is None else c)  # noqa: E731

        def layer(name, inp, out, g_out, g_in):
            if self.layers[name][2]:
                self._relu_bwd(g_out, out)
            self._wgrad(name, inp, g_out)
            if g_in is not None:
                self._dgrad(name, g_out, g_in)
        layer("head", A("d1"), None, A("g_out"), A("g_d1"))
        layer("d1", A("cat1"), A("d1"), A("g_d1"), A("g_cat1"))
        self._up_bwd(A("g_cat1", 0, 32), A("g_d2"))
        layer("d2", A("cat2"), A("d2"), A("g_d2"), A("g_cat2"))
        self._up_bwd(A("g_cat2", 0, 48), A("g_d3"))
        layer("d3", A("cat3"), A("d3"), A("g_d3"), A("g_cat3"))
        self._up_bwd(A("g_cat3", 0, 64), A("g_d4"))
        layer("d4", A("cat4"), A("d4"), A("g_d4"), A("g_cat4"))
        self._up_bwd(A("g_cat4", 0, 64), A("g_e5b"))
        layer("e5b", A("e5a"), A("e5b"), A("g_e5b"), A("g_e5a"))
        layer("e5a", A("p4"), A("e5a"), A("g_e5a"), A("g_p4"))
        self._pool_bwd_acc(A("g_p4"), A("g_cat4", 64, 64))
        layer("e4b", A("e4a"), A("cat4", 64, 64), A("g_cat4", 64, 64), A("g_e4a"))
        layer("e4a", A("p3"), A("e4a"), A("g_e4a"), A("g_p3"))
        self._pool_bwd_acc(A("g_p3"), A("g_cat3", 64, 48))
        layer("e3b", A("e3a"), A("cat3", 64, 48), A("g_cat3", 64, 48), A("g_e3a"))
        layer("e3a", A("p2"), A("e3a"), A("g_e3a"), A("g_p2"))
        self._pool_bwd_acc(A("g_p2"), A("g_cat2", 48, 32))
        layer("e2b", A("e2a"), A("cat2", 48, 32), A("g_cat2", 48, 32), A("g_e2a"))
        layer("e2a", A("p1"), A("e2a"), A("g_e2a"), A("g_p1"))
        self._pool_bwd_acc(A("g_p1"), A("g_cat1", 32, 16))
        layer("e1b", A("e1a"), A("cat1", 32, 16), A("g_cat1", 32, 16), A("g_e1a"))
        layer("e1a", A("x"), A("e1a"), A("g_e1a"), None)

    def loss_and_grad(self, b, target, margin):
        """b["loss"] = MSE over the central box, b["g_out"] its gradient."""
        n, s = b["out"].shape[0], b["out"].shape[1]
        b["loss"].zero_()
        N.call("sw100_nn_mse", _p(b["out"]), _p(target), n, s, s, 16, N_OUT, margin, _p(b["g_out"]), _p(b["loss"]),
               E._stream())

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        N.call("sw100_nn_adam", _p(self.master), _p(self.grad), _p(self.m), _p(self.v), self.n_params,
               C.c_float(lr), C.c_float(b1), C.c_float(b2), C.c_float(eps), self.step, E._stream())
        self.refresh_weights()


# ------------------------------------------------------------------ data
def window_inputs(site: E.DeviceSite, origins, size, out: torch.Tensor):
    """Network inputs of windows at ``origins`` [(r0, c0)] of a site."""
    org = torch.tensor(np.asarray(origins, np.int32).reshape(-1), device=site.device)
    dem = site.t.get("dem")
    N.call("sw100_nn_input", _p(site.t["dsm"]), _p(site.t["vegdsm"]), _p(site.t["vegdsm2"]), _p(dem), site.rows,
           site.cols, _p(org), len(origins), size, _p(out), E._stream())
    return org


def window_targets(planes: torch.Tensor, origins, size, out: torch.Tensor):
    """Exact SVF planes of the windows, NHWC float32 (16 channels, 15 used);
    cells outside the grid are 0 (the loss never reads them: windows lie
    inside the grid where it is measured)."""
    out.zero_()
    rows, cols = planes.shape[1], planes.shape[2]
    for k, (r0, c0) in enumerate(origins):
        ra, rb = max(0, r0), min(rows, r0 + size)
        ca, cb = max(0, c0), min(cols, c0 + size)
        out[k, ra - r0:rb - r0, ca - c0:cb - c0, :N_OUT] = planes[:N_OUT, ra:rb, ca:cb].permute(1, 2, 0)
    return out


@dataclass
class TrainReport:
    steps: int
    windows: int
    seconds: float
    loss_first: float
    loss_last: float


def train(net: UNet, sites, planes, *, steps=600, batch=8, size=256, margin=64, lr=2e-3, seed=0,
          log_every=0) -> TrainReport:
    """Train on random windows of the given sites (``planes[i]`` = the exact
    SVF planes of ``sites[i]``); windows lie fully inside their site."""
    rng = np.random.default_rng(seed)
    b = net.buffers(batch, size)
    target = torch.zeros((batch, size, size, 16), dtype=F32T, device=net.device)
    losses = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(steps):
        k = int(rng.integers(len(sites)))
        s = sites[k]
        origins = [(int(rng.integers(0, s.rows - size + 1)), int(rng.integers(0, s.cols - size + 1)))
                   for _ in range(batch)]
        window_inputs(s, origins, size, b["x"])
        window_targets(planes[k], origins, size, target)
        net.forward(b)
        net.loss_and_grad(b, target, margin)
        net.grad.zero_()
        net.backward(b)
        lr_t = lr * (0.1 + 0.9 * 0.5 * (1 + math.cos(math.pi * it / max(1, steps))))
        net.adam(lr=lr_t)
        if it == 0 or it == steps - 1 or (log_every and it % log_every == 0):
            losses.append(float(b["loss"].item()))
    torch.cuda.synchronize()
    return TrainReport(steps, steps * batch, time.perf_counter() - t0, losses[0], losses[-1])


class SvfPreview:
    """Edit preview on a site whose exact SVF is known.

    For an edited box: the net's change of the 15 SVF planes over the
    central block of a window around the box (net(after) - net(before),
    added to the exact planes before the edit), then the exact windowed
    recompute restricted to the box's own pixels (their planes and patch
    bits exact: the edited cells change most).  Cells of the block outside
    the box keep their patch bits from before the edit.  When the net's
    mean absolute error on the window before the edit -- where the exact
    answer is known -- exceeds ``threshold``, the exact windowed recompute
    runs instead.  The net's forward pass is replayed from a CUDA graph."""

    def __init__(self, net: UNet, size=256, margin=64, threshold=0.02, graph=True):
        self.net, self.size, self.margin, self.threshold = net, size, margin, threshold
        self.use_graph = graph
        self._graph = None

    def window_origin(self, site, r0, c0, h, w):
        """Window whose central block covers the edited box (clipped so the
        whole window lies in the grid when the site is large enough)."""
        cb = self.size - 2 * self.margin
        if h > cb or w > cb:
            raise ValueError(f"edit box {h} x {w} is larger than the preview block {cb} x {cb}")
        rr = r0 + h // 2 - self.size // 2
        cc = c0 + w // 2 - self.size // 2
        rr = min(max(rr, 0), max(0, site.rows - self.size))
        cc = min(max(cc, 0), max(0, site.cols - self.size))
        return rr, cc

    def _forward(self, b):
        if not self.use_graph:
            return self.net.forward(b)
        if self._graph is None:
            self.net.forward(b)                       # warm-up outside the capture
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self.net.forward(b)
            self._graph = g
        self._graph.replay()
        return b["out"]

    def edit(self, site: E.DeviceSite, r0, c0, dsm=None, trees=None, dem=None):
        """Apply a block edit with the preview; returns a record with the
        mode ("preview" or "exact"), the window and the net's error before
        the edit."""
        blk = next(np.asarray(x, np.float32) for x in (dsm, trees, dem) if x is not None)
        h, w = blk.shape
        orr, occ = self.window_origin(site, r0, c0, h, w)
        S, m = self.size, self.margin
        b = self.net.buffers(2, S)
        planes = site.svf_result.planes
        window_inputs(site, [(orr, occ)], S, b["x"][0:1])          # before the edit
        site.update_rasters_block(r0, c0, dsm=dsm, trees=trees, dem=dem)
        if getattr(site, "_pending_full", False):                 # new step tables / bush: exact only
            return {"mode": "exact", "window": (orr, occ), "pre_error": None,
                    "exact": site.refresh_svf_after_block(r0, c0, h, w)}
        window_inputs(site, [(orr, occ)], S, b["x"][1:2])          # after it
        out = self._forward(b)
        ra, ca = orr + m, occ + m
        cs = S - 2 * m
        exact_pre = planes[:N_OUT, ra:ra + cs, ca:ca + cs].permute(1, 2, 0)
        pre = out[0, m:S - m, m:S - m, :N_OUT]
        err = float((pre - exact_pre).abs().mean().item())
        if err > self.threshold:
            return {"mode": "exact", "window": (orr, occ), "pre_error": err,
                    "exact": site.refresh_svf_after_block(r0, c0, h, w)}
        new = (exact_pre + (out[1, m:S - m, m:S - m, :N_OUT] - pre)).clamp_(0.0, 1.0)
        planes[:N_OUT, ra:ra + cs, ca:ca + cs] = new.permute(2, 0, 1)
        refresh_statics(planes, ra, ca, cs, cs, site.params.transVeg)
        site.exact_svf_box(r0, c0, h, w)
        return {"mode": "preview", "window": (orr, occ), "pre_error": err}


# ------------------------------------------------------------ statics
def refresh_statics(planes: torch.Tensor, r0, c0, h, w, trans_veg=0.03):
    """Time-loop statics (planes 16-18) of a block from its SVF planes
    (utci_process.py:864-897): svfbuveg, tan(acos(sqrt(svf))) and
    tan(asin(exp(log(1 - max(svf + svfveg - 1, 0)) / 2)))."""
    sl = (slice(r0, r0 + h), slice(c0, c0 + w))
    svf, svfveg = planes[0][sl], planes[11][sl]
    planes[16][sl] = svf - (1.0 - svfveg) * (1.0 - trans_veg)
    planes[17][sl] = torch.tan(torch.acos(torch.sqrt(svf)))
    tmp = (svf + svfveg - 1.0).clamp(min=0.0)
    planes[18][sl] = torch.tan(torch.asin(torch.exp(torch.log(1.0 - tmp) / 2.0)))


# --------------------------------------------------------- training data
def training_sites(n_sites=8, side=512, seed=77):
    """Seeded synthetic cities with their exact SVF (the sweep is the
    teacher): [(DeviceSite, planes)]."""
    from . import synthetic
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_sites):
        c = synthetic.make_city(side, side, seed=int(seed * 100 + k), density=float(rng.uniform(0.10, 0.45)),
                                canopy_cover=float(rng.uniform(0.0, 0.30)))
        s = E.DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, amaxvalue=48.0)
        res = s.run_svf()
        out.append((s, res.planes))
    return out


def random_edit(site: E.DeviceSite, rng, block=128):
    """A seeded building edit inside a block: add a building, remove the
    built cells of a box, or raise / lower the built cells of a box by
    5-30 m.  Returns (kind, r0, c0, new_dsm_block)."""
    h = int(rng.integers(10, 41))
    w = int(rng.integers(10, 41))
    r0 = int(rng.integers(block, site.rows - block - h))
    c0 = int(rng.integers(block, site.cols - block - w))
    sl = (slice(r0, r0 + h), slice(c0, c0 + w))
    dsm, dem = site.host["dsm"][sl].copy(), site.host["dem"][sl]
    kind = ("add", "remove", "height")[int(rng.integers(3))]
    built = dsm - dem >= 2.0
    if kind == "add" or not built.any():
        kind = "add"
        dsm = np.maximum(dsm, dem + np.float32(rng.uniform(5, 30)))
    elif kind == "remove":
        dsm = np.where(built, dem, dsm).astype(np.float32)
    else:
        dz = np.float32(rng.uniform(5, 30) * (1 if rng.random() < 0.5 else -1))
        dsm = np.where(built, np.maximum(dem + 2.5, dsm + dz), dsm).astype(np.float32)
    return kind, r0, c0, dsm.astype(np.float32)


def evaluate_edits(net: UNet, site: E.DeviceSite, series, n_edits=50, seed=5, threshold=1.0):
    """Seeded edits on a site with exact SVF: per edit, the exact windowed
    recompute, the preview and the stale (unchanged) SVF, with device times
    and, over the edit window's central block, the SVF mean absolute error
    and the Tmrt RMSE of the whole 24-step chain against the exact chain.
    Shadows are recomputed exactly in every variant (the sun march reads the
    edited rasters); the patch cubes stay those before the edit for the
    preview and stale variants."""
    rng = np.random.default_rng(seed)
    prev = SvfPreview(net, threshold=threshold)
    r = site.svf_result
    base_planes, base_bits = r.planes.clone(), r.bits.clone()
    s_struct, s_dev = site.upload_series(series)
    rows = []
    S, m = prev.size, prev.margin
    cs = S - 2 * m

    def tmrt():
        site.state.zero_()
        return site.run_time_loop(series, requested=("tmrt",), series_dev=(s_struct, s_dev))["tmrt"]

    for k in range(n_edits):
        kind, r0, c0, new = random_edit(site, rng)
        h, w = new.shape
        old = site.host["dsm"][r0:r0 + h, c0:c0 + w].copy()
        orr, occ = prev.window_origin(site, r0, c0, h, w)
        win = (slice(orr + m, orr + m + cs), slice(occ + m, occ + m + cs))
        # exact
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        site.edit_svf_block(r0, c0, dsm=new)
        e1.record()
        torch.cuda.synchronize()
        t_exact = e0.elapsed_time(e1)
        exact_planes = r.planes[:N_OUT][(slice(None),) + win].clone()
        t_ex = tmrt()[(slice(None),) + win].clone()
        # stale SVF, edited rasters
        r.planes.copy_(base_planes)
        r.bits.copy_(base_bits)
        t_st = tmrt()[(slice(None),) + win].clone()
        stale_planes = r.planes[:N_OUT][(slice(None),) + win].clone()
        # preview from the state before the edit
        site.update_rasters_block(r0, c0, dsm=old)
        e0.record()
        info = prev.edit(site, r0, c0, dsm=new)
        e1.record()
        torch.cuda.synchronize()
        t_prev = e0.elapsed_time(e1)
        prev_planes = r.planes[:N_OUT][(slice(None),) + win].clone()
        t_pv = tmrt()[(slice(None),) + win].clone()
        # back to the base state for the next edit
        site.update_rasters_block(r0, c0, dsm=old)
        r.planes.copy_(base_planes)
        r.bits.copy_(base_bits)
        valid = torch.isfinite(t_ex) & torch.isfinite(t_pv) & torch.isfinite(t_st)
        rmse = lambda a: float(torch.sqrt(((a - t_ex)[valid] ** 2).mean()).item())  # noqa: E731
        rows.append({"kind": kind, "mode": info["mode"], "ms_exact": t_exact, "ms_preview": t_prev,
                     "svf_mae_preview": float((prev_planes - exact_planes).abs().mean().item()),
                     "svf_mae_stale": float((stale_planes - exact_planes).abs().mean().item()),
                     "tmrt_rmse_preview": rmse(t_pv), "tmrt_rmse_stale": rmse(t_st)})
    return rows


WEIGHTS = __import__("os").path.join(__import__("os").path.dirname(__file__), "data", "preview_weights.npz")


def load_pretrained(path: str = WEIGHTS, seed: int = 0) -> UNet:
    """The network with the weights trained by :func:`main` (the file
    shipped with the package: 3000 steps of 8 windows of 256 x 256 cells
    from 12 seeded 512 x 512 cities)."""
    net = UNet(seed=seed)
    with np.load(path) as z:
        net.load_state_dict({"master": z["master"], "step": int(z["step"])})
    return net


def main(argv=None):
    """Train the preview on seeded cities and save its weights:
    python -m solweig_project_b200.preview --out weights.npz [--steps N]"""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--sites", type=int, default=12)
    ap.add_argument("--side", type=int, default=512)
    args = ap.parse_args(argv)
    from . import build
    build.build()
    data = training_sites(args.sites, args.side)
    net = UNet(seed=0)
    rep = train(net, [s for s, _ in data], [p for _, p in data], steps=args.steps, log_every=100)
    st = net.state_dict()
    np.savez_compressed(args.out, master=st["master"], step=st["step"], loss_first=rep.loss_first,
                        loss_last=rep.loss_last, seconds=rep.seconds, windows=rep.windows)
    print(f"trained {rep.steps} steps ({rep.windows} windows) in {rep.seconds:.1f} s: "
          f"loss {rep.loss_first:.4g} -> {rep.loss_last:.4g}; saved {args.out}")


if __name__ == "__main__":
    main()
