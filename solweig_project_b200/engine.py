"""Device-side driver of the radiation chain for one site.

:class:`DeviceSite` owns the site's rasters in HBM, runs the SVF sweep and the
time loop through the C ABI (``_native``) and hands back device tensors.
torch provides device memory and the stream; all compute is the library's.

Layout in HBM (npix = rows * cols):
  static rasters          float32 planes, row-major
  SVF result              16 float32 planes + 3 x 5 uint32 bit-cube words
  packed march source     float4 {dsm, vegdsm, vegdsm2, bush}  (workspace)
  sun-march records       n_day x npix float4 {shadow, Lup, albedo, flags} (workspace)
  thermal state           6 float32 planes, carried across calls
  outputs                 n_out x n_t x npix float32
"""
from __future__ import annotations

import collections
import ctypes as C
import threading
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from . import tables as T
from . import timeseries as TS

F32 = np.float32
SVF_NAMES = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS", "svfSaveg",
             "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg", "svftotal", "svfbuveg", "hsvf", "tan_alfa")
STATE_NAMES = ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")


def require_cuda():
    if not torch.cuda.is_available():
        raise N.NativeUnavailable("no CUDA device: the B200 backend runs on the GPU only")
    N.load()


class Timeline:
    """Host phases of a call: mark(name) stamps the end of a phase
    (time.perf_counter); with a stream, a CUDA event is recorded there too,
    so the GPU's progress at that point can be read afterwards."""

    def __init__(self, enabled=True):
        import time
        self.enabled = enabled
        self._clock = time.perf_counter
        self.t0 = self._clock() if enabled else 0.0
        self.marks = []
        self.start_event = None
        if enabled and torch.cuda.is_available():
            self.start_event = torch.cuda.Event(enable_timing=True)
            self.start_event.record()

    def mark(self, name, stream=None):
        if not self.enabled:
            return
        ev = None
        if stream is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
        self.marks.append((name, self._clock(), ev))

    def report(self):
        """[(phase, host ms since the previous mark, host ms since the
        start, GPU ms since the start at the recorded event or None)]."""
        out, prev = [], self.t0
        for name, t, ev in self.marks:
            gpu = self.start_event.elapsed_time(ev) if ev is not None and self.start_event is not None else None
            out.append((name, (t - prev) * 1e3, (t - self.t0) * 1e3, gpu))
            prev = t
        return out


# the time loop's dense patch sums on the tensor cores (sw100_patch_sums)
# rather than in the loop kernel
TENSOR_SUMS = True
# Run the time / flux loops over the site's 8 x 4 pixel patches sorted by
# their ground-view walk work (sw100_walk_work), heaviest first: a loop block
# waits at every step for its slowest warp, and blocks of patches that walk
# alike wait least (3.46 -> 3.11 ms at 500 x 500 x 24; identical results).
# Only for sites up to WALK_ORDER_MAX_PIXELS: the sorted blocks that run at
# once lie all over the grid, and once a day's sun-march records (16 B per
# pixel) no longer sit in L2 their gathers miss (4096 x 4096: 187 ms against
# 171 ms in grid order; sorting within row bands instead: 169 ms there but
# 3.7-3.9 ms at 500 x 500).
WALK_ORDER = True
WALK_ORDER_MAX_PIXELS = 1 << 21
# work levels of the order (grid order within a level): exact work values
# 3.12 ms, 24 levels 3.06 ms, 6 levels 3.21 ms at 500 x 500 x 24
WALK_LEVELS = 24

# device copies of the ground-view azimuth table per (device, walk length),
# copied synchronously once (then readable from every stream)
_GVF_DEV = {}
_GVF_LOCK = threading.Lock()


def _gvf_dev(device, second: int) -> torch.Tensor:
    key = (str(device), second)
    with _GVF_LOCK:
        hit = _GVF_DEV.get(key)
        if hit is None:
            raw = np.ascontiguousarray(T.gvf_table(second)).view(np.uint8).reshape(-1).copy()
            TRANSFER["h2d"] += raw.nbytes
            hit = _GVF_DEV[key] = torch.from_numpy(raw).to(device)
            torch.cuda.synchronize(device)
        return hit

# chunks of the chunked time loop whose device buffers are alive at once
CHUNKS_IN_FLIGHT = 3

# default chunk lengths of the chunked time loop (then 8 while steps remain):
# a long first chunk whose tables are built while the SVF sweep runs, a short
# last one whose GPU work and copy-back are the call's tail (500 x 500 x 24 on
# B200, median of 24 interleaved calls: 8.74 ms per call against 8.90 with
# 16 + 8 and 9.21 with 14 + 6 + 4)
DEFAULT_CHUNKS = (16, 6, 2, 8)

# host <-> device bytes moved by this module (inputs, tables, results)
TRANSFER = {"h2d": 0, "d2h": 0}


# The chunked loop's side and copy streams, one of each per device for the
# whole process.  The caching allocator keeps freed blocks per stream, so
# buffers allocated on a stream of a site's own would never be reused by the
# next site's: every call would go back to cudaMalloc, which can wait for
# the device.
_STREAMS = {}
_STREAMS_LOCK = threading.Lock()


def _shared_stream(device, role):
    dev = torch.device(device)
    key = (dev.index if dev.index is not None else torch.cuda.current_device(), role)
    with _STREAMS_LOCK:
        if key not in _STREAMS:
            _STREAMS[key] = torch.cuda.Stream(device=key[0])
        return _STREAMS[key]


def _upload(host: torch.Tensor, device) -> torch.Tensor:
    """Host tensor -> device through a pinned staging buffer."""
    TRANSFER["h2d"] += host.numel() * host.element_size()
    return host.pin_memory().to(device, non_blocking=True)


def _dev(x, device, dtype=torch.float32):
    return _upload(torch.as_tensor(np.ascontiguousarray(x), dtype=dtype), device)


def _table(arr: np.ndarray, device) -> torch.Tensor:
    """Upload a structured numpy table as raw bytes."""
    raw = np.ascontiguousarray(arr).view(np.uint8).reshape(-1)
    if raw.size == 0:
        raw = np.zeros(16, np.uint8)
    return _upload(torch.from_numpy(raw.copy()), device)


def to_host(t: torch.Tensor) -> np.ndarray:
    """Device tensor -> numpy array in page-locked host memory (torch's
    caching host allocator: a repeated call of the same size reuses the
    buffer once the previous result is released)."""
    TRANSFER["d2h"] += t.numel() * t.element_size()
    if t.device.type == "cpu":
        return t.numpy()
    out = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    out.copy_(t)
    return out.numpy()


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def march_inputs(dsm, trees, dem):
    """Derived march rasters exactly as compute_utci / run_utci_window build
    them (utci_process.py:667-681, 1377-1385), float32 IEEE arithmetic."""
    a = np.asarray(dsm, F32)
    t1 = np.asarray(trees, F32).copy()
    t2 = np.asarray(dem, F32)
    t1[t1 < 0.] = 0.
    vegdem = t1 + t2
    vegdem2 = t1 * F32(0.25) + t2
    bush = np.logical_not(vegdem2 * vegdem).astype(F32) * vegdem
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * F32(0.25) + a
    vegdsm2[vegdsm2 == a] = 0
    amax = F32(max(a.max(), vegdem.max()))
    buildings = a - t2
    buildings[buildings < 2.] = 1.
    buildings[buildings >= 2.] = 0.
    return vegdsm, vegdsm2, bush, amax, buildings


@dataclass
class SvfResult:
    planes: torch.Tensor      # (19, rows, cols) float32, SVF_NAMES order
    bits: torch.Tensor        # (3, 5, rows, cols) int32 words (sh, vegsh, vbshvegsh)
    single_step: np.ndarray   # uint32[5] patches with <= 1 march step

    def plane(self, name):
        return self.planes[SVF_NAMES.index(name)]

    def cubes(self, n_patches=153):
        """Dense (rows, cols, P) float32 cubes (shmat, vegshmat, vbshvegshmat)
        as the reference returns them (shadow.py:625)."""
        b = self.bits.view(torch.int32)
        rows, cols = b.shape[2], b.shape[3]
        q = torch.arange(n_patches, device=b.device)
        words = b[:, q // 32]                                   # (3, P, rows, cols)
        shift = (q % 32).view(1, -1, 1, 1)
        bit = ((words >> shift) & 1).to(torch.float32)
        single = torch.tensor([(int(self.single_step[k // 32]) >> (k % 32)) & 1 for k in range(n_patches)],
                              device=b.device, dtype=torch.bool).view(-1, 1, 1)
        sh, veg, vb = bit[0], bit[1], bit[2]
        vb = torch.where(single, 2.0 - vb, vb)
        return tuple(x.permute(1, 2, 0).contiguous() for x in (sh, veg, vb))


class DeviceSite:
    """One site: rasters resident on the device, SVF sweep and time loop."""

    def __init__(self, dsm, trees, dem, walls, aspect_deg, scale, *, landcover=None, lc_class=None,
                 windcoeff=None, amaxvalue=None, params: TS.ModelParams = None, device="cuda"):
        require_cuda()
        self.device = torch.device(device)
        self.params = params or TS.ModelParams()
        a = np.asarray(dsm, F32)
        self.rows, self.cols = a.shape
        if self.rows * self.cols >= 2 ** 31:
            raise ValueError("grid too large")
        for name, x in (("trees", trees), ("dem", dem), ("walls", walls), ("aspect", aspect_deg),
                        ("landcover", landcover), ("windcoeff", windcoeff)):
            if x is not None and np.shape(x) != a.shape:
                raise ValueError(f"{name} must have the shape of the DSM {a.shape}")
        if landcover is not None and lc_class is None:
            raise ValueError("landcover needs lc_class (the land-cover class table)")
        self.scale = float(scale)
        d = self.device
        # the input rasters go up as they are; everything derived from them
        # is computed on the device (sw100_prepare_site)
        self.t = {"dsm": _dev(a, d), "trees": _dev(trees, d), "dem": _dev(dem, d), "walls": _dev(walls, d)}
        aspect_d = _dev(aspect_deg, d)
        lc_d = _dev(landcover, d) if landcover is not None else None
        plane = lambda dtype=torch.float32: torch.empty((self.rows, self.cols), dtype=dtype, device=d)  # noqa: E731
        for k in ("vegdsm", "vegdsm2", "bush", "buildings", "aspect_rad", "tgk", "tstart", "alb", "emis"):
            self.t[k] = plane()
        self.t["class_idx"] = plane(torch.uint8)
        self.t["windcoeff"] = (torch.ones((self.rows, self.cols), dtype=torch.float32, device=d) if windcoeff is None
                               else _dev(windcoeff, d))
        table = N.ClassTable()
        if landcover is not None:
            tab, valid = TS.class_table(lc_class)
            for k in ("tgk", "tstart", "alb", "emis"):
                getattr(table, k)[:] = [float(v) for v in tab[k]]
            table.valid = valid
        stats = torch.empty(N.SITE_STATS_WORDS, dtype=torch.int32, device=d)
        if WALK_ORDER and self.rows * self.cols <= WALK_ORDER_MAX_PIXELS:
            # the loops' azimuth table, copied (and synchronised on, once per
            # process) while the stats read below waits for the device anyway
            _gvf_dev(d, self._walk_second())
        t = self.t
        N.call("sw100_prepare_site", _ptr(t["dsm"]), _ptr(t["trees"]), _ptr(t["dem"]), _ptr(aspect_d), _ptr(lc_d),
               C.byref(table), self.rows, self.cols, _ptr(t["vegdsm"]), _ptr(t["vegdsm2"]), _ptr(t["bush"]),
               _ptr(t["buildings"]), _ptr(t["aspect_rad"]), _ptr(t["tgk"]), _ptr(t["tstart"]), _ptr(t["alb"]),
               _ptr(t["emis"]), _ptr(t["class_idx"]), _ptr(stats), _stream())
        st = to_host(stats).view(np.uint32)
        if st[N.N_SITE_STATS + 3]:
            raise ValueError("landcover holds a code without a row in lc_class")
        v = {s: N.stat_value(st, s) for s in range(N.N_SITE_STATS)}
        # the host computation's reductions, Python max() quirks with NaN included
        amax = F32(max(v[N.STAT_DSM], v[N.STAT_VEGDEM]))
        self.amax_fixed = amaxvalue is not None
        self.amax = F32(amaxvalue) if amaxvalue is not None else amax
        self.bush_any = bool(v[N.STAT_BUSH] > 0)
        self.vmax = F32(max(v[N.STAT_DSM], v[N.STAT_VEGDSM], v[N.STAT_VEGDSM2]))
        self.all_finite = not st[N.N_SITE_STATS + 1]
        self.hmax = float(max(v[N.STAT_ABS_DSM], v[N.STAT_ABS_VEGDSM], v[N.STAT_ABS_VEGDSM2]))
        if not self.bush_any:
            self.t["bush"] = None
        self.props = TS.device_props(lc_class if landcover is not None else None, st[N.N_SITE_STATS + 2])
        self._host = None        # host copies of dsm / trees / dem, made on first use by an edit
        self.svf_result: SvfResult | None = None
        self.state = torch.zeros((6, self.rows, self.cols), dtype=torch.float32, device=d)
        self._keep = []
        self._cache = {}

    @classmethod
    def from_march_rasters(cls, a, vegdsm, vegdsm2, bush, amaxvalue, scale, device="cuda"):
        """A site that only runs the SVF sweep, from the march rasters the
        reference's svf_calculator takes (DSM, canopy top, trunk top, bush)."""
        require_cuda()
        self = cls.__new__(cls)
        self.device = torch.device(device)
        self.params = TS.ModelParams()
        a = np.asarray(a, F32)
        self.rows, self.cols = a.shape
        vegdsm = np.asarray(vegdsm, F32)
        vegdsm2 = np.asarray(vegdsm2, F32)
        bush = np.asarray(bush, F32)
        self.amax = F32(amaxvalue)
        self.amax_fixed = True
        self._set_march_stats(a, vegdsm, vegdsm2, bush)
        self._host = None
        self.scale = float(scale)
        d = self.device
        self.t = {"dsm": _dev(a, d), "vegdsm": _dev(vegdsm, d), "vegdsm2": _dev(vegdsm2, d),
                  "bush": _dev(bush, d) if self.bush_any else None}
        self.props = None
        self.svf_result = None
        self.state = None
        self._keep = []
        self._cache = {}
        return self

    @property
    def host(self):
        """Host copies of the edited inputs (dsm, trees, dem), read back from
        the device on first use; block edits update them in place.  None for
        a site built from march rasters."""
        if self._host is None and "trees" in self.t:
            self._host = {k: to_host(self.t[k]).reshape(self.rows, self.cols).copy() for k in ("dsm", "trees", "dem")}
        return self._host

    @host.setter
    def host(self, value):
        self._host = value

    def _set_march_stats(self, a, vegdsm, vegdsm2, bush):
        self.bush_any = bool(bush.max() > 0)
        self.vmax = F32(max(a.max(), vegdsm.max(), vegdsm2.max()))
        self.all_finite = bool(np.isfinite(a).all() and np.isfinite(vegdsm).all() and np.isfinite(vegdsm2).all())
        self.hmax = float(max(np.abs(a).max(), np.abs(vegdsm).max(), np.abs(vegdsm2).max()))

    # --------------------------------------------------------------- SVF
    def walk_order(self) -> torch.Tensor:
        """The loops' patch order (sw100_site_planes.patch_order): the 8 x 4
        pixel patches by ground-view walk work (sw100_walk_work) in
        WALK_LEVELS levels, heaviest first, grid order within a level (so
        that the blocks at work still gather from neighbouring patches).
        Built on the device on first use and kept until an edit changes the
        buildings raster."""
        hit = self._cache.get("walk_order")
        if hit is None:
            second = self._walk_second()
            gvf = _gvf_dev(self.device, second)
            n = ((self.rows + 3) // 4) * ((self.cols + 7) // 8)
            work = torch.empty(n, dtype=torch.int32, device=self.device)
            N.call("sw100_walk_work", C.byref(self.site_struct()), self.rows, self.cols, _ptr(gvf), second,
                   _ptr(work), _stream())
            q = max(1, (N.N_GVF_AZ * second) // WALK_LEVELS)
            order = torch.argsort(work // q, descending=True, stable=True).to(torch.int32)
            hit = self._cache["walk_order"] = (order, work, gvf)
        return hit[0]

    def _walk_second(self) -> int:
        """Steps of the ground-view walks (`second`, at most the tables'
        MAX_GVF_STEPS)."""
        return min(int(TS.walk_steps(self.params, self.scale)[1]), N.MAX_GVF_STEPS)

    def loop_site_struct(self) -> N.SitePlanes:
        """site_struct() with the patch order of the time / flux loops
        (WALK_ORDER, sites up to WALK_ORDER_MAX_PIXELS)."""
        s = self.site_struct()
        if WALK_ORDER and self.rows * self.cols <= WALK_ORDER_MAX_PIXELS:
            order = self.walk_order()
            s.patch_order, s.n_patch_order = order.data_ptr(), order.numel()
        return s

    def site_struct(self) -> N.SitePlanes:
        s = N.SitePlanes()
        t = self.t
        s.dsm, s.vegdsm, s.vegdsm2 = t["dsm"].data_ptr(), t["vegdsm"].data_ptr(), t["vegdsm2"].data_ptr()
        s.bush = t["bush"].data_ptr() if t["bush"] is not None else 0
        s.vmax = float(self.vmax)
        s.bush_any = int(self.bush_any)
        for k in ("svfbuveg", "hsvf", "tan_alfa", "buildings", "walls", "aspect_rad", "tgk", "tstart", "alb",
                  "emis", "class_idx", "windcoeff", "bits"):
            v = t.get(k)
            setattr(s, k, v.data_ptr() if v is not None else 0)
        if self.svf_result is not None:
            for w in range(N.CUBE_WORDS):
                s.single_step[w] = int(self.svf_result.single_step[w])
        return s

    def svf_tables(self, patch_option=2):
        """Plan and step tables of the SVF sweep, built and uploaded once."""
        key = ("svf", patch_option)
        if key not in self._cache:
            plan, steps, single = T.svf_plan(self.rows, self.cols, self.scale, self.amax, self.bush_any,
                                             patch_option, trans_veg=self.params.transVeg,
                                             all_finite=self.all_finite)
            d = self.device
            ws_bytes = N.workspace_bytes("sw100_svf_workspace_bytes", self.rows, self.cols, len(steps))
            self._cache[key] = (_table(plan, d), _table(steps, d), len(steps), single,
                                torch.empty(ws_bytes, dtype=torch.uint8, device=d))
            self._cache[("svf_host", patch_option)] = (plan, steps)
        return self._cache[key]

    def edit_svf(self, dsm, trees, dem, walls=None, aspect_deg=None, patch_option=2) -> dict:
        """Exact SVF update after an edit of the rasters: the new march
        rasters are diffed against the current ones on the device, and only
        the pixels whose marches can read the changed box re-march, only the
        patches that do (the corridor closure of the reference's incremental
        exact march, solweig_core/sparse_work.py:633-781, spliced into the
        stored result as incremental/solver.py:861-1135 does).  The planes
        and bits equal a full sweep of the new rasters bit for bit.  A full
        sweep runs instead when the step tables would change (a new
        amaxvalue), when either scene has bush, or when a raster holds a
        non-finite value.  Returns {"mode": "window" | "full" | "none",
        "rect", "window", "pixels"}."""
        if self.svf_result is None:
            raise RuntimeError("run_svf() (or set_svf()) must come before edit_svf()")
        a = np.asarray(dsm, F32)
        if a.shape != (self.rows, self.cols):
            raise ValueError(f"edited rasters must keep the grid shape {(self.rows, self.cols)}")
        vegdsm, vegdsm2, bush, amax, buildings = march_inputs(a, trees, dem)
        new_amax = self.amax if self.amax_fixed else amax
        old = {k: self.t[k] for k in ("dsm", "vegdsm", "vegdsm2", "bush")}
        old_site = self.site_struct()
        old_bush, old_hmax = self.bush_any, self.hmax
        d = self.device
        self.t.update(dsm=_dev(a, d), vegdsm=_dev(vegdsm, d), vegdsm2=_dev(vegdsm2, d),
                      bush=_dev(bush, d) if bush.max() > 0 else None, buildings=_dev(buildings, d),
                      dem=_dev(np.asarray(dem, F32), d))
        self._cache.pop("walk_order", None)   # the buildings changed
        if walls is not None:
            self.t["walls"] = _dev(np.asarray(walls, F32), d)
        if aspect_deg is not None:
            self.t["aspect_rad"] = _dev((np.asarray(aspect_deg, F32) * F32(np.pi)) / F32(180.), d)
        self._set_march_stats(a, vegdsm, vegdsm2, bush)
        self.hmax = max(self.hmax, old_hmax)  # a bound over the rasters before and after the edit
        if self.host is not None:
            self.host = {"dsm": a.copy(), "trees": np.asarray(trees, F32).copy(), "dem": np.asarray(dem, F32).copy()}
        if old_bush or self.bush_any or new_amax != self.amax or not self.all_finite:
            self.amax = new_amax
            self._cache = {k: v for k, v in self._cache.items() if k[0] not in ("svf", "svf_host")}
            self.run_svf(patch_option)
            return {"mode": "full", "rect": None, "window": (0, self.rows - 1, 0, self.cols - 1),
                    "pixels": self.rows * self.cols}
        new_site = self.site_struct()
        key = ("diff_ws",)
        ws_bytes = N.workspace_bytes("sw100_diff_bbox_workspace_bytes", self.rows, self.cols)
        if key not in self._cache:
            self._cache[key] = (torch.empty(ws_bytes, dtype=torch.uint8, device=d),
                                torch.empty(4, dtype=torch.int32, device=d))
        ws, box = self._cache[key]
        N.call("sw100_diff_bbox", C.byref(old_site), C.byref(new_site), self.rows, self.cols, _ptr(box), _ptr(ws),
               ws.numel(), _stream())
        rect = tuple(int(v) for v in box.cpu().tolist())
        del old
        if rect[1] < 0:
            return {"mode": "none", "rect": None, "window": None, "pixels": 0}
        return self._window_update(rect, patch_option)

    def _corridor(self, patch_option):
        """Corridor descriptors and per-patch shift bounds, cached while the
        height bound they were built for still holds."""
        key = ("corridor", patch_option)
        hit = self._cache.get(key)
        if hit is None or hit[0] < self.hmax:
            plan_d, steps_d, n_steps, _, _ = self.svf_tables(patch_option)
            plan, steps = self._cache[("svf_host", patch_option)]
            bound = max(64.0, 2.0 * self.hmax)
            desc = T.svf_corridor(plan, steps, bound)
            self._cache[key] = hit = (bound, desc, _upload(torch.from_numpy(desc), self.device),
                                      T.patch_shift_bounds(plan, steps, desc))
        return hit[1], hit[2], hit[3]

    def exact_svf_box(self, r0, c0, h, w, patch_option=2):
        """Exact SVF planes and bits of the box's own pixels after an edit
        of the rasters inside it, one thread per (pixel, patch) march
        (sw100_svf_box); pixels outside keep what they hold."""
        plan_d, steps_d, n_steps, _, _ = self.svf_tables(patch_option)
        _, desc_d, _ = self._corridor(patch_option)
        key = ("window_ws",)
        if key not in self._cache:
            self._cache[key] = torch.empty(N.workspace_bytes("sw100_svf_window_workspace_bytes", self.rows,
                                                             self.cols), dtype=torch.uint8, device=self.device)
        wws = self._cache[key]
        r = self.svf_result
        site = self.site_struct()
        box = (r0, r0 + h - 1, c0, c0 + w - 1)
        N.call("sw100_svf_box", C.byref(site), self.rows, self.cols, _ptr(plan_d), _ptr(steps_d), n_steps, _ptr(desc_d),
               (C.c_int32 * 4)(*box), _ptr(r.planes), _ptr(r.bits), _ptr(wws), wws.numel(), _stream())
        return {"mode": "box", "rect": box, "window": box, "pixels": h * w}

    def _window_update(self, rect, patch_option=2) -> dict:
        plan_d, steps_d, n_steps, _, _ = self.svf_tables(patch_option)
        desc, desc_d, bounds = self._corridor(patch_option)
        window = T.window_from_bounds(rect, bounds, self.rows, self.cols)
        key = ("window_ws",)
        if key not in self._cache:
            self._cache[key] = torch.empty(N.workspace_bytes("sw100_svf_window_workspace_bytes", self.rows,
                                                             self.cols), dtype=torch.uint8, device=self.device)
        wws = self._cache[key]
        r = self.svf_result
        site = self.site_struct()
        N.call("sw100_svf_window", C.byref(site), self.rows, self.cols, _ptr(plan_d), _ptr(steps_d), n_steps,
               _ptr(desc_d), (C.c_int32 * 4)(*rect), (C.c_int32 * 4)(*window), _ptr(r.planes), _ptr(r.bits),
               _ptr(wws), wws.numel(), _stream())
        self._prepare_loop_statics()
        return {"mode": "window", "rect": tuple(rect), "window": window,
                "pixels": (window[1] - window[0] + 1) * (window[3] - window[2] + 1)}

    def edit_svf_block(self, r0, c0, dsm=None, trees=None, dem=None, patch_option=2) -> dict:
        """Exact SVF update after replacing the block of the rasters at
        (r0, c0) with the given arrays (any of dsm / trees / dem, same block
        shape): only the block travels to the device and the block is the
        edit rectangle.  Same result and fallbacks as :meth:`edit_svf`."""
        blk = next(np.asarray(x, F32) for x in (dsm, trees, dem) if x is not None)
        self.update_rasters_block(r0, c0, dsm=dsm, trees=trees, dem=dem)
        return self.refresh_svf_after_block(r0, c0, blk.shape[0], blk.shape[1], patch_option)

    def update_rasters_block(self, r0, c0, dsm=None, trees=None, dem=None):
        """Replace the block at (r0, c0) of the edited inputs (host copies
        and device march rasters); the SVF result is left as it was (see
        :meth:`refresh_svf_after_block`)."""
        if self.svf_result is None or self.host is None:
            raise RuntimeError("block edits need a site built from rasters and a computed SVF")
        blk = next(np.asarray(x, F32) for x in (dsm, trees, dem) if x is not None)
        h, w = blk.shape
        if r0 < 0 or c0 < 0 or r0 + h > self.rows or c0 + w > self.cols or h == 0 or w == 0:
            raise ValueError(f"block {h} x {w} at ({r0}, {c0}) is outside the {self.rows} x {self.cols} grid")
        sl = (slice(r0, r0 + h), slice(c0, c0 + w))
        for name, v in (("dsm", dsm), ("trees", trees), ("dem", dem)):
            if v is not None:
                self.host[name][sl] = np.asarray(v, F32)
        a, t1, t2 = self.host["dsm"], self.host["trees"], self.host["dem"]
        vegdsm_b, vegdsm2_b, bush_b, _, bld_b = march_inputs(a[sl], t1[sl], t2[sl])
        self._pending_full = bool(self.bush_any or bush_b.max() > 0 or not (
            np.isfinite(a[sl]).all() and np.isfinite(vegdsm_b).all() and np.isfinite(vegdsm2_b).all()))
        if not self.amax_fixed:
            amax = F32(max(a.max(), float((np.maximum(t1, 0) + t2).max())))
            self._pending_full = self._pending_full or amax != self.amax
        names = ("dsm", "vegdsm", "vegdsm2", "buildings", "dem")
        stack = np.stack([a[sl], vegdsm_b, vegdsm2_b, bld_b, t2[sl]]).astype(F32)
        TRANSFER["h2d"] += stack.nbytes
        dev = torch.from_numpy(stack).to(self.device)      # one small copy for the five planes
        for k, name in enumerate(names):
            self.t[name].view(self.rows, self.cols)[sl].copy_(dev[k])
        self._cache.pop("walk_order", None)   # the buildings changed
        # bounds only need to stay above the true maxima (early exit, height-blind patches)
        hb = float(max(np.abs(a[sl]).max(), np.abs(vegdsm_b).max(), np.abs(vegdsm2_b).max()))
        self.vmax = F32(max(float(self.vmax), float(a[sl].max()), float(vegdsm_b.max()), float(vegdsm2_b.max())))
        self.hmax = max(self.hmax, hb)

    def refresh_svf_after_block(self, r0, c0, h, w, patch_option=2) -> dict:
        """Exact SVF update for rasters changed inside the block (r0, c0, h,
        w) by :meth:`update_rasters_block`: the windowed recompute, or a full
        sweep when the edit changed the step tables or brought bush."""
        if getattr(self, "_pending_full", False):
            a, t1, t2 = self.host["dsm"], self.host["trees"], self.host["dem"]
            vegdsm, vegdsm2, bush, amax, _ = march_inputs(a, t1, t2)
            self._set_march_stats(a, vegdsm, vegdsm2, bush)
            if bush.max() > 0:
                self.t["bush"] = _dev(bush, self.device)
            if not self.amax_fixed:
                self.amax = amax
            self._cache = {k: v for k, v in self._cache.items() if k[0] not in ("svf", "svf_host", "corridor")}
            self._pending_full = False
            self.run_svf(patch_option)
            return {"mode": "full", "rect": None, "window": (0, self.rows - 1, 0, self.cols - 1),
                    "pixels": self.rows * self.cols}
        return self._window_update((r0, r0 + h - 1, c0, c0 + w - 1), patch_option)

    def launch_svf(self, planes, bits, patch_option=2):
        """The sweep alone into caller buffers (no host work once the tables
        are cached)."""
        plan_d, steps_d, n_steps, _, ws = self.svf_tables(patch_option)
        site = self.site_struct()
        N.call("sw100_svf_sweep", C.byref(site), self.rows, self.cols, _ptr(plan_d), _ptr(steps_d), n_steps,
               _ptr(planes), _ptr(bits), _ptr(ws), ws.numel(), _stream())

    def count_svf_gathers(self, planes, bits, patch_option=2) -> int:
        """The sweep into caller buffers through the counting kernel: the
        number of source gathers its marches execute (12 bytes each), for
        measurement (sw100_svf_sweep_count)."""
        plan_d, steps_d, n_steps, _, ws = self.svf_tables(patch_option)
        site = self.site_struct()
        cnt = torch.zeros(1, dtype=torch.int64, device=self.device)
        N.call("sw100_svf_sweep_count", C.byref(site), self.rows, self.cols, _ptr(plan_d), _ptr(steps_d), n_steps,
               _ptr(planes), _ptr(bits), _ptr(ws), ws.numel(), _ptr(cnt), _stream())
        return int(cnt.item())

    def run_svf(self, patch_option=2) -> SvfResult:
        d = self.device
        planes = torch.empty((N.SVF_PLANES, self.rows, self.cols), dtype=torch.float32, device=d)
        bits = torch.empty((3, N.CUBE_WORDS, self.rows, self.cols), dtype=torch.int32, device=d)
        self.launch_svf(planes, bits, patch_option)
        self.svf_result = SvfResult(planes, bits, self.svf_tables(patch_option)[3])
        self._prepare_loop_statics()
        return self.svf_result

    def set_svf(self, planes, bits, single_step):
        """Install an SVF result computed earlier (a cached bundle)."""
        self.svf_result = SvfResult(planes, bits, np.asarray(single_step, np.uint32))
        self._prepare_loop_statics()

    def _prepare_loop_statics(self):
        """Per-pixel statics of the time loop derived from the SVF planes:
        svfbuveg (utci_process.py:864), tan(asvf) with asvf = acos(sqrt(svf))
        (utci_process.py:865, solweig.py:550) and tan(svfalfa)
        (utci_process.py:892-897), planes 16-18 of the result (written by
        the sweep's epilogue, or by sw100_svf_statics for planes that came
        from elsewhere)."""
        r = self.svf_result
        self.t["svfbuveg"] = r.plane("svfbuveg")
        self.t["bits"] = r.bits
        self.t["hsvf"] = r.plane("hsvf")
        self.t["tan_alfa"] = r.plane("tan_alfa")

    # ---------------------------------------------------------- time loop
    def build_series(self, met_file, altitude, azimuth, zen, jday, dectime, altmax, location, time_start=0,
                     time_stop=None, initial_scalars=None, day_chain=None):
        ser = TS.build_series(met_file=met_file, altitude=altitude, azimuth=azimuth, zen=zen, jday=jday,
                              dectime=dectime, altmax=altmax, location=location, scale=self.scale,
                              amax=self.amax, rows=self.rows, cols=self.cols, props=self.props,
                              params=self.params, time_start=time_start, time_stop=time_stop,
                              initial_scalars=initial_scalars, day_chain=day_chain)
        if ser.class_idx is not None:
            self.t["class_idx"] = _upload(torch.from_numpy(ser.class_idx), self.device)
        return ser

    def upload_series(self, ser: TS.Series):
        """The five tables of a series in one page-locked buffer and one
        host-to-device copy (each table 256-byte aligned); returns the
        Series record of device pointers and the device buffer."""
        parts = [np.ascontiguousarray(a).view(np.uint8).reshape(-1)
                 for a in (ser.steps, ser.sun, ser.sun_table, ser.patch, ser.gvf)]
        offs, total = [], 0
        for a in parts:
            offs.append(total)
            total += (max(a.size, 16) + 255) // 256 * 256
        host = torch.empty(total, dtype=torch.uint8, pin_memory=True)
        hv = host.numpy()
        for a, o in zip(parts, offs):
            hv[o:o + a.size] = a
        TRANSFER["h2d"] += total
        dev = host.to(self.device, non_blocking=True)
        base = dev.data_ptr()
        s = N.Series()
        s.steps, s.sun, s.sun_table, s.patch, s.gvf = (base + o for o in offs)
        s.n_t, s.n_day, s.n_patches = len(ser.steps), len(ser.sun), ser.patch.shape[1]
        return s, {"tables": dev, "staging": host}

    def run_time_loop(self, ser: TS.Series, requested=("utci",), series_dev=None, workspace=None,
                      tensor_sums=None):
        """All steps of the series: the sun marches, the dense patch sums on
        the tensor cores (sw100_patch_sums; with ``tensor_sums=False`` the
        loop kernel computes them itself) and the time loop; returns
        {name: (n_t, rows, cols) device tensor}."""
        if self.svf_result is None:
            raise RuntimeError("run_svf() (or set_svf()) must come before the time loop")
        names = [k for k in N.OUT_BITS if k in requested]
        mask = 0
        for k in names:
            mask |= N.OUT_BITS[k]
        n_t = len(ser.steps)
        d = self.device
        out = torch.empty((len(names), n_t, self.rows, self.cols), dtype=torch.float32, device=d)
        s, dev = series_dev if series_dev is not None else self.upload_series(ser)
        tensor_sums = TENSOR_SUMS if tensor_sums is None else tensor_sums
        if not tensor_sums:
            ws_bytes = N.workspace_bytes("sw100_time_loop_workspace_bytes", self.rows, self.cols, s.n_day)
            ws = workspace if workspace is not None and workspace.numel() >= ws_bytes else \
                torch.empty(ws_bytes, dtype=torch.uint8, device=d)
            site = self.loop_site_struct()
            N.call("sw100_time_loop", C.byref(site), self.rows, self.cols, C.byref(s), _ptr(self.state), mask,
                   _ptr(out), _ptr(ws), ws.numel(), _stream())
            self._keep = [dev, ws]
            return {k: out[i] for i, k in enumerate(names)}
        gsrc = torch.empty((max(1, s.n_day), self.rows, self.cols, 4), dtype=torch.float32, device=d)
        if s.n_day:
            self.launch_sun_march(s, gsrc)
        sums = self.launch_patch_sums(s)
        self.launch_flux_loop(s, gsrc, mask, out, sums=sums)
        self._keep = [dev, gsrc, sums]
        return {k: out[i] for i, k in enumerate(names)}

    def launch_patch_sums(self, series: N.Series, sums=None):
        """The dense patch sums of every step of the series on the tensor
        cores (sw100_patch_sums) into `sums` ((n_t, 4, rows, cols) float32,
        allocated when None); returns it."""
        if sums is None:
            sums = torch.empty((series.n_t, 4, self.rows, self.cols), dtype=torch.float32, device=self.device)
        ws_bytes = N.workspace_bytes("sw100_patch_sums_workspace_bytes", series.n_t)
        key = "sums_ws"
        if self._cache.get(key) is None or self._cache[key].numel() < ws_bytes:
            self._cache[key] = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
        if getattr(self, "tc_err", None) is None:
            self.tc_err = torch.zeros(1, dtype=torch.int32, device=self.device)
        site = self.site_struct()
        N.call("sw100_patch_sums", C.byref(site), self.rows, self.cols, C.byref(series), _ptr(sums), _ptr(self.tc_err),
               _ptr(self._cache[key]), self._cache[key].numel(), _stream())
        return sums

    def check_tensor_error(self):
        """Raise NativeError when a tensor-core kernel of this site gave up a
        bounded wait (reads the device flag: synchronises)."""
        err = getattr(self, "tc_err", None)
        if err is not None and int(err.item()) != 0:
            code = int(err.item())
            err.zero_()
            raise N.NativeError("sw100_patch_sums", code, "a bounded wait of the tensor-core patch sums expired")

    def run_sun_march(self, ser: TS.Series):
        """Sun-march records and the 8 reference planes per daytime row
        (parity / debugging entry)."""
        s, dev = self.upload_series(ser)
        d = self.device
        n_day = max(1, s.n_day)
        gsrc = torch.empty((n_day, self.rows, self.cols, 4), dtype=torch.float32, device=d)
        dbg = torch.empty((n_day, 8, self.rows, self.cols), dtype=torch.float32, device=d)
        self.launch_sun_march(s, gsrc, dbg)
        self._keep = [dev]
        return gsrc[:s.n_day], dbg[:s.n_day]

    def launch_sun_march(self, series: N.Series, gsrc, debug8=None):
        key = "sun_ws"
        ws_bytes = N.workspace_bytes("sw100_sun_march_workspace_bytes", self.rows, self.cols)
        if key not in self._cache:
            self._cache[key] = torch.empty(ws_bytes, dtype=torch.uint8, device=self.device)
        ws = self._cache[key]
        site = self.site_struct()
        N.call("sw100_sun_march", C.byref(site), self.rows, self.cols, C.byref(series), _ptr(gsrc), _ptr(debug8),
               _ptr(ws), ws_bytes, _stream())

    def launch_flux_loop(self, series: N.Series, gsrc, out_mask, outputs, sums=None):
        """The loop kernel over sun-march records `gsrc`; with `sums` (from
        launch_patch_sums) it reads the dense patch sums instead of
        computing them."""
        site = self.loop_site_struct()
        if sums is None:
            N.call("sw100_flux_loop", C.byref(site), self.rows, self.cols, C.byref(series), _ptr(gsrc),
                   _ptr(self.state), out_mask, _ptr(outputs), _stream())
        else:
            N.call("sw100_flux_loop_sums", C.byref(site), self.rows, self.cols, C.byref(series), _ptr(gsrc),
                   _ptr(sums), _ptr(self.state), out_mask, _ptr(outputs), _stream())

    def copy_stream(self) -> torch.cuda.Stream:
        """Stream of the chunked loop's device-to-host output copies (one per
        device, shared by all sites)."""
        return _shared_stream(self.device, "copy")

    def side_stream(self) -> torch.cuda.Stream:
        """Second stream: sun marches, which read only the rasters, run there
        beside the SVF sweep and the flux loops (one per device, shared by
        all sites)."""
        return _shared_stream(self.device, "side")

    def run_chain_chunked(self, met_file, altitude, azimuth, zen, jday, dectime, altmax, location,
                          requested=("utci",), time_start=0, time_stop=None, initial_scalars=None,
                          chunk_steps=DEFAULT_CHUNKS, rasters_ready=None, timeline=None, tables=None):
        """The time loop of steps [time_start, time_stop) with the host tables
        built chunk by chunk while the GPU works: the tables of a chunk
        (`chunk_steps`: one length, or a sequence of lengths, chunk_bounds)
        are built, its sun march and flux loop launched and its
        outputs copied asynchronously into page-locked host arrays; then the
        next chunk's tables are built while those run.  The thermal state
        (device planes) and the carried scalars (CI, timeadd, firstdaytime)
        pass from chunk to chunk exactly as between the reference's
        consecutive windows, so the result equals one launch over all steps
        bit for bit.  Each chunk's tables go up and its sun march runs on the
        side stream, after `rasters_ready` (an event recorded on the current
        stream once the rasters were last written; None: everything queued
        before this call), so it overlaps the SVF sweep and the previous
        chunk's flux loop; the flux loop waits for it on the current stream.
        `timeline` (a Timeline, optional) records the host phases.
        Device memory stays bounded whatever the number of steps: at most
        `CHUNKS_IN_FLIGHT` chunks keep their device buffers (outputs, sun-march
        records, tables); before an older chunk's buffers are released, the
        host waits for the event recorded after that chunk's copies.
        Returns ({name: (T, rows, cols) float32 ndarray}, final carried
        scalars)."""
        if self.svf_result is None:
            raise RuntimeError("run_svf() (or set_svf()) must come before the time loop")
        if time_stop is None:
            time_stop = met_file.shape[0]
        bounds = chunk_bounds(time_start, time_stop, chunk_steps)
        names = [k for k in N.OUT_BITS if k in requested]
        mask = 0
        for k in names:
            mask |= N.OUT_BITS[k]
        n_t = time_stop - time_start
        host = {k: torch.empty((n_t, self.rows, self.cols), dtype=torch.float32, pin_memory=True) for k in names}
        ring = collections.deque()
        main, side, copy = torch.cuda.current_stream(), self.side_stream(), self.copy_stream()
        if rasters_ready is None:
            rasters_ready = torch.cuda.Event()
            rasters_ready.record(main)
        side.wait_event(rasters_ready)
        tl = timeline if timeline is not None else Timeline(enabled=False)
        # the loops' patch order, queued behind the work already on this
        # stream (the SVF sweep) before the host builds the first tables
        self.loop_site_struct()
        if tables is None:
            tables = self.start_tables(met_file, altitude, azimuth, zen, jday, dectime, altmax, location,
                                       time_start, time_stop, chunk_steps, initial_scalars)
        elif tables.span != (time_start, time_stop, tuple(bounds)):
            tables.finish()
            raise ValueError(f"tables were started for steps / chunks {tables.span}, "
                             f"not {(time_start, time_stop, tuple(bounds))}")
        try:
            return self._chunks(tables, names, mask, host, ring, main, side, copy, tl, time_start, bounds)
        finally:
            tables.finish()

    def start_tables(self, met_file, altitude, azimuth, zen, jday, dectime, altmax, location, time_start=0,
                     time_stop=None, chunk_steps=DEFAULT_CHUNKS, initial_scalars=None):
        """The host tables of run_chain_chunked's chunks, in order, each built
        when it is read (ChunkTables)."""
        if time_stop is None:
            time_stop = met_file.shape[0]
        kw = dict(met_file=met_file, altitude=altitude, azimuth=azimuth, zen=zen, jday=jday, dectime=dectime,
                  altmax=altmax, location=location, scale=self.scale, amax=self.amax, rows=self.rows,
                  cols=self.cols, props=self.props, params=self.params)
        return ChunkTables(kw, time_start, time_stop, chunk_steps, initial_scalars)

    def _chunks(self, tables, names, mask, host, ring, main, side, copy, tl, time_start, bounds):
        scalars = None
        for t0, t1 in bounds:
            ser = tables.next()
            if ser.class_idx is not None:
                # the device planes of this site index the tables by the
                # cleaned land-cover code (device_props); a per-pixel class
                # plane from the host would have to be uploaded on the side
                # stream, which this loop does not do
                raise RuntimeError("the chunked time loop expects device-side land-cover classes")
            scalars = ser.final
            tl.mark(f"tables {t0}-{t1}")
            with torch.cuda.stream(side):
                s, dev = self.upload_series(ser)
                gsrc = torch.empty((max(1, s.n_day), self.rows, self.cols, 4), dtype=torch.float32,
                                   device=self.device)
                if s.n_day:
                    self.launch_sun_march(s, gsrc)
                marched = torch.cuda.Event()
                marched.record(side)
            main.wait_event(marched)
            out = torch.empty((len(names), t1 - t0, self.rows, self.cols), dtype=torch.float32, device=self.device)
            sums = self.launch_patch_sums(s) if TENSOR_SUMS else None
            self.launch_flux_loop(s, gsrc, mask, out, sums=sums)
            # outputs go back on a copy stream, overlapping the next chunk
            fluxed = torch.cuda.Event()
            fluxed.record(main)
            copy.wait_event(fluxed)
            with torch.cuda.stream(copy):
                for i, k in enumerate(names):
                    host[k][t0 - time_start:t1 - time_start].copy_(out[i], non_blocking=True)
                    TRANSFER["d2h"] += out[i].numel() * out[i].element_size()
            # the side-stream allocations are read on the current stream and
            # `out` on the copy stream: a chunk's buffers are released only
            # once the event recorded after its copies has completed
            done = torch.cuda.Event()
            done.record(copy)
            ring.append((done, out, dev, gsrc, sums))
            tl.mark(f"launch {t0}-{t1}", main)
            if len(ring) > CHUNKS_IN_FLIGHT:
                old = ring.popleft()
                old[0].synchronize()
                del old
        main.synchronize()
        copy.synchronize()
        tl.mark("wait for the GPU")
        ring.clear()
        self.check_tensor_error()
        return {k: v.numpy() for k, v in host.items()}, scalars

    def load_state(self, state: dict):
        for k, name in enumerate(STATE_NAMES):
            v = state[name]
            if not isinstance(v, torch.Tensor):
                v = torch.as_tensor(np.asarray(v, F32))
            self.state[k].copy_(v.to(dtype=torch.float32))

    def state_dict(self):
        return {name: self.state[k].clone() for k, name in enumerate(STATE_NAMES)}


def chunk_bounds(time_start, time_stop, chunk_steps):
    """The chunks [(t0, t1), ...] of steps [time_start, time_stop):
    `chunk_steps` is one length for every chunk, or a sequence of lengths
    taken in order (the last one repeated while steps remain)."""
    lengths = [chunk_steps] if isinstance(chunk_steps, (int, np.integer)) else list(chunk_steps)
    if not lengths or any(int(n) < 1 for n in lengths):
        raise ValueError("chunk_steps must be >= 1 (or a sequence of lengths >= 1)")
    out, t0, k = [], time_start, 0
    while t0 < time_stop:
        t1 = min(time_stop, t0 + int(lengths[min(k, len(lengths) - 1)]))
        out.append((t0, t1))
        t0, k = t1, k + 1
    return out


class ChunkTables:
    """The host tables (timeseries.build_series) of steps [time_start,
    time_stop) in chunks of `chunk_steps`, built in order as next() is
    called, the carried scalars passed from chunk to chunk and the daytime
    scalar chain evaluated once for the whole range."""

    def __init__(self, kw, time_start, time_stop, chunk_steps, initial_scalars=None):
        self.bounds = chunk_bounds(time_start, time_stop, chunk_steps)
        self.span = (time_start, time_stop, tuple(self.bounds))
        self._kw, self._scalars, self._dc = kw, initial_scalars, None
        self._left = list(self.bounds)

    def next(self):
        if not self._left:
            raise StopIteration
        kw = self._kw
        if self._dc is None:
            self._dc = TS.day_chain(kw["met_file"], kw["altitude"], kw["azimuth"], kw["zen"], kw["jday"],
                                    kw["location"], self.span[0], self.span[1])
        t0, t1 = self._left.pop(0)
        ser = TS.build_series(**kw, time_start=t0, time_stop=t1, initial_scalars=self._scalars, day_chain=self._dc)
        self._scalars = ser.final
        return ser

    def finish(self):
        self._left = []


def utci(ta, rh, tmrt, va) -> torch.Tensor:
    """utci_calculator on device tensors (calculate_utci.py:259-330)."""
    require_cuda()
    ta, rh, tmrt, va = (torch.as_tensor(x, dtype=torch.float32, device="cuda").contiguous() for x in (ta, rh, tmrt, va))
    out = torch.empty_like(ta)
    N.call("sw100_utci", _ptr(ta), _ptr(rh), _ptr(tmrt), _ptr(va), ta.numel(), _ptr(out), _stream())
    return out
