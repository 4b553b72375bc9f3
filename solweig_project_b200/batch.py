"""Many sites in one launch per stage, replayed as a CUDA graph.

The reference runs the chain one site (tile) at a time
(``solweig_gpu/solweig_gpu.py:387-497`` run_utci_tiles ->
``utci_process.py:1472-1651`` compute_utci, each tile a separate
svf_calculator + run_utci_window).  :class:`SiteBatch` keeps every site of a
batch resident in HBM and drives the whole batch with one launch per stage
(pack, [bush flags], SVF sweep, sun march, flux loop) through the
``sw100_batch_*`` entry points: a device array of per-site descriptors and a
device tile list per stage, heaviest sites first.  :meth:`SiteBatch.capture`
records the stage launches in a CUDA graph that :meth:`SiteBatch.replay`
re-issues with one call.

Launch shapes come from :class:`Autotuner`: per stage, it times the block
shapes of 128 threads (8 x 16, 32 x 4, 16 x 8, 4 x 32, 64 x 2, 128 x 1) with one tile per
block or a persistent grid striding over the tile list, and stores the
fastest per grid-size bucket (the batch's pixel-weighted median side) in a
JSON file.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from . import engine as E
from . import timeseries as TS

STAGES = ("pack", "bush", "svf", "sun", "flux")
SHAPES = ((8, 16), (32, 4), (16, 8), (4, 32), (64, 2), (128, 1))
SM_COUNT = 148
# the march and loop stages default to 8 x 16 tiles: a warp covers 8 x 4
# pixels, whose rays and ground-view walks meet similar obstacles (less
# divergence than 32 x 1 rows)
DEFAULT_SHAPE = {"pack": ((32, 4), "tiles"), "bush": ((32, 4), "tiles"), "svf": ((8, 16), "tiles"),
                 "sun": ((8, 16), "tiles"), "flux": ((8, 16), "tiles")}
ENTRY = {"pack": "sw100_batch_pack", "bush": "sw100_batch_bush_flags", "svf": "sw100_batch_svf",
         "sun": "sw100_batch_sun_march", "flux": "sw100_batch_flux_loop"}


class BatchSite(C.Structure):
    """ctypes mirror of sw100_batch_site."""
    _fields_ = [
        ("site", N.SitePlanes), ("rows", C.c_int32), ("cols", C.c_int32), ("plan", C.c_void_p),
        ("steps", C.c_void_p), ("series", N.Series), ("svf_planes", C.c_void_p), ("svf_bits", C.c_void_p),
        ("src4", C.c_void_p), ("bflags", C.c_void_p), ("gsrc", C.c_void_p), ("state", C.c_void_p),
        ("outputs", C.c_void_p), ("out_mask", C.c_uint32), ("svf_steps", C.c_int32), ("skipmap", C.c_void_p),
        ("sums", C.c_void_p),
    ]


TILE_DTYPE = np.dtype([("site", "<i4"), ("tx", "<i4"), ("ty", "<i4"), ("day", "<i4")])


def build_tiles(dims, shape, order) -> np.ndarray:
    """Tile list of the sites ``order`` (indices into ``dims``, in launch
    order): dims[i] = (rows, cols, n_rows_per_pixel), where the last is the
    number of daytime rows for the sun march and 1 otherwise.  Every pixel of
    every listed site is covered once per row."""
    bx, by = shape
    parts = []
    for i in order:
        rows, cols, n_day = dims[i]
        nx, ny = -(-cols // bx), -(-rows // by)
        ty, tx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        for d in range(n_day):
            t = np.zeros(nx * ny, TILE_DTYPE)
            t["site"], t["tx"], t["ty"], t["day"] = i, tx.reshape(-1), ty.reshape(-1), d
            parts.append(t)
    return np.concatenate(parts) if parts else np.zeros(0, TILE_DTYPE)


def partition_sites(costs, n_ranks: int):
    """Longest-processing-time split of sites over ranks: sites in
    decreasing cost, each to the rank with the least work so far (ties to
    the lower rank).  Returns one list of site indices per rank, each in
    increasing index order.  Sites are independent, so no data crosses
    ranks."""
    if n_ranks <= 0:
        raise ValueError("n_ranks must be positive")
    load = [0.0] * n_ranks
    parts = [[] for _ in range(n_ranks)]
    for i in sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k)):
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def size_bucket(sides) -> str:
    """Grid-size bucket of a batch: its pixel-weighted median side."""
    sides = np.sort(np.asarray(sides, np.int64))
    w = np.cumsum(sides.astype(np.float64) ** 2)
    med = int(sides[np.searchsorted(w, w[-1] / 2)])
    for lim in (192, 384, 768, 1536):
        if med <= lim:
            return f"side<={lim}"
    return "side>1536"


@dataclass
class _Member:
    site: E.DeviceSite
    series: TS.Series
    series_struct: N.Series
    series_dev: dict
    names: list
    planes: torch.Tensor
    bits: torch.Tensor
    src4: torch.Tensor
    bflags: torch.Tensor
    gsrc: torch.Tensor
    outputs: torch.Tensor
    n_steps: int
    skipmap: torch.Tensor
    sums: "torch.Tensor | None" = None


class SiteBatch:
    """A batch of sites resident on one GPU.

    ``sites`` are :class:`~solweig_project_b200.engine.DeviceSite` objects
    (rasters uploaded), ``series`` their time series
    (:meth:`DeviceSite.build_series`).  ``requested`` selects the outputs
    (same names and order as :meth:`DeviceSite.run_time_loop`)."""

    def __init__(self, sites, series, requested=("utci", "tmrt"), tuner: "Autotuner | None" = None):
        if len(sites) != len(series) or not sites:
            raise ValueError("one time series per site, at least one site")
        E.require_cuda()
        self.device = sites[0].device
        self.names = [k for k in N.OUT_BITS if k in requested]
        mask = 0
        for k in self.names:
            mask |= N.OUT_BITS[k]
        self.members = []
        for site, ser in zip(sites, series):
            plan_d, steps_d, n_steps, single, _ = site.svf_tables()
            d = self.device
            rows, cols = site.rows, site.cols
            npix = rows * cols
            planes = torch.empty((N.SVF_PLANES, rows, cols), dtype=torch.float32, device=d)
            bits = torch.zeros((3, N.CUBE_WORDS, rows, cols), dtype=torch.int32, device=d)
            site.set_svf(planes, bits, single)           # statics point into planes / bits
            s_struct, s_dev = site.upload_series(ser)
            n_day = max(1, s_struct.n_day)
            self.members.append(_Member(
                site=site, series=ser, series_struct=s_struct, series_dev=s_dev, names=self.names,
                planes=planes, bits=bits, src4=torch.empty((npix, 4), dtype=torch.float32, device=d),
                bflags=torch.zeros(max(1, n_steps), dtype=torch.int32, device=d),
                gsrc=torch.empty((n_day, npix, 4), dtype=torch.float32, device=d),
                outputs=torch.empty((len(self.names), s_struct.n_t, rows, cols), dtype=torch.float32, device=d),
                n_steps=n_steps,
                skipmap=torch.empty(-(-rows // 8) * -(-cols // 8), dtype=torch.float32, device=d)))
            site._plan_steps = (plan_d, steps_d)
        self.mask = mask
        # the dense patch sums of each site on the tensor cores, then the
        # flux loop that reads them (as the single-site chain runs)
        self.tensor_sums = E.TENSOR_SUMS
        for m in self.members:
            m.sums = (torch.empty((m.series_struct.n_t, 4, m.site.rows, m.site.cols), dtype=torch.float32,
                                  device=self.device) if self.tensor_sums else None)
        host = (BatchSite * len(self.members))()
        for i, m in enumerate(self.members):
            b = host[i]
            b.site = m.site.site_struct()
            b.rows, b.cols = m.site.rows, m.site.cols
            b.plan, b.steps = m.site._plan_steps[0].data_ptr(), m.site._plan_steps[1].data_ptr()
            b.series = m.series_struct
            b.svf_planes, b.svf_bits = m.planes.data_ptr(), m.bits.data_ptr()
            b.src4, b.bflags, b.gsrc = m.src4.data_ptr(), m.bflags.data_ptr(), m.gsrc.data_ptr()
            b.state, b.outputs, b.out_mask = m.site.state.data_ptr(), m.outputs.data_ptr(), mask
            b.svf_steps = m.n_steps
            b.skipmap = m.skipmap.data_ptr()
            b.sums = m.sums.data_ptr() if m.sums is not None else 0
        N.call("sw100_batch_validate", C.cast(host, C.c_void_p), len(self.members))
        raw = np.frombuffer(bytes(host), np.uint8).copy()
        self.sites_dev = torch.from_numpy(raw).to(self.device)
        self._host_sites = host
        self.bucket = size_bucket([max(m.site.rows, m.site.cols) for m in self.members])
        self.tuner = tuner or Autotuner()
        self.shapes = {st: self.tuner.lookup(st, self.bucket) for st in STAGES}
        self._tiles = {}
        self.graph = None

    # ------------------------------------------------------------ tiles
    def _site_order(self, stage):
        """Sites heaviest first: SVF steps x pixels for the sweep, daytime
        rows x pixels for the sun march, pixels x steps for the flux loop."""
        def cost(m):
            npix = m.site.rows * m.site.cols
            if stage == "svf" or stage == "bush":
                return npix * m.n_steps
            if stage == "sun":
                return npix * m.series_struct.n_day
            return npix * m.series_struct.n_t
        return sorted(range(len(self.members)), key=lambda i: -cost(self.members[i]))

    def tiles(self, stage, shape):
        key = (stage, shape)
        if key not in self._tiles:
            order = [i for i in self._site_order(stage) if stage != "bush" or self.members[i].site.bush_any]
            dims = [(m.site.rows, m.site.cols, m.series_struct.n_day if stage == "sun" else 1) for m in self.members]
            arr = build_tiles(dims, shape, order)
            dev = torch.from_numpy(arr.view(np.uint8).copy()).to(self.device) if arr.size else None
            self._tiles[key] = (dev, int(arr.size))
        return self._tiles[key]

    # ---------------------------------------------------------- launches
    def launch(self, stage, shape=None, mode=None):
        (bx, by), m = self.shapes[stage]
        if shape is not None:
            bx, by = shape
            m = mode
        dev, n = self.tiles(stage, (bx, by))
        if n == 0:
            return
        grid = n if m == "tiles" else min(n, SM_COUNT * 8)
        entry = "sw100_batch_flux_loop_sums" if stage == "flux" and self.tensor_sums else ENTRY[stage]
        N.call(entry, C.c_void_p(self.sites_dev.data_ptr()), C.c_void_p(dev.data_ptr()), n, bx, by, grid,
               E._stream())

    def run(self, reset_state=True):
        """Every stage of every site: pack, bush flags, sweep, sun march, flux
        loop (with the thermal state zeroed first unless told otherwise)."""
        for m in self.members:
            if m.site.bush_any:
                m.bflags.zero_()
            if reset_state:
                m.site.state.zero_()
        for st in STAGES:
            if st == "flux" and self.tensor_sums:
                for m in self.members:   # after the sweep: the sums read its bit cubes
                    m.site.launch_patch_sums(m.series_struct, m.sums)
            self.launch(st)
            if st == "pack":
                N.call("sw100_batch_skipmap", C.c_void_p(self.sites_dev.data_ptr()), len(self.members),
                       E._stream())

    def capture(self):
        """Record :meth:`run` in a CUDA graph (tile lists and descriptors are
        built first, outside the capture)."""
        for st in STAGES:
            self.tiles(st, self.shapes[st][0])
        self.run()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def replay(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def check_tensor_errors(self):
        """Raise if a bounded wait of a site's patch-sum product ran out
        (reads each site's error flag: synchronises)."""
        if self.tensor_sums:
            for m in self.members:
                m.site.check_tensor_error()

    def outputs(self, i):
        """{name: (n_t, rows, cols) device tensor} of site i."""
        m = self.members[i]
        return {k: m.outputs[j] for j, k in enumerate(self.names)}

    def svf(self, i):
        m = self.members[i]
        return m.planes, m.bits

    @property
    def pixels(self):
        return sum(m.site.rows * m.site.cols for m in self.members)


class Autotuner:
    """Launch shape per (stage, grid-size bucket), timed on the device and
    kept in a JSON file (``SOLWEIG_B200_TUNE`` or
    ``~/.cache/solweig_project_b200/tune.json``)."""

    def __init__(self, path: str | None = None):
        self.path = path or os.environ.get("SOLWEIG_B200_TUNE") or os.path.join(
            os.path.expanduser("~"), ".cache", "solweig_project_b200", "tune.json")
        self.table = {}
        try:
            with open(self.path) as fh:
                self.table = json.load(fh)
        except (OSError, ValueError):
            self.table = {}

    def lookup(self, stage, bucket):
        hit = self.table.get(f"{stage}|{bucket}")
        if hit is None:
            return DEFAULT_SHAPE[stage]
        return tuple(hit["shape"]), hit["mode"]

    def tune(self, batch: SiteBatch, reps: int = 2) -> dict:
        """Time every candidate of every stage on this batch and store the
        fastest; returns {stage: (shape, mode, ms)}."""
        batch.run()
        torch.cuda.synchronize()
        chosen = {}
        for st in STAGES:
            if batch.tiles(st, SHAPES[0])[1] == 0:
                continue
            best = None
            for shape in SHAPES:
                for mode in ("tiles", "persistent"):
                    ts = []
                    for _ in range(reps + 1):
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record()
                        batch.launch(st, shape, mode)
                        e1.record()
                        torch.cuda.synchronize()
                        ts.append(e0.elapsed_time(e1))
                    ms = min(ts[1:])
                    if best is None or ms < best[2]:
                        best = (shape, mode, ms)
            chosen[st] = best
            self.table[f"{st}|{batch.bucket}"] = {"shape": list(best[0]), "mode": best[1], "ms": best[2]}
            batch.shapes[st] = (best[0], best[1])
        batch.graph = None
        self.save()
        return chosen

    def save(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            with open(self.path, "w") as fh:
                json.dump(self.table, fh, indent=1, sort_keys=True)
        except OSError:
            pass
