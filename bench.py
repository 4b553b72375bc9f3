"""Throughput of the exact SOLWEIG chain (SVF sweep + sun march + fluxes +
Tmrt + UTCI) on B200, in pixel x timesteps per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload exact500|tile4096]

One step = one pass of the whole chain over one site: the 153-patch SVF sweep
and the 24 hourly steps of the time loop (sun march of the daytime steps,
ground view factors, K/L fluxes, Tmrt, UTCI).  Inputs are the seeded
synthetic city of the workload (500 x 500 px at 1 m by default).

* ``value``: device throughput with the rasters and tables resident in HBM
  (CUDA events on the launching stream, L2 flushed before every timed step).
* ``e2e``: the same metric through the public entry point
  (:func:`solweig_project_b200.api.run_exact_chain` from host rasters in
  pinned memory), host->device inputs and device->host UTCI/Tmrt included.
* With torchrun (N > 1) every rank runs its own site (weak scaling, no
  collective on the data path); the time is the max over ranks.
* ``--impl reference`` times the CPU oracle (the reference's algorithm
  restated on the host cores) over the whole workload: one full pass whose
  K timed steps are its K pieces.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

METRIC = "px*steps/s shadow->Tmrt->UTCI (exact chain incl. SVF sweep)"
UNIT = "px*steps/s"
N_STEPS_DAY = 24
WORKLOADS = {
    # name: (side, h_max, description)
    "exact500": (500, 40.0, "500x500 px @1 m, 24 hourly steps, SVF sweep + shadows + fluxes + Tmrt + UTCI"),
    "tile4096": (4096, 120.0, "4096x4096 px @1 m, buildings up to 120 m, 24 hourly steps, full exact chain"),
    "preview1024": (1024, 40.0, "learned SVF preview of seeded building edits (add / remove / height change, "
                                "10-40 px boxes) on a held-out 1024x1024 city vs the exact windowed recompute and "
                                "the full sweep; Tmrt of the 24-step chain over the edit window"),
    "batched64": (None, 40.0, "64 seeded sites, sides log-uniform 128-1024 px, density 10-45 %, canopy 0-30 %, "
                              "latitudes 0-60 N, 24 hourly steps each; one launch per stage for all sites, "
                              "replayed as a CUDA graph, autotuned launch shapes"),
}
FLUX_BYTES_PER_PX_STEP = 190      # compulsory HBM bytes per pixel and step of the flux stage
SVF_GATHER_BYTES_PER_STEP = 12    # 3 float32 gathers per march step
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# each kernel, from ncu captures: the flux loop at 500 x 500 x 24 (the default
# workload), the SVF sweep and sun march at 1024 x 1024 scaled to a launch of
# the measured size by pixel count (their traffic is per pixel).
NCU_TRAFFIC = {"flux_loop": (500 * 500, 349_762_816), "svf_sweep": (1024 * 1024, 281_261_824),
               "sun_march": (1024 * 1024, 340_633_088)}
# issue-slot utilisation (smsp__issue_active) of the same captures: the
# binding roofline of these integer / FP32 kernels is instruction issue
NCU_ISSUE_ACTIVE = {"flux_loop": 0.516, "svf_sweep": 0.726, "sun_march": 0.791, "patch_sums_tc": 0.386}
# active lanes per issued warp instruction (of 32) in the same captures
NCU_ACTIVE_LANES = {"flux_loop": 25.05, "svf_sweep": 24.27, "sun_march": 26.50, "patch_sums_tc": 30.67}
# tensor-pipe activity (sm__pipe_tensor_cycles_active) of the patch-sum product at 500 x 500 x 24
NCU_TENSOR_ACTIVE = {"patch_sums_tc": 0.142}
# end-to-end calls timed after 2 warm-up calls; the median is reported (the
# call is host-bound at small sizes, so one slow call from other host load
# should not move the figure)
E2E_TIMED = 7
# reference pins of the 500 x 500 city (seed 1234): Tmrt / UTCI of the
# unmodified reference and of an FP64 re-evaluation at seeded sample pixels
PINS = {"exact500": os.path.join(REPO, "tests", "golden", "large_c2_500.npz")}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="exact500")
    ap.add_argument("--side", type=int, default=None, help="override the workload's square side (px)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--edits", type=int, default=None,
                    help="preview1024: seeded edits in all (default 20 x steps)")
    ap.add_argument("--sites", type=int, default=1, help="preview1024: held-out 1024 x 1024 cities the edits share")
    ap.add_argument("--timeline", action="store_true",
                    help="print the host timeline of one end-to-end call (after the bench line)")
    return ap.parse_args()


def make_workload(name, rank, side=None):
    from solweig_project_b200 import synthetic
    if name == "batched64":   # the first site of the batch (reference arm sample)
        sp = synthetic.multi_site_specs()[0]
        city = synthetic.make_city(side or sp["side"], side or sp["side"], seed=sp["seed"], density=sp["density"],
                                   canopy_cover=sp["canopy"])
        return city, synthetic.make_met(sp["seed"]), synthetic.load_sun_geometry("multi0"), \
            synthetic.default_lc_class()
    side0, hmax, _ = WORKLOADS[name]
    side = side or side0
    city = synthetic.make_city(side, side, seed=1234 + rank, h_max=hmax)
    met = synthetic.make_met(1234)
    geo = synthetic.load_sun_geometry("single")
    return city, met, geo, synthetic.default_lc_class()


class ClockSampler:
    """SM clock and throttle-reason samples during the timed region: an NVML
    polling thread (every ~2 ms, the first sample taken before the region
    starts), nvidia-smi as the fallback when NVML is unavailable."""

    FIELDS = ("clocks.sm", "clocks.max.sm", "clocks_event_reasons.active", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index):
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None
        self.gpu = gpu_index
        self.rows = []
        self.thread = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.gpu)
        bus = getattr(props, "pci_bus_id", None)
        if bus is not None:
            dom, dev = getattr(props, "pci_domain_id", 0), getattr(props, "pci_device_id", 0)
            try:
                return pynvml.nvmlDeviceGetHandleByPciBusId(f"{dom:08x}:{bus:02x}:{dev:02x}.0")
            except pynvml.NVMLError:
                pass
        uuid = str(getattr(props, "uuid", ""))
        if uuid:
            try:
                return pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except pynvml.NVMLError:
                pass
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v for v in vis.split(",") if v.strip()]
        idx = int(ids[self.gpu]) if ids and ids[self.gpu].strip().isdigit() else self.gpu
        return pynvml.nvmlDeviceGetHandleByIndex(idx)

    def _poll(self, handle, ready):
        import pynvml
        bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
        mx = pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM)
        while True:
            sm = pynvml.nvmlDeviceGetClockInfo(handle, pynvml.NVML_CLOCK_SM)
            r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
            self.rows.append((float(sm), float(mx), {k for k, b in bits.items() if r & b}))
            ready.set()
            if self.stop.wait(0.002):
                return

    def __enter__(self):
        import threading
        try:
            handle = self._nvml_handle()
            self.stop, ready = threading.Event(), threading.Event()
            self.thread = threading.Thread(target=self._poll, args=(handle, ready), daemon=True)
            self.thread.start()
            ready.wait(2.0)
            return self
        except Exception:  # noqa: BLE001 - any NVML trouble: fall back to nvidia-smi
            self.thread = None
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + ",".join(self.FIELDS),
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.thread is not None:
            sm = [r[0] for r in self.rows]
            mx = [r[1] for r in self.rows]
            reasons = sorted(set().union(*[r[2] for r in self.rows])) if self.rows else []
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                    "reasons": reasons, "samples": len(sm), "source": "nvml"}
        try:
            rows = [[c.strip() for c in line.split(",")] for line in open(self.path) if line.strip()]
        except OSError:
            rows = []
        sm = [float(r[0]) for r in rows if r and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if len(r) > 1 and r[1].replace(".", "").isdigit()]
        reasons = sorted({self.REASONS[i] for r in rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm), "source": "nvidia-smi"}


def _err(got, want):
    d = np.asarray(got, np.float64) - np.asarray(want, np.float64)
    d = d[~np.isnan(d)]
    return {"max": float(np.abs(d).max()), "rms": float(np.sqrt(np.mean(d * d)))}


def error_vs_fp64(pin_path, tmrt, utci):
    """Tmrt / UTCI of the timed step against the reference pins of the same
    city (tests/golden/make_golden_large.py): the unmodified reference's
    float32 values and an FP64 re-evaluation of the same chain (same shadow
    geometry), at 4096 ground + 256 building sample pixels of every step."""
    with np.load(pin_path) as z:
        d = {k: z[k] for k in z.files}
    T, s = d["sample_tmrt"].shape[0], d["samples"]
    tm, ut = tmrt.reshape(T, -1)[:, s], utci.reshape(T, -1)[:, s]
    tm64 = d["sample_tmrt"].astype(np.float64) + d["sample_tmrt64_delta"]
    ut64 = d["sample_utci"].astype(np.float64) + d["sample_utci64_delta"]
    return {"samples": f"{s.size} px x {T} steps", "tmrt_K": _err(tm, tm64), "utci_C": _err(ut, ut64),
            "reference_tmrt_K": _err(d["sample_tmrt"], tm64), "reference_utci_C": _err(d["sample_utci"], ut64),
            "vs_reference_tmrt_K": _err(tm, d["sample_tmrt"]), "vs_reference_utci_C": _err(ut, d["sample_utci"]),
            "reference_all_px_tmrt_K": {"max": float(d["ref_fp64_tmrt_max"]), "rms": float(d["ref_fp64_tmrt_rms"])},
            "reference_all_px_utci_C": {"max": float(d["ref_fp64_utci_max"]), "rms": float(d["ref_fp64_utci_rms"])}}


# the CPU baseline of the default run: a crop of the workload small enough
# for 10-30 s of host work next to the GPU bench
CPU_BASELINE_CROP = 200


def oracle_pass(city, met, geo, lc_class, n_pieces, march_map):
    """One pass of the CPU oracle over a whole site -- the 153-patch SVF
    sweep, then the 24-step window -- cut into `n_pieces` pieces timed one
    after another; returns the piece times (s), which add up to the pass,
    and the window's outputs.
    The sweep is one piece (its patch marches through `march_map`, the sums
    in patch order) and the window's steps are split over the other pieces
    (one generator, so the window is set up once, as in a single call);
    beyond 1 + 24 pieces the sweep is split into patch groups too.  With one
    piece the whole pass is one."""
    from oracle import svf as osvf, window as ow
    from solweig_project_b200.synthetic import DEFAULT_LOCATION
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(city.dsm, city.trees, city.dem)
    tasks = osvf.patch_tasks(2)
    n_t = met.shape[0]
    n_svf = min(len(tasks), max(1, n_pieces - n_t))
    n_win = max(0, n_pieces - n_svf)
    acc = osvf.SvfAccumulator(2, *city.dsm.shape, vegdsm2)
    window = {}

    def svf_part(group):
        def run():
            for t, res in march_map([tasks[j] for j in group]):
                acc.add(t, *res)
        return run

    def window_part(n, last):
        def run():
            if "steps" not in window:
                window["steps"] = ow.iter_utci_window(
                    a=city.dsm, temp1=city.trees, temp2=city.dem, walls=city.walls, dirwalls=city.aspect,
                    svf_bundle=acc.result(), met_file=met, location=dict(DEFAULT_LOCATION), scale=city.scale,
                    landcover_grid=city.landcover, lc_class=lc_class, requested_variables=("utci", "tmrt"), **geo)
            for _ in range(n):
                next(window["steps"])
            if last:
                try:
                    next(window["steps"])
                except StopIteration as done:
                    window["out"] = done.value
        return run

    svf_runs = [svf_part(g) for g in np.array_split(np.arange(len(tasks)), n_svf)]
    chunks = np.array_split(np.arange(n_t), max(1, n_win))
    win_runs = [window_part(len(c), k == len(chunks) - 1) for k, c in enumerate(chunks)]
    pieces = [[r] for r in svf_runs + win_runs] if n_win else [svf_runs + win_runs]
    times = []
    for piece in pieces:
        t0 = time.perf_counter()
        for run in piece:
            run()
        times.append(time.perf_counter() - t0)
    if "out" not in window:
        raise RuntimeError("the oracle window did not finish")
    return times, window["out"]


def _crop(city, n):
    import dataclasses
    sl = (slice(0, n), slice(0, n))
    return dataclasses.replace(city, **{k: getattr(city, k)[sl] for k in
                                        ("dsm", "trees", "dem", "walls", "aspect", "landcover")})


def _march_map(city, processes):
    """(march_map, close) for oracle_pass: the patch marches of this city
    in a spawn pool of `processes` workers, or in this process."""
    from oracle import svf as osvf
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(city.dsm, city.trees, city.dem)
    if processes <= 1:
        def serial(tasks):
            for t in tasks:
                yield t, osvf.shadow_patch(amax, city.dsm, vegdsm, vegdsm2, bush, t[2], t[3], city.scale)
        return serial, lambda: None
    pool, one = osvf.march_pool(processes, amax, city.dsm, vegdsm, vegdsm2, bush, city.scale)

    def close():
        pool.close()
        pool.join()
    return (lambda tasks: pool.imap(one, tasks)), close


def cpu_baseline(city, met, geo, lc_class, crop=CPU_BASELINE_CROP):
    """The CPU oracle on a crop x crop px corner of the workload, all 24
    steps, SVF sweep included: the patch marches on every host core (spawn
    pool), the window in this process with all cores as torch threads."""
    import torch
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    sub = _crop(city, crop)
    march_map, close = _march_map(sub, cores)
    try:
        dt = sum(oracle_pass(sub, met, geo, lc_class, 1, march_map)[0])
    finally:
        close()
    return {"value": crop * crop * N_STEPS_DAY / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{crop}x{crop} px corner of the {city.shape[0]}x{city.shape[1]} workload, 24 steps, SVF "
                      f"sweep included, {dt:.1f} s: patch marches in a {cores}-process pool, window numpy in one "
                      f"process ({cores} torch threads)"}


def run_reference(args):
    """--impl reference: one pass of the CPU oracle over the whole workload
    (every pixel, the full march lengths), its K timed steps the K pieces of
    that pass (oracle_pass); W warm-up passes over a 32 x 32 corner first."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch
    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    city, met, geo, lc_class = make_workload(args.workload, 0, args.side)
    small = _crop(city, 32)
    serial, _ = _march_map(small, 1)
    for _ in range(args.warmup):
        oracle_pass(small, met, geo, lc_class, 1, serial)
    march_map, close = _march_map(city, cores)
    try:
        times, _ = oracle_pass(city, met, geo, lc_class, args.steps, march_map)
    finally:
        close()
    total = sum(times)
    rows, cols = city.shape
    value = rows * cols * N_STEPS_DAY / total
    sample = (f"one full pass of the {rows}x{cols} workload (SVF sweep + 24 steps) in {args.steps} timed pieces "
              f"(sweep, then the window's steps), {total:.1f} s: patch marches in a {cores}-process spawn pool, "
              f"window numpy in one process ({cores} torch threads)")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded city, 24 h forcing)",
        "config": {"workload": args.workload, "rows": rows, "cols": cols, "timesteps": N_STEPS_DAY,
                   "sample": sample, "piece_s": [round(t, 3) for t in times]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_batched(args, world, rank, local):
    """The batched workload: this rank's share of the 64 sites (LPT split by
    pixels, strong scaling) in one graph-replayed launch per stage."""
    import torch
    import torch.distributed as dist
    from solweig_project_b200 import _native as N
    from solweig_project_b200 import batch as B
    from solweig_project_b200 import build, synthetic
    from solweig_project_b200.engine import DeviceSite
    build.build()
    specs = synthetic.multi_site_specs()
    mine = B.partition_sites([s["side"] ** 2 for s in specs], world)[rank]
    lc_class = synthetic.default_lc_class()
    sites, series, cities, mets, geos, locs = [], [], [], [], [], []
    for i in mine:
        sp = specs[i]
        c = synthetic.make_city(sp["side"], sp["side"], seed=sp["seed"], density=sp["density"],
                                canopy_cover=sp["canopy"])
        met = synthetic.make_met(sp["seed"])
        geo = synthetic.load_sun_geometry(f"multi{i}")
        loc = {"latitude": sp["latitude"], "longitude": sp["longitude"], "altitude": 3.0}
        s = DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, landcover=c.landcover, lc_class=lc_class)
        series.append(s.build_series(met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"], geo["dectime"],
                                     geo["altmax"], loc))
        sites.append(s)
        cities.append(c)
    dev = sites[0].device
    tuner = B.Autotuner()
    batch = B.SiteBatch(sites, series, requested=("utci", "tmrt"), tuner=tuner)
    tuned = tuner.tune(batch)
    batch.capture()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        batch.replay()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
    launches0 = N.launch_count()
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(float(k))
            events[k][0].record(stream)
            batch.replay()
            events[k][1].record(stream)
        torch.cuda.synchronize()
    direct_launches = N.launch_count() - launches0   # launches outside the graph (none expected)
    step_ms = sum(e[0].elapsed_time(e[1]) for e in events) / args.steps
    t_max = torch.tensor([step_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    step_ms = float(t_max.item())
    total_px = sum(s["side"] ** 2 for s in specs)
    value = total_px * N_STEPS_DAY / (step_ms / 1e3)
    batch.check_tensor_errors()
    # stage breakdown (one launch per stage, outside the graph; the patch-sum
    # products one per site)
    stage_ms = {}
    for st in B.STAGES:
        if st == "flux" and batch.tensor_sums:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for m in batch.members:
                m.site.launch_patch_sums(m.series_struct, m.sums)
            e1.record(stream)
            torch.cuda.synchronize()
            stage_ms["patch_sums_tc"] = e0.elapsed_time(e1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.launch(st)
        e1.record(stream)
        torch.cuda.synchronize()
        stage_ms[st] = e0.elapsed_time(e1)
    # e2e: rasters from pinned host memory into the resident batch, the graph,
    # UTCI / Tmrt back to pinned host memory
    # the site's march rasters and wall planes, as the sweep / time loop read them
    pinned_in = []
    for m in batch.members:
        for k in ("dsm", "vegdsm", "vegdsm2", "walls", "aspect_rad"):
            pinned_in.append((m.site.t[k], m.site.t[k].detach().cpu().pin_memory()))
    pinned_out = [torch.empty(tuple(batch.members[i].outputs.shape), dtype=torch.float32).pin_memory()
                  for i in range(len(sites))]
    e2e_times = []
    for it in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for d_t, h in pinned_in:
            d_t.copy_(h, non_blocking=True)
        batch.replay()
        for m, h in zip(batch.members, pinned_out):
            h.copy_(m.outputs, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= 1:
            e2e_times.append(e0.elapsed_time(e1))
    e2e_ms = torch.tensor([float(np.median(e2e_times))], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    h2d = sum(h.numel() * 4 for _, h in pinned_in)
    d2h = sum(h.numel() * 4 for h in pinned_out)
    # the graph replays the non-empty stage launches of the batch once per step
    per_replay = sum(1 for st in B.STAGES if batch.tiles(st, batch.shapes[st][0])[1] > 0)
    launches = args.steps * per_replay + direct_launches
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        except OSError:
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        npix_rank = batch.pixels
        dom = max(("svf", "flux"), key=lambda k: stage_ms[k])
        if dom == "svf":
            # source gathers the sweeps execute, counted site by site with the
            # counting sweep (untimed; the batch kernel runs the same marches)
            gathers = 0
            for m in batch.members:
                tmp_p = torch.empty((N.SVF_PLANES, m.site.rows, m.site.cols), dtype=torch.float32, device=dev)
                tmp_b = torch.empty((3, N.CUBE_WORDS, m.site.rows, m.site.cols), dtype=torch.int32, device=dev)
                gathers += m.site.count_svf_gathers(tmp_p, tmp_b)
            achieved = SVF_GATHER_BYTES_PER_STEP * gathers / (stage_ms["svf"] * 1e6)
            note = "march gather bytes (12 B x source gathers executed, counted by sw100_svf_sweep_count) / " \
                   "launch time"
        else:
            achieved = FLUX_BYTES_PER_PX_STEP * npix_rank * N_STEPS_DAY / (stage_ms["flux"] * 1e6)
            note = "compulsory 190 B per pixel-step / launch time"
        clk = clocks.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (64 seeded cities + 24 h forcing each)",
            "config": {"workload": "batched64", "description": WORKLOADS["batched64"][2], "sites": len(specs),
                       "pixels": total_px, "timesteps": N_STEPS_DAY,
                       "launch_shapes": {k: [list(v[0]), v[1]] for k, v in batch.shapes.items()},
                       "l2": "flushed (256 MiB write) before every timed step; inputs far above L2",
                       "parallelism": f"sites LPT-split over {world} rank(s)"},
            "roofline": {"bound": "hbm", "kernel": dom + "_batch", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": None,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback",
                         "definition": note},
            "stages_ms": stage_ms,
            "autotune_ms": {k: v[2] for k, v in tuned.items()},
            "gpu_launches": int(launches),
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "e2e": {"value": total_px * N_STEPS_DAY / (float(e2e_ms.item()) / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": float(e2e_ms.item()), "timed_calls": len(e2e_times), "statistic": "median"},
        }
        print(json.dumps(line), flush=True)
    batch.graph = None
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_preview(args, world, rank, local):
    """The learned-preview workload: per seeded edit, the preview's device
    latency against the exact windowed recompute and the full sweep, and SVF
    / Tmrt errors against the exact chain (with the stale SVF as the method
    without it), the edits spread over `--sites` held-out cities."""
    import torch
    from solweig_project_b200 import build, synthetic
    from solweig_project_b200 import preview as PV
    from solweig_project_b200.engine import DeviceSite
    build.build()
    if rank != 0:
        return
    net = PV.load_pretrained()
    met = synthetic.make_met(1234)
    geo = synthetic.load_sun_geometry("single")
    n_edits = args.edits or max(20, 20 * args.steps)
    n_sites = max(1, min(args.sites, n_edits))
    rows, per_site, full_all = [], [], []
    with ClockSampler(local) as clocks:
        for i in range(n_sites):
            c = synthetic.make_city(1024, 1024, seed=4242 + i, density=0.3, canopy_cover=0.15)
            site = DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, landcover=c.landcover,
                              lc_class=synthetic.default_lc_class(), amaxvalue=48.0)
            site.run_svf()
            ser = site.build_series(met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"], geo["dectime"],
                                    geo["altmax"], dict(synthetic.DEFAULT_LOCATION))
            if i == 0:   # warm-up (graph capture etc.)
                PV.evaluate_edits(net, site, ser, n_edits=max(1, args.warmup), seed=99)
            n = n_edits // n_sites + (1 if i < n_edits % n_sites else 0)
            got = PV.evaluate_edits(net, site, ser, n_edits=n, seed=5 + i)
            full = []
            for _ in range(3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                site.launch_svf(site.svf_result.planes, site.svf_result.bits)
                e1.record()
                torch.cuda.synchronize()
                full.append(e0.elapsed_time(e1))
            full_all.append(float(np.median(full)))
            per_site.append({"seed": 4242 + i, "edits": n, "full_sweep_ms": full_all[-1],
                             "preview_ms": float(np.median([r["ms_preview"] for r in got])),
                             "exact_window_ms": float(np.median([r["ms_exact"] for r in got])),
                             "tmrt_rmse_K": {"preview": float(np.mean([r["tmrt_rmse_preview"] for r in got])),
                                             "stale": float(np.mean([r["tmrt_rmse_stale"] for r in got]))}})
            rows += got
            del site
            torch.cuda.empty_cache()
    mean = lambda k: float(np.mean([r[k] for r in rows]))  # noqa: E731
    med = lambda k: float(np.median([r[k] for r in rows]))  # noqa: E731
    full_ms = float(np.median(full_all))
    clk = clocks.summary()
    print(json.dumps({
        "metric": "SVF edit latency, learned preview (device ms per edit)", "value": med("ms_preview"), "unit": "ms",
        "n_gpus": 1, "steps": n_edits, "warmup": args.warmup, "ms_per_step": med("ms_preview"),
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
        "data": f"synthetic ({n_sites} held-out seeded 1024x1024 cities, seeded edits)",
        "config": {"workload": "preview1024", "description": WORKLOADS["preview1024"][2], "edits": n_edits,
                   "sites": n_sites, "net_params": net.n_params,
                   "window": "256x256 (128x128 block + 64 px context)"},
        "exact_window_ms": med("ms_exact"), "full_sweep_ms": full_ms,
        "speedup_vs_exact_window": med("ms_exact") / med("ms_preview"),
        "speedup_vs_full_sweep": full_ms / med("ms_preview"),
        "svf_mae": {"preview": mean("svf_mae_preview"), "stale": mean("svf_mae_stale")},
        "tmrt_rmse_K": {"preview": mean("tmrt_rmse_preview"), "stale": mean("tmrt_rmse_stale")},
        "modes": {m: sum(r["mode"] == m for r in rows) for m in ("preview", "exact")},
        "per_site": per_site,
        "gpu_launches": None,
        "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "e2e": {"value": med("ms_preview"), "unit": "ms", "h2d_bytes_per_step": 5 * 4 * 40 * 40,
                "d2h_bytes_per_step": 4},
    }), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    if args.workload == "batched64":
        run_batched(args, world, rank, local)
        return
    if args.workload == "preview1024":
        run_preview(args, world, rank, local)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    from solweig_project_b200 import _native as N
    from solweig_project_b200 import api, build
    from solweig_project_b200.engine import DeviceSite
    build.build()
    city, met, geo, lc_class = make_workload(args.workload, rank, args.side)
    rows, cols = city.shape
    npix = rows * cols
    loc = {"latitude": 30.3, "longitude": -97.7, "altitude": 3.0}

    site = DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale,
                      landcover=city.landcover, lc_class=lc_class)
    res = site.run_svf()
    ser = site.build_series(met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"], geo["dectime"],
                            geo["altmax"], loc)
    series, series_dev = site.upload_series(ser)
    n_day = series.n_day
    dev = site.device
    planes, bits = res.planes, res.bits
    gsrc = torch.empty((max(1, n_day), rows, cols, 4), dtype=torch.float32, device=dev)
    outputs = torch.empty((2, N_STEPS_DAY, rows, cols), dtype=torch.float32, device=dev)
    mask = N.OUT_UTCI | N.OUT_TMRT
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    from solweig_project_b200 import engine as E
    sums = torch.empty((N_STEPS_DAY, 4, rows, cols), dtype=torch.float32, device=dev) if E.TENSOR_SUMS else None

    def step(ev=None):
        if ev is not None:
            ev[0].record(stream)
        site.launch_svf(planes, bits)
        if ev is not None:
            ev[1].record(stream)
        site.launch_sun_march(series, gsrc)
        if ev is not None:
            ev[2].record(stream)
        if sums is not None:
            site.launch_patch_sums(series, sums)
        if ev is not None:
            ev[4].record(stream)
        site.state.zero_()
        site.launch_flux_loop(series, gsrc, mask, outputs, sums=sums)
        if ev is not None:
            ev[3].record(stream)

    for _ in range(args.warmup):
        step()
    # source gathers the sweep's marches execute (counting kernel, untimed)
    svf_gathers = site.count_svf_gathers(planes, bits)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(args.steps)]
    launches0 = N.launch_count()
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(float(k))          # evict L2 between timed steps (not timed)
            step(events[k])
        torch.cuda.synchronize()
    launches = N.launch_count() - launches0
    site.check_tensor_error()
    svf_ms = [e[0].elapsed_time(e[1]) for e in events]
    march_ms = [e[1].elapsed_time(e[2]) for e in events]
    sums_ms = [e[2].elapsed_time(e[4]) for e in events]
    loop_ms = [e[4].elapsed_time(e[3]) for e in events]
    step_ms = sum(e[0].elapsed_time(e[3]) for e in events) / args.steps
    t_max = torch.tensor([step_ms], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
        dist.barrier()
    step_ms = float(t_max.item())
    value = world * npix * N_STEPS_DAY / (step_ms / 1e3)

    # ---------------------------------------------------------------- e2e
    e2e = None
    if not args.no_e2e:
        pinned = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in (
            ("dsm", city.dsm), ("trees", city.trees), ("dem", city.dem), ("walls", city.walls),
            ("aspect", city.aspect), ("landcover", city.landcover))}
        from solweig_project_b200 import engine as E
        e2e_times = []
        moved = []
        for it in range(2 + E2E_TIMED):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            E.TRANSFER.update(h2d=0, d2h=0)
            e0.record(stream)
            out = api.run_exact_chain(dsm=pinned["dsm"].numpy(), trees=pinned["trees"].numpy(),
                                      dem=pinned["dem"].numpy(), walls=pinned["walls"].numpy(),
                                      aspect=pinned["aspect"].numpy(), scale=city.scale, met_file=met,
                                      location=loc, landcover=pinned["landcover"].numpy(), lc_class=lc_class,
                                      requested=("utci", "tmrt"), **geo)
            e1.record(stream)
            torch.cuda.synchronize()
            if it >= 2:
                e2e_times.append(e0.elapsed_time(e1))
                moved.append(dict(E.TRANSFER))
        h2d, d2h = moved[-1]["h2d"], moved[-1]["d2h"]
        e2e_ms = torch.tensor([float(np.median(e2e_times))], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
        if args.timeline and rank == 0:
            tl = E.Timeline()
            torch.cuda.synchronize()
            api.run_exact_chain(dsm=pinned["dsm"].numpy(), trees=pinned["trees"].numpy(), dem=pinned["dem"].numpy(),
                                walls=pinned["walls"].numpy(), aspect=pinned["aspect"].numpy(), scale=city.scale,
                                met_file=met, location=loc, landcover=pinned["landcover"].numpy(),
                                lc_class=lc_class, requested=("utci", "tmrt"), timeline=tl, **geo)
            timeline_rows = tl.report()
        e2e = {"value": world * npix * N_STEPS_DAY / (float(e2e_ms.item()) / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": float(e2e_ms.item()), "timed_calls": len(e2e_times), "statistic": "median"}

    if rank == 0:
        svf_steps = int(site.svf_tables(2)[2])
        loop_t = sum(loop_ms) / len(loop_ms)
        svf_t = sum(svf_ms) / len(svf_ms)
        march_t = sum(march_ms) / len(march_ms)
        sums_t = sum(sums_ms) / len(sums_ms)
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
        except OSError:
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        stages = {
            "svf_sweep": {"ms": svf_t, "table_steps_per_px": svf_steps,
                          "executed_gathers_per_px": svf_gathers / npix,
                          "gbs_gather": SVF_GATHER_BYTES_PER_STEP * svf_gathers / (svf_t * 1e6),
                          "issue_active_frac_ncu": NCU_ISSUE_ACTIVE["svf_sweep"],
                          "active_lanes_ncu": NCU_ACTIVE_LANES["svf_sweep"]},
            "sun_march": {"ms": march_t, "issue_active_frac_ncu": NCU_ISSUE_ACTIVE["sun_march"],
                          "active_lanes_ncu": NCU_ACTIVE_LANES["sun_march"]},
            "patch_sums_tc": {"ms": sums_t,
                              "tflops_bf16": (2.0 * npix * 624 * 96 * ((N_STEPS_DAY + 7) // 8) / (sums_t * 1e9)
                                              if sums is not None and sums_t > 0 else None),
                              "issue_active_frac_ncu": NCU_ISSUE_ACTIVE["patch_sums_tc"],
                              "tensor_active_frac_ncu": NCU_TENSOR_ACTIVE["patch_sums_tc"],
                              "note": "dense 153-patch sums as a one-hot x weight product on tcgen05 (BF16 in 3 "
                                      "parts, FP32 accumulate); includes the weight split kernel"},
            "flux_loop": {"ms": loop_t,
                          "gbs_compulsory": FLUX_BYTES_PER_PX_STEP * npix * N_STEPS_DAY / (loop_t * 1e6),
                          "issue_active_frac_ncu": NCU_ISSUE_ACTIVE["flux_loop"],
                          "active_lanes_ncu": NCU_ACTIVE_LANES["flux_loop"]},
        }
        dom = max(stages, key=lambda k: stages[k]["ms"])
        if dom == "svf_sweep":
            achieved = stages[dom]["gbs_gather"]
            roof_note = "march gather bytes (12 B x source gathers executed, counted by sw100_svf_sweep_count) / " \
                        "launch time"
            bind_note = ("DRAM traffic per launch is about the rasters read once plus the planes and bit cubes "
                         "written (~200 B per pixel): the gathers of a warp's neighbouring rays hit L1 / L2, and "
                         "the marches' step tests bound the launch")
        elif dom == "flux_loop":
            achieved = stages[dom]["gbs_compulsory"]
            roof_note = "compulsory 190 B per pixel-step / launch time"
            bind_note = ("DRAM traffic per launch is far below the algorithmic bytes: each pixel's patch-bit cubes "
                         "are read once per launch and kept on chip (shared memory) across the 24 steps")
        else:
            achieved = None
            roof_note = bind_note = ""
        clk = clocks.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded city + 24 h forcing, random geometry)",
            "config": {"workload": args.workload if args.side is None else f"{args.workload}@{rows}",
                       "description": WORKLOADS[args.workload][2], "rows": rows,
                       "cols": cols, "timesteps": N_STEPS_DAY, "daytime_steps": int(n_day),
                       "svf_march_steps_per_px": svf_steps, "l2": "flushed (256 MiB write) before every timed step",
                       "parallelism": f"site-per-rank x{world}"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": (achieved / hbm) if achieved else None,
                         "traffic": (NCU_TRAFFIC[dom][1] * npix / NCU_TRAFFIC[dom][0]) if dom in NCU_TRAFFIC else None,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback",
                         "definition": roof_note,
                         "binding": {"resource": "SM instruction issue", "kernel": dom,
                                     "issue_active_frac_ncu": NCU_ISSUE_ACTIVE.get(dom),
                                     "active_lanes_ncu": NCU_ACTIVE_LANES.get(dom),
                                     "note": bind_note}},
            "stages": stages,
            "gpu_launches": int(launches),
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        if e2e is not None:
            line["e2e"] = e2e
        pin = PINS.get(args.workload) if args.side is None else None
        if pin is not None and os.path.exists(pin):
            line["error_vs_fp64"] = error_vs_fp64(pin, outputs[1].cpu().numpy(), outputs[0].cpu().numpy())
        if not args.no_cpu_baseline and world == 1:   # rank 0 at N = 1 only
            line["cpu_baseline"] = cpu_baseline(city, met, geo, lc_class)
        print(json.dumps(line), flush=True)
        if args.timeline and e2e is not None:
            print("host timeline of one end-to-end call (ms): phase | host phase | host since start | "
                  "GPU since start at the phase's end", flush=True)
            for name, dt, t, gpu in timeline_rows:
                print(f"  {name:28s} {dt:8.3f} {t:8.3f} {'' if gpu is None else f'{gpu:8.3f}'}", flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
