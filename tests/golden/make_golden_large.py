"""Reference pins at the benchmark sizes: the 200 x 200 and 500 x 500 seeded
cities (the 500 x 500 one is the city ``bench.py`` times), three sites of
the 64-site batched workload and a 512 x 512 city of the 4096 x 4096 tile's
generator (buildings up to 120 m), 24 hourly steps.

    python tests/golden/make_golden_large.py --ref <reference checkout> [--cases c1_200 c2_500 ...]

(``--ref`` may be replaced by the environment variable ``SOLWEIG_REFERENCE``.)

Full planes at these sizes would make fixtures of hundreds of MB, so each
case records, from the unmodified reference run on the host CPU:

* sha256 digests of the inputs the repository regenerates from the seed
  (DSM, trees, DEM, land cover, and the reference's own ``walls_aspect``
  wall height / aspect), so a test first proves it feeds the same rasters;
* sha256 digests of the raw float32 bytes of the 15 SVF planes and
  SVFtotal of ``shadow.svf_calculator`` and of the three patch cubes (bits
  packed along the patch axis, little bit order), plus the SVF values at
  the sample pixels for diagnostics;
* per daytime step, digests of the 8 planes of
  ``shadowingfunction_wallheight_23`` (captured by wrapping the function
  the reference's ``Solweig_2022a_calc`` calls);
* per step, the digest of the ``shadow`` output of ``run_utci_window``;
* Tmrt and UTCI of every step at seeded sample pixels (4096 ground pixels,
  256 building pixels), and per step the float64 sums of Tmrt over all
  pixels and of UTCI over its valid pixels;
* an FP64 re-evaluation of the same run: the reference's
  ``run_utci_window`` again, under ``torch.set_default_dtype(float64)``
  with float64 inputs, the float32-typed constants of ``solweig.py`` and
  ``calculate_utci.py`` read as float64 (a proxy for the ``torch`` name of
  those modules), and the discrete geometry held at the float32 contract:
  the SVF bundle and every sun-march result of the float32 run are fed in
  (cast to float64), so the comparison measures the arithmetic of the flux
  -> Tmrt -> UTCI chain, not predicate flips of the shadow marches.  Tmrt
  and UTCI are captured in float64 before the reference stores them into
  its float32 output arrays.  The fixture stores them at the sample pixels
  as float32 offsets from the float32 reference values, and the max / RMS
  error of the float32 reference against FP64 over all pixels.

Files: ``tests/golden/large_<case>.npz``.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)

from make_golden import SVF_NAMES, install_stubs, reference_path  # noqa: E402
from solweig_project_b200 import synthetic  # noqa: E402

# name: (side, seed, h_max) of a single-site city at lat 30.3 / lon -97.7, or
# ("multi", i): site i of the 64-site batched workload (its own seed,
# density, canopy cover, latitude and forcing)
CASES = {
    "c1_200": (200, 1234, 40.0),
    "c2_500": (500, 1234, 40.0),
    "c3_site37": ("multi", 37),
    "c3_site47": ("multi", 47),
    "c3_site17": ("multi", 17),
    # the 4096 x 4096 tile's generator (buildings up to 120 m) at 512 x 512
    "c4_proxy512": (512, 1234, 120.0),
}
N_GROUND = 4096
N_BUILDING = 256
MARCH_NAMES = ("vegsh", "sh", "vbshvegsh", "wallsh", "wallsun", "wallshve", "facesh", "facesun")


def digest(a, dtype=np.float32):
    a = np.ascontiguousarray(np.asarray(a, dtype))
    return hashlib.sha256(a.tobytes()).hexdigest()


def cube_digest(cube):
    """Digest of a (rows, cols, P) 0/1 cube packed along P, little bit order."""
    c = np.asarray(cube)
    assert np.isin(c, (0, 1)).all()
    return digest(np.packbits(c.astype(np.uint8), axis=2, bitorder="little"), np.uint8)


def sample_pixels(buildings_ground, seed):
    """Seeded sample: N_GROUND ground pixels and N_BUILDING building pixels
    (flat indices, sorted)."""
    rng = np.random.default_rng(seed + 99)
    flat = buildings_ground.reshape(-1)
    ground = np.flatnonzero(flat == 1)
    build = np.flatnonzero(flat == 0)
    g = rng.choice(ground, size=min(N_GROUND, ground.size), replace=False)
    b = rng.choice(build, size=min(N_BUILDING, build.size), replace=False)
    return np.sort(np.concatenate([g, b])).astype(np.int64)


class _Float64Torch:
    """Stand-in for the ``torch`` name of a reference module: every
    attribute is torch's, except ``float32``, which reads as float64."""

    def __init__(self, torch):
        self._torch = torch

    def __getattr__(self, name):
        if name == "float32":
            return self._torch.float64
        return getattr(self._torch, name)


def make_case_inputs(spec):
    """(city, met, location) of a case spec (see CASES)."""
    if spec[0] == "multi":
        sp = synthetic.multi_site_specs()[spec[1]]
        city = synthetic.make_city(sp["side"], sp["side"], seed=sp["seed"], density=sp["density"],
                                   canopy_cover=sp["canopy"], with_walls=False)
        loc = {"latitude": sp["latitude"], "longitude": sp["longitude"], "altitude": 3.0}
        return city, synthetic.make_met(sp["seed"]), loc, sp["seed"]
    side, seed, h_max = spec
    city = synthetic.make_city(side, side, seed=seed, h_max=h_max, with_walls=False)
    return city, synthetic.make_met(seed), dict(synthetic.DEFAULT_LOCATION), seed


def run_case(name, spec, ref):
    import torch
    import solweig_gpu.calculate_utci as rcu
    import solweig_gpu.shadow as rshadow
    import solweig_gpu.solweig as rsolweig
    import solweig_gpu.sun_position as rsun
    import solweig_gpu.utci_process as rup
    import solweig_gpu.walls_aspect as rwa

    city, met, loc, seed = make_case_inputs(spec)
    rows, cols = city.shape
    scale = 1.0
    out = {"spec": np.array([str(x) for x in spec]), "seed": seed}
    if spec[0] != "multi":
        out.update(side=spec[0], h_max=spec[2])
    t0 = time.time()
    walls = rwa.findwalls(city.dsm, 3.0).astype(np.float32)
    aspect = rwa.filter1Goodwin_as_aspect_v3(walls.astype(np.float64), scale, city.dsm).astype(np.float32)
    print(f"[{name}] walls/aspect {time.time() - t0:.1f}s", flush=True)
    for k, v in (("dsm", city.dsm), ("trees", city.trees), ("dem", city.dem), ("landcover", city.landcover),
                 ("walls", walls), ("aspect", aspect)):
        out["digest_in_" + k] = digest(v)

    _, altitude, azimuth, zen, jday, _, dectime, altmax = rsun.Solweig_2015a_metdata_noload(
        met, loc, synthetic.DEFAULT_UTC)
    geo = dict(altitude=altitude, azimuth=azimuth, zen=zen, jday=jday, dectime=dectime, altmax=altmax)
    for k, v in geo.items():
        out[k] = np.asarray(v, np.float64)
    out["met"] = met
    out["latitude"], out["longitude"], out["site_altitude"] = loc["latitude"], loc["longitude"], loc["altitude"]
    lc_class = np.loadtxt(os.path.join(ref, "solweig_gpu", "landcoverclasses_2016a.txt"),
                          skiprows=1, usecols=range(1, 7))

    buildings_ground = np.where(city.dsm - city.dem < 2.0, 1, 0)
    samples = sample_pixels(buildings_ground, seed)
    out["samples"] = samples

    # ---------------- float32: the reference as it runs
    a = torch.tensor(city.dsm)
    temp1 = torch.tensor(city.trees)
    temp2 = torch.tensor(city.dem)
    temp1[temp1 < 0.] = 0.
    vegdem = temp1 + temp2
    vegdem2 = torch.add(temp1 * 0.25, temp2)
    bush = torch.logical_not(vegdem2 * vegdem) * vegdem
    vegdsm = temp1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = temp1 * 0.25 + a
    vegdsm2[vegdsm2 == a] = 0
    amaxvalue = torch.maximum(a.max(), vegdem.max())
    out["amaxvalue"] = np.float32(amaxvalue.item())

    t0 = time.time()
    bundle = rshadow.svf_calculator(2, amaxvalue, a, vegdsm, vegdsm2, bush, scale)
    print(f"[{name}] svf_calculator {time.time() - t0:.1f}s", flush=True)
    bundle_np = {}
    for k, v in zip(SVF_NAMES, bundle):
        arr = v.detach().cpu().numpy()
        bundle_np[k] = arr
        if k.endswith("mat"):
            out["digest_svf_" + k] = cube_digest(arr)
        else:
            out["digest_svf_" + k] = digest(arr)
            out["sample_svf_" + k] = arr.reshape(-1)[samples].astype(np.float32)

    march_log = []
    orig_march = rsolweig.shadowingfunction_wallheight_23

    def march_capture(*args, **kwargs):
        r = orig_march(*args, **kwargs)
        march_log.append((args[3], args[4], tuple(x.detach().cpu().numpy().astype(np.float32) for x in r)))
        return r

    T = met.shape[0]
    rsolweig.shadowingfunction_wallheight_23 = march_capture
    try:
        t0 = time.time()
        outputs = rup.run_utci_window(
            a=a, temp1=torch.tensor(city.trees), temp2=temp2, walls=torch.tensor(walls),
            dirwalls=torch.tensor(aspect), svf_bundle=bundle, met_file=met, location=loc, scale=scale,
            amaxvalue=amaxvalue, landcover_grid=torch.tensor(city.landcover), lc_class=lc_class,
            requested_variables=("utci", "tmrt", "shadow"), **geo)
        print(f"[{name}] run_utci_window float32 {time.time() - t0:.1f}s", flush=True)
    finally:
        rsolweig.shadowingfunction_wallheight_23 = orig_march

    out["march_steps"] = np.array([i for i in range(T) if altitude[0][i] > 0], np.int32)
    assert len(march_log) == len(out["march_steps"])
    out["digest_march"] = np.array([[digest(p) for p in planes] for _, _, planes in march_log])
    out["digest_shadow"] = np.array([digest(outputs["shadow"][t]) for t in range(T)])
    tm32 = outputs["tmrt"].reshape(T, -1)
    ut32 = outputs["utci"].reshape(T, -1)
    out["sample_tmrt"] = tm32[:, samples].copy()
    out["sample_utci"] = ut32[:, samples].copy()
    out["sum_tmrt"] = tm32.astype(np.float64).sum(axis=1)
    out["sum_utci"] = np.nansum(ut32.astype(np.float64), axis=1)
    out["n_utci_valid"] = np.sum(~np.isnan(ut32), axis=1)

    # ---------------- FP64 re-evaluation with the float32 geometry
    captured_tmrt = []
    captured_utci = []
    replay = iter(march_log)
    orig_calc = rup.Solweig_2022a_calc
    orig_utci = rup.utci_calculator
    saved_torch = (rsolweig.torch, rcu.torch)

    def march_replay(*args, **kwargs):
        az, alt, planes = next(replay)
        assert float(args[3]) == float(az) and float(args[4]) == float(alt)
        return tuple(torch.tensor(p, dtype=torch.float64) for p in planes)

    def calc_capture(*args, **kwargs):
        r = orig_calc(*args, **kwargs)
        captured_tmrt.append(r[0].detach().cpu().numpy().astype(np.float64))
        return r

    def utci_capture(*args, **kwargs):
        r = orig_utci(*args, **kwargs)
        captured_utci.append(r.detach().cpu().numpy().astype(np.float64))
        return r

    prev_default = torch.get_default_dtype()
    torch.set_default_dtype(torch.float64)
    rsolweig.torch = _Float64Torch(torch)
    rcu.torch = _Float64Torch(torch)
    rsolweig.shadowingfunction_wallheight_23 = march_replay
    rup.Solweig_2022a_calc = calc_capture
    rup.utci_calculator = utci_capture
    try:
        f64 = lambda x: torch.tensor(np.asarray(x, np.float64))  # noqa: E731
        bundle64 = tuple(f64(bundle_np[k]) for k in SVF_NAMES)
        t0 = time.time()
        rup.run_utci_window(
            a=f64(city.dsm), temp1=f64(city.trees), temp2=f64(city.dem), walls=f64(walls),
            dirwalls=f64(aspect), svf_bundle=bundle64, met_file=met, location=loc, scale=scale,
            amaxvalue=torch.tensor(float(out["amaxvalue"]), dtype=torch.float64),
            landcover_grid=f64(city.landcover), lc_class=lc_class, requested_variables=("utci", "tmrt"), **geo)
        print(f"[{name}] run_utci_window float64 {time.time() - t0:.1f}s", flush=True)
    finally:
        torch.set_default_dtype(prev_default)
        rsolweig.torch, rcu.torch = saved_torch
        rsolweig.shadowingfunction_wallheight_23 = orig_march
        rup.Solweig_2022a_calc = orig_calc
        rup.utci_calculator = orig_utci

    assert len(captured_tmrt) == T and len(captured_utci) == T
    tm64 = np.stack([np.broadcast_to(x, (rows, cols)) for x in captured_tmrt]).reshape(T, -1)
    ut64 = np.stack(captured_utci).reshape(T, -1)
    ut64 = np.where(np.isnan(ut32), np.nan, ut64)
    out["sample_tmrt64_delta"] = (tm64[:, samples] - tm32[:, samples]).astype(np.float32)
    out["sample_utci64_delta"] = (ut64[:, samples] - ut32[:, samples]).astype(np.float32)
    dt = tm32.astype(np.float64) - tm64
    du = ut32.astype(np.float64) - ut64
    out["ref_fp64_tmrt_max"] = float(np.abs(dt).max())
    out["ref_fp64_tmrt_rms"] = float(np.sqrt(np.mean(dt * dt)))
    out["ref_fp64_utci_max"] = float(np.nanmax(np.abs(du)))
    out["ref_fp64_utci_rms"] = float(np.sqrt(np.nanmean(du * du)))
    out["sum_tmrt64"] = tm64.sum(axis=1)
    out["sum_utci64"] = np.nansum(ut64, axis=1)
    print(f"[{name}] reference float32 vs FP64: Tmrt max {out['ref_fp64_tmrt_max']:.3g} rms "
          f"{out['ref_fp64_tmrt_rms']:.3g} K, UTCI max {out['ref_fp64_utci_max']:.3g} rms "
          f"{out['ref_fp64_utci_rms']:.3g} C", flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (or $SOLWEIG_REFERENCE)")
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    args = ap.parse_args()
    ref = reference_path(args.ref)
    install_stubs(ref)
    import torch
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    for name in args.cases:
        data = run_case(name, CASES[name], ref)
        path = os.path.join(HERE, f"large_{name}.npz")
        np.savez_compressed(path, **data)
        print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)", flush=True)


if __name__ == "__main__":
    main()
