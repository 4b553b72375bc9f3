"""Generate the golden fixtures by running the reference implementation.

Run where a read-only checkout of the reference is available:

    python tests/golden/make_golden.py --ref <reference checkout>

(``--ref`` may be replaced by the environment variable ``SOLWEIG_REFERENCE``.)

It imports ``solweig_gpu`` from the reference with I/O-only stubs for GDAL,
timezonefinder and pytz (they are used only for raster I/O and time zones),
builds seeded synthetic cities with :mod:`solweig_project_b200.synthetic`,
and records, per case:

* the inputs (DSM, trees, DEM, land cover, walls/aspect from the reference's
  own ``walls_aspect``, met rows, the sun geometry returned by the reference's
  ``Solweig_2015a_metdata_noload``);
* the SVF bundle of ``shadow.svf_calculator`` (15 planes, 3 patch cubes,
  SVFtotal);
* per daytime step, the 8 outputs of ``shadowingfunction_wallheight_23``;
* per step, the planes and scalars returned by ``Solweig_2022a_calc`` and
  the ground-view-factor planes of ``gvf_2018a`` (captured by wrapping the
  reference functions, which are left unmodified);
* the outputs of ``utci_process.run_utci_window`` for every variable.

The files are written to ``tests/golden/<case>.npz``.  The GPU box never
needs the reference: tests only read these files.
"""
from __future__ import annotations

import argparse
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from solweig_project_b200 import synthetic  # noqa: E402


def reference_path(arg):
    """The reference checkout named by ``--ref`` or ``$SOLWEIG_REFERENCE``."""
    ref = arg or os.environ.get("SOLWEIG_REFERENCE")
    if not ref:
        raise SystemExit("name the reference checkout with --ref or SOLWEIG_REFERENCE")
    if not os.path.isdir(os.path.join(ref, "solweig_gpu")):
        raise SystemExit(f"{ref!r} holds no solweig_gpu package")
    return ref


def install_stubs(ref):
    osgeo = types.ModuleType("osgeo")
    gdal = types.ModuleType("osgeo.gdal")
    gdal.UseExceptions = lambda: None
    osr = types.ModuleType("osgeo.osr")
    osgeo.gdal = gdal
    osgeo.osr = osr
    sys.modules.setdefault("osgeo", osgeo)
    sys.modules.setdefault("osgeo.gdal", gdal)
    sys.modules.setdefault("osgeo.osr", osr)
    tzf = types.ModuleType("timezonefinder")
    tzf.TimezoneFinder = type("TimezoneFinder", (), {})
    sys.modules.setdefault("timezonefinder", tzf)
    sys.modules.setdefault("pytz", types.ModuleType("pytz"))
    if ref not in sys.path:
        sys.path.insert(0, ref)


CASES = {
    # name: (rows, cols, seed, scale, dem_level, full_chain, extra make_city kwargs)
    "city36": (36, 36, 11, 1.0, 0.0, True,
               {"n_buildings": 7, "n_trees": 6, "side_range": (4, 12)}),
    "city24x40_s05": (24, 40, 12, 0.5, 0.0, True,
                      {"n_buildings": 5, "n_trees": 5, "side_range": (3, 10)}),
    "dem_bush": (24, 24, 13, 1.0, 2.0, True,
                 {"n_buildings": 4, "n_trees": 4, "side_range": (3, 8)}),
    "strip1x16": (1, 16, 14, 1.0, 0.0, False,
                  {"n_buildings": 2, "n_trees": 3, "side_range": (1, 3)}),
    # bush: ground lowered to -0.25 x canopy under the trees of the left half,
    # so that vegdem2 == 0 != vegdem there and the reference's bush raster
    # (utci_process.py:669-672) is non-zero
    "bush24": (24, 28, 16, 1.0, 0.0, True,
               {"n_buildings": 3, "n_trees": 7, "side_range": (3, 8), "bush_left_half": True}),
    # low vegetation only: patches of the 78 degree ring stop after one step,
    # which is where vbshvegsh can take the value 2
    "lowveg16": (16, 16, 15, 1.0, 0.0, False,
                 {"n_buildings": 0, "n_trees": 8, "tree_peak": (2.5, 4.0)}),
}

STEP_PLANES = ("Tmrt", "Kdown", "Kup", "Ldown", "Lup", "Tg", "shadow", "Keast", "Ksouth",
               "Kwest", "Knorth", "Least", "Lsouth", "Lwest", "Lnorth", "KsideI", "TgOut",
               "Lside", "KsideD", "dRad", "Kside", "Tgmap1", "TgOut1")
STEP_SCALARS = ("esky", "CI", "radI", "radD", "CI_Tg", "CI_TgG", "timeadd", "firstdaytime", "I0")
GVF_NAMES = ("gvfLup", "gvfalb", "gvfalbnosh", "gvfLupE", "gvfalbE", "gvfalbnoshE", "gvfLupS",
             "gvfalbS", "gvfalbnoshS", "gvfLupW", "gvfalbW", "gvfalbnoshW", "gvfLupN",
             "gvfalbN", "gvfalbnoshN", "gvfSum", "gvfNorm")
SVF_NAMES = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg",
             "svfS", "svfSaveg", "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg",
             "vegshmat", "vbshvegshmat", "shmat", "svftotal")


def _np(x):
    import torch
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def run_case(name, spec, ref):
    import torch
    import solweig_gpu.shadow as rshadow
    import solweig_gpu.solweig as rsolweig
    import solweig_gpu.utci_process as rup
    import solweig_gpu.sun_position as rsun
    import solweig_gpu.walls_aspect as rwa

    rows, cols, seed, scale, dem_level, full, kw = spec
    kw = dict(kw)
    bush_left_half = kw.pop("bush_left_half", False)
    city = synthetic.make_city(rows, cols, seed, scale=scale, dem_level=dem_level,
                               with_walls=False, **kw)
    if bush_left_half:
        sel = (city.trees > 0) & (np.arange(cols)[None, :] < cols // 2)
        city.dem[sel] = np.float32(-0.25) * city.trees[sel]
        city.dsm = np.maximum(city.dsm, city.dem).astype(np.float32)
    out = {"rows": rows, "cols": cols, "seed": seed, "scale": scale, "dem_level": dem_level,
           "dsm": city.dsm, "trees": city.trees, "dem": city.dem, "landcover": city.landcover}
    t0 = time.time()
    if rows >= 3 and cols >= 3:
        walls = rwa.findwalls(city.dsm, 3.0)
        aspect = rwa.filter1Goodwin_as_aspect_v3(walls, scale, city.dsm)
    else:
        walls = np.zeros((rows, cols))
        aspect = np.zeros((rows, cols))
    out["walls_ref"] = walls.astype(np.float32)
    out["aspect_ref"] = aspect.astype(np.float32)
    out["walls_ref64"] = walls
    out["aspect_ref64"] = aspect
    print(f"[{name}] walls/aspect {time.time() - t0:.1f}s", flush=True)

    met = synthetic.make_met(seed)
    loc = dict(synthetic.DEFAULT_LOCATION)
    YYYY, altitude, azimuth, zen, jday, leafon, dectime, altmax = rsun.Solweig_2015a_metdata_noload(
        met, loc, synthetic.DEFAULT_UTC)
    out.update(met=met, altitude=altitude, azimuth=azimuth, zen=zen, jday=jday,
               dectime=dectime, altmax=altmax, latitude=loc["latitude"],
               longitude=loc["longitude"], site_altitude=loc["altitude"],
               utc=synthetic.DEFAULT_UTC)

    # --- inputs exactly as compute_utci builds them (utci_process.py:1377-1385)
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
    for k, v in zip(SVF_NAMES, bundle):
        arr = _np(v)
        if k.endswith("mat"):
            out["svf_" + k] = arr.astype(np.uint8)
            assert np.array_equal(out["svf_" + k].astype(np.float32), arr), k
        else:
            out["svf_" + k] = arr.astype(np.float32)

    # --- the sun march for every daytime step
    walls_t = torch.tensor(out["walls_ref"])
    dirwalls_t = torch.tensor(out["aspect_ref"])
    march = {k: [] for k in ("vegsh", "sh", "vbshvegsh", "wallsh", "wallsun", "wallshve", "facesh", "facesun")}
    march_steps = []
    if full:
        for i in range(met.shape[0]):
            if altitude[0][i] > 0:
                r = rsolweig.shadowingfunction_wallheight_23(
                    a, vegdsm, vegdsm2, torch.tensor(azimuth[0][i]).item(),
                    torch.tensor(altitude[0][i]).item(), scale, amaxvalue.item(), bush,
                    walls_t, dirwalls_t * np.pi / 180.)
                for k, v in zip(march, r):
                    march[k].append(_np(v).astype(np.float32))
                march_steps.append(i)
        out["march_steps"] = np.array(march_steps, np.int32)
        for k, v in march.items():
            out["march_" + k] = np.stack(v) if v else np.zeros((0, rows, cols), np.float32)

    if not full:
        return out

    # --- the time loop with captured intermediates
    captured = []
    gvf_captured = []
    orig_calc = rup.Solweig_2022a_calc
    orig_gvf = rsolweig.gvf_2018a

    def calc_wrap(*args, **kwargs):
        r = orig_calc(*args, **kwargs)
        names = ("Tmrt", "Kdown", "Kup", "Ldown", "Lup", "Tg", "ea", "esky", "I0", "CI", "shadow",
                 "firstdaytime", "timestepdec", "timeadd", "Tgmap1", "Tgmap1E", "Tgmap1S",
                 "Tgmap1W", "Tgmap1N", "Keast", "Ksouth", "Kwest", "Knorth", "Least", "Lsouth",
                 "Lwest", "Lnorth", "KsideI", "TgOut1", "TgOut", "radI", "radD", "Lside",
                 "L_patches", "CI_Tg", "CI_TgG", "KsideD", "dRad", "Kside")
        captured.append(dict(zip(names, r)))
        return r

    def gvf_wrap(*args, **kwargs):
        r = orig_gvf(*args, **kwargs)
        gvf_captured.append((len(captured), r))
        return r

    rup.Solweig_2022a_calc = calc_wrap
    rsolweig.gvf_2018a = gvf_wrap
    try:
        lc_class = np.loadtxt(os.path.join(ref, "solweig_gpu", "landcoverclasses_2016a.txt"),
                              skiprows=1, usecols=range(1, 7))
        t0 = time.time()
        outputs, final_state = rup.run_utci_window(
            a=a, temp1=torch.tensor(city.trees), temp2=temp2, walls=walls_t, dirwalls=dirwalls_t,
            svf_bundle=bundle, met_file=met, altitude=altitude, azimuth=azimuth, zen=zen,
            jday=jday, dectime=dectime, altmax=altmax, location=loc, scale=scale,
            amaxvalue=amaxvalue, landcover_grid=torch.tensor(city.landcover), lc_class=lc_class,
            requested_variables=("utci", "tmrt", "kup", "kdown", "lup", "ldown", "shadow", "ta", "wind"),
            return_final_state=True)
        print(f"[{name}] run_utci_window {time.time() - t0:.1f}s", flush=True)
    finally:
        rup.Solweig_2022a_calc = orig_calc
        rsolweig.gvf_2018a = orig_gvf

    out["lc_class"] = lc_class
    for k, v in outputs.items():
        out["out_" + k] = v
    for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1"):
        out["final_" + k] = _np(final_state[k]).astype(np.float32)
    for k in ("CI", "firstdaytime", "timeadd"):
        out["final_" + k] = np.float64(final_state[k])
    out["final_Twater"] = np.float64(np.nan if final_state["Twater"] is None else final_state["Twater"])
    T = met.shape[0]
    for k in STEP_PLANES:
        planes = []
        for c in captured:
            v = _np(c[k]).astype(np.float32)
            planes.append(np.broadcast_to(v, (rows, cols)).copy())
        out["step_" + k] = np.stack(planes)
    for k in STEP_SCALARS:
        out["step_" + k] = np.array([float(_np(c[k]).reshape(-1)[0]) if np.size(_np(c[k])) else np.nan
                                     for c in captured], np.float64)
    lp = np.zeros((T, 153, 3), np.float32)
    for i, c in enumerate(captured):
        if c["L_patches"] is not None:
            lp[i] = _np(c["L_patches"]).astype(np.float32)
    out["step_L_patches"] = lp
    gsteps = []
    gvals = {k: [] for k in GVF_NAMES}
    for idx, r in gvf_captured:
        gsteps.append(idx)
        for k, v in zip(GVF_NAMES, r):
            gvals[k].append(_np(v).astype(np.float32))
    out["gvf_steps"] = np.array(gsteps, np.int32)
    for k, v in gvals.items():
        out["gvf_" + k] = np.stack(v)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="reference checkout (or $SOLWEIG_REFERENCE)")
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    args = ap.parse_args()
    args.ref = reference_path(args.ref)
    install_stubs(args.ref)
    import torch
    torch.set_num_threads(max(1, os.cpu_count() or 1))
    for name in args.cases:
        data = run_case(name, CASES[name], args.ref)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"wrote {path} ({os.path.getsize(path) / 1e6:.2f} MB)", flush=True)


if __name__ == "__main__":
    main()
