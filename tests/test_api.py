"""Drop-in API and the solweig_core-style seam.

CPU tests cover argument validation and dispatch (they raise before any GPU
work); GPU tests run the drop-ins against the reference goldens."""
import dataclasses

import numpy as np
import pytest

from conftest import golden_location, load_golden
from golden_util import assert_bits_equal, max_abs

from solweig_project_b200 import api
from solweig_project_b200.core import (ArrayView, DispatchBlockedError, PhysicalWindow, RefusalReason,
                                       RequestValidationError, SolveRequestView, StaleBufferError, TimeCoverage)
from solweig_project_b200.core.dispatch import BACKEND_EXACT_CHAIN, resolve


def _request(**kw):
    base = dict(logical_domain_id="site", rows=10, cols=12, origin_x_m=0.0, origin_y_m=0.0, pixel_size_m=1.0,
                read_window=PhysicalWindow(0, 10, 0, 12), write_window=PhysicalWindow(2, 8, 3, 9),
                time=TimeCoverage(0, 24, 24), profile_id="b200")
    base.update(kw)
    return SolveRequestView(**base)


def test_cuda_request_resolves_to_the_exact_chain():
    res = resolve(_request())
    assert res.ready and res.plan.backend == BACKEND_EXACT_CHAIN and res.plan.device == "cuda"


def test_cpu_request_is_refused_not_retargeted():
    res = resolve(_request(device="cpu"))
    assert not res.ready and res.plan is None
    assert res.refusal.reason is RefusalReason.UNSUPPORTED_DEVICE
    with pytest.raises(DispatchBlockedError):
        res.raise_if_blocked()


def test_unknown_backend_preference_is_refused():
    res = resolve(_request(), prefer_backend="numba-full-solve")
    assert res.refusal.reason is RefusalReason.UNKNOWN_BACKEND


@pytest.mark.parametrize("bad", [
    dict(write_window=PhysicalWindow(0, 11, 0, 12)),
    dict(read_window=PhysicalWindow(3, 8, 3, 9), write_window=PhysicalWindow(2, 8, 3, 9)),
    dict(time=TimeCoverage(5, 30, 24)),
    dict(rows=0),
    dict(profile_id=""),
    dict(device="tpu"),
])
def test_request_validation_refuses(bad):
    with pytest.raises(RequestValidationError) as err:
        _request(**bad).validate()
    assert err.value.refusal.reason is RefusalReason.REQUEST_INVALID


def test_frozen_view_detects_mutation():
    a = np.zeros((4, 4), np.float32)
    v = ArrayView.from_numpy(a, freeze=True, logical_domain_id="site")
    v.assert_not_mutated()
    a[1, 1] = 2
    with pytest.raises(StaleBufferError):
        v.assert_not_mutated()


def test_run_utci_window_validates_before_gpu_work():
    d = load_golden("city36")
    common = dict(a=d["dsm"], temp1=d["trees"].copy(), temp2=d["dem"], walls=d["walls_ref"],
                  dirwalls=d["aspect_ref"], svf_bundle=(), met_file=d["met"], altitude=d["altitude"],
                  azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"], dectime=d["dectime"], altmax=d["altmax"],
                  location=golden_location(d), scale=1.0)
    with pytest.raises(ValueError, match="unknown requested variables"):
        api.run_utci_window(**common, requested_variables=("utci", "wbgt"))
    with pytest.raises(ValueError, match="invalid time range"):
        api.run_utci_window(**common, time_start=4, time_stop=2)
    with pytest.raises(ValueError, match="out_window"):
        api.run_utci_window(**common, out_window=(0, 99, 0, 5))
    with pytest.raises(ValueError, match="requires out_window"):
        api.run_utci_window(**common, svf_bundle_cubes_cropped=True)
    with pytest.raises(ValueError, match="unknown model parameters"):
        api.run_utci_window(**common, model_parameters={"albedo": 0.3})


def test_svf_calculator_requires_its_inputs():
    with pytest.raises(ValueError, match="must be provided"):
        api.svf_calculator(2, amaxvalue=10.0, a=np.zeros((4, 4), np.float32))


@pytest.mark.gpu
def test_dropins_against_reference(cuda):
    d = load_golden("city36")
    import torch
    from oracle.svf import scene_from_rasters
    vegdsm, vegdsm2, bush, amax = scene_from_rasters(d["dsm"], d["trees"], d["dem"])
    bundle = api.svf_calculator(2, amax, d["dsm"], vegdsm, vegdsm2, bush, 1.0)
    names = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS", "svfSaveg",
             "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg", "vegshmat", "vbshvegshmat", "shmat", "svftotal")
    for name, v in zip(names, bundle):
        assert isinstance(v, torch.Tensor) and v.is_cuda
        assert_bits_equal(v.cpu().numpy(), d["svf_" + name].astype(np.float32), name)
    kw = dict(a=d["dsm"], temp1=d["trees"].copy(), temp2=d["dem"], walls=d["walls_ref"], dirwalls=d["aspect_ref"],
              met_file=d["met"], altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"],
              dectime=d["dectime"], altmax=d["altmax"], location=golden_location(d), scale=1.0,
              amaxvalue=d["amaxvalue"], landcover_grid=d["landcover"], lc_class=d["lc_class"],
              requested_variables=("utci", "tmrt", "shadow", "ta", "wind"))
    # the dense 19-tuple, as the reference returns it
    out, final = api.run_utci_window(svf_bundle=bundle, return_final_state=True, **kw)
    assert_bits_equal(out["shadow"], d["out_shadow"], "shadow")
    assert_bits_equal(out["ta"], d["out_ta"], "ta")
    assert_bits_equal(out["wind"], d["out_wind"], "wind")
    assert max_abs(out["tmrt"], d["out_tmrt"]) <= 1e-3
    assert max_abs(out["utci"], d["out_utci"]) <= 1e-3
    assert final["CI"] == float(d["final_CI"]) and final["next_step"] == 24
    # the packed form gives the same numbers
    packed = api.svf_calculator(2, amax, d["dsm"], vegdsm, vegdsm2, bush, 1.0, packed=True)
    out2 = api.run_utci_window(svf_bundle=packed, **dict(kw, temp1=d["trees"].copy()))
    assert_bits_equal(out2["shadow"], out["shadow"], "packed shadow")
    assert max_abs(out2["tmrt"], out["tmrt"]) <= 1e-4
    # warm start at step 10 resumes the cold trajectory
    first, state = api.run_utci_window(svf_bundle=packed, time_stop=10, return_final_state=True,
                                       **dict(kw, temp1=d["trees"].copy()))
    rest = api.run_utci_window(svf_bundle=packed, time_start=10, initial_state=state,
                               **dict(kw, temp1=d["trees"].copy()))
    assert max_abs(rest["tmrt"], out2["tmrt"][10:]) <= 1e-4
    with pytest.raises(ValueError, match="next_step"):
        api.run_utci_window(svf_bundle=packed, time_start=11, initial_state=state,
                            **dict(kw, temp1=d["trees"].copy()))
    # out_window crops the full-window result
    win = api.run_utci_window(svf_bundle=packed, out_window=(5, 30, 2, 20), **dict(kw, temp1=d["trees"].copy()))
    assert_bits_equal(win["shadow"], out["shadow"][:, 5:30, 2:20], "window shadow")


@pytest.mark.gpu
def test_water_temperature_and_warm_start_against_reference(cuda):
    """final_state["Twater"] is the reference's (utci_process.py:917-922,
    1085) and a warm start carries it."""
    d = load_golden("city36")
    bundle = tuple(d["svf_" + k].astype(np.float32) for k in
                   ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS",
                    "svfSaveg", "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg", "vegshmat", "vbshvegshmat",
                    "shmat", "svftotal"))
    kw = dict(a=d["dsm"], temp2=d["dem"], walls=d["walls_ref"], dirwalls=d["aspect_ref"], svf_bundle=bundle,
              met_file=d["met"], altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"],
              dectime=d["dectime"], altmax=d["altmax"], location=golden_location(d), scale=1.0,
              amaxvalue=d["amaxvalue"], landcover_grid=d["landcover"], lc_class=d["lc_class"],
              requested_variables=("utci", "tmrt"))
    out, final = api.run_utci_window(temp1=d["trees"].copy(), return_final_state=True, **kw)
    assert final["Twater"] == float(d["final_Twater"])
    assert max_abs(out["tmrt"], d["out_tmrt"]) <= 1e-3
    first, state = api.run_utci_window(temp1=d["trees"].copy(), time_stop=7, return_final_state=True, **kw)
    assert state["Twater"] == float(d["final_Twater"])      # established at the first (midnight) row
    state["Twater"] = None
    rest, final2 = api.run_utci_window(temp1=d["trees"].copy(), time_start=7, initial_state=state,
                                       return_final_state=True, **kw)
    assert final2["Twater"] is None                         # no midnight row in 7..23: stays unestablished
    assert max_abs(rest["tmrt"], out["tmrt"][7:]) <= 1e-4
    # without land cover the reference never establishes it
    nolc = dict(kw, landcover_grid=None, lc_class=None)
    _, f3 = api.run_utci_window(temp1=d["trees"].copy(), return_final_state=True, **nolc)
    assert f3["Twater"] is None


@pytest.mark.gpu
def test_pre_cropped_cube_bundle(cuda):
    """svf_bundle_cubes_cropped=True (the solver's mode,
    incremental/solver.py:2080; utci_process.py:651-663): cubes cut to the
    write window give the window of the full-bundle run bit for bit, and the
    reference's outputs there within the tolerances."""
    d = load_golden("city36")
    names = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS", "svfSaveg",
             "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg", "vegshmat", "vbshvegshmat", "shmat", "svftotal")
    full = tuple(d["svf_" + k].astype(np.float32) for k in names)
    w = (5, 30, 2, 20)
    cropped = full[:15] + tuple(c[w[0]:w[1], w[2]:w[3], :] for c in full[15:18]) + full[18:]
    kw = dict(a=d["dsm"], temp2=d["dem"], walls=d["walls_ref"], dirwalls=d["aspect_ref"], met_file=d["met"],
              altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"], dectime=d["dectime"],
              altmax=d["altmax"], location=golden_location(d), scale=1.0, amaxvalue=d["amaxvalue"],
              landcover_grid=d["landcover"], lc_class=d["lc_class"], out_window=w,
              requested_variables=("utci", "tmrt", "shadow", "kdown", "lup"))
    a = api.run_utci_window(temp1=d["trees"].copy(), svf_bundle=full, **kw)
    b = api.run_utci_window(temp1=d["trees"].copy(), svf_bundle=cropped, svf_bundle_cubes_cropped=True, **kw)
    sl = (slice(None), slice(w[0], w[1]), slice(w[2], w[3]))
    for k in a:
        assert b[k].shape == (24, w[1] - w[0], w[3] - w[2])
        assert_bits_equal(b[k], a[k], f"cropped {k}")
    assert_bits_equal(b["shadow"], d["out_shadow"][sl], "shadow vs reference")
    assert max_abs(b["tmrt"], d["out_tmrt"][sl]) <= 1e-3
    assert max_abs(b["utci"], d["out_utci"][sl]) <= 1e-3
    with pytest.raises(ValueError, match="do not cover"):
        api.run_utci_window(temp1=d["trees"].copy(), svf_bundle=full, svf_bundle_cubes_cropped=True, **kw)


def _utci_f64(ta, rh, tmrt, va):
    """UTCI of calculate_utci.py:259-330 re-evaluated in float64 (the float32
    regression coefficients, every other operation in double), with the
    largest magnitude the running sum `Ta + t_0 + ... + t_j` reaches."""
    from oracle.radiation import _utci_terms
    ta, rh, tmrt, va = (np.asarray(x, np.float64) for x in (ta, rh, tmrt, va))
    g = [-2.8365744E3, -6.028076559E3, 1.954263612E1, -2.737830188E-2, 1.6261698E-5, 7.0229056E-10,
         -1.8680009E-13, 2.7150305]
    tk = ta + 273.15
    es = g[7] * np.log(tk) + sum(g[i] * tk ** (i - 2.0) for i in range(7))
    pa = np.exp(es) * 0.01 * rh / 100.0 / 10.0
    d = tmrt - ta
    acc = ta.copy()
    peak = np.abs(acc)
    for c, pt, pv, pd, pp in _utci_terms():
        acc = acc + float(c) * ta ** pt * va ** pv * d ** pd * pa ** pp
        peak = np.maximum(peak, np.abs(acc))
    return acc, peak


@pytest.mark.gpu
def test_utci_calculator_against_oracle(cuda):
    """The standalone UTCI against the oracle's float32 evaluation.

    The 210-term sum is ill-conditioned for windy, hot inputs: its running
    sum reaches ~1e4 while the result is ~10-50, so a one-ulp difference in
    one float32 power (torch's vectorised pow is not correctly rounded)
    moves the result by ulp(running sum).  Each value must be within 1e-3 C
    of the oracle or within 4 ulp of its largest running sum, and the
    device's error against a float64 re-evaluation may not exceed the
    oracle's own by more than that bound."""
    from oracle.radiation import utci_calculator as oracle_utci
    rng = np.random.default_rng(0)
    n = 20000
    ta = rng.uniform(-20, 45, n).astype(np.float32)
    rh = rng.uniform(5, 100, n).astype(np.float32)
    tmrt = (ta + rng.uniform(-10, 40, n)).astype(np.float32)
    va = rng.uniform(0.5, 15, n).astype(np.float32)
    ta[:5] = -999.0
    got = api.utci_calculator(ta, rh, tmrt, va).cpu().numpy()
    want = oracle_utci(ta, rh, tmrt, va)
    assert (got[:5] == -999).all()
    got, want = got[5:].astype(np.float64), want[5:].astype(np.float64)
    exact, peak = _utci_f64(ta[5:], rh[5:], tmrt[5:], va[5:])
    bound = np.maximum(1e-3, 4 * np.spacing(peak.astype(np.float32)).astype(np.float64))
    diff = np.abs(got - want)
    assert (diff <= bound).all(), f"worst excess {float((diff - bound).max())}"
    assert (np.abs(got - exact) <= np.abs(want - exact) + bound).all()
    # calm, mild conditions (the chain's usual range) stay within 1e-3 C
    calm = (va[5:] <= 4) & (ta[5:] <= 35)
    assert diff[calm].max() <= 1e-3


def test_recompute_utci_steps_validates_like_the_reference():
    d = load_golden("city36")
    planes = {0: np.zeros((36, 36), np.float32)}
    with pytest.raises(ValueError, match="non-empty"):
        api.recompute_utci_steps(d["met"], [], planes, d["dsm"], d["dem"])
    with pytest.raises(ValueError, match="outside the met table"):
        api.recompute_utci_steps(d["met"], [99], planes, d["dsm"], d["dem"])
    with pytest.raises(ValueError, match="no published tmrt plane"):
        api.recompute_utci_steps(d["met"], [0, 1], planes, d["dsm"], d["dem"])
    with pytest.raises(ValueError, match="shape"):
        api.recompute_utci_steps(d["met"], [0], {0: np.zeros((5, 5), np.float32)}, d["dsm"], d["dem"])
    with pytest.raises(ValueError, match="dem shape"):
        api.recompute_utci_steps(d["met"], [0], planes, d["dsm"], d["dem"][:5])


@pytest.mark.gpu
def test_recompute_utci_steps_equals_a_full_run(cuda):
    """Wind speed and urban heat island enter only the UTCI tail: the
    fast path from the first run's Tmrt equals a full run with the edited
    forcing, bit for bit."""
    from oracle.svf import scene_from_rasters
    d = load_golden("city36")
    vegdsm, vegdsm2, bush, amax = scene_from_rasters(d["dsm"], d["trees"], d["dem"])
    packed = api.svf_calculator(2, amax, d["dsm"], vegdsm, vegdsm2, bush, 1.0, packed=True)
    kw = dict(a=d["dsm"], temp2=d["dem"], walls=d["walls_ref"], dirwalls=d["aspect_ref"], svf_bundle=packed,
              altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"], dectime=d["dectime"],
              altmax=d["altmax"], location=golden_location(d), scale=1.0, amaxvalue=d["amaxvalue"],
              landcover_grid=d["landcover"], lc_class=d["lc_class"], requested_variables=("utci", "tmrt"))
    base = api.run_utci_window(temp1=d["trees"].copy(), met_file=d["met"], **kw)
    met2 = np.array(d["met"], copy=True)
    if met2.shape[1] <= 24:
        met2 = np.concatenate([met2, np.zeros((met2.shape[0], 25 - met2.shape[1]))], axis=1)
    met2[:, 9] = met2[:, 9] * 1.7 + 0.3          # wind speed
    met2[:, 24] = 1.25                            # urban heat island
    edited = api.run_utci_window(temp1=d["trees"].copy(), met_file=met2, **kw)
    assert_bits_equal(edited["tmrt"], base["tmrt"], "tmrt unchanged by wind / uhii")
    idx = [3, 11, 12, 20]
    fast = api.recompute_utci_steps(met2, idx, {i: base["tmrt"][i] for i in idx}, d["dsm"], d["dem"])
    assert_bits_equal(fast, edited["utci"][idx], "utci fast path")
    # against the CPU oracle (the reference's chain restated) run with the edited forcing
    from oracle import window as ow
    names = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS", "svfSaveg",
             "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg", "vegshmat", "vbshvegshmat", "shmat", "svftotal")
    want = ow.run_utci_window(a=d["dsm"], temp1=d["trees"], temp2=d["dem"], walls=d["walls_ref"],
                              dirwalls=d["aspect_ref"], svf_bundle=tuple(d["svf_" + k].astype(np.float32)
                                                                          for k in names),
                              met_file=met2, altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"],
                              jday=d["jday"], dectime=d["dectime"], altmax=d["altmax"],
                              location=golden_location(d), scale=1.0, amaxvalue=d["amaxvalue"],
                              landcover_grid=d["landcover"], lc_class=d["lc_class"], requested_variables=("utci",))
    assert max_abs(fast, want["utci"][idx]) <= 1e-3


def test_svf_calculator_save_rasters_argument_checks(tmp_path):
    z = np.zeros((4, 4), np.float32)
    with pytest.raises(ValueError, match="output_dir must be provided"):
        api.svf_calculator(2, 1.0, z, z, z, z, 1.0, save_rasters=True)
    with pytest.raises(ValueError, match="gdal_dsm or building_dsm_path"):
        api.svf_calculator(2, 1.0, z, z, z, z, 1.0, save_rasters=True, output_dir=str(tmp_path))
    with pytest.raises(ValueError, match="building_dsm_path, tree_path, and dem_path"):
        api.svf_calculator(2, save_rasters=True, output_dir=str(tmp_path), building_dsm_path="x.tif")


@pytest.mark.gpu
def test_svf_calculator_writes_the_reference_cache(cuda, tmp_path):
    """save_rasters=True (shadow.py:100-164, 444-487): the cache it writes
    holds the reference's planes and cubes bit for bit, georeferenced; the
    standalone form reads the three rasters and gives the same cache."""
    from solweig_project_b200 import formats as FM
    d = load_golden("city36")
    from oracle.svf import scene_from_rasters
    vegdsm, vegdsm2, bush, amax = scene_from_rasters(d["dsm"], d["trees"], d["dem"])
    gt = (600000.0, 1.0, 0.0, 3300000.0, 0.0, -1.0)
    api.svf_calculator(2, amax, d["dsm"], vegdsm, vegdsm2, bush, 1.0, save_rasters=True,
                       output_dir=str(tmp_path / "a"), number="0_0", gdal_dsm=gt)
    for name, tif in (("Building_DSM.tif", d["dsm"]), ("Trees.tif", d["trees"]), ("DEM.tif", d["dem"])):
        with open(tmp_path / name, "wb") as fh:
            fh.write(FM.tiff_bytes(tif, gt, epsg=32614))
    api.svf_calculator(2, save_rasters=True, output_dir=str(tmp_path / "b"), number="0_0",
                       building_dsm_path=str(tmp_path / "Building_DSM.tif"), tree_path=str(tmp_path / "Trees.tif"),
                       dem_path=str(tmp_path / "DEM.tif"))
    for sub in ("a", "b"):
        planes, (sh, veg, vb) = FM.read_svf_cache(str(tmp_path / sub), number="0_0")
        for k, v in planes.items():
            assert_bits_equal(v, d["svf_" + k], f"{sub} {k}")
        assert_bits_equal(sh, d["svf_shmat"].astype(np.float32), "shmat")
        assert_bits_equal(veg, d["svf_vegshmat"].astype(np.float32), "vegshmat")
        assert_bits_equal(vb, d["svf_vbshvegshmat"].astype(np.float32), "vbshvegshmat")
        assert FM.svf_cache_extent_matches((36, 36), gt, str(tmp_path / sub), number="0_0")
