"""Host-side tables and input preparation (no GPU): march step tables, patch
layout, predicate bounds, the walls/aspect restatement, the per-step scalars
and the C struct layouts shared with the library."""
import os
import subprocess

import numpy as np
import pytest
import torch

from conftest import FULL_CASES, REPO, golden_location, load_golden

from oracle import march as om
from oracle import svf as osvf
from solweig_project_b200 import _native as N
from solweig_project_b200 import tables as T
from solweig_project_b200 import timeseries as TS
from solweig_project_b200.walls_aspect import filter1Goodwin_as_aspect_v3, findwalls


def test_patch_layout_matches_oracle():
    assert np.array_equal(T.sweep_azimuths(), osvf.patch_azimuths())
    alt, azi = T.sky_patches()
    a2, z2 = osvf.create_patches(2)[:2]
    assert np.array_equal(alt, a2) and np.array_equal(azi, z2)
    # the reference's band count truncation leaves the last sweep azimuths at 0
    assert (T.sweep_azimuths()[-4:] == 0).all()


@pytest.mark.parametrize("seed", [0, 1])
def test_step_tables_match_oracle(seed):
    rng = np.random.default_rng(seed)
    _, altint, _, nband = T.PATCH_LAYOUT[2]
    azs = T.sweep_azimuths()
    for _ in range(3):
        rows, cols = int(rng.integers(1, 300)), int(rng.integers(1, 300))
        scale = float(rng.choice([1.0, 0.5, 2.0]))
        amax = float(rng.uniform(1, 120))
        q = 0
        for i in range(len(altint)):
            for _ in range(nband[i]):
                got = T.svf_patch_table(azs[q], altint[i], scale, amax, rows, cols)
                want = osvf.shadow_step_table(azs[q], altint[i], scale, amax, rows, cols)
                for g, w in zip(got, want):
                    assert np.array_equal(g, w)
                q += 1
        for _ in range(10):
            az, al = float(rng.uniform(0, 360)), float(rng.uniform(0.3, 89.9))
            got = T.sun_table(az, al, scale, amax, rows, cols)
            want = om.sun_step_table(az, al, scale, amax, rows, cols)
            for g, w in zip(got[:3], want[:3]):
                assert np.array_equal(g, w)
            assert got[3] == want[3]


@pytest.mark.parametrize("palt", [5.9999995, 6.0, 17.999998, 30.0, 42.000004, 54.0, 66.0, 78.0, 89.99999, 90.0])
def test_atan_bounds_reproduce_predicate(palt):
    lo, hi = T.atan_degree_bounds(palt)
    rng = np.random.default_rng(7)
    x0 = np.float32(np.tan(np.deg2rad(palt)))
    x = np.concatenate([x0 + np.linspace(-2e-5, 2e-5, 40001), rng.uniform(-50, 50, 100000),
                        [lo, hi, np.nextafter(lo, -np.inf), np.nextafter(hi, np.inf)]]).astype(np.float32)
    x = x[np.isfinite(x)]
    deg = (torch.atan(torch.from_numpy(x)) * (180.0 / torch.pi)).numpy()
    assert np.array_equal(deg < np.float32(palt), x < lo)
    assert np.array_equal(deg > np.float32(palt), x > hi)


@pytest.mark.parametrize("case", FULL_CASES)
def test_walls_aspect_restatement(case):
    d = load_golden(case)
    w = findwalls(d["dsm"], 3.0)
    assert np.array_equal(w, d["walls_ref64"])
    a = filter1Goodwin_as_aspect_v3(w, float(d["scale"]), d["dsm"])
    assert np.array_equal(a, d["aspect_ref64"])


@pytest.mark.parametrize("case", FULL_CASES)
def test_series_scalars_match_reference(case):
    d = load_golden(case)
    rows, cols = d["dsm"].shape
    props = TS.landcover_props(d["landcover"], d["lc_class"], rows, cols)
    ser = TS.build_series(met_file=d["met"], altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"],
                          jday=d["jday"], dectime=d["dectime"], altmax=d["altmax"], location=golden_location(d),
                          scale=float(d["scale"]), amax=float(d["amaxvalue"]), rows=rows, cols=cols, props=props)
    day = ser.steps["is_day"] == 1
    assert np.array_equal(day, d["altitude"][0] > 0)
    assert np.array_equal(ser.steps["radI"][day], d["step_radI"][day].astype(np.float32))
    assert np.array_equal(ser.steps["radD"][day], d["step_radD"][day].astype(np.float32))
    assert np.array_equal(ser.steps["cig"][day], d["step_CI_TgG"][day].astype(np.float32))
    assert ser.final["CI"] == float(d["final_CI"])
    assert ser.final["timeadd"] == float(d["final_timeadd"])
    assert ser.final["firstdaytime"] == float(d["final_firstdaytime"])
    assert len(ser.sun) == len(d["march_steps"])
    assert np.array_equal(ser.sun["t"], d["march_steps"])
    # Perez luminance of the patches reaches the kernel through anilum[sh=1, veg=1]
    lp = d["step_L_patches"]
    assert np.array_equal(ser.patch["anilum"][day][:, :, 3], lp[day][:, :, 2])


def test_struct_layouts_match_c_header(tmp_path):
    src = tmp_path / "layout.c"
    names = list(N.EXPECTED_SIZES)
    body = "".join(f'printf("%zu\\n", sizeof({n}));' for n in names)
    body += 'printf("%zu\\n", sizeof(sw100_site_planes)); printf("%zu\\n", sizeof(sw100_series));'
    body += ('printf("%zu\\n", sizeof(sw100_batch_site)); printf("%zu\\n", offsetof(sw100_batch_site, skipmap));'
             'printf("%zu\\n", sizeof(sw100_class_table)); printf("%zu\\n", sizeof(sw100_site_stats));'
             'printf("%zu\\n", sizeof(sw100_tile));')
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "solweig_b200.h"\nint main(void){' + body +
                   'return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    import ctypes
    for n, s in zip(names, sizes):
        assert N.DTYPES[n].itemsize == s == N.EXPECTED_SIZES[n], n
    assert sizes[len(names)] == ctypes.sizeof(N.SitePlanes)
    assert sizes[len(names) + 1] == ctypes.sizeof(N.Series)
    from solweig_project_b200 import batch as B
    bs, skip_off, ct, st, tile = sizes[len(names) + 2:len(names) + 7]
    assert bs == ctypes.sizeof(B.BatchSite) and skip_off == B.BatchSite.skipmap.offset
    assert ct == ctypes.sizeof(N.ClassTable)
    assert st == 4 * N.SITE_STATS_WORDS
    assert tile == B.TILE_DTYPE.itemsize


def _series_step(pa_pows, k, ta, va, d):
    """The device's per-step UTCI sum (csrc/utci_series.cuh utci_series_step)
    restated in numpy float32."""
    from oracle.radiation import _utci_terms
    vp = [None] + [np.array([TS.utci_pow(x, p) for x in va], np.float32) for p in range(1, 7)]
    dp = [None] + [np.array([TS.utci_pow(x, p) for x in d], np.float32) for p in range(1, 7)]
    acc = np.full(va.shape, ta, np.float32)
    for j, (_, pt, pv, pd, pp) in enumerate(_utci_terms()):
        t = np.full(va.shape, k[j], np.float32)
        if pv:
            t = t * vp[pv]
        if pd:
            t = t * dp[pd]
        if pp:
            t = t * pa_pows[pp - 1]
        acc = acc + t
    return acc


def test_utci_step_table_reproduces_the_reference_sum():
    """The per-step table (Pa powers, c * Ta^pt per term) gives the
    reference's float32 running sum: bit-equal on most pixels, and within
    1e-3 C everywhere at the chain's wind speeds."""
    from oracle.radiation import utci_calculator
    rng = np.random.default_rng(3)
    for ta, rh in ((np.float32(31.7), np.float32(48.0)), (np.float32(24.25), np.float32(70.0)),
                   (np.float32(36.0), np.float32(35.0))):
        pa_pows, k = TS._utci_table(ta, rh)
        assert pa_pows.dtype == np.float32 and k.shape == (210,)
        tmrt = rng.uniform(15, 75, 3000).astype(np.float32)
        va = rng.uniform(0.15, 6, 3000).astype(np.float32)
        want = utci_calculator(np.full(3000, ta, np.float32), np.full(3000, rh, np.float32), tmrt, va)
        got = _series_step(pa_pows, k, ta, va, (tmrt - ta).astype(np.float32))
        assert np.abs(got.astype(np.float64) - want).max() <= 1e-3
        assert (got == want).mean() >= 0.9


def test_utci_vapour_pressure_matches_the_reference_chain():
    """Pa of calculate_utci.py:273-282: float32, log / exp rounded once."""
    import torch
    ta = np.linspace(-30, 50, 4001).astype(np.float32)
    rh = np.float32(55.0)
    tk = torch.from_numpy(ta + np.float32(273.15))
    g = torch.tensor([-2.8365744E3, -6.028076559E3, 1.954263612E1, -2.737830188E-2,
                      1.6261698E-5, 7.0229056E-10, -1.8680009E-13, 2.7150305], dtype=torch.float32)
    es = g[7] * torch.log(tk)
    for i in range(0, 7):
        es = es + g[i] * tk ** (i + 1 - 3.)
    want = ((torch.exp(es) * 0.01) * float(rh) / 100. / 10.0).numpy()
    got = np.array([TS.utci_vapour_pressure(t, rh) for t in ta], np.float32)
    rel = np.abs(got.astype(np.float64) - want) / np.abs(want)
    assert rel.max() <= 4e-7 and (got == want).mean() >= 0.95
