"""The series builder evaluates the daytime scalar chain for all daytime
steps at once (timeseries._day_chain); every value must equal the 0-dim,
step-by-step evaluation of the reference's helpers bit for bit, dtype and
sign of zero included, across the branches (missing Ta / RH / pressure,
the three clearness regimes of the diffuse split, radD <= 10, sun below
10 degrees and below 1 degree, every Perez clearness bin)."""
import numpy as np
import pytest
import torch

from solweig_project_b200 import timeseries as TS


def _same(a, b):
    a = torch.as_tensor(a).double().reshape(-1)
    b = torch.as_tensor(b).double().reshape(-1)
    return bool((((a == b) | (torch.isnan(a) & torch.isnan(b))) & (torch.signbit(a) == torch.signbit(b))).all())


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_day_chain_equals_stepwise_helpers(seed):
    rng = np.random.default_rng(seed)
    n = 160
    alt = rng.uniform(0.01, 89, n)
    alt[:12] = rng.uniform(0.01, 1.5, 12)
    met = np.zeros((n, 25))
    met[:, 11] = rng.uniform(-20, 45, n)
    met[::37, 11] = -999.0
    met[5, 11] = np.nan
    met[:, 10] = rng.uniform(5, 100, n)
    met[::41, 10] = -999.0
    met[:, 14] = rng.uniform(0, 1100, n)
    met[::7, 14] = rng.uniform(0, 15, len(met[::7, 14]))
    met[:, 12] = rng.uniform(90, 105, n)
    met[::5, 12] = -999.0
    altitude = alt[None, :]
    zen = np.radians(90 - alt + rng.normal(0, 0.01, n))[None, :]
    azimuth = rng.uniform(0, 360, n)[None, :]
    jday = rng.integers(1, 366, n).astype(np.float64)[None, :]
    lat = float(rng.uniform(-60, 89))
    days = list(range(n))
    with torch.inference_mode():
        dc = TS._day_chain(days, met, altitude, azimuth, zen, jday, lat)
        bins = set()
        for d, i in enumerate(days):
            Ta, RH, radG = met[i, 11], met[i, 10], met[i, 14]
            jd = jday[0][i]
            snup = TS._snup(torch.tensor(jd.item()), torch.tensor(lat))
            I0, CI, Kt = TS._clearness(torch.tensor(zen[0][i].item()), torch.tensor(jd.item()), Ta.item(),
                                       torch.tensor(RH.item()) / 100., torch.tensor(radG.item()), lat,
                                       torch.tensor(met[i, 12].item()))
            radI, radD = TS._diffuse(torch.tensor(radG.item()), torch.tensor(alt[i].item()), Kt,
                                     torch.tensor(Ta.item()), torch.tensor(RH.item()))
            radI0, radD0 = TS._diffuse(I0, alt[i].item(), 1., Ta.item(), RH.item())
            for name, want in (("snup", snup), ("I0", I0), ("CI", CI), ("Kt", Kt), ("radI", radI), ("radD", radD),
                               ("radI0", radI0), ("radD0", radD0)):
                got = dc[name][d]
                assert got.dtype == want.dtype and _same(got, want), (seed, i, name, got, want)
            zen_deg = (torch.tensor(zen[0][i]) * (180 / np.pi)).item()
            lv = TS._perez(zen_deg, azimuth[0][i].item(), radD, radI, jd.item())
            assert dc["lv"][d] is not None
            assert torch.equal(lv.view(torch.int32), dc["lv"][d].view(torch.int32)), (seed, i, "lv")
            bins.add(float(radD) <= 10)
        assert bins == {True, False}


@pytest.mark.parametrize("chunk", [1, 5, 7])
def test_chunked_series_equal_one_build(chunk):
    """Building a day in chunks (carried scalars passed on, one day chain for
    the whole window) gives the tables of one build: only the daytime-row
    numbering restarts in each chunk."""
    from conftest import load_golden, golden_location
    from solweig_project_b200.engine import march_inputs
    d = load_golden("city36")
    rows, cols = d["dsm"].shape
    props = TS.landcover_props(d["landcover"], d["lc_class"], rows, cols)
    kw = dict(met_file=d["met"], altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"],
              dectime=d["dectime"], altmax=d["altmax"], location=golden_location(d), scale=float(d["scale"]),
              amax=march_inputs(d["dsm"], d["trees"], d["dem"])[3], rows=rows, cols=cols, props=props)
    full = TS.build_series(**kw)
    dc = TS.day_chain(d["met"], d["altitude"], d["azimuth"], d["zen"], d["jday"], golden_location(d))
    n, sc, parts = d["met"].shape[0], None, []
    for t0 in range(0, n, chunk):
        s = TS.build_series(**kw, time_start=t0, time_stop=min(n, t0 + chunk), initial_scalars=sc, day_chain=dc)
        sc = s.final
        parts.append(s)
    a, b = full.steps.copy(), np.concatenate([p.steps for p in parts])
    a["day_row"] = 0
    b["day_row"] = 0
    assert a.tobytes() == b.tobytes()
    assert full.patch.tobytes() == np.concatenate([p.patch for p in parts]).tobytes()
    assert full.sun_table.tobytes() == np.concatenate([p.sun_table for p in parts]).tobytes()
    assert full.final == sc


@pytest.mark.parametrize("scale,amax,rows,cols", [(1.0, 40.0, 500, 500), (0.5, 12.0, 36, 80), (2.0, 120.0, 300, 100)])
def test_sun_tables_equal_one_step_form(scale, amax, rows, cols):
    from solweig_project_b200 import tables as T
    rng = np.random.default_rng(3)
    az = rng.uniform(0, 360, 120).tolist() + [0.0, 90.0, 180.0, 270.0, 359.999, 45.0, 135.0, 225.0, 315.0]
    alt = rng.uniform(0.5, 89, len(az)).tolist()
    got = T.sun_tables(az, alt, scale, np.float32(amax), rows, cols)
    for k in range(len(az)):
        dx, dy, dz, azf = T.sun_table(az[k], alt[k], scale, float(np.float32(amax)), rows, cols)
        mode, lo, hi = T.facesh_thresholds(azf)
        v = got[k]
        assert np.array_equal(dx, v[0]) and np.array_equal(dy, v[1]) and dz.tobytes() == v[2].tobytes()
        assert np.float32(azf).tobytes() == np.float32(v[3]).tobytes()
        assert (mode, np.float32(lo).tobytes(), np.float32(hi).tobytes()) == \
            (v[4][0], np.float32(v[4][1]).tobytes(), np.float32(v[4][2]).tobytes())


def test_utci_tables_equal_one_step_form():
    """The UTCI step tables built for all steps at once equal the one-step
    form bit for bit (float32 chain, float64 log / exp / high powers rounded
    once), over the forcing range and its edges."""
    rng = np.random.default_rng(23)
    ta = np.concatenate([rng.uniform(-60, 70, 20000), [-50.0, 0.0, -0.0, 46.0, 70.0, np.nan]]).astype(np.float32)
    rh = np.concatenate([rng.uniform(0, 100, 20000), [0.0, 100.0, 5.0, 50.0, np.nan, 30.0]]).astype(np.float32)
    pa_v, k_v = TS._utci_tables(ta, rh)
    for j in range(len(ta)):
        pa, k = TS._utci_table(ta[j], rh[j])
        assert pa.tobytes() == pa_v[j].tobytes() and k.tobytes() == k_v[j].tobytes(), (j, ta[j], rh[j])


@pytest.mark.parametrize("e", [4, 0.3, -1.6364])
def test_float64_powers_match_torch_0dim(e):
    """The float fast path of _pow_each / _rpow_each returns the 0-dim
    torch bits (the C library's pow in both)."""
    import torch
    from solweig_project_b200 import timeseries as TS
    rng = np.random.default_rng(7)
    x = torch.tensor(rng.uniform(0.01, 400.0, 20000), dtype=torch.float64)
    want = torch.stack([x[k] ** e for k in range(x.shape[0])])
    assert torch.equal(TS._pow_each(x, e).view(torch.int64), want.view(torch.int64))
    y = torch.tensor(rng.uniform(-3.0, 3.0, 20000), dtype=torch.float64)
    for base in (10, 0.935):
        want = torch.stack([base ** y[k] for k in range(y.shape[0])])
        assert torch.equal(TS._rpow_each(base, y).view(torch.int64), want.view(torch.int64))
    # values the float path leaves to torch: zero, negative, overflow
    z = torch.tensor([0.0, -2.0, 1e300], dtype=torch.float64)
    assert torch.equal(TS._pow_each(z, 4), torch.stack([z[k] ** 4 for k in range(3)]))
    big = torch.tensor([400.0, 1.0], dtype=torch.float64)
    assert torch.equal(TS._rpow_each(10, big), torch.stack([10 ** big[k] for k in range(2)]))


@pytest.mark.parametrize("e", [4, 0.3, -1.6364])
def test_float32_powers_match_torch_0dim(e):
    rng = np.random.default_rng(11)
    x = torch.tensor(rng.uniform(0.01, 400.0, 20000), dtype=torch.float32)
    want = torch.stack([x[k] ** e for k in range(x.shape[0])])
    got = TS._pow_each(x, e)
    assert got.dtype == torch.float32 and torch.equal(got.view(torch.int32), want.view(torch.int32))
    y = torch.tensor(rng.uniform(-3.0, 40.0, 20000), dtype=torch.float32)
    for base in (10, 0.935):
        want = torch.stack([base ** y[k] for k in range(y.shape[0])])
        got = TS._rpow_each(base, y)
        assert got.dtype == torch.float32 and torch.equal(got.view(torch.int32), want.view(torch.int32))
