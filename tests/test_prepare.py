"""Device site preparation (sw100_prepare_site) against the host restatement.

The derived rasters (vegdsm, vegdsm2, bush, buildings, aspect in radians,
land-cover property planes) must equal the host computation of
engine.march_inputs / timeseries.landcover_props bit for bit, and the
reductions must give the same amaxvalue, march bound, bush flag, finiteness
flag and height bound, on plain, bush, NaN, negative-canopy and
no-land-cover inputs.
"""
import numpy as np
import pytest

from solweig_project_b200 import _native as N
from solweig_project_b200 import timeseries as TS

F32 = np.float32


def test_stat_keys_round_trip():
    vals = np.array([0.0, -0.0, 1.5, -2.25, 3.4e38, -3.4e38, 1e-45, np.inf, -np.inf], F32)
    for x in vals:
        u = int(x.view(np.uint32))
        k = (u | 0x80000000) if not (u & 0x80000000) else (~u & 0xffffffff)
        st = np.zeros(N.SITE_STATS_WORDS, np.uint32)
        st[0] = k
        assert N.stat_value(st, 0).view(np.uint32) == x.view(np.uint32)
    st = np.zeros(N.SITE_STATS_WORDS, np.uint32)
    st[2] = st[3] = 0x80000000          # +0
    st[N.N_SITE_STATS] = 1 << 3
    assert np.isnan(N.stat_value(st, 3)) and N.stat_value(st, 2) == 0
    # order: larger float, larger key
    keys = []
    for x in np.sort(vals):
        u = int(x.view(np.uint32))
        keys.append((u | 0x80000000) if not (u & 0x80000000) else (~u & 0xffffffff))
    assert keys == sorted(keys)


def test_class_table_matches_landcover_props():
    from solweig_project_b200 import synthetic
    lc_class = synthetic.default_lc_class()
    tab, valid = TS.class_table(lc_class)
    lc = np.array([[1, 2, 3, 4, 5, 6, 7, 0, 9, -1]], F32)
    props = TS.landcover_props(lc, lc_class, 1, lc.shape[1])
    clean = np.array([[1, 2, 5, 5, 5, 6, 7, 6, 6, 6]])
    for k, arr in (("tgk", props.tgk), ("tstart", props.tstart), ("alb", props.alb), ("emis", props.emis),
                   ("tmax", props.tmaxlst)):
        assert np.array_equal(tab[k][clean].view(np.uint32), np.asarray(arr, F32).view(np.uint32)), k
    assert all((valid >> c) & 1 for c in (1, 2, 5, 6, 7))


def _inputs(kind):
    from solweig_project_b200 import synthetic
    c = synthetic.make_city(96, 80, seed=17, n_buildings=12, n_trees=20)
    dsm, trees, dem, lc = c.dsm.copy(), c.trees.copy(), c.dem.copy(), c.landcover.copy()
    if kind == "bush":      # ground at -0.25 x canopy: vegdem2 == 0 there
        sel = trees > 0
        dem[sel] = F32(-0.25) * trees[sel]
        dsm = np.maximum(dsm, dem).astype(F32)
    elif kind == "nan":
        dsm[10, 11] = np.nan
        trees[50, 40] = np.nan
    elif kind == "negative":
        trees[trees > 0] *= F32(-1)
        dem = dem - F32(2.5)
        lc[0:5, 0:5] = 3
        lc[6:9, 0:5] = 11
    return c, dsm, trees, dem, lc


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["plain", "bush", "nan", "negative", "no_landcover"])
def test_prepare_site_matches_host(cuda, kind):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite, march_inputs
    c, dsm, trees, dem, lc = _inputs(kind)
    lc_class = synthetic.default_lc_class()
    use_lc = kind != "no_landcover"
    s = DeviceSite(dsm, trees, dem, c.walls, c.aspect, c.scale, landcover=lc if use_lc else None,
                   lc_class=lc_class if use_lc else None)
    vegdsm, vegdsm2, bush, amax, buildings = march_inputs(dsm, trees, dem)

    def same(name, got, want):
        g = got.cpu().numpy().reshape(want.shape)
        w = np.asarray(want, F32)
        ok = (g.view(np.uint32) == w.view(np.uint32)) | (np.isnan(g) & np.isnan(w))
        assert ok.all(), (kind, name, int((~ok).sum()))

    same("vegdsm", s.t["vegdsm"], vegdsm)
    same("vegdsm2", s.t["vegdsm2"], vegdsm2)
    same("buildings", s.t["buildings"], buildings)
    same("aspect_rad", s.t["aspect_rad"], (np.asarray(c.aspect, F32) * F32(np.pi)) / F32(180.))
    assert s.bush_any == bool(bush.max() > 0)
    if s.bush_any:
        same("bush", s.t["bush"], bush)
    assert (s.amax.view(np.uint32) == F32(amax).view(np.uint32)) or (np.isnan(s.amax) and np.isnan(amax))
    vmax = F32(max(dsm.max(), vegdsm.max(), vegdsm2.max()))
    assert (s.vmax.view(np.uint32) == vmax.view(np.uint32)) or (np.isnan(s.vmax) and np.isnan(vmax))
    assert s.all_finite == bool(np.isfinite(dsm).all() and np.isfinite(vegdsm).all() and np.isfinite(vegdsm2).all())
    hmax = float(max(np.abs(dsm).max(), np.abs(vegdsm).max(), np.abs(vegdsm2).max()))
    assert s.hmax == hmax or (np.isnan(s.hmax) and np.isnan(hmax))
    props = TS.landcover_props(lc if use_lc else None, lc_class if use_lc else None, *dsm.shape)
    for k in ("tgk", "tstart", "alb", "emis"):
        same(k, s.t[k], getattr(props, k))
    if use_lc:
        # the per-code tg_factor slots hold the factors of the classes
        geo = synthetic.load_sun_geometry("single")
        kw = dict(met_file=synthetic.make_met(3), location=dict(synthetic.DEFAULT_LOCATION), scale=1.0,
                  amax=float(amax), rows=dsm.shape[0], cols=dsm.shape[1], **geo)
        host = TS.build_series(props=props, **kw)
        dev = TS.build_series(props=s.props, **kw)
        codes = s.t["class_idx"].cpu().numpy().reshape(dsm.shape)
        day = host.steps["is_day"] == 1
        got = dev.steps["tg_factor"][day][:, codes]
        want = host.steps["tg_factor"][day][:, host.class_idx]
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        for k in host.steps.dtype.names:
            if k != "tg_factor":
                a, b = (np.ascontiguousarray(x.steps[k]).view(np.uint8) for x in (dev, host))
                assert np.array_equal(a, b), k


@pytest.mark.gpu
def test_prepare_site_refuses_unknown_codes(cuda):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    c, dsm, trees, dem, lc = _inputs("plain")
    lc[3, 3] = 2.5
    with pytest.raises(ValueError, match="lc_class"):
        DeviceSite(dsm, trees, dem, c.walls, c.aspect, c.scale, landcover=lc, lc_class=synthetic.default_lc_class())
