"""thermal_comfort (solweig_gpu/solweig_gpu.py:500-670) on this library:
argument refusals, raster checks and coordinate conversion on CPU; on the
GPU, a tiled run from GeoTIFF inputs on disk against the library's own
drop-in per tile (bit for bit), one tile against the CPU oracle, and a
second run that reuses the SVF cache."""
import math
import os

import numpy as np
import pytest

from solweig_project_b200 import comfort as CF
from solweig_project_b200 import formats as FM
from solweig_project_b200 import synthetic

GT = (621000.0, 1.0, 0.0, 3352000.0, 0.0, -1.0)     # UTM 14N, 1 m pixels
EPSG = 32614


def _utm_forward(lon, lat, zone):
    """Transverse Mercator forward series (Snyder 1987, eqs. 8-9, 8-10) on
    WGS84, the inverse's counterpart for a round trip."""
    a, f, k0 = 6378137.0, 1 / 298.257223563, 0.9996
    e2 = f * (2 - f)
    ep2 = e2 / (1 - e2)
    phi, lam = math.radians(lat), math.radians(lon - (zone * 6 - 183))
    n = a / math.sqrt(1 - e2 * math.sin(phi) ** 2)
    t = math.tan(phi) ** 2
    c = ep2 * math.cos(phi) ** 2
    A = lam * math.cos(phi)
    m = a * ((1 - e2 / 4 - 3 * e2 ** 2 / 64 - 5 * e2 ** 3 / 256) * phi
             - (3 * e2 / 8 + 3 * e2 ** 2 / 32 + 45 * e2 ** 3 / 1024) * math.sin(2 * phi)
             + (15 * e2 ** 2 / 256 + 45 * e2 ** 3 / 1024) * math.sin(4 * phi)
             - (35 * e2 ** 3 / 3072) * math.sin(6 * phi))
    x = k0 * n * (A + (1 - t + c) * A ** 3 / 6 + (5 - 18 * t + t * t + 72 * c - 58 * ep2) * A ** 5 / 120)
    y = k0 * (m + n * math.tan(phi) * (A * A / 2 + (5 - t + 9 * c + 4 * c * c) * A ** 4 / 24
                                       + (61 - 58 * t + t * t + 600 * c - 330 * ep2) * A ** 6 / 720))
    return x + 500000.0, y + (10000000.0 if lat < 0 else 0.0)


@pytest.mark.parametrize("lon,lat", [(-97.7, 30.3), (-95.2, 12.0), (-99.9, 55.5), (-97.0, -33.9)])
def test_utm_inverse_round_trip(lon, lat):
    zone = 14
    e, n = _utm_forward(lon, lat, zone)
    got = CF._utm_to_lonlat(e, n, zone, lat < 0)
    assert abs(got[0] - lon) < 1e-7 and abs(got[1] - lat) < 1e-7


def test_centre_of_geographic_and_web_mercator_rasters():
    assert CF.centre_lonlat((-98.0, 0.001, 0.0, 30.5, 0.0, -0.001), 400, 600, 4326) == \
        pytest.approx((-97.7, 30.3))
    x = 6378137.0 * math.radians(-97.7)
    y = 6378137.0 * math.log(math.tan(math.pi / 4 + math.radians(30.3) / 2))
    lon, lat = CF.centre_lonlat((x - 50, 1.0, 0.0, y + 50, 0.0, -1.0), 100, 100, 3857)
    assert abs(lon + 97.7) < 1e-9 and abs(lat - 30.3) < 1e-9
    assert CF.centre_lonlat(GT, 10, 10, 2154) is None


def _write_inputs(folder, city, met):
    os.makedirs(folder, exist_ok=True)
    for name, arr in (("Building_DSM.tif", city.dsm), ("DEM.tif", city.dem), ("Trees.tif", city.trees),
                      ("Landcover.tif", city.landcover)):
        with open(os.path.join(folder, name), "wb") as fh:
            fh.write(FM.tiff_bytes(arr, GT, epsg=EPSG))
    path = os.path.join(folder, "met.txt")
    header = "%iy id it imin qn qh qe qs qf U RH Tair press rain kdown snow ldown fcld wuh xsmd lai kdiff kdir wdir uhii"
    np.savetxt(path, met, fmt="%.10g", delimiter=" ", header=header, comments="")
    return path


def test_refusals(tmp_path):
    city = synthetic.make_city(20, 20, seed=1, with_walls=False)
    met_path = _write_inputs(str(tmp_path), city, synthetic.make_met(1))
    base = dict(base_path=str(tmp_path), selected_date_str="2024-07-14", ERA_5_z0_find=False,
                own_met_file=met_path, utc_offset=-5)
    with pytest.raises(NotImplementedError, match="WBGT"):
        CF.thermal_comfort(**base, save_wbgt=True)
    with pytest.raises(NotImplementedError, match="ERA5"):
        CF.thermal_comfort(**dict(base, use_own_met=False))
    with pytest.raises(ValueError, match="met file"):
        CF.thermal_comfort(**dict(base, own_met_file=None))
    with pytest.raises(ValueError, match="utc_offset"):
        CF.thermal_comfort(**dict(base, utc_offset=None))
    with pytest.raises(FileNotFoundError):
        CF.thermal_comfort(**dict(base, dem_filename="missing.tif"))
    with open(tmp_path / "Small.tif", "wb") as fh:
        fh.write(FM.tiff_bytes(city.dem[:10], GT, epsg=EPSG))
    with pytest.raises(ValueError, match="dimensions"):
        CF.thermal_comfort(**dict(base, dem_filename="Small.tif"))
    with open(tmp_path / "Other.tif", "wb") as fh:
        fh.write(FM.tiff_bytes(city.dem, GT, epsg=32615))
    with pytest.raises(ValueError, match="CRS"):
        CF.thermal_comfort(**dict(base, dem_filename="Other.tif"))


@pytest.mark.gpu
def test_tiled_run_from_rasters(cuda, tmp_path):
    from golden_util import max_abs
    from oracle import svf as osvf
    from oracle import window as ow
    from solweig_project_b200 import api, sunpos
    from solweig_project_b200 import tiles as TL
    from solweig_project_b200.walls_aspect import filter1Goodwin_as_aspect_v3, findwalls
    city = synthetic.make_city(90, 70, seed=31, n_buildings=14, n_trees=10, side_range=(4, 14), with_walls=False)
    met = synthetic.make_met(31)
    folder = str(tmp_path / "area")
    met_path = _write_inputs(folder, city, met)
    kw = dict(landcover_filename="Landcover.tif", ERA_5_z0_find=False, tile_size=48, overlap=8,
              own_met_file=met_path, utc_offset=-5, save_shadow=True, save_svf=True)
    assert CF.thermal_comfort(folder, "2024-07-14", **kw) is None
    lc_class = synthetic.default_lc_class()
    wins = TL.tile_windows(90, 70, 48, 8)
    assert len(wins) == 4
    first = {}
    for n, (key, r0, r1, c0, c1) in enumerate(wins):
        sl = (slice(r0, r1), slice(c0, c1))
        out = {}
        for name in ("UTCI", "TMRT", "Shadow", "SVF"):
            arr, gt, md = FM.read_tiff(open(os.path.join(folder, "output_folder", key, f"{name}_{key}.tif"),
                                            "rb").read(), with_metadata=True)
            out[name] = arr
            assert gt == (GT[0] + c0, 1.0, 0.0, GT[3] - r0, 0.0, -1.0)
        assert md[0] == {} and out["UTCI"].shape == (24, r1 - r0, c1 - c0)
        first[key] = out
        # the same tile through the library's own drop-in
        dsm, dem, trees = city.dsm[sl], city.dem[sl], city.trees[sl]
        w64 = findwalls(dsm, 3.0)
        aspect = filter1Goodwin_as_aspect_v3(w64, 1.0, dsm).astype(np.float32)
        lon, lat = CF.centre_lonlat(CF._tile_geotransform(GT, r0, c0), r1 - r0, c1 - c0, EPSG)
        loc = {"longitude": lon, "latitude": lat, "altitude": 0.0}
        _, alt, azi, zen, jday, _, dectime, altmax = sunpos.metdata_noload(met, loc, -5.0)
        geo = dict(altitude=alt, azimuth=azi, zen=zen, jday=jday, dectime=dectime, altmax=altmax)
        want = api.run_exact_chain(dsm=dsm, trees=trees, dem=dem, walls=w64.astype(np.float32), aspect=aspect,
                                   scale=1.0, met_file=met, location=loc, landcover=city.landcover[sl],
                                   lc_class=lc_class, requested=("utci", "tmrt", "shadow"), **geo)
        for name, k in (("UTCI", "utci"), ("TMRT", "tmrt"), ("Shadow", "shadow")):
            assert np.array_equal(out[name].view(np.uint32), want[k].view(np.uint32)), (key, name)
        if n == 1:   # one tile against the CPU oracle
            vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(dsm, trees, dem)
            bundle = osvf.svf_calculator(2, amax, dsm, vegdsm, vegdsm2, bush, 1.0)
            assert np.array_equal(out["SVF"].view(np.uint32), np.asarray(bundle[18], np.float32).view(np.uint32))
            ref = ow.run_utci_window(a=dsm, temp1=trees, temp2=dem, walls=w64.astype(np.float32), dirwalls=aspect,
                                     svf_bundle=bundle, met_file=met, location=loc, scale=1.0,
                                     landcover_grid=city.landcover[sl], lc_class=lc_class,
                                     requested_variables=("utci", "tmrt", "shadow"), **geo)
            assert np.array_equal(out["Shadow"].view(np.uint32), ref["shadow"].view(np.uint32))
            assert max_abs(out["TMRT"], ref["tmrt"]) <= 1e-3
            assert max_abs(out["UTCI"], ref["utci"]) <= 1e-3
    # a second run reads the SVF cache (no SVF_<key>.tif rewrite) and gives the same outputs
    for key, *_ in wins:
        os.remove(os.path.join(folder, "output_folder", key, f"SVF_{key}.tif"))
    CF.thermal_comfort(folder, "2024-07-14", **kw)
    for key, *_ in wins:
        assert not os.path.exists(os.path.join(folder, "output_folder", key, f"SVF_{key}.tif"))
        for name in ("UTCI", "TMRT", "Shadow"):
            arr, _ = FM.read_tiff(open(os.path.join(folder, "output_folder", key, f"{name}_{key}.tif"), "rb").read())
            assert np.array_equal(arr.view(np.uint32), first[key][name].view(np.uint32)), (key, name)
