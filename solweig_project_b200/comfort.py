"""``thermal_comfort``: the reference's top-level entry point
(solweig_gpu/solweig_gpu.py:500-670) on this library.

The reference's pipeline, step by step:

1. rasters (building DSM, DEM, trees, optional land cover) are checked for
   equal size, pixel size and coordinate system (preprocessor.py:237-279);
2. the area is cut into tiles of ``tile_size`` pixels plus ``overlap`` to the
   right / bottom, keyed "i_j" (preprocessor.py:341-385);
3. per tile: wall height and aspect from the tile's own DSM
   (walls_aspect.py:190-208, wall limit 3 m, scale = 1 / pixel size), the
   site at the tile centre (longitude / latitude from the raster's
   coordinate system, altitude 3 m where the median ground is above 0,
   utci_process.py:1325-1360), the sun geometry of the forcing rows
   (sun_position.py:905-1010), the SVF from the tile's cache
   ``<base>/processed_inputs/SVF`` when its size and geotransform match, else
   computed and cached (utci_process.py:1391-1411), the time loop, and one
   multi-band GeoTIFF per output in ``<base>/output_folder/<key>/``, a band
   per forcing row with a "Time" item (utci_process.py:1472-1651).

Everything per pixel runs in the CUDA library, tile after tile.
Differences from the reference, each refused with an error rather than
approximated:

* GDAL / PROJ and the time-zone database are absent: rasters are read with
  this library's GeoTIFF reader (or ``.npy``); the tile centre is converted
  to longitude / latitude for geographic WGS84 (EPSG:4326), UTM on WGS84
  (EPSG:326xx / 327xx) and Web Mercator (EPSG:3857) rasters, otherwise the
  keyword ``location`` must name the site; the UTC offset of the selected
  date must be given as ``utc_offset`` (hours).
* ERA5 / WRF forcing (``use_own_met=False``), directional wind coefficients
  from an ERA5 roughness file and WBGT are not part of this library.
"""
from __future__ import annotations

import datetime as _dt
import math
import os

import numpy as np

from . import formats as FM
from . import sunpos
from . import tiles as TL
from .walls_aspect import filter1Goodwin_as_aspect_v3, findwalls

F32 = np.float32
ERA5_ROUGHNESS_FILE = "data_stream-oper_stepType-instant.nc"


# ------------------------------------------------------------ coordinates
def _utm_to_lonlat(easting, northing, zone, south):
    """Inverse transverse Mercator on WGS84 (UTM: k0 0.9996, false easting
    500 km, false northing 10 000 km in the south), the series of Snyder
    (1987), Map Projections -- A Working Manual, USGS PP 1395, eqs. 8-18 to
    8-25: sub-millimetre within a zone."""
    a, f, k0 = 6378137.0, 1 / 298.257223563, 0.9996
    e2 = f * (2 - f)
    ep2 = e2 / (1 - e2)
    x = easting - 500000.0
    y = northing - (10000000.0 if south else 0.0)
    m = y / k0
    mu = m / (a * (1 - e2 / 4 - 3 * e2 ** 2 / 64 - 5 * e2 ** 3 / 256))
    e1 = (1 - math.sqrt(1 - e2)) / (1 + math.sqrt(1 - e2))
    phi1 = (mu + (3 * e1 / 2 - 27 * e1 ** 3 / 32) * math.sin(2 * mu)
            + (21 * e1 ** 2 / 16 - 55 * e1 ** 4 / 32) * math.sin(4 * mu)
            + (151 * e1 ** 3 / 96) * math.sin(6 * mu) + (1097 * e1 ** 4 / 512) * math.sin(8 * mu))
    s1, c1, t1 = math.sin(phi1), math.cos(phi1), math.tan(phi1)
    n1 = a / math.sqrt(1 - e2 * s1 * s1)
    r1 = a * (1 - e2) / (1 - e2 * s1 * s1) ** 1.5
    cc = ep2 * c1 * c1
    tt = t1 * t1
    d = x / (n1 * k0)
    lat = phi1 - (n1 * t1 / r1) * (d ** 2 / 2 - (5 + 3 * tt + 10 * cc - 4 * cc ** 2 - 9 * ep2) * d ** 4 / 24
                                   + (61 + 90 * tt + 298 * cc + 45 * tt ** 2 - 252 * ep2 - 3 * cc ** 2) * d ** 6 / 720)
    lon = (d - (1 + 2 * tt + cc) * d ** 3 / 6
           + (5 - 2 * cc + 28 * tt - 3 * cc ** 2 + 8 * ep2 + 24 * tt ** 2) * d ** 5 / 120) / c1
    return math.degrees(lon) + (zone * 6 - 183), math.degrees(lat)


def centre_lonlat(geotransform, rows, cols, epsg):
    """Longitude / latitude (degrees) of a raster's centre, taken as the
    reference takes it (x0 + dx * cols / 2, y0 + dy * rows / 2), for the
    coordinate systems this library converts; None for others."""
    if geotransform is None or epsg is None:
        return None
    cx = geotransform[0] + geotransform[1] * cols / 2.0
    cy = geotransform[3] + geotransform[5] * rows / 2.0
    if epsg == 4326:
        return cx, cy
    if 32601 <= epsg <= 32660:
        return _utm_to_lonlat(cx, cy, epsg - 32600, False)
    if 32701 <= epsg <= 32760:
        return _utm_to_lonlat(cx, cy, epsg - 32700, True)
    if epsg == 3857:
        r = 6378137.0
        return math.degrees(cx / r), math.degrees(2 * math.atan(math.exp(cy / r)) - math.pi / 2)
    return None


def _tile_geotransform(gt, r0, c0):
    if gt is None:
        return None
    return (gt[0] + c0 * gt[1] + r0 * gt[2], gt[1], gt[2], gt[3] + c0 * gt[4] + r0 * gt[5], gt[4], gt[5])


def _lower_median(x):
    """torch.median's value: the lower of the two middle elements."""
    v = np.sort(np.asarray(x, np.float32).reshape(-1))
    return float(v[(v.size - 1) // 2])


def _resolve(base_path, name):
    if name is None:
        return None
    return name if os.path.isabs(name) else os.path.join(base_path, name)


def check_rasters(rasters):
    """Equal size, pixel size and coordinate system (preprocessor.py:237-279)."""
    ref = rasters[0]
    for r in rasters[1:]:
        if r.shape != ref.shape:
            raise ValueError("Error: Raster dimensions do not match.")
        if (r.geotransform is None) != (ref.geotransform is None) or (
                r.geotransform is not None and (r.geotransform[1] != ref.geotransform[1] or
                                                r.geotransform[5] != ref.geotransform[5])):
            raise ValueError("Error: Pixel sizes do not match.")
        if r.epsg != ref.epsg:
            raise ValueError("Error: CRS does not match.")


# ------------------------------------------------------------- the entry
def thermal_comfort(base_path, selected_date_str, building_dsm_filename="Building_DSM.tif",
                    dem_filename="DEM.tif", trees_filename="Trees.tif", landcover_filename=None,
                    ERA_5_z0_find=True, tile_size=3600, overlap=20, use_own_met=True, start_time=None,
                    end_time=None, data_source_type=None, data_folder=None, own_met_file=None, use_uhi=True,
                    save_tmrt=True, save_svf=False, save_kup=False, save_kdown=False, save_lup=False,
                    save_ldown=False, save_shadow=False, save_wbgt=False, save_ta=False, save_wind=False, *,
                    utc_offset=None, location=None, scale=None):
    """Urban thermal comfort of a raster area for one day of forcing
    (solweig_gpu/solweig_gpu.py:500-670, same arguments and outputs).
    Writes ``<base_path>/output_folder/<i_j>/UTCI_<i_j>.tif`` (and TMRT,
    Kup, Kdown, Lup, Ldown, Shadow, Ta, Wind, SVF as selected), one band per
    forcing row.  Keywords beyond the reference's: ``utc_offset`` (hours,
    required: no time-zone database), ``location`` ({"latitude",
    "longitude"} of the area, needed when the rasters' coordinate system is
    not one this library converts) and ``scale`` (pixels per metre, needed
    for .npy rasters).  Returns None."""
    from .engine import DeviceSite
    from . import synthetic
    if save_wbgt:
        raise NotImplementedError("WBGT is not part of this library")
    if not use_own_met:
        raise NotImplementedError("ERA5 / WRF forcing preprocessing is not part of this library; "
                                  "pass use_own_met=True with own_met_file")
    if own_met_file is None:
        raise ValueError("Error: Please provide the path to your own met file.")
    if ERA_5_z0_find:
        era5 = os.path.join(data_folder, ERA5_ROUGHNESS_FILE) if data_folder else None
        if era5 is not None and os.path.exists(era5):
            raise NotImplementedError("directional wind coefficients from ERA5 roughness are not part of this "
                                      "library; pass ERA_5_z0_find=False")
        print("Could not find ERA-5 file with roughness length")
    if utc_offset is None:
        raise ValueError("utc_offset (hours) is required: the time-zone database the reference consults is not "
                         "available to this library")
    paths = [_resolve(base_path, building_dsm_filename), _resolve(base_path, dem_filename),
             _resolve(base_path, trees_filename)]
    lc_path = _resolve(base_path, landcover_filename)
    if lc_path is not None:
        paths.append(lc_path)
    for p in paths:
        if not os.path.exists(p):
            raise FileNotFoundError(f"Could not open {p}")
    rasters = [FM.read_raster(p) for p in paths]
    check_rasters(rasters)
    dsm_r = rasters[0]
    gt = dsm_r.geotransform
    if scale is None:
        if gt is None:
            raise ValueError("scale (pixels per metre) is required for rasters without a geotransform")
        scale = 1.0 / gt[1]
    met = np.loadtxt(own_met_file, skiprows=1, delimiter=" ")
    met = np.atleast_2d(met)
    base_date = _dt.datetime.strptime(selected_date_str, "%Y-%m-%d")
    rows, cols = dsm_r.shape
    wins = TL.tile_windows(rows, cols, int(tile_size), int(overlap))
    requested = ["utci"] + [k for k, on in (("tmrt", save_tmrt), ("kup", save_kup), ("kdown", save_kdown),
                                            ("lup", save_lup), ("ldown", save_ldown), ("shadow", save_shadow))
                            if on]
    lc_class = synthetic.default_lc_class() if lc_path is not None else None
    svf_dir = os.path.join(base_path, "processed_inputs", "SVF")
    out_root = os.path.join(base_path, "output_folder")
    names = dict(TL.FILE_NAMES, ta="Ta", wind="Wind")
    times = [{"Time": base_date.replace(hour=int(met[t, 2]), minute=int(met[t, 3])).isoformat()}
             for t in range(met.shape[0])]
    uh = met[:, 24] if met.shape[1] > 24 else np.zeros(met.shape[0])
    for key, r0, r1, c0, c1 in wins:
        sl = (slice(r0, r1), slice(c0, c1))
        dsm, dem, trees = (r.data[sl] for r in rasters[:3])
        lc = rasters[3].data[sl] if lc_path is not None else None
        walls64 = findwalls(dsm, 3.0)
        aspect = filter1Goodwin_as_aspect_v3(walls64, scale, dsm).astype(F32)   # stored as float32 rasters
        walls = walls64.astype(F32)
        tgt = _tile_geotransform(gt, r0, c0)
        lonlat = centre_lonlat(tgt, r1 - r0, c1 - c0, dsm_r.epsg)
        if lonlat is None:
            if location is None:
                raise ValueError(f"the rasters' coordinate system (EPSG {dsm_r.epsg}) is not one this library "
                                 "converts to longitude / latitude; pass location={'latitude', 'longitude'}")
            lonlat = (float(location["longitude"]), float(location["latitude"]))
        alt = _lower_median(dem)
        if alt > 0:
            alt = 3.
        loc = {"longitude": lonlat[0], "latitude": lonlat[1], "altitude": alt}
        _, altitude, azimuth, zen, jday, _, dectime, altmax = sunpos.metdata_noload(met, loc, float(utc_offset))
        site = DeviceSite(dsm, trees, dem, walls, aspect, scale, landcover=lc, lc_class=lc_class)
        cached = FM.svf_cache_extent_matches(dsm.shape, tgt, svf_dir, number=key)
        if cached:
            planes, cubes = FM.read_svf_cache(svf_dir, number=key)
            _install_cached_svf(site, planes, cubes)
        else:
            res = site.run_svf()
            FM.write_svf_cache(svf_dir, res.planes, res.cubes(), tgt, number=key, epsg=dsm_r.epsg)
        outs, _ = site.run_chain_chunked(met, altitude, azimuth, zen, jday, dectime, altmax, loc,
                                         requested=tuple(requested))
        if save_ta:
            ta = [(F32(0) + F32(met[t, 11])) + F32(uh[t]) for t in range(met.shape[0])]
            outs["ta"] = np.broadcast_to(np.array(ta, F32)[:, None, None], (met.shape[0], r1 - r0, c1 - c0)).copy()
        if save_wind:
            outs["wind"] = np.stack([np.maximum(np.ones((r1 - r0, c1 - c0), F32) * F32(met[t, 9]), F32(0.15))
                                     for t in range(met.shape[0])])
        folder = os.path.join(out_root, key)
        os.makedirs(folder, exist_ok=True)
        for name, arr in outs.items():
            with open(os.path.join(folder, f"{names[name]}_{key}.tif"), "wb") as fh:
                fh.write(FM.tiff_bytes(arr, tgt, times[:arr.shape[0]], epsg=dsm_r.epsg))
        if save_svf and not cached:
            with open(os.path.join(folder, f"SVF_{key}.tif"), "wb") as fh:
                fh.write(FM.tiff_bytes(site.svf_result.plane("svftotal").cpu().numpy(), tgt, epsg=dsm_r.epsg))
        elif save_svf:
            print(f"[INFO] SVF cache already exists for tile {key}; skipping duplicate SVF_{key}.tif write.")
    return None


def _install_cached_svf(site, planes, cubes):
    """The SVF of a tile from its cache (15 planes, SVFtotal, dense cubes)."""
    from .api import _pack_bundle
    order = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS", "svfSaveg",
             "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg")
    sh, veg, vb = cubes
    _pack_bundle(site, tuple(planes[k] for k in order) + (veg, vb, sh, planes["svftotal"]))
