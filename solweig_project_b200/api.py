"""Drop-in entry points with the reference's names, arguments and errors.

* :func:`svf_calculator`   <- ``solweig_gpu/shadow.py:409-625``
* :func:`run_utci_window`  <- ``solweig_gpu/utci_process.py:477-1090``
* :func:`utci_calculator`  <- ``solweig_gpu/calculate_utci.py:259-330``
* :func:`recompute_utci_steps` <- ``solweig_gpu/utci_process.py:1093-1196``
* :func:`run_exact_chain`  -- the whole chain for one site from host rasters
  (what ``compute_utci`` does between its raster I/O, utci_process.py:1376-1470)
* :func:`thermal_comfort`  <- ``solweig_gpu/solweig_gpu.py:500-670`` (rasters
  on disk -> tiled GeoTIFF outputs; :mod:`solweig_project_b200.comfort`)

All of them run on the CUDA library; there is no CPU path.  A missing GPU or
library raises :class:`~solweig_project_b200._native.NativeUnavailable`.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N
from . import engine as E
from . import formats as FM
from . import tables as T
from . import timeseries as TS

from .comfort import thermal_comfort  # noqa: E402,F401  (re-exported drop-in)

F32 = np.float32
VALID_VARIABLES = frozenset({"utci", "tmrt", "kup", "kdown", "lup", "ldown", "shadow", "ta", "wind"})
STATE_PLANES = E.STATE_NAMES


def _np32(x):
    if isinstance(x, torch.Tensor):
        return x.detach().to("cpu").numpy().astype(F32, copy=False)
    return np.asarray(x, F32)


class PackedSvf:
    """SVF result kept on the device: 15 planes + SVFtotal + time-loop
    statics, and the packed patch cubes (60 B per pixel instead of three
    (rows, cols, 153) float32 cubes)."""

    def __init__(self, result: E.SvfResult):
        self.result = result

    def bundle(self):
        """The reference's 19-tuple with dense cubes (shadow.py:625)."""
        r = self.result
        sh, veg, vb = r.cubes()
        p = [r.plane(k) for k in ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg",
                                  "svfS", "svfSaveg", "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg")]
        return (*p, veg, vb, sh, r.plane("svftotal"))


def _geotransform_of(gdal_dsm, building_dsm_path):
    """Georeferencing to copy into the cache rasters: a dataset-like object
    with GetGeoTransform(), a 6-tuple, or the building DSM raster on disk."""
    if gdal_dsm is not None:
        if hasattr(gdal_dsm, "GetGeoTransform"):
            return tuple(gdal_dsm.GetGeoTransform()), None
        gt = tuple(float(v) for v in gdal_dsm)
        if len(gt) != 6:
            raise ValueError("gdal_dsm must be a dataset with GetGeoTransform() or a 6-value geotransform")
        return gt, None
    r = FM.read_raster(building_dsm_path)
    return r.geotransform, r.epsg


def svf_calculator(patch_option, amaxvalue=None, a=None, vegdem=None, vegdem2=None, bush=None, scale=None,
                   save_rasters=False, building_dsm_path=None, tree_path=None, dem_path=None, output_dir=None,
                   number=None, gdal_dsm=None, packed=False):
    """153-patch sky-view-factor sweep.  Arguments as the reference:
    ``a`` the building DSM, ``vegdem``/``vegdem2`` the canopy/trunk tops
    (0 where no vegetation), ``bush``, ``amaxvalue`` the domain height bound,
    ``scale`` pixels per metre.  Returns the 19-tuple (svf, svfaveg, svfE,
    svfEaveg, svfEveg, svfN, svfNaveg, svfNveg, svfS, svfSaveg, svfSveg,
    svfveg, svfW, svfWaveg, svfWveg, vegshmat, vbshvegshmat, shmat, SVFtotal)
    of CUDA tensors, or a :class:`PackedSvf` with ``packed=True``.

    ``save_rasters=True`` also writes the reference's cache
    (shadow.py:100-164, 444-487): ``svfs[_<number>].zip`` (15 GeoTIFFs),
    ``shadowmats[_<number>].npz`` and ``SkyViewFactor[_<number>].tif`` in
    ``output_dir``, georeferenced from ``gdal_dsm`` (a dataset with
    GetGeoTransform() or a geotransform) or the raster at
    ``building_dsm_path``.  Without the march rasters it reads the building
    DSM, trees and DEM rasters from the three paths and derives them as
    compute_utci does (scale = 1 / pixel size)."""
    geo, epsg = None, None
    if save_rasters:
        if output_dir is None:
            raise ValueError("When save_rasters=True, output_dir must be provided.")
        if any(x is None for x in (amaxvalue, a, vegdem, vegdem2, bush, scale)):
            if building_dsm_path is None or tree_path is None or dem_path is None:
                raise ValueError("When save_rasters=True and SVF tensors are not provided, "
                                 "building_dsm_path, tree_path, and dem_path must be provided.")
            dsm_r = FM.read_raster(building_dsm_path)
            if dsm_r.geotransform is None:
                raise ValueError(f"{building_dsm_path} carries no geotransform (the scale comes from it)")
            a = dsm_r.data
            trees = FM.read_raster(tree_path).data.copy()
            dem = FM.read_raster(dem_path).data
            scale = 1.0 / dsm_r.geotransform[1]
            vegdem, vegdem2, bush, amaxvalue, _ = E.march_inputs(a, trees, dem)
            geo, epsg = dsm_r.geotransform, dsm_r.epsg
        elif gdal_dsm is None and building_dsm_path is None:
            raise ValueError("When save_rasters=True with precomputed tensors, provide either gdal_dsm or "
                             "building_dsm_path so GeoTIFF metadata can be copied.")
        else:
            geo, epsg = _geotransform_of(gdal_dsm, building_dsm_path)
    required = {"amaxvalue": amaxvalue, "a": a, "vegdem": vegdem, "vegdem2": vegdem2, "bush": bush, "scale": scale}
    missing = [k for k, v in required.items() if v is None]
    if missing:
        raise ValueError("When save_rasters=False, these arguments must be provided: " + ", ".join(missing))
    if patch_option not in T.PATCH_LAYOUT or patch_option != 2:
        raise ValueError(f"patch_option {patch_option} is not supported (the time loop uses option 2)")
    site = E.DeviceSite.from_march_rasters(_np32(a), _np32(vegdem), _np32(vegdem2), _np32(bush),
                                           float(_np32(amaxvalue)), float(scale))
    res = site.run_svf(patch_option)
    if save_rasters:
        FM.write_svf_cache(output_dir, res.planes, res.cubes(), geo, number=number, epsg=epsg)
    return PackedSvf(res) if packed else PackedSvf(res).bundle()


def _pack_bundle(site: E.DeviceSite, svf_bundle, cubes_window=None):
    """Accept a PackedSvf or the reference's 19-tuple (torch / numpy).
    ``cubes_window`` = (r0, r1, c0, c1): the tuple's three patch cubes cover
    only that window of the site (the reference's pre-cropped bundles,
    utci_process.py:651-663); the site's bit cubes are zero outside it,
    where no output is kept (a pixel's patch sums read its own cubes only)."""
    if isinstance(svf_bundle, PackedSvf):
        if cubes_window is not None:
            raise ValueError("svf_bundle_cubes_cropped=True needs the reference's 19-tuple, not a PackedSvf")
        r = svf_bundle.result
        site.set_svf(r.planes, r.bits, r.single_step)
        return
    if len(svf_bundle) != 19:
        raise ValueError("svf_bundle must be the 19-tuple of svf_calculator")
    (svf, svfaveg, svfE, svfEaveg, svfEveg, svfN, svfNaveg, svfNveg, svfS, svfSaveg, svfSveg, svfveg, svfW,
     svfWaveg, svfWveg, vegshmat, vbshvegshmat, shmat, svftotal) = svf_bundle
    d = site.device
    planes = torch.empty((N.SVF_PLANES, site.rows, site.cols), dtype=torch.float32, device=d)
    for k, v in enumerate((svf, svfaveg, svfE, svfEaveg, svfEveg, svfN, svfNaveg, svfNveg, svfS, svfSaveg, svfSveg,
                           svfveg, svfW, svfWaveg, svfWveg, svftotal)):
        planes[k] = torch.as_tensor(_np32(v) if not isinstance(v, torch.Tensor) else v, dtype=torch.float32).to(d)
    # time-loop statics (utci_process.py:864-897), on the device as the sweep's epilogue writes them
    N.call("sw100_svf_statics", E._ptr(planes), site.rows, site.cols, float(site.params.transVeg), E._stream())
    _, _, _, single, _ = site.svf_tables(2)
    cubes = [torch.as_tensor(_np32(c) if not isinstance(c, torch.Tensor) else c, dtype=torch.float32).to(d).contiguous()
             for c in (shmat, vegshmat, vbshvegshmat)]
    r0, r1, c0, c1 = cubes_window if cubes_window is not None else (0, site.rows, 0, site.cols)
    crows, ccols, P = cubes[0].shape
    if (crows, ccols) != (r1 - r0, c1 - c0) or any(tuple(c.shape) != (crows, ccols, P) for c in cubes):
        raise ValueError(f"patch cubes of shape {tuple(cubes[0].shape)} do not cover the "
                         f"{'write window' if cubes_window is not None else 'grid'} {(r1 - r0, c1 - c0)}")
    single_c = (C.c_uint32 * N.CUBE_WORDS)(*[int(x) for x in single])
    if cubes_window is None:
        bits = torch.empty((3, N.CUBE_WORDS, site.rows, site.cols), dtype=torch.int32, device=d)
        N.call("sw100_pack_cubes", E._ptr(cubes[0]), E._ptr(cubes[1]), E._ptr(cubes[2]), site.rows, site.cols, P,
               single_c, E._ptr(bits), E._stream())
    else:
        crop = torch.empty((3, N.CUBE_WORDS, crows, ccols), dtype=torch.int32, device=d)
        N.call("sw100_pack_cubes", E._ptr(cubes[0]), E._ptr(cubes[1]), E._ptr(cubes[2]), crows, ccols, P,
               single_c, E._ptr(crop), E._stream())
        bits = torch.zeros((3, N.CUBE_WORDS, site.rows, site.cols), dtype=torch.int32, device=d)
        bits[:, :, r0:r1, c0:c1] = crop
    site.svf_result = E.SvfResult(planes, bits, np.asarray(single, np.uint32))
    site.t["svfbuveg"], site.t["hsvf"], site.t["tan_alfa"] = planes[16], planes[17], planes[18]
    site.t["bits"] = bits


def _check_variables(requested_variables):
    requested = set(requested_variables) | {"utci"}
    if not requested.issubset(VALID_VARIABLES):
        raise ValueError(f"unknown requested variables: {sorted(requested - VALID_VARIABLES)}")
    return requested


def _model_params(model_parameters) -> TS.ModelParams:
    if not model_parameters:
        return TS.ModelParams()
    unknown = sorted(set(model_parameters) - TS.PARAM_NAMES)
    if unknown:
        raise ValueError(f"unknown model parameters {unknown}; accepted names are {sorted(TS.PARAM_NAMES)}")
    return TS.ModelParams(**dict(model_parameters))


def run_utci_window(*, a, temp1, temp2, walls, dirwalls, svf_bundle, met_file, altitude, azimuth, zen, jday,
                    dectime, altmax, location, scale, amaxvalue=None, landcover_grid=None, lc_class=None,
                    windcoeff=None, windcoeff_by_dir=None, time_start=0, time_stop=None,
                    requested_variables=("utci",), save_wbgt=False, out_window=None, model_parameters=None,
                    svf_bundle_cubes_cropped=False, initial_state=None, return_final_state=False):
    """Windowed temporal core (utci_process.py:477-1090) on the GPU.

    Returns ``{name: ndarray (T, rows, cols) float32}`` or
    ``(outputs, final_state)``; raises ``ValueError`` for unknown variables,
    model parameters, time ranges, windows or warm-start states as the
    reference does.  ``temp1`` is clamped at 0 in place like the reference."""
    requested = _check_variables(requested_variables)
    if time_stop is None:
        time_stop = met_file.shape[0]
    if not 0 <= time_start < time_stop <= met_file.shape[0]:
        raise ValueError(f"invalid time range [{time_start}, {time_stop}) for {met_file.shape[0]} forcing rows")
    a_np = _np32(a)
    rows, cols = a_np.shape
    if out_window is not None:
        r0, r1, c0, c1 = out_window
        if not (0 <= r0 < r1 <= rows and 0 <= c0 < c1 <= cols):
            raise ValueError(f"out_window {out_window} outside tensor shape {(rows, cols)}")
    elif svf_bundle_cubes_cropped:
        raise ValueError("svf_bundle_cubes_cropped=True requires out_window: the pre-cropped cube extent must "
                         "match a declared write window")
    if save_wbgt:
        raise NotImplementedError("WBGT is not part of this library")
    if windcoeff_by_dir is not None:
        raise NotImplementedError("directional wind coefficients are not supported; pass windcoeff")
    params = _model_params(model_parameters)
    if isinstance(temp1, torch.Tensor):
        temp1[temp1 < 0.] = 0.
    elif isinstance(temp1, np.ndarray):
        temp1[temp1 < 0.] = 0.
    site = E.DeviceSite(a_np, _np32(temp1), _np32(temp2), _np32(walls), _np32(dirwalls), float(scale),
                        landcover=None if landcover_grid is None else _np32(landcover_grid), lc_class=lc_class,
                        windcoeff=None if windcoeff is None else _np32(windcoeff),
                        amaxvalue=None if amaxvalue is None else float(_np32(amaxvalue)), params=params)
    _pack_bundle(site, svf_bundle, cubes_window=out_window if svf_bundle_cubes_cropped else None)
    init_scalars = None
    if initial_state is not None:
        init_scalars = _validate_state(initial_state, rows, cols, time_start, out_window)
        site.load_state(initial_state)
    gpu_vars = [k for k in N.OUT_BITS if k in requested]
    outputs, final_scalars = site.run_chain_chunked(met_file, altitude, azimuth, zen, jday, dectime, altmax,
                                                    location, requested=gpu_vars, time_start=time_start,
                                                    time_stop=time_stop, initial_scalars=init_scalars)
    n_t = time_stop - time_start
    if "ta" in requested:
        uh = met_file[:, 24] if met_file.shape[1] > 24 else np.zeros(met_file.shape[0])
        ta = [(F32(0) + F32(met_file[i, 11])) + F32(uh[i]) for i in range(time_start, time_stop)]
        outputs["ta"] = np.broadcast_to(np.array(ta, F32)[:, None, None], (n_t, rows, cols)).copy()
    if "wind" in requested:
        wc = np.ones((rows, cols), F32) if windcoeff is None else _np32(windcoeff)
        outputs["wind"] = np.stack([np.maximum(wc * F32(met_file[i, 9]), F32(0.15))
                                    for i in range(time_start, time_stop)])
    if out_window is not None:
        r0, r1, c0, c1 = out_window
        outputs = {k: np.ascontiguousarray(v[:, r0:r1, c0:c1]) for k, v in outputs.items()}
    if not return_final_state:
        return outputs
    st = site.state_dict()
    final = {k: (v[r0:r1, c0:c1].clone() if out_window is not None else v) for k, v in st.items()}
    twater = water_temperature(met_file, jday, dectime, time_start, time_stop, landcover_grid is not None,
                               None if initial_state is None else initial_state.get("Twater"))
    final.update(CI=final_scalars["CI"], firstdaytime=final_scalars["firstdaytime"],
                 timeadd=final_scalars["timeadd"], Twater=twater, next_step=int(time_stop))
    return outputs, final


def water_temperature(met_file, jday, dectime, time_start, time_stop, landcover_on, carried=None):
    """The water temperature the reference carries across steps
    (utci_process.py:841-846, 917-922): with land cover on, at every
    midnight row (and the first row) it becomes the mean air temperature of
    that day's forcing rows; a warm start resumes the carried value (None:
    not yet established).  Returns a float, or None while not established.
    Land-cover cleaning maps code 3 (the class whose ground takes it) to 5
    before the chain runs, so the value never reaches a pixel; it is carried
    for the state contract."""
    twater = None if carried is None else float(carried)
    if not landcover_on:
        return twater
    ta = np.asarray(met_file[:, 11], np.float64)
    day_of = np.asarray(jday)[0]
    for i in range(time_start, time_stop):
        if (dectime[i] - np.floor(dectime[i])) == 0 or i == 0:
            twater = float(np.mean(ta[day_of == np.floor(dectime[i])]))
    return twater


def _validate_state(state, rows, cols, time_start, out_window):
    """Warm-start checks of utci_process.py:425-474."""
    if not isinstance(state, dict):
        raise ValueError(f"initial_state must be a dict of thermal planes + scalars, got {type(state).__name__}")
    rec = state.get("next_step")
    if rec is not None and int(rec) != int(time_start):
        raise ValueError(f"initial_state was captured at next_step={rec!r} but time_start={time_start!r}")
    if out_window is not None:
        raise NotImplementedError("warm starts of a windowed run are not supported")
    for name in STATE_PLANES:
        if name not in state:
            raise ValueError(f"initial_state is missing the plane {name!r}")
        plane = state[name]
        dtype_ok = (plane.dtype == torch.float32) if isinstance(plane, torch.Tensor) else \
            (isinstance(plane, np.ndarray) and plane.dtype == np.float32)
        if not dtype_ok:
            raise ValueError(f"initial_state plane {name!r} must be float32")
        if tuple(plane.shape) != (rows, cols):
            raise ValueError(f"initial_state plane {name!r} shape {tuple(plane.shape)} does not match the working "
                             f"extent {(rows, cols)}")
    for name in ("CI", "firstdaytime", "timeadd"):
        if name not in state:
            raise ValueError(f"initial_state is missing the carried scalar {name!r}")
    return {"CI": float(state["CI"]), "firstdaytime": float(state["firstdaytime"]),
            "timeadd": float(state["timeadd"])}


def utci_calculator(Ta, RH, Tmrt, va10m):
    """UTCI (calculate_utci.py:259-330) on the GPU; -999 where any input is
    <= -999.  Accepts tensors or arrays of one shape; returns a CUDA tensor."""
    shape = np.shape(Ta)
    flat = [torch.as_tensor(np.asarray(x, F32) if not isinstance(x, torch.Tensor) else x,
                            dtype=torch.float32).reshape(-1) for x in (Ta, RH, Tmrt, va10m)]
    return E.utci(*flat).reshape(shape)


def recompute_utci_steps(met_file, time_indices, tmrt_planes, buildings_dsm, dem):
    """UTCI-only recompute of the steps ``time_indices`` from stored Tmrt
    planes (utci_process.py:1093-1196, the met fast path for wind speed /
    urban-heat-island edits): same arguments, errors and result
    ((len(time_indices), rows, cols) float32, NaN outside buildings == 1) as
    the reference, computed by the library's UTCI tail on the GPU."""
    a = _np32(buildings_dsm)
    rows, cols = a.shape
    d = _np32(dem)
    if d.shape != a.shape:
        raise ValueError(f"dem shape {d.shape} != buildings_dsm shape {a.shape}")
    indices = tuple(int(i) for i in time_indices)
    if not indices:
        raise ValueError("time_indices must be non-empty")
    met_file = np.asarray(met_file)
    for i in indices:
        if not 0 <= i < met_file.shape[0]:
            raise ValueError(f"time index {i} outside the met table ({met_file.shape[0]} steps)")
        plane = tmrt_planes.get(i)
        if plane is None:
            raise ValueError(f"no published tmrt plane for timestep {i}")
        if tuple(plane.shape) != (rows, cols):
            raise ValueError(f"tmrt plane t={i} shape {tuple(plane.shape)} != tile {(rows, cols)}")
    E.require_cuda()
    dev = torch.device("cuda")
    buildings = a - d
    buildings[buildings < 2.] = 1.
    buildings[buildings >= 2.] = 0.
    rec = TS.utci_step_records(met_file, indices)
    steps_d = E._table(rec, dev)
    tmrt = torch.stack([torch.as_tensor(_np32(tmrt_planes[i])) for i in indices]).pin_memory().to(dev)
    bld = E._dev(buildings, dev)
    out = torch.empty((len(indices), rows, cols), dtype=torch.float32, device=dev)
    N.call("sw100_utci_steps", E._ptr(steps_d), len(indices), E._ptr(tmrt), E._ptr(bld), None, rows * cols,
           E._ptr(out), E._stream())
    return E.to_host(out)


def run_exact_chain(*, dsm, trees, dem, walls, aspect, scale, met_file, altitude, azimuth, zen, jday, dectime,
                    altmax, location, landcover=None, lc_class=None, windcoeff=None, requested=("utci", "tmrt"),
                    model_parameters=None, return_device=False, timeline=None, chunk_steps=E.DEFAULT_CHUNKS):
    """SVF sweep + time loop for one site from host rasters: the work
    compute_utci does between reading and writing rasters
    (utci_process.py:1376-1470).  The time loop runs in chunks
    (``chunk_steps``: one length or a sequence of lengths) whose host tables
    are built while the GPU runs the previous chunk; ``timeline`` (an
    engine.Timeline) records the host phases of the call."""
    requested = _check_variables(requested)
    tl = timeline if timeline is not None else E.Timeline(enabled=False)
    site = E.DeviceSite(dsm, trees, dem, walls, aspect, scale, landcover=landcover, lc_class=lc_class,
                        windcoeff=windcoeff, params=_model_params(model_parameters))
    tl.mark("upload + prepare site", torch.cuda.current_stream())
    if return_device:
        site.run_svf()
        ser = site.build_series(met_file, altitude, azimuth, zen, jday, dectime, altmax, location)
        return site.run_time_loop(ser, requested=[k for k in N.OUT_BITS if k in requested])
    # host tables of later steps are built while the GPU runs earlier ones
    tables = site.start_tables(met_file, altitude, azimuth, zen, jday, dectime, altmax, location,
                               chunk_steps=chunk_steps)
    try:
        rasters_ready = torch.cuda.Event()   # the sun marches need the rasters only, not the SVF
        rasters_ready.record()
        site.run_svf()
        tl.mark("svf tables + sweep launch", torch.cuda.current_stream())
        out, _ = site.run_chain_chunked(met_file, altitude, azimuth, zen, jday, dectime, altmax, location,
                                        requested=requested, rasters_ready=rasters_ready, timeline=timeline,
                                        chunk_steps=chunk_steps, tables=tables)
    finally:
        tables.finish()
    return out
