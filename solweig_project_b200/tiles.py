"""Tile orchestration of a large raster, all tiles as one batch.

The reference cuts the study area into tiles of ``tile_size`` pixels plus
``overlap`` on the right / bottom (``solweig_gpu/preprocessor.py:341-385``
create_tiles_to_folder: windows [i, j, min(tile_size + overlap, W - i),
min(tile_size + overlap, H - j)] for i, j stepping by tile_size, keyed
"i_j" with i the column offset), then runs the chain tile by tile and
writes one multi-band GeoTIFF per output and tile, one band per step with
a "Time" item (``solweig_gpu/solweig_gpu.py:387-497`` run_utci_tiles,
``utci_process.py:1472-1651``).

:func:`run_tiles` keeps every tile resident and runs them as one
:class:`~solweig_project_b200.batch.SiteBatch` (one launch per stage for
all tiles); each tile is computed exactly as the reference computes it, on
its own window, so results equal single-tile runs bit for bit.
"""
from __future__ import annotations

import datetime as _dt
import os

import numpy as np

from . import batch as B
from . import formats as FM
from .engine import DeviceSite

F32 = np.float32
FILE_NAMES = {"utci": "UTCI", "tmrt": "TMRT", "kup": "Kup", "kdown": "Kdown", "lup": "Lup", "ldown": "Ldown",
              "shadow": "Shadow"}


def tile_windows(rows: int, cols: int, tile_size: int, overlap: int):
    """[(key, r0, r1, c0, c1)] of the reference's tiling (half-open windows)."""
    if overlap < 0 or overlap >= tile_size:
        raise ValueError("overlap must be 0 <= overlap < tilesize")
    if tile_size >= cols and tile_size >= rows:
        return [("0_0", 0, rows, 0, cols)]
    out = []
    for i in range(0, cols, tile_size):
        for j in range(0, rows, tile_size):
            w = min(tile_size + overlap, cols - i)
            h = min(tile_size + overlap, rows - j)
            out.append((f"{i}_{j}", j, j + h, i, i + w))
    return out


def _tile_geotransform(gt, r0, c0):
    if gt is None:
        return None
    x0, dx, rx, y0, ry, dy = gt
    return (x0 + c0 * dx + r0 * rx, dx, rx, y0 + c0 * ry + r0 * dy, ry, dy)


def run_tiles(*, dsm, trees, dem, walls, aspect, scale, met_file, altitude, azimuth, zen, jday, dectime, altmax,
              location, tile_size=3600, overlap=20, landcover=None, lc_class=None, requested=("utci", "tmrt"),
              output_dir=None, selected_date=None, geotransform=None, graph=False):
    """The chain for every tile of the reference's tiling, as one batch.
    Returns {key: {name: (T, h, w) float32}}; with ``output_dir`` also
    writes ``output_dir/<key>/<NAME>_<key>.tif`` (one band per step, "Time"
    = the selected date at the forcing row's hour and minute)."""
    rows, cols = np.asarray(dsm).shape
    wins = tile_windows(rows, cols, tile_size, overlap)
    sites, series = [], []
    for _, r0, r1, c0, c1 in wins:
        sl = (slice(r0, r1), slice(c0, c1))
        s = DeviceSite(np.asarray(dsm, F32)[sl], np.asarray(trees, F32)[sl], np.asarray(dem, F32)[sl],
                       np.asarray(walls, F32)[sl], np.asarray(aspect, F32)[sl], scale,
                       landcover=None if landcover is None else np.asarray(landcover, F32)[sl], lc_class=lc_class)
        series.append(s.build_series(met_file, altitude, azimuth, zen, jday, dectime, altmax, location))
        sites.append(s)
    batch = B.SiteBatch(sites, series, requested=requested)
    if graph:
        batch.replay()
    else:
        batch.run()
    results = {}
    for i, (key, r0, r1, c0, c1) in enumerate(wins):
        outs = {k: v.cpu().numpy() for k, v in batch.outputs(i).items()}
        results[key] = outs
        if output_dir is not None:
            folder = os.path.join(output_dir, key)
            os.makedirs(folder, exist_ok=True)
            base = _dt.datetime.fromisoformat(selected_date) if selected_date else _dt.datetime(2000, 1, 1)
            times = [{"Time": base.replace(hour=int(met_file[t, 2]), minute=int(met_file[t, 3])).isoformat()}
                     for t in range(len(met_file))]
            for name, arr in outs.items():
                path = os.path.join(folder, f"{FILE_NAMES[name]}_{key}.tif")
                with open(path, "wb") as fh:
                    fh.write(FM.tiff_bytes(arr, _tile_geotransform(geotransform, r0, c0), times[:arr.shape[0]]))
    return results
