"""Seeded synthetic cities and meteorological forcing.

The workloads the project is measured on are synthetic: flat DEM, axis-aligned
rectangular buildings, Gaussian tree canopies, a land-cover grid derived from
the masks and 24 hourly forcing rows.  The shapes follow the reference's raster
contract (``Building_DSM``, ``Trees`` (canopy height above ground), ``DEM``,
land cover codes from ``solweig_gpu/landcoverclasses_2016a.txt``) and its met
file column layout (``solweig_gpu/utci_process.py:796-815``: 1 DOY, 2 hour,
3 minute, 9 wind, 10 RH, 11 Ta, 12 P [kPa], 14 global radiation, 21 diffuse,
22 direct, 23 wind direction, 24 urban heat island increment).

Everything is driven by ``numpy.random.default_rng(seed)`` so every caller
(tests, bench, fixtures) regenerates bit-identical inputs from a seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# Land-cover codes (solweig_gpu/landcoverclasses_2016a.txt)
LC_PAVED = 1
LC_BUILDING = 2
LC_GRASS = 5

# Default site (Austin, TX) used by the single-site workloads.
DEFAULT_LOCATION = {"latitude": 30.3, "longitude": -97.7, "altitude": 3.0}
DEFAULT_UTC = -5.0
DEFAULT_YEAR = 2024
DEFAULT_DOY = 196


@dataclass
class City:
    """Raster inputs of one site, all float32 (rows, cols)."""

    dsm: np.ndarray          # building DSM (ground + buildings), m
    trees: np.ndarray        # canopy height above ground, m (``temp1``)
    dem: np.ndarray          # ground elevation, m (``temp2``)
    landcover: np.ndarray    # land-cover codes (float32)
    scale: float = 1.0       # pixels per metre
    walls: np.ndarray | None = None    # wall height, m
    aspect: np.ndarray | None = None   # wall aspect, degrees
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return self.dsm.shape


def _paint_buildings(rng, rows, cols, dsm, n_buildings, side_lo, side_hi, h_lo, h_hi,
                     density=None):
    """Axis-aligned rectangles painted with ``max``.

    With ``density`` set, rectangles are added until the built-up fraction
    reaches it (bounded by ``n_buildings`` * 50 attempts as a safety net).
    """
    placed = 0
    attempts = 0
    built = int(np.count_nonzero(dsm > 0))
    limit = n_buildings if density is None else max(1, n_buildings) * 50
    while attempts < limit:
        attempts += 1
        h = int(rng.integers(side_lo, side_hi + 1))
        w = int(rng.integers(side_lo, side_hi + 1))
        r0 = int(rng.integers(0, rows))
        c0 = int(rng.integers(0, cols))
        height = np.float32(rng.uniform(h_lo, h_hi))
        blk = dsm[r0:r0 + h, c0:c0 + w]
        before = int(np.count_nonzero(blk > 0)) if density is not None else 0
        np.maximum(blk, height, out=blk)
        placed += 1
        if density is not None:
            built += int(np.count_nonzero(blk > 0)) - before   # running count of (dsm > 0)
            if built / dsm.size >= density:
                break
    return placed


def _paint_trees(rng, rows, cols, canopy, n_trees, r_lo, r_hi, p_lo, p_hi, cover=None):
    """Gaussian canopies truncated at their radius (sigma = radius / 2)."""
    yy = np.arange(rows, dtype=np.float64)[:, None]
    xx = np.arange(cols, dtype=np.float64)[None, :]
    attempts = 0
    covered = int(np.count_nonzero(canopy > 0))
    limit = n_trees if cover is None else max(1, n_trees) * 50
    while attempts < limit:
        attempts += 1
        cy = rng.uniform(0, rows)
        cx = rng.uniform(0, cols)
        rad = rng.uniform(r_lo, r_hi)
        peak = rng.uniform(p_lo, p_hi)
        r0, r1 = max(0, int(cy - rad) - 1), min(rows, int(cy + rad) + 2)
        c0, c1 = max(0, int(cx - rad) - 1), min(cols, int(cx + rad) + 2)
        if r0 >= r1 or c0 >= c1:
            continue
        d2 = (yy[r0:r1] - cy) ** 2 + (xx[:, c0:c1] - cx) ** 2
        sigma = rad / 2.0
        h = peak * np.exp(-d2 / (2.0 * sigma * sigma))
        h[d2 > rad * rad] = 0.0
        blk = canopy[r0:r1, c0:c1]
        before = int(np.count_nonzero(blk > 0)) if cover is not None else 0
        np.maximum(blk, h.astype(np.float32), out=blk)
        if cover is not None:
            covered += int(np.count_nonzero(blk > 0)) - before   # running count of (canopy > 0)
            if covered / canopy.size >= cover:
                break


def make_city(rows: int, cols: int | None = None, seed: int = 1234, *,
              n_buildings: int | None = None, n_trees: int | None = None,
              h_max: float = 40.0, density: float | None = None,
              canopy_cover: float | None = None, scale: float = 1.0,
              dem_level: float = 0.0, with_walls: bool = True,
              side_range: tuple[int, int] | None = None,
              tree_peak: tuple[float, float] = (5.0, 15.0)) -> City:
    """Seeded synthetic city.

    Defaults follow the single-site workloads: 40 buildings (sides 10-40 px,
    heights U(5, ``h_max``)) and 30 canopies (radius U(2, 6), peak U(5, 15))
    per 200x200 px, scaled by area; canopies are zeroed on buildings.  With
    ``density`` / ``canopy_cover`` the painters run until those fractions are
    reached (batched multi-site workload).
    """
    cols = rows if cols is None else cols
    rng = np.random.default_rng(seed)
    area = rows * cols / (200.0 * 200.0)
    if n_buildings is None:
        n_buildings = max(1, int(round(40 * area)))
    if n_trees is None:
        n_trees = int(round(30 * area))
    dsm = np.zeros((rows, cols), np.float32)
    if side_range is None:
        side_hi = max(2, min(40, rows, cols))
        side_lo = min(10, side_hi)
    else:
        side_lo, side_hi = side_range
    _paint_buildings(rng, rows, cols, dsm, n_buildings, side_lo, side_hi, 5.0, h_max, density)
    canopy = np.zeros((rows, cols), np.float32)
    if n_trees > 0 or (canopy_cover or 0) > 0:
        _paint_trees(rng, rows, cols, canopy, max(n_trees, 1), 2.0, 6.0, tree_peak[0], tree_peak[1],
                     canopy_cover)
    canopy[dsm > 0] = 0.0
    dem = np.full((rows, cols), np.float32(dem_level), np.float32)
    dsm = (dsm + dem).astype(np.float32)
    lc = np.full((rows, cols), LC_PAVED, np.float32)
    lc[canopy > 0] = LC_GRASS
    lc[(dsm - dem) > 0] = LC_BUILDING
    city = City(dsm=dsm, trees=canopy, dem=dem, landcover=lc, scale=float(scale),
                meta={"seed": seed, "h_max": h_max, "density": density,
                      "canopy_cover": canopy_cover})
    if with_walls:
        from .walls_aspect import findwalls, filter1Goodwin_as_aspect_v3
        city.walls = findwalls(dsm, 3.0).astype(np.float32)
        city.aspect = filter1Goodwin_as_aspect_v3(city.walls, city.scale, dsm).astype(np.float32)
    return city


def make_met(seed: int = 1234, year: int = DEFAULT_YEAR, doy: int = DEFAULT_DOY,
             hours: int = 24, uhii: float = 0.0) -> np.ndarray:
    """24 hourly forcing rows in the reference's met-file column layout.

    Ta = 30 + 6 cos(2 pi (h - 15) / 24) (24-36 C, peak 15:00); RH inverse
    (70 -> 35 %); clear-sky global radiation peaking at 900 W/m2; wind
    U(0.5, 4) m/s; P = 100 kPa; diffuse/direct/wind direction = -999.
    """
    rng = np.random.default_rng(seed + 7919)
    met = np.full((hours, 25), -999.0, np.float64)
    h = np.arange(hours, dtype=np.float64)
    phase = np.cos(2.0 * math.pi * (h - 15.0) / 24.0)
    met[:, 0] = year
    met[:, 1] = doy
    met[:, 2] = h
    met[:, 3] = 0.0
    met[:, 9] = np.round(rng.uniform(0.5, 4.0, hours), 2)
    met[:, 10] = np.round(52.5 - 17.5 * phase, 2)
    met[:, 11] = np.round(30.0 + 6.0 * phase, 2)
    met[:, 12] = 100.0
    met[:, 14] = np.round(np.maximum(0.0, 900.0 * np.sin(math.pi * (h - 6.0) / 14.0)), 2)
    met[:, 21] = -999.0
    met[:, 22] = -999.0
    met[:, 23] = -999.0
    met[:, 24] = uhii
    return met


def multi_site_specs(n_sites: int = 64, seed: int = 2024):
    """Seeded specs of the batched workload: square sides log-uniform in
    [128, 1024] px, building density U(10, 45) %, canopy cover U(0, 30) %,
    latitude U(0, 60) N (longitude -97.7, UTC-5)."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_sites):
        side = int(round(math.exp(rng.uniform(math.log(128), math.log(1024)))))
        specs.append({"seed": int(seed * 1000 + i), "side": side, "density": float(rng.uniform(0.10, 0.45)),
                      "canopy": float(rng.uniform(0.0, 0.30)), "latitude": float(rng.uniform(0.0, 60.0)),
                      "longitude": DEFAULT_LOCATION["longitude"]})
    return specs


def default_lc_class() -> np.ndarray:
    """Land-cover class table (code, albedo, emissivity, TgK, Tstart, TmaxLST)
    as the reference loads landcoverclasses_2016a.txt (utci_process.py:1310-1316)."""
    import json
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "landcover_classes.json")
    with open(path) as fh:
        rows = json.load(fh)["classes"]
    return np.array([r[1:] for r in rows], np.float64)


def load_sun_geometry(prefix: str, path: str | None = None):
    """Sun geometry arrays (float64, (1, 24)) recorded for a workload."""
    import os
    if path is None:
        path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden",
                            "sun_geometry.npz")
    with np.load(path) as z:
        return {k: z[f"{prefix}_{k}"] for k in ("altitude", "azimuth", "zen", "jday", "dectime", "altmax")}
