"""Wall height and wall aspect from a DSM (host-side input preparation).

Vectorised restatement of ``solweig_gpu/walls_aspect.py``: the reference
visits every pixel in Python loops (180 filter rotations x rows x cols); here
each rotation is one pass of shifted-plane sums over the whole grid, with the
same per-pixel update rule and the same summation order, so the outputs are
identical on the same DSM.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.ndimage import rotate

WALL_LIMIT = 3.0


def findwalls(dem_array: np.ndarray, walllimit: float = WALL_LIMIT) -> np.ndarray:
    """Wall height = max of the 4-neighbours minus the cell, zeroed below
    ``walllimit`` and on the one-pixel border (walls_aspect.py:27-56)."""
    dem = np.asarray(dem_array)
    rows, cols = dem.shape
    walls = np.zeros((rows, cols), np.float64)
    if rows >= 3 and cols >= 3:
        nb = np.maximum(np.maximum(dem[0:-2, 1:-1], dem[2:, 1:-1]),
                        np.maximum(dem[1:-1, 0:-2], dem[1:-1, 2:]))
        walls[1:-1, 1:-1] = nb
    walls = walls - dem
    walls[walls < walllimit] = 0
    walls[:, 0] = 0
    walls[:, -1] = 0
    walls[0, :] = 0
    walls[-1, :] = 0
    return walls


def get_ders(dsm: np.ndarray, scale: float):
    """Slope and aspect of the DSM (walls_aspect.py:78-97)."""
    dx = 1 / scale
    fy, fx = np.gradient(dsm, dx, dx)
    theta = np.arctan2(fx, fy)
    grad = np.arctan(np.sqrt(fy ** 2 + fx ** 2))
    asp = -theta
    asp[asp < 0] += 2 * np.pi
    return grad, asp


def filter1Goodwin_as_aspect_v3(walls: np.ndarray, scale: float, a: np.ndarray) -> np.ndarray:
    """Wall aspect in degrees by a rotating line filter
    (walls_aspect.py:99-161): for each of 180 orientations the number of wall
    pixels under the rotated line is compared with the best so far; the side
    with the higher summed DSM decides between the two opposite aspects."""
    rows, cols = a.shape
    filtersize = int(np.floor((scale + 1e-10) * 9))
    if filtersize <= 2:
        filtersize = 3
    elif filtersize != 9 and filtersize % 2 == 0:
        filtersize += 1
    n = filtersize - 1
    hc = int(np.ceil(filtersize / 2.))
    hf = int(np.floor(filtersize / 2.))

    filtmatrix = np.zeros((filtersize, filtersize))
    buildfilt = np.zeros((filtersize, filtersize))
    filtmatrix[:, hc - 1] = 1
    buildfilt[hc - 1, :hf] = 1
    buildfilt[hc - 1, hc:] = 2

    y = np.zeros((rows, cols))
    x = np.zeros((rows, cols))
    wall_u8 = (walls > 0).astype(np.uint8)
    a32 = np.asarray(a, np.float32)

    # pixel block visited by the reference loops
    i0, i1 = hc - 1, rows - hc - 1
    j0, j1 = hc - 1, cols - hc - 1
    if i1 > i0 and j1 > j0:
        # only wall pixels of the block are ever updated: evaluate the
        # filters there (same per-pixel sums, in the same order)
        wr, wc = np.nonzero(wall_u8[i0:i1, j0:j1] == 1)
        wr, wc = wr + i0, wc + j0
        zw = np.zeros(wr.size, np.float64)
        for h in range(0, 180):
            filt1 = np.round(rotate(filtmatrix, h, order=1, reshape=False, mode='nearest'))
            filtb = np.round(rotate(buildfilt, h, order=0, reshape=False, mode='nearest'))
            index = 270 - h
            if h in (150, 30):
                filtb[:, n] = 0
            if index == 225:
                filt1[0, 0] = filt1[n, n] = 1
            if index == 135:
                filt1[0, n] = filt1[n, 0] = 1
            # wall count under the rotated line (exact small integers)
            offs = [(di - hf, dj - hf) for di in range(filtersize) for dj in range(filtersize)
                    if filt1[di, dj] != 0]
            weights = [filt1[di + hf, dj + hf] for di, dj in offs]
            cnt = np.zeros(wr.size, np.float64)
            for (di, dj), w in zip(offs, weights):
                cnt = cnt + wall_u8[wr + di, wc + dj] * w
            upd = zw < cnt
            if not upd.any():
                continue
            o1 = [(di - hf, dj - hf) for di in range(filtersize) for dj in range(filtersize)
                  if filtb[di, dj] == 1]
            o2 = [(di - hf, dj - hf) for di in range(filtersize) for dj in range(filtersize)
                  if filtb[di, dj] == 2]
            ur, uc = wr[upd], wc[upd]
            s1 = np.zeros(ur.size, np.float32)
            for di, dj in o1:
                s1 = s1 + a32[ur + di, uc + dj]
            s2 = np.zeros(ur.size, np.float32)
            for di, dj in o2:
                s2 = s2 + a32[ur + di, uc + dj]
            zw[upd] = cnt[upd]
            x[ur, uc] = np.where(s1 > s2, 1, 2)
            y[ur, uc] = index

    y[x == 1] -= 180
    y[y < 0] += 360
    _, asp = get_ders(a32, scale)
    y += ((wall_u8 == 1) & (y == 0)) * (asp / (math.pi / 180.))
    return y
