"""Spatial split of one large site across ranks with a static halo.

A pixel's results depend on the rasters within a bounded distance:

* its SVF marches read sources along 153 rays whose step tables end where
  the drop exceeds the height bound amaxvalue (shadow.py:241-300) -- except
  the zenith patch, whose result is "shaded iff any source up the column
  is in the grid" (its drop is negative at every step), so one in-grid row
  above settles it;
* its sun marches (solweig.py:1092-1149) end the same way, at every
  daytime step;
* its ground view factors walk `second` pixels over the sun-march records
  of its neighbours (solweig.py:136-192), which in turn read their own sun
  marches.

So with ``halo = max(longest SVF march, longest sun march + second) + 1``
pixels of the neighbouring parts around each part's core, and the site's
own amaxvalue for every part, each part's step tables equal the whole
site's (a march table ends by the height bound, not by the part's size)
and every source a core pixel reads lies in its window whenever it lies in
the site: the core results are the whole site's, bit for bit.  Walls and
aspect are taken from the whole site, cropped.  Bush scenes are refused:
their per-step bush flags test the whole grid (shadow.py:295).

The split needs no exchange between ranks while it runs; the rasters of a
window are copied to its rank once, and the cores are gathered at the end.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import tables as T

F32 = np.float32


@dataclass(frozen=True)
class Part:
    """A rank's share: its core rows [r0, r1) (all columns) and the window
    [w0, w1) of rows it computes (core plus halo, clipped to the site)."""
    r0: int
    r1: int
    w0: int
    w1: int

    @property
    def core_in_window(self):
        return slice(self.r0 - self.w0, self.r1 - self.w0)


def march_reach(rows, cols, scale, amax, sun_azimuths, sun_altitudes, second, patch_option=2):
    """Longest march (pixels along either axis) of the site's SVF tables
    (zenith patch excepted) and of the daytime sun tables, and the halo
    they ask for.  Returns (svf_reach, sun_reach, halo)."""
    plan, steps, _ = T.svf_plan(rows, cols, scale, F32(amax), False, patch_option)
    P = int(plan["n_patches"][0])
    svf = 0
    for q in range(P - 1):                       # the last patch is the zenith
        o, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
        if n:
            svf = max(svf, int(np.abs(steps["dx"][o:o + n]).max()), int(np.abs(steps["dy"][o:o + n]).max()))
    sun = 0
    for dx, dy, *_ in T.sun_tables(list(sun_azimuths), list(sun_altitudes), scale, F32(amax), rows, cols):
        if len(dx):
            sun = max(sun, int(np.abs(dx).max()), int(np.abs(dy).max()))
    return svf, sun, max(svf, sun + int(second)) + 1


def split_rows(rows, parts, halo):
    """Row bands of nearly equal size, each with `halo` rows of its
    neighbours on either side (clipped at the site's edges)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    bounds = np.linspace(0, rows, parts + 1).round().astype(int)
    out = []
    for k in range(parts):
        r0, r1 = int(bounds[k]), int(bounds[k + 1])
        out.append(Part(r0, r1, max(0, r0 - halo), min(rows, r1 + halo)))
    return out


def plan(dsm, trees, dem, scale, met, geometry, parts, second=None):
    """The parts of a site for `parts` ranks, the site's amaxvalue and the
    halo.  `geometry`: the sun-geometry arrays of the forcing
    (altitude / azimuth (1, T), as run_utci_window takes them).  A halo that
    covers the whole site means no split helps: every part is then the
    whole site."""
    from .engine import march_inputs
    _, _, bush, amax, _ = march_inputs(dsm, trees, dem)
    if bush.max() > 0:
        raise ValueError("sites with bush are not split: their bush step flags test the whole grid")
    rows, cols = np.shape(dsm)
    alt = np.asarray(geometry["altitude"])[0]
    azi = np.asarray(geometry["azimuth"])[0]
    day = alt > 0
    if second is None:
        second = int(round(22 * float(scale)))    # round(height 1.1 m * 20 * scale), solweig.py:2051-2058
    _, _, halo = march_reach(rows, cols, scale, amax, azi[day].tolist(), alt[day].tolist(), second)
    return split_rows(rows, parts, halo), amax, halo


def stitch(parts, cores, rows):
    """{name: (T, rows, cols)} from each part's core outputs."""
    out = {}
    for p, c in zip(parts, cores):
        for k, v in c.items():
            if k not in out:
                out[k] = np.empty((v.shape[0], rows) + v.shape[2:], v.dtype)
            out[k][:, p.r0:p.r1] = v
    return out
