"""Oracle: ground view factors (reference ``solweig_gpu/solweig.py:75-402``,
``sunonsurface_2018a`` and ``gvf_2018a``)."""
from __future__ import annotations

import numpy as np
import torch

from .svf import F32


def _pow4(x):
    """``x ** 4`` with torch's CPU pow (the reference's rounding)."""
    return torch.from_numpy(np.ascontiguousarray(x, F32)).pow(4).numpy()


def gvf_offsets(azimuth_deg_f32, second):
    """Per-step shifts of one ground-view-factor walk (solweig.py:136-178):
    index 0..second-1, float32 tensor trigonometry, ``.int()`` truncation."""
    az = torch.tensor(azimuth_deg_f32, dtype=torch.float32) * (torch.pi / 180)
    pb4 = torch.pi / 4
    sin_a, cos_a, tan_a = torch.sin(az), torch.cos(az), torch.tan(az)
    ssin, scos = torch.sign(sin_a), torch.sign(cos_a)
    branch_y = bool((pb4 <= az) & (az < 3 * pb4)) or bool((5 * pb4 <= az) & (az < 7 * pb4))
    tan_a, ssin, scos = F32(tan_a.item()), F32(ssin.item()), F32(scos.item())
    m_scos = F32(-1) * scos
    out = []
    for index in range(int(second)):
        fi = F32(index)
        if branch_y:
            dy = ssin * fi
            dx = m_scos * np.abs(np.rint(fi / tan_a))
        else:
            dy = ssin * np.abs(np.rint(fi * tan_a))
            dx = m_scos * fi
        out.append((int(dx), int(dy)))
    return out, F32(az.item())


def _shift_into(dst, src, dx, dy):
    """``dst[r, c] = src[r + dx, c + dy]`` inside the valid window only; the
    rest of ``dst`` keeps its previous content (the reference allocates the
    temporaries once per azimuth and never clears them)."""
    rows, cols = src.shape
    r0, r1 = max(0, -dx), min(rows, rows - dx)
    c0, c1 = max(0, -dy), min(cols, cols - dy)
    if r0 < r1 and c0 < c1:
        dst[r0:r1, c0:c1] = src[r0 + dx:r1 + dx, c0 + dy:c1 + dy]


def _facesh(az_rad_f32, aspect, wallbol):
    azt = torch.tensor(az_rad_f32)
    azilow = azt - torch.pi / 2
    azihigh = azt + torch.pi / 2
    if azilow >= 0 and azihigh < 2 * torch.pi:
        lo, hi = F32(azilow.item()), F32(azihigh.item())
        return np.logical_or(aspect < lo, aspect >= hi).astype(F32) - wallbol + F32(1)
    if azilow < 0 and azihigh <= 2 * torch.pi:
        azilow = azilow + 2 * torch.pi
    elif azilow > 0 and azihigh >= 2 * torch.pi:
        azihigh = azihigh - 2 * torch.pi
    lo, hi = F32(azilow.item()), F32(azihigh.item())
    return np.logical_or(aspect > lo, aspect <= hi).astype(F32) * F32(-1) + F32(1)


def sunonsurface(azimuth_deg, scale, buildings, shadow, sunwall, first, second, aspect, walls,
                 Tg, Tgwall, Ta, emis_grid, ewall, alb_grid, SBC, albedo_b):
    """One search azimuth of the GVF walk (solweig.py:75-288).  ``Ta`` is the
    float64 forcing value, ``Tgwall`` a float32 array broadcastable to the
    grid, ``first``/``second`` the rounded float32 walk lengths."""
    rows, cols = walls.shape
    wallbol = (walls > 0).astype(F32)
    sunwall = sunwall.copy()
    sunwall[sunwall > 0] = 1
    ta32 = F32(Ta)
    sbc = F32(SBC)
    ta4 = F32((torch.tensor(Ta, dtype=torch.float64) + 273.15) ** 4)
    Lup = sbc * emis_grid * _pow4(Tg * shadow + ta32 + F32(273.15)) - sbc * emis_grid * ta4
    ewall32 = F32(ewall)
    sbc_ewall = F32(torch.tensor(SBC) * torch.tensor(ewall))
    lwall_b = F32((torch.tensor(SBC) * torch.tensor(ewall)) * (torch.tensor(Ta, dtype=torch.float64) + 273.15) ** 4)
    Lwall = sbc_ewall * _pow4(Tgwall + ta32 + F32(273.15)) - lwall_b
    del ewall32
    albshadow = alb_grid * shadow
    alb = alb_grid
    z = lambda: np.zeros((rows, cols), F32)  # noqa: E731
    tempsh, tempbu, tempbub, tempbubwall, tempwallsun = z(), z(), z(), z(), z()
    weightsumsh, weightsumwall = z(), z()
    weightsumLupsh, weightsumLwall, weightsumalbsh, weightsumalbwall = z(), z(), z(), z()
    weightsumalbnosh, weightsumalbwallnosh = z(), z()
    tempLupsh, tempalbsh, tempalbnosh = z(), z(), z()
    first = F32(np.rint(F32(first) * F32(scale)))
    if first < 1:
        first = F32(1)
    second = F32(np.rint(F32(second) * F32(scale)))
    alb_b = F32(albedo_b)
    offsets, az_rad = gvf_offsets(F32(azimuth_deg), second)
    f = buildings
    snap = None
    for n, (dx, dy) in enumerate(offsets):
        _shift_into(tempbu, buildings, dx, dy)
        _shift_into(tempsh, shadow, dx, dy)
        _shift_into(tempLupsh, Lup, dx, dy)
        _shift_into(tempalbsh, albshadow, dx, dy)
        _shift_into(tempalbnosh, alb, dx, dy)
        f = np.minimum(f, tempbu)
        weightsumsh = weightsumsh + tempsh * f
        weightsumLupsh = weightsumLupsh + tempLupsh * f
        weightsumalbsh = weightsumalbsh + tempalbsh * f
        weightsumalbnosh = weightsumalbnosh + tempalbnosh * f
        _shift_into(tempwallsun, sunwall, dx, dy)
        tempb = tempwallsun * f
        tempbwall = f * F32(-1) + F32(1)
        tempbub = ((tempb + tempbub) > 0).astype(F32)
        tempbubwall = ((tempbwall + tempbubwall) > 0).astype(F32)
        weightsumLwall = weightsumLwall + tempbub * Lwall
        weightsumalbwall = weightsumalbwall + tempbub * alb_b
        weightsumwall = weightsumwall + tempbub
        weightsumalbwallnosh = weightsumalbwallnosh + tempbubwall * alb_b
        if (n + 1) <= first:
            snap = dict(wall=weightsumwall.copy(), sh=weightsumsh.copy(), Lwall=weightsumLwall.copy(),
                        Lupsh=weightsumLupsh.copy(), albwall=weightsumalbwall.copy(),
                        albsh=weightsumalbsh.copy(), albwallnosh=weightsumalbwallnosh.copy(),
                        albnosh=weightsumalbnosh.copy())
    wsi_f = (snap["wall"] > 0).astype(F32)
    wi_f = (snap["albwallnosh"] > 0).astype(F32)
    wsi_s = (weightsumwall > 0).astype(F32)
    wi_s = (weightsumalbwallnosh > 0).astype(F32)
    facesh = _facesh(az_rad, aspect, wallbol)
    keep = (weightsumwall == second).astype(F32) - facesh
    keep[keep == -1] = 0
    f1 = first + F32(1)
    s1 = second + F32(1)
    gvf1 = ((snap["wall"] + snap["sh"]) / f1) * wsi_f + (snap["sh"]) / first * (F32(1) - wsi_f)
    weightsumwall[keep == 1] = 0
    gvf2 = ((weightsumwall + weightsumsh) / s1) * wsi_s + (weightsumsh) / second * (F32(1) - wsi_s)
    gvf2[gvf2 > 1.] = 1.
    gvfLup1 = ((snap["Lwall"] + snap["Lupsh"]) / f1) * wsi_f + (snap["Lupsh"]) / first * (F32(1) - wsi_f)
    weightsumLwall[keep == 1] = 0
    gvfLup2 = ((weightsumLwall + weightsumLupsh) / s1) * wsi_s + (weightsumLupsh) / second * (F32(1) - wsi_s)
    gvfalb1 = ((snap["albwall"] + snap["albsh"]) / f1) * wsi_f + (snap["albsh"]) / first * (F32(1) - wsi_f)
    weightsumalbwall[keep == 1] = 0
    gvfalb2 = ((weightsumalbwall + weightsumalbsh) / s1) * wsi_s + (weightsumalbsh) / second * (F32(1) - wsi_s)
    gvfalbnosh1 = ((snap["albwallnosh"] + snap["albnosh"]) / f1) * wi_f + (snap["albnosh"]) / first * (F32(1) - wi_f)
    gvfalbnosh2 = ((weightsumalbwallnosh + weightsumalbnosh) / second) * wi_s + \
        (weightsumalbnosh) / second * (F32(1) - wi_s)
    gvf = (gvf1 * F32(0.5) + gvf2 * F32(0.4)) / F32(0.9)
    gvfLup = (gvfLup1 * F32(0.5) + gvfLup2 * F32(0.4)) / F32(0.9)
    nb = buildings * F32(-1) + F32(1)
    gvfLup = gvfLup + ((sbc * emis_grid * _pow4(Tg * shadow + ta32 + F32(273.15))) - sbc * emis_grid * ta4) * nb
    gvfalb = (gvfalb1 * F32(0.5) + gvfalb2 * F32(0.4)) / F32(0.9)
    gvfalb = gvfalb + alb_grid * nb * shadow
    gvfalbnosh = (gvfalbnosh1 * F32(0.5) + gvfalbnosh2 * F32(0.4)) / F32(0.9)
    gvfalbnosh = gvfalbnosh * buildings + alb_grid * nb
    return gvf, gvfLup, gvfalb, gvfalbnosh, gvf2


GVF_ORDER = ("gvfLup", "gvfalb", "gvfalbnosh", "gvfLupE", "gvfalbE", "gvfalbnoshE", "gvfLupS",
             "gvfalbS", "gvfalbnoshS", "gvfLupW", "gvfalbW", "gvfalbnoshW", "gvfLupN",
             "gvfalbN", "gvfalbnoshN", "gvfSum", "gvfNorm")


def gvf_2018a(wallsun, walls, buildings, scale, shadow, first, second, dirwalls, Tg, Tgwall, Ta,
              emis_grid, ewall, alb_grid, SBC, albedo_b):
    """18 search azimuths 5, 25, ..., 345 (solweig.py:291-402)."""
    rows, cols = walls.shape
    azimuthA = np.arange(5, 359, 20, dtype=np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        sunwall = ((wallsun / walls * buildings) == 1).astype(F32)
    aspect = (dirwalls * F32(np.pi)) / F32(180)
    z = lambda: np.zeros((rows, cols), F32)  # noqa: E731
    acc = {k: z() for k in GVF_ORDER[:-2]}
    gvfSum = z()
    for az in azimuthA:
        _, gLup, galb, galbnosh, gvf2 = sunonsurface(az, scale, buildings, shadow, sunwall, first, second,
                                                     aspect, walls, Tg, Tgwall, Ta, emis_grid, ewall,
                                                     alb_grid, SBC, albedo_b)
        acc["gvfLup"] = acc["gvfLup"] + gLup
        acc["gvfalb"] = acc["gvfalb"] + galb
        acc["gvfalbnosh"] = acc["gvfalbnosh"] + galbnosh
        gvfSum = gvfSum + gvf2
        for d, inside in (("E", 0 <= az < 180), ("S", 90 <= az < 270), ("W", 180 <= az < 360),
                          ("N", 270 <= az or az < 90)):
            if inside:
                acc["gvfLup" + d] = acc["gvfLup" + d] + gLup
                acc["gvfalb" + d] = acc["gvfalb" + d] + galb
                acc["gvfalbnosh" + d] = acc["gvfalbnosh" + d] + galbnosh
    lup_air = F32(SBC) * emis_grid * F32((torch.tensor(Ta, dtype=torch.float64) + 273.15) ** 4)
    n = F32(len(azimuthA))
    h = F32(len(azimuthA) / 2)
    out = {}
    out["gvfLup"] = acc["gvfLup"] / n + lup_air
    out["gvfalb"] = acc["gvfalb"] / n
    out["gvfalbnosh"] = acc["gvfalbnosh"] / n
    for d in "ESWN":
        out["gvfLup" + d] = acc["gvfLup" + d] / h + lup_air
        out["gvfalb" + d] = acc["gvfalb" + d] / h
        out["gvfalbnosh" + d] = acc["gvfalbnosh" + d] / h
    out["gvfSum"] = gvfSum
    norm = gvfSum / n
    norm[buildings == 0] = 1
    out["gvfNorm"] = norm
    return tuple(out[k].astype(F32) for k in GVF_ORDER)
