"""Oracle: wall-height sun march (reference ``solweig_gpu/solweig.py:1079-1224``,
``shadowingfunction_wallheight_23``)."""
from __future__ import annotations

import numpy as np
import torch

from .svf import F32, _shift, torch_max


def sun_step_table(azimuth, altitude, scale, amaxvalue, rows, cols):
    """Executed (dx, dy, dz) of the sun march: index starts at 0 (the self
    comparison), no azimuth-zero substitution, float32 tensor branch bounds
    (solweig.py:1092-1149).  ``azimuth``/``altitude`` are python floats in
    degrees (the reference passes ``.item()`` of float64 tensors)."""
    degrees = torch.tensor(np.pi / 180.0)
    az = torch.tensor(azimuth) * degrees
    alt = torch.tensor(altitude) * degrees
    pb4 = torch.tensor(np.pi / 4.0)
    sin_a, cos_a, tan_a = torch.sin(az), torch.cos(az), torch.tan(az)
    ssin, scos = torch.sign(sin_a), torch.sign(cos_a)
    dssin = torch.abs(1 / sin_a)
    dscos = torch.abs(1 / cos_a)
    tanalt = torch.tan(alt) / scale
    branch_y = bool((pb4 <= az) & (az < 3 * pb4)) or bool((5 * pb4 <= az) & (az < 7 * pb4))
    tan_a, ssin, scos = F32(tan_a.item()), F32(ssin.item()), F32(scos.item())
    ds = F32(dssin.item()) if branch_y else F32(dscos.item())
    tanalt = F32(tanalt.item())
    amax = F32(amaxvalue)
    m_scos = F32(-1) * scos
    dxs, dys, dzs = [], [], []
    dx = dy = dz = F32(0.)
    index = 0
    while amax >= dz and abs(dx) < rows and abs(dy) < cols:
        fi = F32(index)
        if branch_y:
            dy = ssin * fi
            dx = m_scos * np.abs(np.rint(fi / tan_a))
        else:
            dy = ssin * np.abs(np.rint(fi * tan_a))
            dx = m_scos * fi
        dz = (ds * fi) * tanalt
        dxs.append(int(dx))
        dys.append(int(dy))
        dzs.append(dz)
        index += 1
    az_f = F32(az.item())
    return np.array(dxs, np.int64), np.array(dys, np.int64), np.array(dzs, np.float32), az_f


def facesh_plane(az_rad, aspect_rad, wallbol):
    """Wall faces turned away from the sun (solweig.py:1187-1196)."""
    azt = torch.tensor(az_rad)
    azilow = azt - torch.pi / 2
    azihigh = azt + torch.pi / 2
    if azilow >= 0 and azihigh < 2 * torch.pi:
        lo, hi = F32(azilow.item()), F32(azihigh.item())
        return (np.logical_or(aspect_rad < lo, aspect_rad >= hi).astype(F32) - wallbol + F32(1))
    if azilow < 0 and azihigh <= 2 * torch.pi:
        azilow = azilow + 2 * torch.pi
    elif azilow > 0 and azihigh >= 2 * torch.pi:
        azihigh = azihigh - 2 * torch.pi
    else:  # pragma: no cover - the reference leaves facesh undefined here
        raise ValueError("azimuth outside the reference's facesh branches")
    lo, hi = F32(azilow.item()), F32(azihigh.item())
    return np.logical_or(aspect_rad > lo, aspect_rad <= hi).astype(F32) * F32(-1) + F32(1)


def wallheight_23(a, vegdem, vegdem2, azimuth, altitude, scale, amaxvalue, bush, walls, aspect_rad):
    """Sun march + wall tail; returns (vegsh, sh, vbshvegsh, wallsh, wallsun,
    wallshve, facesh, facesun) as float32 planes."""
    a = np.asarray(a, F32)
    rows, cols = a.shape
    dxs, dys, dzs, az_f = sun_step_table(azimuth, altitude, scale, amaxvalue, rows, cols)
    bushplant = (bush > 1).astype(F32)
    sh = np.zeros_like(a)
    vbshvegsh = np.zeros_like(a)
    vegsh = np.zeros_like(a) + bushplant
    f = a
    shvoveg = vegdem
    wallbol = (walls > 0).astype(F32)
    dzprev = F32(0.)
    ones = np.ones_like(a)
    for dx, dy, dz in zip(dxs, dys, dzs):
        inb = _shift(ones, dx, dy) > 0
        tempvegdem = np.where(inb, _shift(vegdem, dx, dy) - dz, F32(0.)).astype(F32)
        tempvegdem2 = np.where(inb, _shift(vegdem2, dx, dy) - dz, F32(0.)).astype(F32)
        temp = np.where(inb, _shift(a, dx, dy) - dz, F32(0.)).astype(F32)
        f = torch_max(f, temp)
        shvoveg = torch_max(shvoveg, tempvegdem)
        sh = np.where(f > a, F32(1.), F32(0.))
        fabovea = (tempvegdem > a).astype(F32)
        gabovea = (tempvegdem2 > a).astype(F32)
        tlf = np.where(inb, _shift(vegdem, dx, dy) - dzprev, F32(0.)).astype(F32)
        tlg = np.where(inb, _shift(vegdem2, dx, dy) - dzprev, F32(0.)).astype(F32)
        lastfabovea = tlf > a
        lastgabovea = tlg > a
        dzprev = dz
        vegsh2 = fabovea + gabovea + lastfabovea.astype(F32) + lastgabovea.astype(F32)
        vegsh2 = np.where(vegsh2 == 4, F32(0.), vegsh2)
        vegsh2 = np.where(vegsh2 > 0, F32(1.), vegsh2)
        vegsh = torch_max(vegsh, vegsh2)
        vegsh = np.where(vegsh * sh > 0, F32(0.), vegsh)
        vbshvegsh = vbshvegsh + vegsh
    facesh = facesh_plane(az_f, aspect_rad, wallbol)
    sh = F32(1) - sh
    vbshvegsh = np.where(vbshvegsh > 0, F32(1.), vbshvegsh)
    vbshvegsh = vbshvegsh - vegsh
    vegsh = np.where(vegsh > 0, F32(1.), vegsh)
    shvoveg = (shvoveg - a) * vegsh
    vegsh = F32(1) - vegsh
    vbshvegsh = F32(1) - vbshvegsh
    shvo = f - a
    facesun = np.logical_and(facesh + wallbol == 1, walls > 0).astype(F32)
    wallsun = walls - shvo
    wallsun = np.where(wallsun < 0, F32(0.), wallsun)
    wallsun = np.where(facesh == 1, F32(0.), wallsun)
    wallsh = walls - wallsun
    wallshve = shvoveg * wallbol
    wallshve = wallshve - wallsh
    wallshve = np.where(wallshve < 0, F32(0.), wallshve)
    wallsun = wallsun - wallshve
    wallsun = np.where(wallsun < 0, F32(0.), wallsun)
    wallshve = np.where(wallshve > walls, walls, wallshve)
    res = (vegsh, sh, vbshvegsh, wallsh, wallsun, wallshve, facesh, facesun)
    return tuple(np.asarray(x, F32) for x in res)


def aspect_radians(dirwalls):
    """``dirwalls * np.pi / 180.`` as the time loop passes it (solweig.py:2083)."""
    return (np.asarray(dirwalls, F32) * F32(np.pi)) / F32(180.)
