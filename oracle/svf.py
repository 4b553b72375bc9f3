"""Oracle: SVF patch sweep (reference ``solweig_gpu/shadow.py``).

* :func:`create_patches` -- ``shadow.py:352-406`` (sky vault patch layout)
* :func:`annulus_weight` -- ``shadow.py:324-350``
* :func:`shadow_step_table` -- the scalar part of ``shadow.py:166-247``
  (per-step shifts and height drops of one patch march)
* :func:`shadow_patch` -- ``shadow.py:166-322`` (one patch march over planes)
* :func:`svf_calculator` -- ``shadow.py:409-625`` (153-patch sweep + sums)
"""
from __future__ import annotations

import numpy as np
import torch

F32 = np.float32

_PATCH_LAYOUT = {
    # option: (annulino, altitude bands, azimuth start, patches per band)
    1: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [30, 30, 24, 24, 18, 12, 6, 1]),
    2: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [31, 30, 28, 24, 19, 13, 7, 1]),
    3: ([0, 12, 24, 36, 48, 60, 72, 84, 90], [6, 18, 30, 42, 54, 66, 78, 90],
        [0, 4, 2, 5, 8, 0, 10, 0], [62, 60, 56, 48, 38, 26, 14, 1]),
}


def create_patches(patch_option: int = 2):
    """Patch altitudes/azimuths (float32) and band layout (shadow.py:352-406)."""
    annulino, altint, azistart, nband = _PATCH_LAYOUT[patch_option]
    nband_t = torch.tensor(nband)
    aziint = 360 / nband_t  # float32 band widths
    alt, azi = [], []
    for j in range(len(altint)):
        for k in range(nband[j]):
            alt.append(torch.tensor([altint[j]], dtype=torch.float32))
            azi.append((k * aziint[j] + torch.tensor(azistart[j])).reshape(1).float())
    return (torch.cat(alt).numpy(), torch.cat(azi).numpy(), np.array(annulino), np.array(altint),
            np.array(nband), aziint.numpy(), np.array(azistart))


def annulus_weight(k: int, n) -> np.float32:
    """Solid-angle weight of annulus ``k`` split over ``n`` azimuth bins
    (shadow.py:324-350); ``n`` is an int64 (iso) or float32 (aniso) 0-dim
    tensor as in the reference."""
    nn = torch.tensor(90.0)
    altitude = torch.tensor(k)
    steprad = (360.0 / n) * (torch.pi / 180.0)
    annulus = 91.0 - altitude
    w = (1.0 / (2.0 * torch.pi)) * torch.sin(torch.pi / (2.0 * nn)) * \
        torch.sin((torch.pi * (2.0 * annulus - 1.0)) / (2.0 * nn))
    return F32((steprad * w).item())


def patch_azimuths(patch_option: int = 2) -> np.ndarray:
    """``iazimuth`` of svf_calculator (shadow.py:530-541), float32.

    The per-band count is ``int(360 / float32(360 / n))``, which truncates to
    ``n - 1`` for several bands; the vector is pre-filled with zeros, so the
    later patches take shifted azimuths and the last few keep azimuth 0."""
    annulino, altint, azistart, nband = _PATCH_LAYOUT[patch_option]
    aziint = torch.tensor([360 / p for p in torch.tensor(nband)])
    out = np.zeros(int(sum(nband)), np.float32)
    index = 0
    for j in range(len(altint)):
        for k in range(int(360 / aziint[j])):
            v = k * aziint[j] + torch.tensor(azistart[j])
            if v > 360.:
                v = v - 360.
            out[index] = F32(v.item())
            index += 1
    return out


def shadow_step_table(azimuth_deg, altitude_deg, scale, amaxvalue, rows, cols):
    """Executed (dx, dy, dz) sequence of one ``shadow()`` march.

    ``azimuth_deg`` is the float32 patch azimuth, ``altitude_deg`` the integer
    band altitude.  Trigonometry runs on 0-dim float32 torch tensors exactly as
    in shadow.py:196-226; the per-step arithmetic is IEEE float32
    (shadow.py:230-239).  Returns int arrays dx, dy and float32 dz.
    """
    degrees = torch.pi / 180.
    if float(azimuth_deg) == 0.0:
        az = torch.tensor(1e-12)
    else:
        az = torch.tensor(F32(azimuth_deg))
    alt = torch.tensor(int(altitude_deg)) if float(altitude_deg).is_integer() \
        else torch.tensor(F32(altitude_deg))
    az = az * degrees
    alt = alt * degrees
    sin_a, cos_a, tan_a = torch.sin(az), torch.cos(az), torch.tan(az)
    ssin, scos = torch.sign(sin_a), torch.sign(cos_a)
    dssin = torch.abs(1. / sin_a)
    dscos = torch.abs(1. / cos_a)
    tanalt = torch.tan(alt) / scale
    pb4 = torch.pi / 4.
    branch_y = bool((pb4 <= az) & (az < 3. * pb4)) or bool((5. * pb4 <= az) & (az < 7. * pb4))
    tan_a, ssin, scos = F32(tan_a.item()), F32(ssin.item()), F32(scos.item())
    ds = F32(dssin.item()) if branch_y else F32(dscos.item())
    tanalt = F32(tanalt.item())
    amax = F32(amaxvalue)
    m_scos = F32(-1.) * scos
    dxs, dys, dzs = [], [], []
    dx = dy = dz = F32(0.)
    index = 1
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
    return np.array(dxs, np.int64), np.array(dys, np.int64), np.array(dzs, np.float32)


def _shift(plane, dx, dy, fill=0.0):
    """``out[r, c] = plane[r + dx, c + dy]`` where in bounds, else ``fill``."""
    rows, cols = plane.shape
    out = np.full_like(plane, fill)
    r0, r1 = max(0, -dx), min(rows, rows - dx)
    c0, c1 = max(0, -dy), min(cols, cols - dy)
    if r0 < r1 and c0 < c1:
        out[r0:r1, c0:c1] = plane[r0 + dx:r1 + dx, c0 + dy:c1 + dy]
    return out


def torch_max(x, y):
    """``torch.max(x, y)``: NaN propagates; on ties the second operand wins."""
    return np.where((x > y) | np.isnan(x), x, y)


def shadow_patch(amaxvalue, a, vegdem, vegdem2, bush, azimuth_deg, altitude_deg, scale):
    """One SVF patch march (shadow.py:166-322) -> (sh, vegsh, vbshvegsh)."""
    rows, cols = a.shape
    dxs, dys, dzs = shadow_step_table(azimuth_deg, altitude_deg, scale, amaxvalue, rows, cols)
    f = a.copy()
    g = np.zeros_like(a)
    sh = np.zeros_like(a)
    vbshvegsh = np.zeros_like(a)
    bushplant = (bush > 1.).astype(F32)
    vegsh = np.zeros_like(a) + bushplant
    bush_any = bool(bush.max() > 0.) if bush.size else False
    for step, (dx, dy, dz) in enumerate(zip(dxs, dys, dzs)):
        inb = _shift(np.ones_like(a), dx, dy)
        tempvegdem = np.where(inb > 0, _shift(vegdem, dx, dy) - dz, F32(0.)).astype(F32)
        tempvegdem2 = np.where(inb > 0, _shift(vegdem2, dx, dy) - dz, F32(0.)).astype(F32)
        temp = np.where(inb > 0, _shift(a, dx, dy) - dz, F32(0.)).astype(F32)
        f = torch_max(f, temp)
        sh = np.where(f > a, F32(1.), np.where(f <= a, F32(0.), sh)).astype(F32)
        fabovea = tempvegdem > a
        gabovea = tempvegdem2 > a
        vegsh2 = fabovea.astype(F32) - gabovea.astype(F32)
        vegsh = torch_max(vegsh, vegsh2)
        vegsh[(vegsh * sh) > 0.] = 0.
        vbshvegsh = vegsh + vbshvegsh
        if step == 0:
            firstvegdem = tempvegdem - temp
            firstvegdem[firstvegdem <= 0.] = 1000.
            vegsh[firstvegdem < dz] = 1.
            vegsh = vegsh * (vegdem2 > a).astype(F32)
            vbshvegsh[...] = 0.
        if bush_any and float(np.max(fabovea * bush)) > 0.:
            tempbush = np.where(inb > 0, _shift(bush, dx, dy) - dz, F32(0.)).astype(F32)
            g = torch_max(g, tempbush)
            g = g * bushplant
    sh = F32(1.) - sh
    vbshvegsh[vbshvegsh > 0.] = 1.
    vbshvegsh = vbshvegsh - vegsh
    if bush_any:
        g = g - bush
        g[g > 0.] = 1.
        g[g < 0.] = 0.
        vegsh = vegsh - bushplant + g
        vegsh[vegsh < 0.] = 0.
    vegsh[vegsh > 0.] = 1.
    vegsh = F32(1.) - vegsh
    vbshvegsh = F32(1.) - vbshvegsh
    return sh.astype(F32), vegsh.astype(F32), vbshvegsh.astype(F32), len(dzs)


SVF_ORDER = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg",
             "svfS", "svfSaveg", "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg",
             "vegshmat", "vbshvegshmat", "shmat", "svftotal")


def svf_calculator(patch_option, amaxvalue, a, vegdem, vegdem2, bush, scale, return_steps=False):
    """153-patch sweep (shadow.py:409-625); returns the reference's 19-tuple
    (15 SVF planes, 3 (rows, cols, P) cubes, SVFtotal)."""
    a = np.asarray(a, F32)
    vegdem = np.asarray(vegdem, F32)
    vegdem2 = np.asarray(vegdem2, F32)
    bush = np.asarray(bush, F32)
    rows, cols = a.shape
    z = lambda: np.zeros((rows, cols), F32)  # noqa: E731
    svf, svfE, svfS, svfW, svfN = z(), z(), z(), z(), z()
    svfveg, svfEveg, svfSveg, svfWveg, svfNveg = z(), z(), z(), z(), z()
    svfaveg, svfEaveg, svfSaveg, svfWaveg, svfNaveg = z(), z(), z(), z(), z()
    annulino, altint, _, nband = _PATCH_LAYOUT[patch_option]
    P = int(sum(nband))
    iaz = patch_azimuths(patch_option)
    shmat = np.zeros((rows, cols, P), F32)
    vegshmat = np.zeros((rows, cols, P), F32)
    vbshmat = np.zeros((rows, cols, P), F32)
    nband_t = torch.tensor(nband)
    aniso_t = torch.ceil(nband_t / 2.0)
    steps = []
    index = 0
    for i in range(len(altint)):
        w_iso = {k: annulus_weight(k, nband_t[i]) for k in range(annulino[i] + 1, annulino[i + 1] + 1)}
        w_an = {k: annulus_weight(k, aniso_t[i]) for k in range(annulino[i] + 1, annulino[i + 1] + 1)}
        for _ in range(nband[i]):
            az = iaz[index]
            sh, vegsh, vbsh, nst = shadow_patch(amaxvalue, a, vegdem, vegdem2, bush, az, altint[i], scale)
            steps.append(nst)
            shmat[:, :, index] = sh
            vegshmat[:, :, index] = vegsh
            vbshmat[:, :, index] = vbsh
            inE = 0 <= az < 180
            inS = 90 <= az < 270
            inW = 180 <= az < 360
            inN = az >= 270 or az < 90
            for k in range(annulino[i] + 1, annulino[i + 1] + 1):
                wi, wa = w_iso[k], w_an[k]
                svf = svf + wi * sh
                wsh = wa * sh
                if inE:
                    svfE = svfE + wsh
                if inS:
                    svfS = svfS + wsh
                if inW:
                    svfW = svfW + wsh
                if inN:
                    svfN = svfN + wsh
                svfveg = svfveg + wi * vegsh
                svfaveg = svfaveg + wi * vbsh
                if inE:
                    svfEveg = svfEveg + wa * vegsh
                    svfEaveg = svfEaveg + wa * vbsh
                if inS:
                    svfSveg = svfSveg + wa * vegsh
                    svfSaveg = svfSaveg + wa * vbsh
                if inW:
                    svfWveg = svfWveg + wa * vegsh
                    svfWaveg = svfWaveg + wa * vbsh
                if inN:
                    svfNveg = svfNveg + wa * vegsh
                    svfNaveg = svfNaveg + wa * vbsh
            index += 1
    tail = F32(3.0459e-004)
    svfS = svfS + tail
    svfW = svfW + tail
    for p in (svf, svfE, svfS, svfW, svfN):
        p[p > 1.] = 1.
    last = z()
    last[vegdem2 == 0.] = tail
    svfSveg = svfSveg + last
    svfWveg = svfWveg + last
    svfSaveg = svfSaveg + last
    svfWaveg = svfWaveg + last
    for p in (svfveg, svfEveg, svfSveg, svfWveg, svfNveg, svfaveg, svfEaveg, svfSaveg, svfWaveg, svfNaveg):
        p[p > 1.] = 1.
    trans = F32(0.03)
    svftotal = svf - (F32(1) - svfveg) * (F32(1) - trans)
    out = (svf, svfaveg, svfE, svfEaveg, svfEveg, svfN, svfNaveg, svfNveg, svfS, svfSaveg, svfSveg,
           svfveg, svfW, svfWaveg, svfWveg, vegshmat, vbshmat, shmat, svftotal)
    if return_steps:
        return out, np.array(steps)
    return out


def scene_from_rasters(dsm, trees, dem):
    """Derived march inputs exactly as compute_utci builds them
    (utci_process.py:1377-1385): vegdsm, vegdsm2, bush, amaxvalue."""
    a = np.asarray(dsm, F32)
    t1 = np.asarray(trees, F32).copy()
    t2 = np.asarray(dem, F32)
    t1[t1 < 0.] = 0.
    vegdem = t1 + t2
    vegdem2 = t1 * F32(0.25) + t2
    bush = np.logical_not(vegdem2 * vegdem).astype(F32) * vegdem
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * F32(0.25) + a
    vegdsm2[vegdsm2 == a] = 0
    amax = F32(max(a.max(), vegdem.max()))
    return vegdsm.astype(F32), vegdsm2.astype(F32), bush.astype(F32), amax
