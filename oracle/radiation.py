"""Oracle: per-timestep scalars and the flux chain of ``Solweig_2022a_calc``
(reference ``solweig_gpu/solweig.py``) plus UTCI (``calculate_utci.py``).

Scalars that the reference keeps as 0-dim tensors are evaluated with 0-dim
torch tensors of the same dtype; plane arithmetic is numpy float32 in the
reference's association order.  Transcendental functions on planes go through
torch's CPU kernels (``_t``) so their rounding is that of the reference.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from .svf import F32, create_patches

F64 = np.float64
SBC = 5.67051e-8


def _t(fn, x, *args):
    """Apply a torch elementwise function to a numpy array (same shape)."""
    arr = np.ascontiguousarray(x)
    return fn(torch.from_numpy(arr), *args).numpy()


# ----------------------------------------------------------------- scalars
def daylen(doy_f32, lat_f32):
    """solweig.py:47-73 on float32 0-dim tensors; returns SNUP."""
    RAD = torch.pi / 180.0
    DEC = -23.45 * torch.cos(2.0 * torch.pi * (doy_f32 + 10.0) / 365.0)
    SOC = torch.tan(RAD * DEC) * torch.tan(RAD * lat_f32)
    SOC = torch.clamp(SOC, -1.0, 1.0)
    DAYL = 12.0 + 24.0 * torch.arcsin(SOC) / torch.pi
    return 12.0 - DAYL / 2.0


def sun_distance(jday):
    b = 2. * torch.pi * jday / 365.
    return torch.sqrt(1.00011 + 0.034221 * torch.cos(b) + 0.001280 * torch.sin(b)
                      + 0.000719 * torch.cos(2. * b) + 0.000077 * torch.sin(2. * b))


_G_TABLE = ((10.0, [3.37, 2.85, 2.80, 2.64]), (20.0, [2.99, 3.02, 2.70, 2.93]),
            (30.0, [3.60, 3.00, 2.98, 2.93]), (40.0, [3.04, 3.11, 2.92, 2.94]),
            (50.0, [2.70, 2.95, 2.77, 2.71]), (60.0, [2.52, 3.07, 2.67, 2.93]),
            (70.0, [1.76, 2.69, 2.61, 2.61]), (80.0, [1.60, 1.67, 2.24, 2.63]),
            (90.0, [1.11, 1.44, 1.94, 2.02]))


def clearness_index(zen, jday, Ta, RH, radG, latitude, P):
    """solweig.py:851-926 -> (I0, CI, Kt)."""
    p = 1013.0 if P == -999.0 else P * 10.0
    Itoa = 1370.0
    D = sun_distance(jday)
    m = 35.0 * torch.cos(zen) * ((1224.0 * (torch.cos(zen) ** 2) + 1.0) ** (-1 / 2.0))
    Trpg = 1.021 - 0.084 * (m * (0.000949 * p + 0.051)) ** 0.5
    G = None
    for hi, g in _G_TABLE:
        if latitude < hi:
            G = g
            break
    if jday > 335 or jday <= 60:
        G = G[0]
    elif 60 < jday <= 152:
        G = G[1]
    elif 152 < jday <= 244:
        G = G[2]
    elif 244 < jday <= 335:
        G = G[3]
    a2 = torch.tensor(17.27)
    b2 = torch.tensor(237.7)
    Td = (b2 * (((a2 * Ta) / (b2 + Ta)) + torch.log(RH))) / (a2 - (((a2 * Ta) / (b2 + Ta)) + torch.log(RH)))
    Td = (Td * 1.8) + 32
    u = torch.exp(0.1133 - torch.log(torch.tensor(G + 1.)) + 0.0393 * Td)
    Tw = 1 - 0.077 * ((u * m) ** 0.3)
    Tar = 0.935 ** m
    I0 = Itoa * torch.cos(zen) * Trpg * Tw * D * Tar
    I0 = torch.where(torch.abs(zen) > torch.pi / 2, torch.tensor(0.0), I0)
    I0 = torch.where(torch.isnan(I0), torch.tensor(0.0), I0)
    corr = 0.1473 * torch.log(90 - (zen / torch.pi * 180)) + 0.3454
    CI = radG / I0 + (1 - corr)
    Kt = radG / (Itoa * torch.cos(zen) * D)
    return I0, CI, Kt


def diffuse_fraction(radG, altitude, Kt, Ta, RH):
    """solweig.py:928-983 (Reindl et al. 1990) -> (radI, radD)."""
    Ta = Ta if isinstance(Ta, torch.Tensor) else torch.tensor(Ta)
    RH = RH if isinstance(RH, torch.Tensor) else torch.tensor(RH)
    alfa = altitude * (torch.pi / 180.0)
    alfa = alfa if isinstance(alfa, torch.Tensor) else torch.tensor(alfa)
    if Ta <= -999.00 or RH <= -999.00 or torch.isnan(Ta) or torch.isnan(RH):
        if Kt <= 0.3:
            radD = radG * (1.020 - 0.248 * Kt)
        elif 0.3 < Kt < 0.78:
            radD = radG * (1.45 - 1.67 * Kt)
        else:
            radD = radG * 0.147
    else:
        RH = RH / 100
        if Kt <= 0.3:
            radD = radG * (1 - 0.232 * Kt + 0.0239 * torch.sin(alfa) - 0.000682 * Ta + 0.0195 * RH)
        elif 0.3 < Kt < 0.78:
            radD = radG * (1.329 - 1.716 * Kt + 0.267 * torch.sin(alfa) - 0.00357 * Ta + 0.106 * RH)
        else:
            radD = radG * (0.426 * Kt - 0.256 * torch.sin(alfa) + 0.00349 * Ta + 0.0734 * RH)
    radI = (radG - radD) / torch.sin(alfa)
    radI = torch.where(radI < 0, torch.tensor(0.0), radI)
    radI = torch.where((altitude < 1) & (radI > radG), radG, radI)
    radD = torch.where(radD > radG, radG, radD)
    return radI, radD


_PEREZ = {
    "a": ([1.3525, -1.2219, -1.1000, -0.5484, -0.6000, -1.0156, -1.0000, -1.0500],
          [-0.2576, -0.7730, -0.2515, -0.6654, -0.3566, -0.3670, 0.0211, 0.0289],
          [-0.2690, 1.4148, 0.8952, -0.2672, -2.5000, 1.0078, 0.5025, 0.4260],
          [-1.4366, 1.1016, 0.0156, 0.7117, 2.3250, 1.4051, -0.5119, 0.3590]),
    "b": ([-0.7670, -0.2054, 0.2782, 0.7234, 0.2937, 0.2875, -0.3000, -0.3250],
          [0.0007, 0.0367, -0.1812, -0.6219, 0.0496, -0.5328, 0.1922, 0.1156],
          [1.2734, -3.9128, -4.5000, -5.6812, -5.6812, -3.8500, 0.7023, 0.7781],
          [-0.1233, 0.9156, 1.1766, 2.6297, 1.8415, 3.3750, -1.6317, 0.0025]),
    "c": ([2.8000, 6.9750, 24.7219, 33.3389, 21.0000, 14.0000, 19.0000, 31.0625],
          [0.6004, 0.1774, -13.0812, -18.3000, -4.7656, -0.9999, -5.0000, -14.5000],
          [1.2375, 6.4477, -37.7000, -62.2500, -21.5906, -7.1406, 1.2438, -46.1148],
          [1.0000, -0.1239, 34.8438, 52.0781, 7.2492, 7.5469, -1.9094, 55.3750]),
    "d": ([1.8734, -1.5798, -5.0000, -3.5000, -3.5000, -3.4000, -4.0000, -7.2312],
          [0.6297, -0.5081, 1.5218, 0.0016, -0.1554, -0.1078, 0.0250, 0.4050],
          [0.9738, -1.7812, 3.9229, 1.1477, 1.4062, -1.0750, 0.3844, 13.3500],
          [0.2809, 0.1080, -2.6204, 0.1062, 0.3988, 1.5702, 0.2656, 0.6234]),
    "e": ([0.0356, 0.2624, -0.0156, 0.4659, 0.0032, -0.0672, 1.0468, 1.5000],
          [-0.1246, 0.0672, 0.1597, -0.3296, 0.0766, 0.4016, -0.3788, -0.6426],
          [-0.5718, -0.2190, 0.4199, -0.0876, -0.0656, 0.3017, -2.4517, 1.8564],
          [0.9938, -0.4285, -0.5562, -0.0329, -0.1294, -0.4844, 1.4656, 0.5636]),
}


def perez_v3(zen_deg, azimuth_deg, radD, radI, jday, patch_option=2):
    """Perez et al. (1993) relative sky luminance per patch (solweig.py:1227-1356,
    patchchoice 1).  Returns lv (P, 3) float32 tensor [alt, azi, lum]."""
    coeff = {k: torch.stack([torch.tensor(c) for c in v], dim=1) for k, v in _PEREZ.items()}
    deg2rad = torch.tensor(np.pi / 180)
    rad2deg = torch.tensor(180 / np.pi)
    altitude = 90 - zen_deg
    zen = torch.tensor(zen_deg) * deg2rad
    azimuth = torch.tensor(azimuth_deg) * deg2rad
    altitude = torch.tensor(altitude) * deg2rad
    Idh, Ibn = radD, radI
    clearness = ((Idh + Ibn) / (Idh + 1.041 * torch.pow(zen, 3))) / (1 + 1.041 * torch.pow(zen, 3))
    day_angle = jday * 2 * torch.pi / 365
    da = torch.tensor(day_angle)
    I0 = 1367 * (1.00011 + 0.034221 * torch.cos(da) + 0.00128 * torch.sin(da) + 0.000719 *
                 torch.cos(2 * da) + 0.000077 * torch.sin(2 * da))
    if altitude >= 10 * deg2rad:
        airmass = 1 / torch.sin(altitude)
    elif altitude < 0:
        airmass = 1 / torch.sin(altitude) + 0.50572 * torch.pow(
            180 * torch.complex(altitude, torch.tensor(0.)) / torch.pi + 6.07995, -1.6364)
    else:
        airmass = 1 / torch.sin(altitude) + 0.50572 * torch.pow(180 * altitude / torch.pi + 6.07995, -1.6364)
    brightness = (airmass * Idh) / I0
    if Idh <= 10:
        brightness = torch.tensor(0.0)
    bins = (1.065, 1.230, 1.500, 1.950, 2.800, 4.500, 6.200)
    ic = 7
    for j, b in enumerate(bins):
        if clearness < b:
            ic = j
            break
    A, B, C, Dc, E = (coeff[k] for k in "abcde")
    m_a = A[ic, 0] + A[ic, 1] * zen + brightness * (A[ic, 2] + A[ic, 3] * zen)
    m_b = B[ic, 0] + B[ic, 1] * zen + brightness * (B[ic, 2] + B[ic, 3] * zen)
    m_e = E[ic, 0] + E[ic, 1] * zen + brightness * (E[ic, 2] + E[ic, 3] * zen)
    if ic > 0:
        m_c = C[ic, 0] + C[ic, 1] * zen + brightness * (C[ic, 2] + C[ic, 3] * zen)
        m_d = Dc[ic, 0] + Dc[ic, 1] * zen + brightness * (Dc[ic, 2] + Dc[ic, 3] * zen)
    else:
        m_c = torch.exp(torch.pow(brightness * (C[ic, 0] + C[ic, 1] * zen), C[ic, 2])) - 1
        m_d = -torch.exp(brightness * (Dc[ic, 0] + Dc[ic, 1] * zen)) + Dc[ic, 2] + brightness * Dc[ic, 3] * brightness
    alt_p, azi_p = (torch.from_numpy(v) for v in create_patches(patch_option)[:2])
    skyzen = (90 - alt_p) * deg2rad
    skyalt = alt_p * deg2rad
    skyazi = azi_p * deg2rad
    cos_ss = torch.sin(skyalt) * torch.sin(altitude) + \
        torch.cos(altitude) * torch.cos(skyalt) * torch.cos(torch.abs(skyazi - azimuth))
    lv = (1 + m_a * torch.exp(m_b / torch.cos(skyzen))) * ((1 + m_c * torch.exp(m_d * torch.arccos(cos_ss)) +
                                                          m_e * cos_ss * cos_ss))
    lv = lv / torch.sum(lv)
    return torch.stack([skyalt * rad2deg, skyazi * rad2deg, lv], dim=1)


def steradians(patch_altitude, skyalt, skyalt_c):
    """Solid angle per patch (solweig.py:688-697 and 1707-1718)."""
    deg2rad = torch.tensor(np.pi / 180)
    n = patch_altitude.shape[0]
    ster = torch.zeros(n)
    for i in range(n):
        cnt = skyalt_c[skyalt == patch_altitude[i]]
        if cnt > 1:
            ster[i] = ((360 / cnt) * deg2rad) * (torch.sin((patch_altitude[i] + patch_altitude[0]) * deg2rad)
                                                 - torch.sin((patch_altitude[i] - patch_altitude[0]) * deg2rad))
        else:
            ster[i] = ((360 / cnt) * deg2rad) * (torch.sin((patch_altitude[i]) * deg2rad)
                                                 - torch.sin((patch_altitude[i - 1] + patch_altitude[0]) * deg2rad))
    return ster


# ------------------------------------------------------------------ planes
def cylindric_wedge(zen, svfalfa):
    """Fraction of shaded wall seen by a cylinder (solweig.py:404-449), with
    the NaN -> 0.5 replacement of solweig.py:2168."""
    beta = torch.tensor(zen, dtype=torch.float32)
    alfa = torch.from_numpy(np.ascontiguousarray(svfalfa, F32)).clone()
    tb = torch.tan(beta)
    ta = torch.tan(alfa)
    xa = 1 - 2. / (ta * tb)
    ha = 2. / (ta * tb)
    ba = (1. / ta)
    hkil = 2. * ba * ha
    m = xa < 0
    qa = torch.zeros_like(alfa)
    qa[m] = tb / 2
    Za = torch.zeros_like(alfa)
    Za[m] = (ba[m] ** 2 - (qa[m] ** 2) / 4) ** 0.5
    phi = torch.zeros_like(alfa)
    phi[m] = torch.atan(Za[m] / qa[m])
    A = torch.zeros_like(alfa)
    A[m] = (torch.sin(phi[m]) - phi[m] * torch.cos(phi[m])) / (1 - torch.cos(phi[m]))
    ukil = torch.zeros_like(alfa)
    ukil[m] = 2 * ba[m] * xa[m] * A[m]
    Ssurf = hkil + ukil
    F_sh = (2 * torch.pi * ba - Ssurf) / (2 * torch.pi * ba)
    F_sh[torch.isnan(F_sh)] = 0.5
    return F_sh.numpy()


def ts_wave_delay(gvfLup, firstdaytime, timeadd, timestepdec, Tgmap1):
    """Surface temperature lag (solweig.py:451-488) -> (Lup, timeadd, Tgmap1)."""
    Tgmap0 = gvfLup
    if firstdaytime == 1:
        Tgmap1 = Tgmap0
    if timeadd >= (59 / 1440):
        w = torch.exp(-33.27 * torch.tensor(timeadd))
        Tgmap1 = Tgmap0 * F32((1 - w).item()) + Tgmap1 * F32(w.item())
        Lup = Tgmap1
        timeadd = timestepdec if timestepdec > (59 / 1440) else 0
    else:
        timeadd = timeadd + timestepdec
        w = torch.exp(-33.27 * torch.tensor(timeadd))
        Lup = Tgmap0 * F32((1 - w).item()) + Tgmap1 * F32(w.item())
    return Lup, timeadd, Tgmap1


def shaded_or_sunlit(solar_altitude, solar_azimuth, patch_altitude, patch_azimuth, hsvf):
    """Patch sunlit/shaded predicate (solweig.py:524-562).  The solar angles
    keep the caller's types (float32 tensor / python float in Kside, float64
    tensors in define_patch_characteristics); ``hsvf = tan(asvf)``."""
    deg2rad = torch.pi / 180.0
    rad2deg = 180.0 / torch.pi
    p2s = torch.abs(solar_azimuth - patch_azimuth)
    xi = torch.cos(p2s * deg2rad)
    yi = 2 * xi * torch.tan(solar_altitude * deg2rad)
    yi_ = torch.where(yi > 0, 0.0, yi)
    tan_delta = hsvf + F32(yi_.item())
    deg = _t(torch.atan, tan_delta) * F32(rad2deg)
    palt = F32(patch_altitude.item())
    return deg < palt, deg > palt


def _acc64(acc, term):
    """``f32_plane += f64_plane``: computed in float64, stored as float32."""
    return (acc.astype(F64) + term).astype(F32)


def kside_aniso_cyl(radI, radD, shadow, azimuth, altitude, albedo, lv, diffsh, hsvf, shmat, vegshmat,
                    vbshmat, KupE, KupS, KupW, KupN):
    """Kside_veg_v2022a, ``cyl == 1`` anisotropic branch (solweig.py:564-832)."""
    deg2rad = torch.tensor(np.pi / 180.0)
    altitude = torch.tensor(altitude)
    rows, cols = shadow.shape
    KsideI = shadow * F32(radI) * F32(torch.cos(altitude * deg2rad).item())
    palt, pazi, plum = lv[:, 0], lv[:, 1], lv[:, 2]
    skyalt, skyalt_c = torch.unique(palt, return_counts=True)
    ster = steradians(palt, skyalt, skyalt_c)
    radTot = torch.zeros(1)
    for i in range(palt.shape[0]):
        radTot += (plum[i] * ster[i] * torch.sin(palt[i] * deg2rad))
    lumChi = (plum * radD) / radTot
    z = lambda: np.zeros((rows, cols), F32)  # noqa: E731
    KsideD, Kref_sun, Kref_sh, Kref_veg = z(), z(), z(), z()
    sunlit_surface = F32(((albedo * (radI * torch.cos(altitude * deg2rad)) + (radD * 0.5)) / torch.pi).item())
    shaded_surface = F32(((albedo * radD * 0.5) / torch.pi).item())
    for idx in range(pazi.shape[0]):
        ang = F32((torch.cos(palt[idx] * deg2rad) * torch.cos(torch.tensor(0.))).item())
        KsideD = KsideD + diffsh[:, :, idx] * F32(lumChi[idx].item()) * ang * F32(ster[idx].item())
        cos_a = F32(torch.cos(palt[idx] * deg2rad).item())
        s = F32(ster[idx].item())
        temp_vegsh = ((vegshmat[:, :, idx] == 0) | (vbshmat[:, :, idx] == 0)).astype(F32)
        Kref_veg = Kref_veg + shaded_surface * temp_vegsh * s * cos_a
        temp_sh = (((F32(1) - shmat[:, :, idx]) * vbshmat[:, :, idx]) == 1).astype(F32)
        sunlit, shaded = shaded_or_sunlit(altitude, azimuth, palt[idx], pazi[idx], hsvf)
        Kref_sun = Kref_sun + sunlit_surface * sunlit.astype(F32) * temp_sh * s * cos_a
        Kref_sh = Kref_sh + shaded_surface * shaded.astype(F32) * temp_sh * s * cos_a
    Kside = KsideI + KsideD + Kref_sun + Kref_sh + Kref_veg
    half = F32(0.5)
    return KupE * half, KupS * half, KupW * half, KupN * half, KsideI, KsideD, Kside, lumChi, ster


def _cardinal(paz):
    return ((paz > 360) or (paz < 180), (paz > 90) and (paz < 270),
            (paz > 180) and (paz < 360), (paz > 270) or (paz < 90))


def lcyl(esky, L_patches, Ta, Tgwall, ewall, Lup, shmat, vegshmat, vbshmat, solar_altitude,
         solar_azimuth, hsvf):
    """Lcyl_v2022a + define_patch_characteristics (solweig.py:1439-1760):
    returns Ldown, Lside, Least_, Lwest_, Lnorth_, Lsouth_.

    ``Tgwall`` is a float32 array (daytime) or the int64 0-dim zero the
    reference uses at night; ``Ta`` the float64 forcing value."""
    sbc = torch.tensor(SBC)
    deg2rad = torch.tensor(np.pi / 180)
    Ta_t = torch.tensor(Ta, dtype=torch.float64)
    sky_np = L_patches.numpy()
    skyalt_np, skyalt_c_np = np.unique(sky_np[:, 0], return_counts=True)
    skyalt = torch.tensor(skyalt_np)
    skyalt_c = torch.tensor(skyalt_c_np)
    palt = L_patches[:, 0]
    pazi = L_patches[:, 1]
    # Martin & Berdahl (1984) band emissivities (model2, solweig.py:1394-1413)
    u_alt, _ = torch.unique(palt, return_counts=True)
    esky_band = 1 - (1 - esky) * torch.exp(0.308 * (1.7 - (1 / torch.cos((90 - u_alt) * deg2rad))))
    ster = steradians(palt, skyalt, skyalt_c)
    P = palt.shape[0]
    Ld = torch.zeros(P)
    Ls = torch.zeros(P)
    ta4 = (Ta_t + 273.15) ** 4
    for alt in skyalt:
        te = esky_band[u_alt == alt]
        msk = palt == alt
        base = (te * sbc * ta4) / torch.tensor(np.pi)
        Ld[msk] = base * ster[msk] * torch.sin(alt * deg2rad)
        Ls[msk] = base * ster[msk] * torch.cos(alt * deg2rad)
    rows, cols = Lup.shape
    z = lambda: np.zeros((rows, cols), F32)  # noqa: E731
    Ldown_sky, Ldown_veg, Ldown_sun, Ldown_sh, Ldown_ref = z(), z(), z(), z(), z()
    Lside_sky, Lside_veg, Lside_sun, Lside_sh, Lside_ref = z(), z(), z(), z(), z()
    card = {"E": z(), "S": z(), "W": z(), "N": z()}
    card_off = {"E": 90, "S": 180, "W": 270, "N": 0}
    ew = torch.tensor(0.9) if ewall is None else torch.tensor(ewall)
    veg_surf = ((ew * sbc * ta4) / torch.tensor(np.pi)).item()  # float64
    if isinstance(Tgwall, np.ndarray):
        tw = _t(torch.pow, np.asarray(Tgwall + F32(Ta) + F32(273.15), F32), 4)
        sun_surf = ((F32((ew * sbc).item()) * tw) / F32(np.pi)).astype(F32)
    else:
        sun_surf = ((ew * sbc * ((Ta_t + Tgwall + 273.15) ** 4)) / torch.tensor(np.pi)).item()
    sh_surf = veg_surf
    sa = solar_altitude
    for idx in range(P):
        shm, vgm, vbm = shmat[:, :, idx], vegshmat[:, :, idx], vbshmat[:, :, idx]
        temp_sky = ((shm == 1) & (vgm == 1)).astype(F32)
        ld = F32(Ld[idx].item())
        ls = F32(Ls[idx].item())
        Ldown_sky = Ldown_sky + temp_sky * ld
        Lside_sky = Lside_sky + temp_sky * ls
        temp_veg = ((vgm == 0) | (vbm == 0)).astype(F32)
        s = ster[idx]
        cos_a = torch.cos(palt[idx] * deg2rad)
        sin_a = torch.sin(palt[idx] * deg2rad)
        vs_cos = (torch.tensor(veg_surf, dtype=torch.float64) * s * cos_a).item()
        vs_sin = (torch.tensor(veg_surf, dtype=torch.float64) * s * sin_a).item()
        Lside_veg = _acc64(Lside_veg, vs_cos * temp_veg.astype(F64))
        Ldown_veg = _acc64(Ldown_veg, vs_sin * temp_veg.astype(F64))
        paz = float(pazi[idx])
        flags = dict(zip("ESWN", _cardinal(paz)))
        cdir = {d: torch.cos((card_off[d] - pazi[idx]) * deg2rad) for d in "ESWN"}
        for d in "ESWN":
            if flags[d]:
                card[d] = card[d] + temp_sky * ls * F32(cdir[d].item())
                card[d] = _acc64(card[d], (torch.tensor(vs_cos, dtype=torch.float64)).item()
                                 * temp_veg.astype(F64) * F64(F32(cdir[d].item())))
        temp_sh = (((F32(1) - shm) * vbm) == 1).astype(F32)
        azdiff = torch.abs(solar_azimuth - pazi[idx])
        s32 = F32(s.item())
        cos32 = F32(cos_a.item())
        sin32 = F32(sin_a.item())
        if (azdiff > 90) and (azdiff < 270) and (sa > 0):
            sunlit, shaded = shaded_or_sunlit(solar_altitude, solar_azimuth, palt[idx], pazi[idx], hsvf)
            sunlit = sunlit.astype(F32)
            shaded = shaded.astype(F32)
            Lside_sun = Lside_sun + sun_surf * sunlit * s32 * cos32 * temp_sh
            Lside_sh = _acc64(Lside_sh, sh_surf * shaded.astype(F64) * F64(s32) * F64(cos32) * temp_sh)
            Ldown_sun = Ldown_sun + sun_surf * sunlit * s32 * sin32 * temp_sh
            Ldown_sh = _acc64(Ldown_sh, sh_surf * shaded.astype(F64) * F64(s32) * F64(sin32) * temp_sh)
            for d in "ESWN":
                if flags[d]:
                    c = F32(cdir[d].item())
                    card[d] = card[d] + sun_surf * sunlit * s32 * cos32 * temp_sh * c
                    card[d] = _acc64(card[d], sh_surf * shaded.astype(F64) * F64(s32) * F64(cos32) * temp_sh * F64(c))
        else:
            k_cos = (torch.tensor(sh_surf, dtype=torch.float64) * s * cos_a).item()
            k_sin = (torch.tensor(sh_surf, dtype=torch.float64) * s * sin_a).item()
            Lside_sh = _acc64(Lside_sh, k_cos * temp_sh.astype(F64))
            Ldown_sh = _acc64(Ldown_sh, k_sin * temp_sh.astype(F64))
            for d in "ESWN":
                if flags[d]:
                    c = F32(cdir[d].item())
                    card[d] = _acc64(card[d], k_cos * temp_sh.astype(F64) * F64(c))
    refl = (((Ldown_sky + Lup) * F32((1 - ew).item()) * F32(0.5)) / F32(np.pi)).astype(F32)
    for idx in range(P):
        temp_sh = ((shmat[:, :, idx] == 0) | (vegshmat[:, :, idx] == 0) | (vbshmat[:, :, idx] == 0)).astype(F32)
        s32 = F32(ster[idx].item())
        cos32 = F32(torch.cos(palt[idx] * deg2rad).item())
        sin32 = F32(torch.sin(palt[idx] * deg2rad).item())
        Lside_ref = Lside_ref + refl * s32 * cos32 * temp_sh
        Ldown_ref = Ldown_ref + refl * s32 * sin32 * temp_sh
        paz = float(pazi[idx])
        for d, inside in zip("ESWN", _cardinal(paz)):
            if inside:
                c = F32(torch.cos((card_off[d] - pazi[idx]) * deg2rad).item())
                card[d] = card[d] + refl * s32 * cos32 * temp_sh * c
    Lside = Lside_sky + Lside_veg + Lside_sh + Lside_sun + Lside_ref
    Ldown = Ldown_sky + Ldown_veg + Ldown_sh + Ldown_sun + Ldown_ref
    return Ldown, Lside, card["E"], card["W"], card["N"], card["S"]


# ------------------------------------------------------------------- UTCI
_TERMS = None


def _utci_terms():
    global _TERMS
    if _TERMS is None:
        here = os.path.dirname(os.path.abspath(__file__))
        path = os.path.join(os.path.dirname(here), "solweig_project_b200", "data", "utci_terms.json")
        with open(path) as fh:
            _TERMS = [(F32(float(c)), a, b, d, e) for c, a, b, d, e in json.load(fh)["terms"]]
    return _TERMS


def utci_calculator(Ta, RH, Tmrt, va10m):
    """UTCI (calculate_utci.py:24-330) on float32 planes; -999 where invalid."""
    Ta = np.asarray(Ta, F32)
    invalid = (Ta <= -999) | (RH <= -999) | (va10m <= -999) | (Tmrt <= -999)
    valid = ~invalid
    tk = torch.from_numpy(Ta[valid] + F32(273.15))
    g = torch.tensor([-2.8365744E3, -6.028076559E3, 1.954263612E1, -2.737830188E-2,
                      1.6261698E-5, 7.0229056E-10, -1.8680009E-13, 2.7150305], dtype=torch.float32)
    es = g[7] * torch.log(tk)
    for i in range(0, 7):
        es = es + g[i] * tk ** (i + 1 - 3.)
    es = torch.exp(es) * 0.01
    ehPa = es * torch.from_numpy(RH[valid]) / 100.
    D = torch.from_numpy(Tmrt[valid] - Ta[valid])
    Pa = ehPa / 10.0
    va = torch.from_numpy(va10m[valid])
    ta = torch.from_numpy(Ta[valid])
    acc = ta.clone()
    for c, pt, pv, pd, pp in _utci_terms():
        term = torch.tensor(c)
        first = True
        for base, pw in ((ta, pt), (va, pv), (D, pd), (Pa, pp)):
            if pw == 0:
                continue
            f = base if pw == 1 else base ** pw
            term = (float(c) * f) if first else term * f
            first = False
        if first:
            term = torch.full_like(acc, float(c))
        acc = acc + term
    out = np.full(Ta.shape, -999, F32)
    out[valid] = acc.numpy()
    return out
