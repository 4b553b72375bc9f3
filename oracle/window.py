"""Oracle: the windowed time loop (reference ``solweig_gpu/utci_process.py:477-1090``
``run_utci_window`` and ``solweig_gpu/solweig.py:1950-2311``
``Solweig_2022a_calc``), full-window case (``out_window=None``), with
``cyl = 1``, ``anisotropic_sky = 1``, ``usevegdem = 1``, ``onlyglobal = 1``
(the reference defaults).
"""
from __future__ import annotations

import numpy as np
import torch

from .svf import F32, create_patches
from . import radiation as rad
from .gvf import gvf_2018a
from .march import aspect_radians, wallheight_23
from .radiation import _t

VARIABLES = ("utci", "tmrt", "kup", "kdown", "lup", "ldown", "shadow", "ta", "wind")
STATE_PLANES = ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1")


def tgmaps(lc_grid, lc_class):
    """Land-cover property grids (solweig_gpu/Tgmaps_v1.py:15-53)."""
    ids = np.unique(lc_grid)
    TgK, Tstart, alb, emis, TmaxLST = (np.copy(lc_grid) for _ in range(5))
    for v in ids:
        row = lc_class[:, 0] == v
        Tstart[Tstart == v] = lc_class[row, 4]
        alb[alb == v] = lc_class[row, 1]
        emis[emis == v] = lc_class[row, 2]
        TmaxLST[TmaxLST == v] = lc_class[row, 5]
        TgK[TgK == v] = lc_class[row, 3]
    wall = np.where(lc_class[:, 0] == 99)
    return (TgK, Tstart, alb, emis, lc_class[wall, 3], lc_class[wall, 4], TmaxLST, lc_class[wall, 5])


def clean_landcover(lc):
    """Codes outside 1..7 -> 6, codes 3/4 -> 5 (utci_process.py:738-744)."""
    lc = np.array(lc, F32, copy=True)
    lc[(lc < 1) | (lc > 7)] = 6
    lc[(lc == 3) | (lc == 4)] = 5
    return lc


def iter_utci_window(*, a, temp1, temp2, walls, dirwalls, svf_bundle, met_file, altitude, azimuth,
                    zen, jday, dectime, altmax, location, scale, amaxvalue=None, landcover_grid=None,
                    lc_class=None, windcoeff=None, time_start=0, time_stop=None,
                    requested_variables=("utci",), initial_state=None, return_final_state=False,
                    capture=None):
    """Full-window time loop.  Inputs are numpy float32 planes, the SVF bundle
    in the reference's 19-tuple order (cubes (rows, cols, P) float32 or uint8),
    ``met_file`` float64 rows and the float64 (1, T) sun-geometry arrays of
    ``Solweig_2015a_metdata_noload``.  Returns ``{name: (T, rows, cols)}``.
    ``capture`` (a list) receives per-step intermediate planes.

    A generator: yields each step's index after the step, and returns what
    run_utci_window returns (the CPU timing cuts the loop between steps)."""
    requested = set(requested_variables) | {"utci"}
    unknown = requested - set(VARIABLES)
    if unknown:
        raise ValueError(f"unknown requested variables: {sorted(unknown)}")
    if time_stop is None:
        time_stop = met_file.shape[0]
    if not 0 <= time_start < time_stop <= met_file.shape[0]:
        raise ValueError(f"invalid time range [{time_start}, {time_stop}) for {met_file.shape[0]} forcing rows")
    a = np.asarray(a, F32)
    rows, cols = a.shape
    (svf, svfaveg, svfE, svfEaveg, svfEveg, svfN, svfNaveg, svfNveg, svfS, svfSaveg, svfSveg, svfveg,
     svfW, svfWaveg, svfWveg, vegshmat, vbshmat, shmat, _svftotal) = svf_bundle
    shmat = np.asarray(shmat, F32)
    vegshmat = np.asarray(vegshmat, F32)
    vbshmat = np.asarray(vbshmat, F32)
    t1 = np.asarray(temp1, F32).copy()
    t2 = np.asarray(temp2, F32)
    t1[t1 < 0.] = 0.
    vegdem = t1 + t2
    vegdem2 = t1 * F32(0.25) + t2
    bush = np.logical_not(vegdem2 * vegdem).astype(F32) * vegdem
    vegdsm = t1 + a
    vegdsm[vegdsm == a] = 0
    vegdsm2 = t1 * F32(0.25) + a
    vegdsm2[vegdsm2 == a] = 0
    if amaxvalue is None:
        amaxvalue = F32(max(a.max(), vegdem.max()))
    buildings = a - t2
    buildings[buildings < 2.] = 1.
    buildings[buildings >= 2.] = 0.
    if windcoeff is None:
        windcoeff = np.ones((rows, cols), F32)
    valid_mask = buildings == 1
    if initial_state is None:
        state = {k: np.zeros((rows, cols), F32) for k in STATE_PLANES}
    else:
        state = {k: np.asarray(initial_state[k], F32).copy() for k in STATE_PLANES}
    walls = np.asarray(walls, F32)
    dirwalls = np.asarray(dirwalls, F32)

    if landcover_grid is not None:
        landcover = 1
        lc = clean_landcover(landcover_grid)
        TgK, Tstart, alb_grid, emis_grid, TgK_wall, Tstart_wall, TmaxLST, TmaxLST_wall = (
            np.asarray(x, F32) for x in tgmaps(lc, lc_class))
    else:
        landcover = 0
        z = np.zeros((rows, cols), F32)
        TgK, Tstart = z + F32(0.37), z - F32(3.41)
        alb_grid, emis_grid = z + F32(0.15), z + F32(0.95)
        TgK_wall, Tstart_wall, TmaxLST, TmaxLST_wall = F32(0.37), F32(-3.41), F32(15.), F32(15.)

    transVeg = 3. / 100.
    albedo_b, ewall, absK, absL = 0.2, 0.9, 0.7, 0.95
    Fside, Fup, Fcyl = 0.22, 0.06, 0.28
    elvis = 0
    Ta_all = met_file[:, 11]
    RH_all = met_file[:, 10]
    radG_all = met_file[:, 14]
    P_all = met_file[:, 12]
    Ws_all = met_file[:, 9]
    uhii_all = met_file[:, 24] if met_file.shape[1] > 24 else np.zeros(met_file.shape[0])
    DOY = met_file[:, 1]
    leafon = np.zeros((1, DOY.shape[0]), F32)
    leafon[0, (DOY > 97) & (DOY < 300)] = 1
    psi = leafon * F32(transVeg)
    psi[leafon == 0] = 0.5
    height = torch.tensor(1.1)
    first = torch.round(height)
    if first == 0.:
        first = torch.tensor(1.)
    second = torch.round(height * 20.)
    first, second = F32(first.item()), F32(second.item())
    timestepdec = 0 if len(Ta_all) == 1 else dectime[1] - dectime[0]
    if initial_state is None:
        timeadd, firstdaytime, CI = 0., 1., 1.0
    else:
        timeadd = float(initial_state["timeadd"])
        firstdaytime = float(initial_state["firstdaytime"])
        CI = float(initial_state["CI"])

    svfbuveg = svf - (F32(1.0) - svfveg) * F32(1.0 - transVeg)
    asvf = _t(torch.acos, _t(torch.sqrt, svf))
    hsvf = _t(torch.tan, asvf)
    diffsh = shmat - (F32(1) - vegshmat) * F32(1 - transVeg)
    tmp = svf + svfveg - F32(1.0)
    tmp[tmp < 0.0] = 0.0
    svfalfa = _t(torch.asin, _t(torch.exp, _t(torch.log, F32(1.0) - tmp) / F32(2.0)))
    aspect_rad = aspect_radians(dirwalls)
    lat = location["latitude"]

    n_out = time_stop - time_start
    outputs = {k: np.empty((n_out, rows, cols), F32) for k in requested}
    sbc32 = F32(rad.SBC)
    for i in range(time_start, time_stop):
        o = i - time_start
        if (dectime[i] - np.floor(dectime[i])) == 0:
            CI = 1.  # utci_process.py:444-455 (single-day np.where tuple -> else branch)
        alt64 = torch.tensor(altitude[0][i])
        azi64 = torch.tensor(azimuth[0][i])
        zen64 = torch.tensor(zen[0][i])
        Ta64 = torch.tensor(Ta_all[i])
        RH64 = torch.tensor(RH_all[i])
        radG64 = torch.tensor(radG_all[i])
        jd = jday[0][i]
        dect = torch.tensor(dectime[i])
        altmax64 = torch.tensor(altmax[0][i])
        SNUP = rad.daylen(torch.tensor(jd.item()), torch.tensor(lat))
        ea = 6.107 * 10 ** ((7.5 * Ta64) / (237.3 + Ta64)) * (RH64 / 100.)
        msteg = 46.5 * (ea / (Ta64 + 273.15))
        esky = (1 - (1 + msteg) * torch.exp(-((1.2 + 3.0 * msteg) ** 0.5))) + elvis
        cap = {}
        if alt64 > 0:
            I0, CI, Kt = rad.clearness_index(torch.tensor(zen64.item()), torch.tensor(jd.item()), Ta64.item(),
                                             torch.tensor(RH64.item()) / 100., torch.tensor(radG64.item()),
                                             lat, torch.tensor(P_all[i].item()))
            CI = min(CI, 1.0)
            radI, radD = rad.diffuse_fraction(torch.tensor(radG64.item()), torch.tensor(alt64.item()), Kt,
                                              torch.tensor(Ta64.item()), torch.tensor(RH64.item()))
            zen_deg = zen64 * (180 / np.pi)
            lv = rad.perez_v3(zen_deg.item(), azi64.item(), radD, radI, jd.item())
            aniLum = np.zeros((rows, cols), F32)
            for idx in range(lv.shape[0]):
                aniLum = aniLum + diffsh[:, :, idx] * F32(lv[idx, 2].item())
            dRad = aniLum * F32(radD.item())
            vegsh, sh, _, wallsh, wallsun, wallshve, _, facesun = wallheight_23(
                a, vegdsm, vegdsm2, azi64.item(), alt64.item(), scale, float(amaxvalue), bush, walls, aspect_rad)
            shadow = sh - (F32(1) - vegsh) * F32(1 - psi[0][i])
            Tgamp = TgK * F32(altmax64.item()) + Tstart
            Tgampwall = TgK_wall * F32(altmax64.item()) + Tstart_wall
            phase = ((dect - torch.floor(dect)) - SNUP / 24)
            phase32 = F32(phase.item())
            snup24 = F32((SNUP / 24).item())
            Tg = Tgamp * _t(torch.sin, ((phase32 / (TmaxLST / F32(24) - snup24)) * F32(np.pi)) / F32(2))
            Tgwall = Tgampwall * _t(torch.sin, ((phase32 / (TmaxLST_wall / F32(24) - snup24)) * F32(np.pi)) / F32(2))
            Tgwall = np.maximum(Tgwall, F32(0))
            radI0, radD0 = rad.diffuse_fraction(I0, alt64.item(), 1., Ta64.item(), RH64.item())
            corr = 0.1473 * torch.log(90 - (zen64 / np.pi * 180)) + 0.3454
            CI_Tg = min((radG64 / radI0) + (1 - corr), 1.0)
            radG0 = radI0 * (torch.sin(alt64 * (np.pi / 180))) + radD0
            CI_TgG = min((radG64 / radG0) + (1 - corr), 1.0)
            cig = F32(float(CI_TgG))
            Tg = Tg * cig
            Tgwall = Tgwall * cig
            if landcover == 1:
                Tg = np.maximum(Tg, F32(0))
            gvf = gvf_2018a(wallsun, walls, buildings, scale, shadow, first, second, dirwalls, Tg, Tgwall,
                            float(Ta64), emis_grid, ewall, alb_grid, rad.SBC, albedo_b)
            (gvfLup, gvfalb, gvfalbnosh, gvfLupE, gvfalbE, gvfalbnoshE, gvfLupS, gvfalbS, gvfalbnoshS,
             gvfLupW, gvfalbW, gvfalbnoshW, gvfLupN, gvfalbN, gvfalbnoshN, gvfSum, gvfNorm) = gvf
            cap["gvf"] = gvf
            Lup, _, state["Tgmap1"] = rad.ts_wave_delay(gvfLup, firstdaytime, timeadd, timestepdec, state["Tgmap1"])
            LupE, _, state["Tgmap1E"] = rad.ts_wave_delay(gvfLupE, firstdaytime, timeadd, timestepdec, state["Tgmap1E"])
            LupS, _, state["Tgmap1S"] = rad.ts_wave_delay(gvfLupS, firstdaytime, timeadd, timestepdec, state["Tgmap1S"])
            LupW, _, state["Tgmap1W"] = rad.ts_wave_delay(gvfLupW, firstdaytime, timeadd, timestepdec, state["Tgmap1W"])
            LupN, _, state["Tgmap1N"] = rad.ts_wave_delay(gvfLupN, firstdaytime, timeadd, timestepdec, state["Tgmap1N"])
            TgTemp = Tg * shadow + F32(Ta64.item())
            TgOut, timeadd, state["TgOut1"] = rad.ts_wave_delay(TgTemp, firstdaytime, timeadd, timestepdec,
                                                                state["TgOut1"])
            F_sh = rad.cylindric_wedge(zen64.item(), svfalfa)
            radI32, radD32, radG32 = F32(radI.item()), F32(radD.item()), F32(radG64.item())
            sin_alt = F32(torch.sin(alt64 * (np.pi / 180)).item())
            albF = (F32(albedo_b) * (F32(1) - svfbuveg)) * (radG32 * (F32(1) - F_sh) + radD32 * F_sh)
            Kdown = radI32 * shadow * sin_alt + dRad + albF
            kup_b = (radD32 * svfbuveg + F32(albedo_b) * (F32(1) - svfbuveg) *
                     (radG32 * (F32(1) - F_sh) + radD32 * F_sh))
            Kup = (gvfalb * radI32 * sin_alt) + kup_b * gvfalbnosh
            KupE = (gvfalbE * radI32 * sin_alt) + kup_b * gvfalbnoshE
            KupS = (gvfalbS * radI32 * sin_alt) + kup_b * gvfalbnoshS
            KupW = (gvfalbW * radI32 * sin_alt) + kup_b * gvfalbnoshW
            KupN = (gvfalbN * radI32 * sin_alt) + kup_b * gvfalbnoshN
            Keast, Ksouth, Kwest, Knorth, KsideI, KsideD, Kside, _, _ = rad.kside_aniso_cyl(
                radI, radD, shadow, azi64.item(), alt64.item(), albedo_b, lv, diffsh, hsvf, shmat, vegshmat,
                vbshmat, KupE, KupS, KupW, KupN)
            firstdaytime = 0
            L_patches = lv
            cap.update(radI=float(radI), radD=float(radD), CI_Tg=float(CI_Tg), CI_TgG=float(CI_TgG),
                       I0=float(I0), dRad=dRad, KsideD=KsideD, KsideI=KsideI, Kside=Kside, Tg=Tg, F_sh=F_sh)
        else:
            Tgwall = torch.tensor(0)
            z = np.zeros((rows, cols), F32)
            Kdown = Kwest = Kup = Keast = Ksouth = Knorth = z
            KsideI = KsideD = F_sh = Tg = shadow = dRad = Kside = z
            Lup = sbc32 * emis_grid * _t(torch.pow, z + F32(Ta64.item()) + Tg + F32(273.15), 4)
            LupE = LupS = LupW = LupN = Lup
            TgOut = F32(Ta64.item()) + Tg
            timeadd = 0
            firstdaytime = 1
            alt_p, azi_p = create_patches(2)[:2]
            L_patches = torch.stack([torch.from_numpy(alt_p), torch.from_numpy(azi_p),
                                     torch.zeros(alt_p.shape[0])], dim=1)
        if CI < 0.95:
            esky = CI * esky + (1 - CI) * 1.
        Ldown, Lside, Least_, Lwest_, Lnorth_, Lsouth_ = rad.lcyl(
            esky, L_patches, float(Ta64), Tgwall, ewall, Lup, shmat, vegshmat, vbshmat, alt64, azi64, hsvf)
        half = F32(0.5)
        Least, Lsouth, Lwest, Lnorth = LupE * half, LupS * half, LupW * half, LupN * half
        Sstr = F32(absK) * (Kside * F32(Fcyl) + (Kdown + Kup) * F32(Fup) + (Knorth + Keast + Ksouth + Kwest) * F32(Fside)) \
            + F32(absL) * ((Ldown + Lup) * F32(Fup) + Lside * F32(Fcyl) + (Lnorth + Least + Lsouth + Lwest) * F32(Fside))
        absl_sbc = F32((absL * torch.tensor(rad.SBC)).item())
        Tmrt = _t(torch.sqrt, _t(torch.sqrt, Sstr / absl_sbc)) - F32(273.2)
        RH_mat = np.zeros((rows, cols), F32) + F32(RH_all[i])
        va = np.maximum(windcoeff * F32(Ws_all[i]), F32(0.15))
        Ta_mat = np.zeros((rows, cols), F32) + F32(Ta_all[i]) + F32(uhii_all[i])
        UTCI_mat = rad.utci_calculator(Ta_mat, RH_mat, Tmrt, va)
        UTCI = np.full((rows, cols), np.nan, F32)
        UTCI[valid_mask] = UTCI_mat[valid_mask]
        res = {"utci": UTCI, "tmrt": Tmrt, "kup": Kup, "kdown": Kdown, "lup": Lup, "ldown": Ldown,
               "shadow": shadow, "ta": Ta_mat, "wind": va}
        for k in outputs:
            outputs[k][o] = res[k]
        if capture is not None:
            cap.update(Tmrt=Tmrt, Kdown=Kdown, Kup=Kup, Ldown=Ldown, Lup=Lup, shadow=shadow, Lside=Lside,
                       Keast=Keast, Least=Least + Least_, Lsouth=Lsouth + Lsouth_, Lwest=Lwest + Lwest_,
                       Lnorth=Lnorth + Lnorth_, TgOut=TgOut, esky=float(esky), CI=float(CI),
                       timeadd=float(timeadd), firstdaytime=float(firstdaytime),
                       Tgmap1=state["Tgmap1"].copy(), TgOut1=state["TgOut1"].copy())
            capture.append(cap)
        yield i
    if return_final_state:
        # water temperature (utci_process.py:841-846, 917-922): with land
        # cover on, the mean air temperature of the day at every midnight row
        twater = None if initial_state is None or initial_state.get("Twater") is None \
            else float(initial_state["Twater"])
        if landcover == 1:
            for i in range(time_start, time_stop):
                if (dectime[i] - np.floor(dectime[i])) == 0 or i == 0:
                    twater = float(np.mean(Ta_all[jday[0] == np.floor(dectime[i])]))
        final = {k: state[k] for k in STATE_PLANES}
        final.update(CI=float(CI), firstdaytime=float(firstdaytime), timeadd=float(timeadd),
                     Twater=twater, next_step=int(time_stop))
        return outputs, final
    return outputs


def run_utci_window(**kwargs):
    """Full-window time loop (utci_process.py:477-1090); the arguments and
    return value of iter_utci_window, run to the end."""
    steps = iter_utci_window(**kwargs)
    while True:
        try:
            next(steps)
        except StopIteration as done:
            return done.value
