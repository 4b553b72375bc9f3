"""Per-step scalar chain of the time loop, packed into the kernel tables.

Everything that does not vary across pixels is evaluated here, once per step,
with 0-dim torch CPU tensors of the dtypes the reference uses (float64 met
scalars, float32 sun geometry), so that every scalar the kernels read has the
reference's float32/float64 bits:

* sky emissivity, clearness index, diffuse fraction and the Perez sky
  luminance per patch (``solweig_gpu/solweig.py:2038-2073, 851-983, 1227-1356``)
* the ground temperature wave and CI_TgG (``solweig.py:2101-2122``)
* wall temperature and the wall longwave terms (``solweig.py:118-121,
  1594-1597``)
* TsWaveDelay weights (``solweig.py:451-488``)
* steradians, luminance shares and the sky longwave per patch
  (``solweig.py:683-731, 1651-1760``)
* the bounds of the shaded/sunlit patch predicate (``solweig.py:524-562``)
* UTCI polynomial coefficients in (D_Tmrt, va) (``calculate_utci.py:24-330``)
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from . import tables as T

F32 = np.float32
SBC = 5.67051e-8
PKG = os.path.dirname(os.path.abspath(__file__))


@dataclass
class ModelParams:
    """Model and receptor constants (utci_process.py:49-69) with the
    override names run_utci_window accepts (utci_process.py:78-82)."""

    albedo_b: float = 0.2
    ewall: float = 0.9
    absK: float = 0.7
    absL: float = 0.95
    Fside: float = 0.22
    Fup: float = 0.06
    Fcyl: float = 0.28
    cyl: bool = True
    elvis: float = 0
    anisotropic_sky: int = 1
    transVeg: float = 3. / 100.
    height: float = 1.1
    firstdayleaf: int = 97
    lastdayleaf: int = 300


PARAM_NAMES = frozenset(ModelParams.__dataclass_fields__)

_G = ((10.0, (3.37, 2.85, 2.80, 2.64)), (20.0, (2.99, 3.02, 2.70, 2.93)), (30.0, (3.60, 3.00, 2.98, 2.93)),
      (40.0, (3.04, 3.11, 2.92, 2.94)), (50.0, (2.70, 2.95, 2.77, 2.71)), (60.0, (2.52, 3.07, 2.67, 2.93)),
      (70.0, (1.76, 2.69, 2.61, 2.61)), (80.0, (1.60, 1.67, 2.24, 2.63)), (90.0, (1.11, 1.44, 1.94, 2.02)))

# Perez et al. (1993) coefficient sets, rows = clearness bins, columns = the
# four terms of each of a..e (the published table, as solweig.py:1250-1269)
_PEREZ = {
    "a": ((1.3525, -0.2576, -0.2690, -1.4366), (-1.2219, -0.7730, 1.4148, 1.1016), (-1.1000, -0.2515, 0.8952, 0.0156),
          (-0.5484, -0.6654, -0.2672, 0.7117), (-0.6000, -0.3566, -2.5000, 2.3250), (-1.0156, -0.3670, 1.0078, 1.4051),
          (-1.0000, 0.0211, 0.5025, -0.5119), (-1.0500, 0.0289, 0.4260, 0.3590)),
    "b": ((-0.7670, 0.0007, 1.2734, -0.1233), (-0.2054, 0.0367, -3.9128, 0.9156), (0.2782, -0.1812, -4.5000, 1.1766),
          (0.7234, -0.6219, -5.6812, 2.6297), (0.2937, 0.0496, -5.6812, 1.8415), (0.2875, -0.5328, -3.8500, 3.3750),
          (-0.3000, 0.1922, 0.7023, -1.6317), (-0.3250, 0.1156, 0.7781, 0.0025)),
    "c": ((2.8000, 0.6004, 1.2375, 1.0000), (6.9750, 0.1774, 6.4477, -0.1239), (24.7219, -13.0812, -37.7000, 34.8438),
          (33.3389, -18.3000, -62.2500, 52.0781), (21.0000, -4.7656, -21.5906, 7.2492), (14.0000, -0.9999, -7.1406, 7.5469),
          (19.0000, -5.0000, 1.2438, -1.9094), (31.0625, -14.5000, -46.1148, 55.3750)),
    "d": ((1.8734, 0.6297, 0.9738, 0.2809), (-1.5798, -0.5081, -1.7812, 0.1080), (-5.0000, 1.5218, 3.9229, -2.6204),
          (-3.5000, 0.0016, 1.1477, 0.1062), (-3.5000, -0.1554, 1.4062, 0.3988), (-3.4000, -0.1078, -1.0750, 1.5702),
          (-4.0000, 0.0250, 0.3844, 0.2656), (-7.2312, 0.4050, 13.3500, 0.6234)),
    "e": ((0.0356, -0.1246, -0.5718, 0.9938), (0.2624, 0.0672, -0.2190, -0.4285), (-0.0156, 0.1597, 0.4199, -0.5562),
          (0.4659, -0.3296, -0.0876, -0.0329), (0.0032, 0.0766, -0.0656, -0.1294), (-0.0672, 0.4016, 0.3017, -0.4844),
          (1.0468, -0.3788, -2.4517, 1.4656), (1.5000, -0.6426, 1.8564, 0.5636)),
}
_CLEAR_BINS = (1.065, 1.230, 1.500, 1.950, 2.800, 4.500, 6.200)


def _utci_terms():
    with open(os.path.join(PKG, "data", "utci_terms.json")) as fh:
        return [(float(F32(float(c))), a, b, d, e) for c, a, b, d, e in json.load(fh)["terms"]]


_TERMS = _utci_terms()
_TERM_C = np.array([F32(c) for c, _, _, _, _ in _TERMS], F32)      # coefficient of each term
_TERM_PT = np.array([pt for _, pt, _, _, _ in _TERMS], np.int64)  # its power of Ta
_ES_G = (-2.8365744E3, -6.028076559E3, 1.954263612E1, -2.737830188E-2, 1.6261698E-5, 7.0229056E-10,
         -1.8680009E-13, 2.7150305)


# --------------------------------------------------------------- scalars
def _snup(jday_f32, lat_f32):
    """Sunrise hour of daylen (solweig.py:47-73)."""
    rad = torch.pi / 180.0
    dec = -23.45 * torch.cos(2.0 * torch.pi * (jday_f32 + 10.0) / 365.0)
    soc = torch.clamp(torch.tan(rad * dec) * torch.tan(rad * lat_f32), -1.0, 1.0)
    return 12.0 - (12.0 + 24.0 * torch.arcsin(soc) / torch.pi) / 2.0


def _clearness(zen, jday, Ta, RH, radG, latitude, P):
    """clearnessindex_2013b (solweig.py:851-926) -> I0, CI, Kt."""
    p = 1013.0 if P == -999.0 else P * 10.0
    b = 2. * torch.pi * jday / 365.
    D = torch.sqrt(1.00011 + 0.034221 * torch.cos(b) + 0.001280 * torch.sin(b) + 0.000719 * torch.cos(2. * b)
                   + 0.000077 * torch.sin(2. * b))
    cz = torch.cos(zen)
    m = 35.0 * cz * ((1224.0 * (cz ** 2) + 1.0) ** (-1 / 2.0))
    trpg = 1.021 - 0.084 * (m * (0.000949 * p + 0.051)) ** 0.5
    G = next(g for hi, g in _G if latitude < hi)
    if jday > 335 or jday <= 60:
        G = G[0]
    elif 60 < jday <= 152:
        G = G[1]
    elif 152 < jday <= 244:
        G = G[2]
    else:
        G = G[3]
    a2, b2 = torch.tensor(17.27), torch.tensor(237.7)
    inner = ((a2 * Ta) / (b2 + Ta)) + torch.log(RH)
    Td = (b2 * inner) / (a2 - inner)
    Td = (Td * 1.8) + 32
    u = torch.exp(0.1133 - torch.log(torch.tensor(G + 1.)) + 0.0393 * Td)
    Tw = 1 - 0.077 * ((u * m) ** 0.3)
    I0 = 1370.0 * torch.cos(zen) * trpg * Tw * D * (0.935 ** m)
    I0 = torch.where(torch.abs(zen) > torch.pi / 2, torch.tensor(0.0), I0)
    I0 = torch.where(torch.isnan(I0), torch.tensor(0.0), I0)
    corr = 0.1473 * torch.log(90 - (zen / torch.pi * 180)) + 0.3454
    return I0, radG / I0 + (1 - corr), radG / (1370.0 * torch.cos(zen) * D)


def _diffuse(radG, altitude, Kt, Ta, RH):
    """diffusefraction, Reindl et al. (1990) (solweig.py:928-983)."""
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
        s = torch.sin(alfa)
        if Kt <= 0.3:
            radD = radG * (1 - 0.232 * Kt + 0.0239 * s - 0.000682 * Ta + 0.0195 * RH)
        elif 0.3 < Kt < 0.78:
            radD = radG * (1.329 - 1.716 * Kt + 0.267 * s - 0.00357 * Ta + 0.106 * RH)
        else:
            radD = radG * (0.426 * Kt - 0.256 * s + 0.00349 * Ta + 0.0734 * RH)
    radI = (radG - radD) / torch.sin(alfa)
    radI = torch.where(radI < 0, torch.tensor(0.0), radI)
    radI = torch.where((altitude < 1) & (radI > radG), radG, radI)
    radD = torch.where(radD > radG, radG, radD)
    return radI, radD


# ------------------------------------------- the day-step chain, batched
# The helpers above evaluate one daytime step at a time on 0-dim tensors, as
# the reference does.  _day_chain evaluates the same operations for every
# daytime step at once on 1-D tensors.  Each element is bit-identical to the
# 0-dim evaluation: torch's elementwise arithmetic, sqrt, exp, log, sin, cos,
# tan, asin, acos and the special powers (x**2, x**3, x**0.5, x**-0.5) give
# the same bits for a 0-dim tensor and for a vector element; the general
# powers (x**0.3, x**-1.6364, c**x, x**c) do not, so they are evaluated on
# 0-dim elements one at a time; and where two 0-dim tensors of different
# dtypes meet, the vector form casts explicitly to the dtype torch's
# promotion of the 0-dim pair gives.
# 0-dim torch powers with a general exponent, reproduced without a tensor per
# element (checked on 20k random inputs per case in
# tests/test_series_batched.py; torch special-cases only the exponents
# below): a float64 x ** e is the C library's pow(), which Python's float **
# calls; a float32 x ** e is that double pow() of x and e rounded once to
# float32; c ** x for a float32 x is powf of float32(c), which numpy's
# float32 scalar ** calls.
_TORCH_SPECIAL_EXPONENTS = (0.5, -0.5, 1.0, 2.0, 3.0, -1.0, -2.0, 0.0)


def _pow_each(x, e):
    """x ** e element by element on 0-dim tensors (e a number or a vector)."""
    if isinstance(e, torch.Tensor):
        return torch.stack([torch.pow(x[k], e[k]) for k in range(x.shape[0])]) if x.shape[0] else x
    if x.dtype in (torch.float64, torch.float32) and float(e) not in _TORCH_SPECIAL_EXPONENTS:
        vals = x.tolist()
        if all(v > 0.0 and v != float("inf") for v in vals):
            try:
                r = [v ** e for v in vals]
            except OverflowError:   # torch gives inf there: its own path below
                r = None
            if r is not None:
                if x.dtype == torch.float64:
                    return torch.tensor(r, dtype=torch.float64)
                return torch.from_numpy(np.array(r, np.float64).astype(np.float32))
    return torch.stack([x[k] ** e for k in range(x.shape[0])]) if x.shape[0] else x


def _rpow_each(base, x):
    """base ** x (a number to a tensor power) element by element."""
    if x.dtype == torch.float64 and isinstance(base, (int, float)) and base > 0:
        vals = x.tolist()
        if all(abs(v) != float("inf") and v == v for v in vals):
            try:
                return torch.tensor([float(base) ** v for v in vals], dtype=torch.float64)
            except OverflowError:
                pass
    if x.dtype == torch.float32 and isinstance(base, (int, float)) and base > 0:
        xs = x.numpy()
        if np.isfinite(xs).all():
            b32 = np.float32(base)
            with np.errstate(over="ignore", under="ignore"):
                return torch.from_numpy(np.array([b32 ** v for v in xs], np.float32))
    return torch.stack([base ** x[k] for k in range(x.shape[0])]) if x.shape[0] else x


def _season_g(latitude, jd32):
    G = next(g for hi, g in _G if latitude < hi)
    out = []
    for j in jd32.tolist():
        if j > 335 or j <= 60:
            out.append(G[0])
        elif 60 < j <= 152:
            out.append(G[1])
        elif 152 < j <= 244:
            out.append(G[2])
        else:
            out.append(G[3])
    return out


def _clearness_v(zen, jday, Ta32, RH, radG, latitude, P):
    """_clearness for vectors: zen, jday, RH, radG, P float32 (as the 0-dim
    call receives them), Ta32 the float32 values of the Python Ta."""
    missing = P == -999.0
    q_known = 0.000949 * (P * 10.0) + 0.051
    q = torch.where(missing, torch.tensor(F32(0.000949 * 1013.0 + 0.051)), q_known)
    b = 2. * torch.pi * jday / 365.
    D = torch.sqrt(1.00011 + 0.034221 * torch.cos(b) + 0.001280 * torch.sin(b) + 0.000719 * torch.cos(2. * b)
                   + 0.000077 * torch.sin(2. * b))
    cz = torch.cos(zen)
    m = 35.0 * cz * ((1224.0 * (cz ** 2) + 1.0) ** (-1 / 2.0))
    trpg = 1.021 - 0.084 * (m * q) ** 0.5
    Gp1 = torch.tensor([g + 1. for g in _season_g(latitude, jday)])
    a2, b2 = torch.tensor(17.27), torch.tensor(237.7)
    inner = ((a2 * Ta32) / (b2 + Ta32)) + torch.log(RH)
    Td = (b2 * inner) / (a2 - inner)
    Td = (Td * 1.8) + 32
    u = torch.exp(0.1133 - torch.log(Gp1) + 0.0393 * Td)
    Tw = 1 - 0.077 * _pow_each(u * m, 0.3)
    I0 = 1370.0 * torch.cos(zen) * trpg * Tw * D * _rpow_each(0.935, m)
    I0 = torch.where(torch.abs(zen) > torch.pi / 2, torch.tensor(0.0), I0)
    I0 = torch.where(torch.isnan(I0), torch.tensor(0.0), I0)
    corr = 0.1473 * torch.log(90 - (zen / torch.pi * 180)) + 0.3454
    return I0, radG / I0 + (1 - corr), radG / (1370.0 * torch.cos(zen) * D)


def _diffuse_v(radG, alfa, low_alt, Kt, Ta, RH):
    """_diffuse for vectors.  alfa: the altitude in radians as the 0-dim call
    makes it; low_alt: altitude < 1 per element; Kt a vector or a number;
    Ta, RH float32 vectors."""
    missing = (Ta <= -999.00) | (RH <= -999.00) | torch.isnan(Ta) | torch.isnan(RH)
    if isinstance(Kt, torch.Tensor):
        k1, k2 = Kt <= 0.3, (0.3 < Kt) & (Kt < 0.78)
    else:
        k1 = torch.full(radG.shape, Kt <= 0.3)
        k2 = torch.full(radG.shape, 0.3 < Kt < 0.78)
    m1, m2, m3 = radG * (1.020 - 0.248 * Kt), radG * (1.45 - 1.67 * Kt), radG * 0.147
    RHc = RH / 100
    s = torch.sin(alfa)
    n1 = radG * (1 - 0.232 * Kt + 0.0239 * s - 0.000682 * Ta + 0.0195 * RHc)
    n2 = radG * (1.329 - 1.716 * Kt + 0.267 * s - 0.00357 * Ta + 0.106 * RHc)
    n3 = radG * (0.426 * Kt - 0.256 * s + 0.00349 * Ta + 0.0734 * RHc)
    radD = torch.where(missing, torch.where(k1, m1, torch.where(k2, m2, m3)),
                       torch.where(k1, n1, torch.where(k2, n2, n3)))
    radI = (radG - radD) / torch.sin(alfa)
    radI = torch.where(radI < 0, torch.tensor(0.0), radI)
    radI = torch.where(low_alt & (radI > radG), radG, radI)
    radD = torch.where(radD > radG, radG, radD)
    return radI, radD


def _perez_v(zen_deg, azimuth_deg, radD, radI, jday):
    """_perez for every daytime step: lists of the Python-float arguments,
    radD / radI float32 vectors; returns the (P, 3) tables in a list, or None
    for a step the batched form does not cover (sun below the horizon)."""
    n = len(zen_deg)
    deg2rad = torch.tensor(np.pi / 180)          # float32, as in _perez
    zen = torch.tensor(zen_deg) * deg2rad
    azimuth = torch.tensor(azimuth_deg) * deg2rad
    altitude = torch.tensor([90 - z for z in zen_deg]) * deg2rad
    z3 = 1.041 * torch.pow(zen, 3)
    clearness = ((radD + radI) / (radD + z3)) / (1 + z3)
    da = torch.tensor([j * 2 * torch.pi / 365 for j in jday], dtype=torch.float32)
    I0 = 1367 * (1.00011 + 0.034221 * torch.cos(da) + 0.00128 * torch.sin(da) + 0.000719 * torch.cos(2 * da)
                 + 0.000077 * torch.sin(2 * da))
    high = altitude >= 10 * deg2rad
    low = 1 / torch.sin(altitude) + 0.50572 * _pow_each(180 * altitude / torch.pi + 6.07995, -1.6364)
    airmass = torch.where(high, 1 / torch.sin(altitude), low)
    bright = (airmass * radD) / I0
    bright = torch.where(radD <= 10, torch.tensor(0.0), bright)
    ic = [next((j for j, b in enumerate(_CLEAR_BINS) if c < b), 7) for c in clearness.tolist()]
    ict = torch.tensor(ic)
    co = {k: torch.tensor(v, dtype=torch.float32)[ict] for k, v in _PEREZ.items()}

    def lin(c):
        return c[:, 0] + c[:, 1] * zen + bright * (c[:, 2] + c[:, 3] * zen)

    m_a, m_b, m_e = lin(co["a"]), lin(co["b"]), lin(co["e"])
    m_c, m_d = lin(co["c"]), lin(co["d"])
    clear0 = [k for k in range(n) if ic[k] == 0]
    if clear0:
        c, d = co["c"], co["d"]
        for k in clear0:
            m_c[k] = torch.exp(torch.pow(bright[k] * (c[k, 0] + c[k, 1] * zen[k]), c[k, 2])) - 1
            m_d[k] = -torch.exp(bright[k] * (d[k, 0] + d[k, 1] * zen[k])) + d[k, 2] + bright[k] * d[k, 3] * bright[k]
    g = _perez_geometry()
    f32 = torch.float32
    cs = g["sin_alt"][None, :] * torch.sin(altitude).to(f32)[:, None] + \
        torch.cos(altitude).to(f32)[:, None] * g["cos_alt"][None, :] * \
        torch.cos(torch.abs(g["skyazi"][None, :] - azimuth.to(f32)[:, None]))
    lv = (1 + m_a.to(f32)[:, None] * torch.exp(m_b.to(f32)[:, None] / g["cos_zen"][None, :])) * \
        ((1 + m_c.to(f32)[:, None] * torch.exp(m_d.to(f32)[:, None] * torch.arccos(cs)) +
          m_e.to(f32)[:, None] * cs * cs))
    out = []
    for k in range(n):
        if altitude[k] < 0:
            out.append(None)
            continue
        row = lv[k].contiguous()
        row = row / torch.sum(row)
        out.append(torch.stack([g["alt_deg"], g["azi_deg"], row], dim=1))
    return out


def day_chain(met_file, altitude, azimuth, zen, jday, location, time_start=0, time_stop=None):
    """The daytime scalar chain of the forcing rows [time_start, time_stop),
    for build_series(..., day_chain=...) calls over parts of that range."""
    if time_stop is None:
        time_stop = met_file.shape[0]
    with torch.inference_mode():
        return _day_chain([i for i in range(time_start, time_stop) if altitude[0][i] > 0], met_file, altitude,
                          azimuth, zen, jday, location["latitude"])


def _day_chain(days, met_file, altitude, azimuth, zen, jday, lat):
    """The per-daytime-step scalars of build_series for the forcing rows
    `days`, each element bit-identical to the 0-dim helpers' result for that
    step (tests/test_series_batched.py): sunrise, clearness (I0, CI, Kt),
    diffuse split, Perez luminances and the diffuse split of I0."""
    if not days:
        return {"pos": {}}
    alt_py = [float(altitude[0][i]) for i in days]
    zen_py = [float(zen[0][i]) for i in days]
    jd_py = [float(jday[0][i]) for i in days]
    ta_py = [float(met_file[i, 11]) for i in days]
    rh_py = [float(met_file[i, 10]) for i in days]
    rg_py = [float(met_file[i, 14]) for i in days]
    jd32 = torch.tensor(jd_py)
    Ta32, RH32, radG32 = torch.tensor(ta_py), torch.tensor(rh_py), torch.tensor(rg_py)
    alt32 = torch.tensor(alt_py)
    out = {"pos": {i: k for k, i in enumerate(days)}, "snup": _snup_v(jd32, torch.tensor(lat))}
    I0, CI, Kt = _clearness_v(torch.tensor(zen_py), jd32, Ta32, RH32 / 100., radG32, lat,
                              torch.tensor([float(met_file[i, 12]) for i in days]))
    out.update(I0=I0, CI=CI, Kt=Kt)
    out["radI"], out["radD"] = _diffuse_v(radG32, alt32 * (torch.pi / 180.0), alt32 < 1, Kt, Ta32, RH32)
    zen_deg = [float(np.float64(z) * (180 / np.pi)) for z in zen_py]
    out["lv"] = _perez_v(zen_deg, [float(azimuth[0][i]) for i in days], out["radD"], out["radI"], jd_py)
    alfa0 = torch.tensor([a * (torch.pi / 180.0) for a in alt_py])
    out["radI0"], out["radD0"] = _diffuse_v(I0, alfa0, torch.tensor([a < 1 for a in alt_py]), 1., Ta32, RH32)
    return out


def _yi_tables(days, azimuth, altitude, pazi):
    """yi_ of shaded_or_sunlit for the Kside call (float32) and the Lcyl call
    (float64 -> float32), and the Lcyl branch flags, for the daytime rows
    `days` against the patch azimuths `pazi` (solweig.py:524-562, the
    expressions of the step-by-step form evaluated as (days, patches)
    arrays, element by element the same operations)."""
    azi = [float(azimuth[0][i]) for i in days]
    alt = [float(altitude[0][i]) for i in days]
    alt32 = torch.tensor(alt)
    yk = 2 * torch.cos(torch.abs(torch.tensor(azi)[:, None] - pazi[None, :]) * (torch.pi / 180.0)) * \
        torch.tan(alt32 * (torch.pi / 180.0))[:, None]
    yi_k = torch.where(yk > 0, 0.0, yk).numpy()
    pz64 = pazi.double()
    azi64 = torch.tensor(azi, dtype=torch.float64)
    yl = 2 * torch.cos(torch.abs(azi64[:, None] - pz64[None, :]) * (torch.pi / 180.0)) * \
        torch.tan(torch.tensor(alt, dtype=torch.float64) * (torch.pi / 180.0))[:, None]
    yi_l = torch.where(yl > 0, 0.0, yl).numpy().astype(F32)
    azd = torch.abs(azi64[:, None] - pz64[None, :])
    flags = ((azd > 90) & (azd < 270)).numpy().astype(np.int32)
    return yi_k, yi_l, flags, pazi.clone()


def _snup_v(jday_f32, lat_f32):
    """_snup for a vector of float32 days."""
    rad = torch.pi / 180.0
    dec = -23.45 * torch.cos(2.0 * torch.pi * (jday_f32 + 10.0) / 365.0)
    soc = torch.clamp(torch.tan(rad * dec) * torch.tan(rad * lat_f32), -1.0, 1.0)
    return 12.0 - (12.0 + 24.0 * torch.arcsin(soc) / torch.pi) / 2.0


_PEREZ_GEOM: dict = {}
_PEREZ_CO: dict = {}


def _perez_geometry():
    """Patch angles of the Perez distribution and their step-independent
    trigonometry (the same tensors every step evaluates)."""
    if not _PEREZ_GEOM:
        deg2rad = torch.tensor(np.pi / 180)
        rad2deg = torch.tensor(180 / np.pi)
        alt_p, azi_p = (torch.from_numpy(v) for v in T.sky_patches(2))
        skyzen = (90 - alt_p) * deg2rad
        skyalt = alt_p * deg2rad
        skyazi = azi_p * deg2rad
        _PEREZ_GEOM.update(skyazi=skyazi, sin_alt=torch.sin(skyalt), cos_alt=torch.cos(skyalt),
                           cos_zen=torch.cos(skyzen), alt_deg=skyalt * rad2deg, azi_deg=skyazi * rad2deg)
    return _PEREZ_GEOM


def _perez(zen_deg, azimuth_deg, radD, radI, jday):
    """Perez_v3 with patchchoice 1 (solweig.py:1227-1356): (P, 3) float32."""
    deg2rad = torch.tensor(np.pi / 180)
    zen = torch.tensor(zen_deg) * deg2rad
    azimuth = torch.tensor(azimuth_deg) * deg2rad
    altitude = torch.tensor(90 - zen_deg) * deg2rad
    z3 = 1.041 * torch.pow(zen, 3)
    clearness = ((radD + radI) / (radD + z3)) / (1 + z3)
    da = torch.tensor(jday * 2 * torch.pi / 365)
    I0 = 1367 * (1.00011 + 0.034221 * torch.cos(da) + 0.00128 * torch.sin(da) + 0.000719 * torch.cos(2 * da)
                 + 0.000077 * torch.sin(2 * da))
    if altitude >= 10 * deg2rad:
        airmass = 1 / torch.sin(altitude)
    elif altitude < 0:
        airmass = 1 / torch.sin(altitude) + 0.50572 * torch.pow(
            180 * torch.complex(altitude, torch.tensor(0.)) / torch.pi + 6.07995, -1.6364)
    else:
        airmass = 1 / torch.sin(altitude) + 0.50572 * torch.pow(180 * altitude / torch.pi + 6.07995, -1.6364)
    bright = (airmass * radD) / I0
    if radD <= 10:
        bright = torch.tensor(0.0)
    ic = next((j for j, b in enumerate(_CLEAR_BINS) if clearness < b), 7)
    co = _PEREZ_CO.get(ic)
    if co is None:
        co = _PEREZ_CO.setdefault(ic, {k: torch.tensor(v[ic]) for k, v in _PEREZ.items()})

    def lin(c):
        return c[0] + c[1] * zen + bright * (c[2] + c[3] * zen)

    m_a, m_b, m_e = lin(co["a"]), lin(co["b"]), lin(co["e"])
    if ic > 0:
        m_c, m_d = lin(co["c"]), lin(co["d"])
    else:
        c, d = co["c"], co["d"]
        m_c = torch.exp(torch.pow(bright * (c[0] + c[1] * zen), c[2])) - 1
        m_d = -torch.exp(bright * (d[0] + d[1] * zen)) + d[2] + bright * d[3] * bright
    g = _perez_geometry()
    cs = g["sin_alt"] * torch.sin(altitude) + torch.cos(altitude) * g["cos_alt"] * \
        torch.cos(torch.abs(g["skyazi"] - azimuth))
    lv = (1 + m_a * torch.exp(m_b / g["cos_zen"])) * ((1 + m_c * torch.exp(m_d * torch.arccos(cs)) +
                                                      m_e * cs * cs))
    lv = lv / torch.sum(lv)
    return torch.stack([g["alt_deg"], g["azi_deg"], lv], dim=1)


_STER_CACHE: dict = {}


def _steradians(palt):
    """Solid angle of each patch (solweig.py:688-697, 1707-1718); a pure
    function of the patch altitudes, which repeat from step to step."""
    key = palt.numpy().tobytes()
    hit = _STER_CACHE.get(key)
    if hit is None:
        hit = _STER_CACHE.setdefault(key, _steradians_uncached(palt))
    return hit.clone()


def _steradians_uncached(palt):
    deg2rad = torch.tensor(np.pi / 180)
    skyalt, cnt = torch.unique(palt, return_counts=True)
    ster = torch.zeros(palt.shape[0])
    for i in range(palt.shape[0]):
        c = cnt[skyalt == palt[i]]
        if c > 1:
            ster[i] = ((360 / c) * deg2rad) * (torch.sin((palt[i] + palt[0]) * deg2rad)
                                               - torch.sin((palt[i] - palt[0]) * deg2rad))
        else:
            ster[i] = ((360 / c) * deg2rad) * (torch.sin(palt[i] * deg2rad)
                                               - torch.sin((palt[i - 1] + palt[0]) * deg2rad))
    return ster


_LSKY_CACHE: dict = {}
_TRIG_CACHE: dict = {}


def _patch_trig(palt):
    """cos / sin of the patch altitudes in radians (the tensors every step
    evaluates from the same altitude vector) and cos(alt) * cos(0)."""
    key = (palt.numpy().tobytes(), str(palt.dtype))
    hit = _TRIG_CACHE.get(key)
    if hit is None:
        deg2rad = torch.tensor(np.pi / 180)
        cos_t, sin_t = torch.cos(palt * deg2rad), torch.sin(palt * deg2rad)
        hit = _TRIG_CACHE.setdefault(key, (cos_t, sin_t, cos_t * torch.cos(torch.tensor(0.))))
    return hit
_THR_CACHE: dict = {}


def _thr_bounds(palt):
    """atan_degree_bounds of every patch altitude, as two float32 vectors."""
    key = palt.numpy().tobytes()
    hit = _THR_CACHE.get(key)
    if hit is None:
        b = np.array([T.atan_degree_bounds(float(pa)) for pa in palt.numpy()], F32).reshape(-1, 2)
        hit = _THR_CACHE.setdefault(key, (b[:, 0].copy(), b[:, 1].copy()))
    return hit


def _lsky_geometry(palt):
    """The step-independent part of _lsky for a patch-altitude vector: the
    distinct altitudes u, the band exponential of each, the patch -> u index,
    the solid angles and sin / cos of each altitude (0-dim evaluations, as
    the per-altitude loop makes them), rounded to the planes' dtype."""
    key = (palt.numpy().tobytes(), str(palt.dtype))
    hit = _LSKY_CACHE.get(key)
    if hit is None:
        deg2rad = torch.tensor(np.pi / 180)
        u, _ = torch.unique(palt, return_counts=True)
        expo = torch.exp(0.308 * (1.7 - (1 / torch.cos((90 - u) * deg2rad))))
        idx = torch.searchsorted(u, palt.contiguous())
        sin_u = torch.stack([torch.sin(alt * deg2rad) for alt in u])
        cos_u = torch.stack([torch.cos(alt * deg2rad) for alt in u])
        hit = _LSKY_CACHE.setdefault(key, (u, expo, idx, _steradians(palt), sin_u, cos_u))
    return hit


_LCYL_CACHE: dict = {}


def _lcyl_geometry(palt):
    """Per patch layout: solid angles, cos / sin of the altitudes (float32
    and float64) and the shaded_or_sunlit bounds, as the Lcyl tables use
    them every step."""
    key = (palt.numpy().tobytes(), str(palt.dtype))
    hit = _LCYL_CACHE.get(key)
    if hit is None:
        ster = _steradians(palt)
        cos_t, sin_t, _ = _patch_trig(palt)
        hit = _LCYL_CACHE.setdefault(key, {
            "ster_n": ster.numpy().copy(), "cos_n": cos_t.numpy().copy(), "sin_n": sin_t.numpy().copy(),
            "s64": ster.double(), "cos64": cos_t.double(), "sin64": sin_t.double(), "thr": _thr_bounds(palt)})
    return hit


def _kside_tables(patch, kside_rows, diff_vals, albedo_b, azimuth, altitude):
    """The Kside columns of the patch table (diffuse, anisotropic luminance,
    reflected terms, the shaded_or_sunlit yi_ and branch flags) for the
    daytime steps `kside_rows` = [(step, forcing row, Perez table, radD,
    radI, float32 altitude)], as (steps, patches) arrays per patch layout;
    each element is the per-step form's operation sequence (radTot is a
    sequential float32 sum along each row, as np.add.accumulate makes it)."""
    groups = {}
    for item in kside_rows:
        lv = item[2]
        key = (lv[:, 0].numpy().tobytes(), lv[:, 1].numpy().tobytes(), str(lv.dtype))
        groups.setdefault(key, []).append(item)
    deg2rad_t = torch.tensor(np.pi / 180)
    for items in groups.values():
        rows_ = [it[0] for it in items]
        palt, pazi = items[0][2][:, 0], items[0][2][:, 1]
        plum = torch.stack([it[2][:, 2] for it in items])
        radD = torch.stack([it[3] for it in items])
        radI = torch.stack([it[4] for it in items])
        alt32 = torch.stack([it[5] for it in items])
        ster = _steradians(palt)
        cos_pt, sin_pt, ang_t = _patch_trig(palt)
        # radTot += lum * ster * sin(alt), one float32 add per patch in order
        terms = (plum * ster[None, :] * sin_pt[None, :]).numpy()
        radTot = torch.from_numpy(np.add.accumulate(terms, axis=1, dtype=F32)[:, -1].copy())
        lumChi = (plum * radD[:, None]) / radTot[:, None]
        sun_k = ((albedo_b * (radI * torch.cos(alt32 * deg2rad_t)) + (radD * 0.5)) / torch.pi).numpy()
        sh_k = ((albedo_b * radD * 0.5) / torch.pi).numpy()
        cos_p, ang, ster_n = cos_pt.numpy(), ang_t.numpy(), ster.numpy()
        lum_n, lvz = lumChi.numpy(), plum.numpy()
        # the four (sh, vegsh) codes as a last axis, one whole-field write each
        # (a slice when the rows are consecutive, as daytime rows are)
        sel = slice(rows_[0], rows_[-1] + 1) if rows_ == list(range(rows_[0], rows_[-1] + 1)) else rows_
        dv = np.asarray(diff_vals, F32)[None, None, :]
        patch["kside_d"][sel] = ((dv * lum_n[:, :, None]) * ang[None, :, None]) * ster_n[None, :, None]
        patch["anilum"][sel] = dv * lvz[:, :, None]
        kref_sh = (sh_k[:, None] * ster_n[None, :]) * cos_p[None, :]
        patch["kref_veg"][sel] = kref_sh
        patch["kref_sh"][sel] = kref_sh
        patch["kref_sun"][sel] = (sun_k[:, None] * ster_n[None, :]) * cos_p[None, :]
        yk, yl, fl, _ = _yi_tables([it[1] for it in items], azimuth, altitude, pazi)
        patch["yi_k"][sel], patch["yi_l"][sel], patch["flags"][sel] = yk, yl, fl


def _lcyl_tables(patch, lcyl_rows, ta4_v, ewall_t, sbc_t):
    """The Lcyl columns of the patch table (sky longwave per patch, solid
    angles, altitude cos / sin, the float64 vegetation / shaded-wall terms,
    the sunlit-wall terms and the shaded_or_sunlit bounds) for the steps
    `lcyl_rows` = [(step, patch altitudes, esky, sunlit wall surface)], as
    (steps, patches) arrays per patch layout: each element is the
    per-step form's operation sequence (_lsky), the 0-dim float64 esky and
    Ta^4 cast to float32 where they meet float32 vectors, as torch does."""
    groups = {}
    for o, palt, esky, sun_surf in lcyl_rows:
        key = (palt.numpy().tobytes(), str(palt.dtype))
        groups.setdefault(key, (palt, []))[1].append((o, esky, sun_surf))
    f32 = torch.float32
    for palt, items in groups.values():
        rows_ = [it[0] for it in items]
        sel = slice(rows_[0], rows_[-1] + 1) if rows_ == list(range(rows_[0], rows_[-1] + 1)) else rows_
        E = torch.stack([it[1] for it in items])
        ta4 = ta4_v[rows_]
        _, expo, idx, ster, sin_u, cos_u = _lsky_geometry(palt)
        band = 1 - (1 - E).to(f32)[:, None] * expo[None, :]
        base = ((band * torch.tensor(SBC) * ta4.to(f32)[:, None]) / torch.tensor(np.pi))[:, idx]
        bs = base * ster[None, :]
        G = _lcyl_geometry(palt)
        patch["ld_sky"][sel] = (bs * sin_u[idx].to(f32)[None, :]).numpy()
        patch["ls_sky"][sel] = (bs * cos_u[idx].to(f32)[None, :]).numpy()
        patch["ster"][sel] = G["ster_n"]
        patch["cos_alt"][sel] = G["cos_n"]
        patch["sin_alt"][sel] = G["sin_n"]
        surf = ((ewall_t * sbc_t * ta4) / torch.tensor(np.pi))  # float64
        vc = ((surf[:, None] * G["s64"][None, :]) * G["cos64"][None, :]).numpy()
        vs = ((surf[:, None] * G["s64"][None, :]) * G["sin64"][None, :]).numpy()
        patch["veg_cos"][sel], patch["veg_sin"][sel] = vc, vs
        patch["sh_cos"][sel], patch["sh_sin"][sel] = vc, vs
        S = np.array([it[2] for it in items], F32)[:, None]
        patch["sun_cos"][sel] = (S * G["ster_n"][None, :]) * G["cos_n"][None, :]
        patch["sun_sin"][sel] = (S * G["ster_n"][None, :]) * G["sin_n"][None, :]
        patch["thr_sun"][sel], patch["thr_shd"][sel] = G["thr"]


def _lsky(esky, palt, Ta64, ta4=None):
    """Sky longwave per patch on horizontal / vertical surfaces with the
    Martin & Berdahl band emissivities (model2, solweig.py:1394-1413, 1725-1737).
    Per distinct altitude: base = (band * sbc * Ta^4) / pi, then per patch
    base * ster * sin(alt) (cos for the vertical); evaluated here as whole
    vectors, each element by the same float32 operations."""
    u, expo, idx, ster, sin_u, cos_u = _lsky_geometry(palt)
    sbc = torch.tensor(SBC)
    band = 1 - (1 - esky) * expo
    if ta4 is None:
        ta4 = (Ta64 + 273.15) ** 4
    base = ((band * sbc * ta4) / torch.tensor(np.pi))[idx]
    bs = base * ster
    dt = bs.dtype
    ld = torch.zeros(palt.shape[0])
    ls = torch.zeros(palt.shape[0])
    ld[:] = bs * sin_u[idx].to(dt)
    ls[:] = bs * cos_u[idx].to(dt)
    return ld, ls, ster.clone()


def utci_pow(x, p: int) -> np.float32:
    """x ** p of a float32 value as torch evaluates a float32 tensor ** int:
    float32 products for p <= 3, the correctly rounded power for p = 4..6
    (a float64 product chain rounded once); the device uses the same
    arithmetic (csrc/utci_series.cuh)."""
    x = F32(x)
    if p == 1:
        return x
    if p == 2:
        return x * x
    if p == 3:
        return (x * x) * x
    d = np.float64(x)
    d2 = d * d
    d4 = d2 * d2
    return F32(d4 if p == 4 else (d4 * d if p == 5 else d4 * d2))


def utci_vapour_pressure(ta, rh) -> np.float32:
    """Pa (kPa) of calculate_utci.py:273-282 in float32, log / exp rounded
    once from float64."""
    g = [F32(v) for v in _ES_G]
    tk = F32(ta) + F32(273.15)
    es = g[7] * F32(np.log(np.float64(tk)))
    es = es + g[0] * (F32(1) / (tk * tk))
    es = es + g[1] * (F32(1) / tk)
    es = es + g[2] * F32(1)
    es = es + g[3] * tk
    es = es + g[4] * (tk * tk)
    es = es + g[5] * ((tk * tk) * tk)
    es = es + g[6] * utci_pow(tk, 4)
    es = F32(np.exp(np.float64(es))) * F32(0.01)
    return ((es * F32(rh)) / F32(100.0)) / F32(10.0)


def _utci_table(ta_mat: np.float32, rh32: np.float32):
    """Per-step UTCI table (calculate_utci.py:259-330): Pa^1..Pa^6 and, per
    regression term, the float32 product c * Ta^pt that starts the term."""
    pa = utci_vapour_pressure(ta_mat, rh32)
    pa_pows = np.array([utci_pow(pa, p) for p in range(1, 7)], F32)
    ta_pows = [F32(1)] + [utci_pow(ta_mat, p) for p in range(1, 7)]
    # c * Ta^pt per term in float32 (c * 1 for the Ta-free terms is c itself)
    k = _TERM_C * np.array(ta_pows, F32)[_TERM_PT]
    return pa_pows, k


def _utci_pow_v(x, p: int):
    """utci_pow of every element of a float32 array (the same operations)."""
    if p == 1:
        return x
    if p == 2:
        return x * x
    if p == 3:
        return (x * x) * x
    d = x.astype(np.float64)
    d2 = d * d
    d4 = d2 * d2
    return (d4 if p == 4 else (d4 * d if p == 5 else d4 * d2)).astype(F32)


def _utci_tables(ta_mat, rh32):
    """_utci_table of many steps at once: (Pa^1..Pa^6, c * Ta^pt) per step,
    each element by the operations of the one-step form."""
    ta = np.asarray(ta_mat, F32).reshape(-1)
    rh = np.asarray(rh32, F32).reshape(-1)
    g = [F32(v) for v in _ES_G]
    tk = ta + F32(273.15)
    es = g[7] * np.log(tk.astype(np.float64)).astype(F32)
    es = es + g[0] * (F32(1) / (tk * tk))
    es = es + g[1] * (F32(1) / tk)
    es = es + g[2] * F32(1)
    es = es + g[3] * tk
    es = es + g[4] * (tk * tk)
    es = es + g[5] * ((tk * tk) * tk)
    es = es + g[6] * _utci_pow_v(tk, 4)
    es = np.exp(es.astype(np.float64)).astype(F32) * F32(0.01)
    pa = ((es * rh) / F32(100.0)) / F32(10.0)
    pa_pows = np.stack([_utci_pow_v(pa, p) for p in range(1, 7)], axis=1)
    ta_pows = np.stack([np.ones_like(ta)] + [_utci_pow_v(ta, p) for p in range(1, 7)], axis=1)
    return pa_pows, _TERM_C[None, :] * ta_pows[:, _TERM_PT]


def utci_step_records(met_file, indices) -> np.ndarray:
    """Time-step records carrying only what the UTCI tail reads (ta_mat,
    rh32, ws32 and the UTCI table) for the forcing rows ``indices``, with
    the reference's met reads and float32 roundings
    (utci_process.py:1158-1191)."""
    met_file = np.asarray(met_file)
    uhii = met_file[:, 24] if met_file.shape[1] > 24 else np.zeros(met_file.shape[0])
    rec = np.zeros(len(indices), N.TIME_STEP_DTYPE)
    for k, i in enumerate(indices):
        S = rec[k]
        S["rh32"] = F32(met_file[i, 10])
        S["ws32"] = F32(met_file[i, 9])
        S["ta_mat"] = (F32(0) + F32(met_file[i, 11])) + F32(uhii[i])
    if len(rec):
        rec["utci_pa"], rec["utci_k"] = _utci_tables(rec["ta_mat"], rec["rh32"])
    return rec


# -------------------------------------------------------------- the series
@dataclass
class LandCoverProps:
    """Per-pixel surface properties and the wall class (Tgmaps_v1.py:15-53)."""

    tgk: np.ndarray
    tstart: np.ndarray
    alb: np.ndarray
    emis: np.ndarray
    tmaxlst: np.ndarray
    tgk_wall: object
    tstart_wall: object
    tmaxlst_wall: object
    landcover: int
    # Sites prepared on the device (sw100_prepare_site) keep no property
    # rasters on the host: their pixels carry the cleaned land-cover code,
    # `codes` has bit c set when code c occurs and `code_tmax[c]` is that
    # class's TmaxLST.
    codes: int = 0
    code_tmax: np.ndarray | None = None
    device_classes: bool = False


_PROP_COLS = {"tstart": 4, "alb": 1, "emis": 2, "tmax": 5, "tgk": 3}


def class_table(lc_class):
    """Per cleaned land-cover code 1..7 the float32 TgK, Tstart, albedo,
    emissivity and TmaxLST of its class row, and the mask of codes that have
    exactly one row (landcover_props gives every pixel of such a code that
    row's values; a code without its row is refused)."""
    lc_class = np.asarray(lc_class)
    tab = {k: np.zeros(8, F32) for k in _PROP_COLS}
    valid = 0
    for c in range(1, 8):
        hit = np.flatnonzero(lc_class[:, 0] == c)
        if len(hit) == 1:
            valid |= 1 << c
            for k, j in _PROP_COLS.items():
                tab[k][c] = F32(lc_class[hit[0], j])
    return tab, valid


def wall_class(lc_class):
    """TgK, Tstart and TmaxLST of the wall class (code 99)."""
    lc_class = np.asarray(lc_class)
    wall = np.where(lc_class[:, 0] == 99)
    return (np.asarray(lc_class[wall, 3], F32), np.asarray(lc_class[wall, 4], F32),
            np.asarray(lc_class[wall, 5], F32))


def device_props(lc_class, codes) -> LandCoverProps:
    """Land-cover description of a device-prepared site (no host rasters);
    lc_class None: the default properties."""
    if lc_class is None:
        return LandCoverProps(None, None, None, None, None, 0.37, -3.41, 15., 0, device_classes=True)
    tab, _ = class_table(lc_class)
    return LandCoverProps(None, None, None, None, None, *wall_class(lc_class), 1, codes=int(codes),
                          code_tmax=tab["tmax"], device_classes=True)


def landcover_props(lc_grid, lc_class, rows, cols) -> LandCoverProps:
    """Cleaned land-cover codes -> property grids (utci_process.py:733-766)."""
    if lc_grid is None:
        z = np.zeros((rows, cols), F32)
        return LandCoverProps(z + F32(0.37), z - F32(3.41), z + F32(0.15), z + F32(0.95), None, 0.37, -3.41, 15., 0)
    lc = np.array(lc_grid, F32, copy=True)
    lc[(lc < 1) | (lc > 7)] = 6
    lc[(lc == 3) | (lc == 4)] = 5
    ids = np.unique(lc)
    out = {k: np.copy(lc) for k in ("tgk", "tstart", "alb", "emis", "tmax")}
    cols_ = {"tstart": 4, "alb": 1, "emis": 2, "tmax": 5, "tgk": 3}
    for v in ids:
        row = lc_class[:, 0] == v
        for k in ("tstart", "alb", "emis", "tmax", "tgk"):
            arr = out[k]
            arr[arr == v] = lc_class[row, cols_[k]]
    wall = np.where(lc_class[:, 0] == 99)
    return LandCoverProps(out["tgk"], out["tstart"], out["alb"], out["emis"], out["tmax"],
                          np.asarray(lc_class[wall, 3], F32), np.asarray(lc_class[wall, 4], F32),
                          np.asarray(lc_class[wall, 5], F32), 1)


@dataclass
class Series:
    steps: np.ndarray         # TIME_STEP_DTYPE (n_t)
    sun: np.ndarray           # SUN_STEP_DTYPE (n_day)
    sun_table: np.ndarray     # STEP_DTYPE
    patch: np.ndarray         # PATCH_STEP_DTYPE (n_t, P)
    gvf: np.ndarray           # GVF_AZ_DTYPE (18)
    final: dict               # carried scalars after the last step
    class_idx: np.ndarray     # uint8 per pixel (None: the site's device plane holds the classes)


def walk_steps(params: "ModelParams", scale) -> tuple:
    """`first` and `second` of the ground-view walks in pixels, as float32:
    the person height rounded (at least 1) and height * 20 rounded
    (utci_process.py:847-853), each times the scale and rounded, first at
    least 1 (solweig.py:143-146)."""
    height = torch.tensor(params.height)
    first = torch.round(height)
    if first == 0.:
        first = torch.tensor(1.)
    second = torch.round(height * 20.)
    sc = torch.tensor(scale)
    first_g = torch.round(first * sc)
    first_g = torch.tensor(1.) if first_g < 1 else first_g
    second_g = torch.round(second * sc)
    return F32(first_g.item()), F32(second_g.item())


@torch.inference_mode()
def build_series(*, met_file, altitude, azimuth, zen, jday, dectime, altmax, location, scale, amax, rows, cols,
                 props: LandCoverProps, params: ModelParams = None, time_start=0, time_stop=None,
                 initial_scalars=None, patch_option=2, day_chain=None) -> Series:
    """Tables for steps [time_start, time_stop) of run_utci_window's loop
    (utci_process.py:917-1067).  `day_chain` (from day_chain() over a range
    holding these steps) spares recomputing the daytime scalar chain when a
    day is built in parts."""
    if params is None:
        params = ModelParams()
    if params.anisotropic_sky != 1 or not params.cyl:
        raise NotImplementedError("only the reference defaults cyl=1, anisotropic_sky=1 are implemented")
    if time_stop is None:
        time_stop = met_file.shape[0]
    n_t = time_stop - time_start
    lat = location["latitude"]
    Ta_all, RH_all, radG_all = met_file[:, 11], met_file[:, 10], met_file[:, 14]
    P_all, Ws_all = met_file[:, 12], met_file[:, 9]
    uhii_all = met_file[:, 24] if met_file.shape[1] > 24 else np.zeros(met_file.shape[0])
    DOY = met_file[:, 1]
    fdl, ldl = params.firstdayleaf, params.lastdayleaf
    leaf = ((DOY > fdl) | (DOY < ldl)) if fdl > ldl else ((DOY > fdl) & (DOY < ldl))
    psi = np.where(leaf, F32(1) * F32(params.transVeg), F32(0.5)).astype(F32)
    first_f, second_f = walk_steps(params, scale)
    timestepdec = 0 if met_file.shape[0] == 1 else dectime[1] - dectime[0]
    if initial_scalars is None:
        timeadd, firstdaytime, CI = 0., 1., 1.0
    else:
        timeadd = float(initial_scalars["timeadd"])
        firstdaytime = float(initial_scalars["firstdaytime"])
        CI = float(initial_scalars["CI"])

    # pixel classes of the ground temperature wave: the distinct TmaxLST
    # values in ascending order (np.unique of the raster); a device-prepared
    # site indexes tg_factor by land-cover code instead, each code's slot
    # holding its TmaxLST value's factor
    code_slot = None
    if props.landcover and props.device_classes:
        present = [c for c in range(1, 8) if (props.codes >> c) & 1]
        tvals = np.unique(np.asarray(props.code_tmax, F32)[present])
        code_slot = {c: int(np.searchsorted(tvals, props.code_tmax[c])) for c in present}
        class_idx = None
    elif props.landcover:
        tvals, class_idx = np.unique(props.tmaxlst, return_inverse=True)
        if len(tvals) > N.MAX_CLASSES:
            raise ValueError(f"more than {N.MAX_CLASSES} distinct TmaxLST classes")
        class_idx = class_idx.reshape(rows, cols).astype(np.uint8)
    else:
        tvals = np.array([15.], F32)
        class_idx = None if props.device_classes else np.zeros((rows, cols), np.uint8)

    P = int(sum(T.PATCH_LAYOUT[patch_option][3]))
    steps = np.zeros(n_t, N.TIME_STEP_DTYPE)
    patch = np.zeros((n_t, P), N.PATCH_STEP_DTYPE)
    sbc_t = torch.tensor(SBC)
    ewall_t = torch.tensor(params.ewall)
    deg2rad_t = torch.tensor(np.pi / 180)
    alt_n, azi_n = T.sky_patches(patch_option)
    night_patches = torch.stack([torch.from_numpy(alt_n), torch.from_numpy(azi_n), torch.zeros(P)], dim=1)
    diff_vals = np.array([F32(s) - (F32(1) - F32(v)) * F32(1 - params.transVeg) for s in (0, 1) for v in (0, 1)], F32)
    # step-independent fields, evaluated once
    steps["sbc"] = F32(SBC)
    steps["albedo_b"] = F32(params.albedo_b)
    steps["first"], steps["second"] = first_f, second_f
    steps["refl_k"] = F32((1 - ewall_t).item())
    for k in ("absK", "absL", "Fside", "Fup", "Fcyl"):
        steps[k] = F32(getattr(params, k))
    steps["absl_sbc"] = F32((params.absL * sbc_t).item())
    steps["landcover"] = props.landcover
    idx_t = np.arange(time_start, time_stop)
    steps["rh32"] = np.asarray(RH_all[idx_t], F32)
    steps["ws32"] = np.asarray(Ws_all[idx_t], F32)
    steps["ta_mat"] = (F32(0) + np.asarray(Ta_all[idx_t], F32)) + np.asarray(uhii_all[idx_t], F32)
    steps["utci_pa"], steps["utci_k"] = _utci_tables(steps["ta_mat"], steps["rh32"])

    # per-step air temperature chain for every step at once (elementwise
    # float64; the general powers 10 ** x and x ** 4 element by element)
    Ta64v = torch.tensor(np.asarray(Ta_all[idx_t]))
    RH64v = torch.tensor(np.asarray(RH_all[idx_t]))
    ea_v = 6.107 * _rpow_each(10, (7.5 * Ta64v) / (237.3 + Ta64v)) * (RH64v / 100.)
    msteg_v = 46.5 * (ea_v / (Ta64v + 273.15))
    esky_v = (1 - (1 + msteg_v) * torch.exp(-((1.2 + 3.0 * msteg_v) ** 0.5))) + params.elvis
    ta4_v = _pow_each(Ta64v + 273.15, 4)
    rows_day = [i for i in range(time_start, time_stop) if altitude[0][i] > 0]
    dc = day_chain if day_chain is not None and all(i in day_chain["pos"] for i in rows_day) else \
        _day_chain(rows_day, met_file, altitude, azimuth, zen, jday, lat)
    # ground temperature wave inputs of every daytime row (solweig.py:2101-2122)
    if rows_day:
        pos = [dc["pos"][i] for i in rows_day]
        snup_d = dc["snup"][pos]
        dect_v = torch.tensor(np.asarray(dectime)[rows_day])
        phase_v = (dect_v - torch.floor(dect_v)) - snup_d / 24
        zen64_v = torch.tensor(np.asarray(zen[0])[rows_day])
        alt64_v = torch.tensor(np.asarray(altitude[0])[rows_day])
        corr_v = 0.1473 * torch.log(90 - (zen64_v / np.pi * 180)) + 0.3454
        cig_v = (torch.tensor(np.asarray(radG_all)[rows_day]) /
                 (dc["radI0"][pos] * (torch.sin(alt64_v * (np.pi / 180))) + dc["radD0"][pos])) + (1 - corr_v)
        if props.landcover:
            tm = torch.from_numpy(np.asarray(tvals, F32))
            # float64 phase / float32 class plane -> float32 (solweig.py:2103)
            fac_v = torch.sin(((phase_v.to(torch.float32)[:, None] / (tm[None, :] / 24 - snup_d[:, None] / 24)) *
                               np.pi) / 2).numpy().astype(F32)
        else:
            wave_v = torch.sin((phase_v / (15. / 24 - snup_d / 24)) * np.pi / 2)
            fac_v = wave_v.numpy().astype(F32)[:, None]
        # wall temperature, wall longwave and sunlit wall surface of every
        # daytime row (solweig.py:2101-2122, :1596), as (rows, wall classes)
        # arrays.  With a land-cover table the wall class is a 1-D float32
        # tensor, so each step's 0-dim float64 operands are rounded to
        # float32 first and the chain runs in float32; without one it runs in
        # float64.  x ** 4 element by element, as the step form evaluates it.
        f32 = torch.float32
        offs_day = [i - time_start for i in rows_day]
        alt_d = torch.tensor(np.asarray(altmax[0])[rows_day])
        ta_d = Ta64v[offs_day]
        ci_d = torch.where(1.0 < cig_v, torch.tensor(1.0, dtype=torch.float64), cig_v)  # min(cig, 1.0)
        se_t = sbc_t * ewall_t
        if props.landcover:
            tgk_w = torch.from_numpy(np.asarray(props.tgk_wall, F32).reshape(-1))[None, :]
            tst_w = torch.from_numpy(np.asarray(props.tstart_wall, F32).reshape(-1))[None, :]
            tmx_w = torch.from_numpy(np.asarray(props.tmaxlst_wall, F32).reshape(-1))[None, :]
            den = tmx_w / 24 - snup_d[:, None] / 24
            tgwall_d = (tgk_w * alt_d.to(f32)[:, None] + tst_w) * \
                torch.sin((phase_v.to(f32)[:, None] / den) * np.pi / 2)
            tgwall_d = torch.maximum(tgwall_d, torch.tensor(0)) * ci_d.to(f32)[:, None]
            base = (tgwall_d + ta_d.to(f32)[:, None]) + 273.15
        else:
            tgwall_d = (0.37 * alt_d + -3.41) * wave_v
            tgwall_d = (torch.maximum(tgwall_d, torch.tensor(0)) * ci_d)[:, None]
            base = (tgwall_d + ta_d[:, None]) + 273.15
        p4 = _pow_each(base.reshape(-1), 4).reshape(base.shape)
        lwall_d = (se_t * p4 - (se_t * ta4_v[offs_day]).to(p4.dtype)[:, None])[:, 0].numpy().astype(F32)
        sunsurf_d = ((se_t * p4) / torch.tensor(np.pi))[:, 0].numpy().astype(F32)
    day_k = {i: k for k, i in enumerate(rows_day)}
    # shortwave geometry of the daytime rows (sin / cos of the altitude,
    # tan of the zenith and its half), each element the per-step operations
    sw_v = {}
    if rows_day:
        alt32_v = torch.tensor([float(altitude[0][i]) for i in rows_day])
        beta_v = torch.tensor([float(zen[0][i]) for i in rows_day], dtype=torch.float32)
        sw_v = {"sin_alt": torch.sin(torch.tensor(np.asarray(altitude[0])[rows_day]) * (np.pi / 180)).numpy().astype(F32),
                "cos_alt": torch.cos(alt32_v * torch.tensor(np.pi / 180.0)).numpy().astype(F32),
                "tan_beta": torch.tan(beta_v).numpy().astype(F32),
                "qa": (torch.tan(beta_v) / 2).numpy().astype(F32), "alt32": alt32_v}
    suntab = T.sun_tables([float(azimuth[0][i]) for i in rows_day], [float(altitude[0][i]) for i in rows_day],
                          scale, float(amax), rows, cols)
    lcyl_rows, kside_rows = [], []
    # per-step fields that are elementwise roundings of the vectors above
    ta32_v = np.asarray(Ta_all[idx_t], np.float64).astype(F32)
    steps["ta32"] = ta32_v
    steps["ta4"] = ta4_v.numpy().astype(F32)
    steps["night_lup_base"] = ((F32(0) + ta32_v) + F32(0)) + F32(273.15)
    esky_py = esky_v.tolist()
    lag_rows, lag_timeadd = [], []    # thermal-lag exponent of each daytime step, evaluated after the loop
    # the daytime clearness index min(CI, 1.0) of each daytime row: the
    # float32 tensor element unless 1.0 < CI (then the float 1.0)
    n_dr = len(rows_day)
    pos_day = [dc["pos"][i] for i in rows_day]
    ci_vals = dc["CI"][pos_day].tolist() if n_dr else []
    day_o = [i - time_start for i in rows_day]
    ci_f32 = False   # the carried CI is a float until a daytime row sets it
    for o, i in enumerate(range(time_start, time_stop)):
        S = steps[o]
        if (dectime[i] - np.floor(dectime[i])) == 0:
            CI, ci_f32 = 1., False
        esky = esky_py[o]
        if altitude[0][i] > 0:
            kd = day_k[i]
            d = pos_day[kd]
            CI, ci_f32 = (1.0, False) if 1.0 < ci_vals[kd] else (ci_vals[kd], True)
            lv = dc["lv"][d]
            if lv is None:   # sun below the horizon in the Perez geometry: the 0-dim form
                lv = _perez((torch.tensor(zen[0][i]) * (180 / np.pi)).item(), torch.tensor(azimuth[0][i]).item(),
                            dc["radD"][d], dc["radI"][d], jday[0][i].item())
            # thermal lag weights (solweig.py:451-488), one timeadd for all six planes
            S["tw_first"] = int(firstdaytime == 1)
            lag_rows.append(o)
            if timeadd >= (59 / 1440):
                lag_timeadd.append(timeadd)
                S["tw_mode"] = 1
                timeadd = timestepdec if timestepdec > (59 / 1440) else 0
            else:
                timeadd = timeadd + timestepdec
                lag_timeadd.append(timeadd)
                S["tw_mode"] = 0
            firstdaytime = 0
            # Kside per patch (solweig.py:683-724): after the loop, all daytime
            # steps of each patch layout at once
            kside_rows.append((o, i, lv, dc["radD"][d], dc["radI"][d], sw_v["alt32"][kd]))
            L_patches = lv
            # sunlit wall surface of define_patch_characteristics (solweig.py:1596)
            sun_surf = sunsurf_d[kd]
        else:
            timeadd = 0
            firstdaytime = 1
            L_patches = night_patches
            sun_surf = F32(0)
        if CI < 0.95:
            # the 0-dim form's promotions: CI (float32 tensor or float) times
            # the float64 esky in float64; 1 - CI in CI's own precision
            one_minus = float(F32(1) - F32(CI)) if ci_f32 else 1 - CI
            esky = float(CI) * esky + one_minus * 1.
        # Lcyl per patch (solweig.py:1651-1760): evaluated after the loop for
        # all steps of each patch layout at once
        lcyl_rows.append((o, L_patches[:, 0], torch.tensor(esky, dtype=torch.float64), sun_surf))
    # the per-daytime-step fields, as columns (each element the value the
    # step form stored: float32 roundings of the same float64 / float32 values)
    steps["day_row"] = -1
    if n_dr:
        steps["is_day"][day_o] = 1
        steps["day_row"][day_o] = np.arange(n_dr)
        counts = np.array([len(suntab[k][2]) for k in range(n_dr)], np.int64)
        offs = np.concatenate([[0], np.cumsum(counts)[:-1]])
        sun_rows = np.zeros(n_dr, N.SUN_STEP_DTYPE)
        sun_rows["step_offset"], sun_rows["step_count"], sun_rows["t"] = offs, counts, day_o
        sun_rows["facesh_mode"] = [suntab[k][4][0] for k in range(n_dr)]
        sun_rows["facesh_lo"] = [suntab[k][4][1] for k in range(n_dr)]
        sun_rows["facesh_hi"] = [suntab[k][4][2] for k in range(n_dr)]
        sun_rows["psi_term"] = F32(1) - np.asarray(psi, F32)[rows_day]
        tables = [np.zeros(int(counts.sum()), N.STEP_DTYPE)]
        tables[0]["dx"] = np.concatenate([suntab[k][0] for k in range(n_dr)])
        tables[0]["dy"] = np.concatenate([suntab[k][1] for k in range(n_dr)])
        tables[0]["dz"] = np.concatenate([suntab[k][2] for k in range(n_dr)])
        # ground temperature wave (solweig.py:2101-2122)
        cig = cig_v.numpy()
        steps["cig"][day_o] = np.where(1.0 < cig, 1.0, cig).astype(F32)
        steps["altmax32"][day_o] = np.asarray(altmax[0], np.float64)[rows_day].astype(F32)
        if code_slot is None:
            steps["tg_factor"][day_o, :len(tvals)] = fac_v
        else:
            for code, k in code_slot.items():
                steps["tg_factor"][day_o, code] = fac_v[:, k]
        steps["lwall"][day_o] = lwall_d
        # shortwave scalars
        steps["radI"][day_o] = dc["radI"][pos_day].numpy().astype(F32)
        steps["radD"][day_o] = dc["radD"][pos_day].numpy().astype(F32)
        steps["radG"][day_o] = np.asarray(radG_all, np.float64)[rows_day].astype(F32)
        for k in ("sin_alt", "cos_alt", "tan_beta", "qa"):
            steps[k][day_o] = sw_v[k]
    # TsWaveDelay weights (solweig.py:451-488): exp(-33.27 * timeadd) with
    # timeadd made a tensor as the 0-dim form makes it (float32 from a
    # Python float, float64 from a numpy float64 such as a dectime
    # difference: torch.tensor's own dtype choice, per element) and rounded
    # to float32 at the end; a vector element has the 0-dim bits
    kinds = [torch.tensor(v).dtype for v in lag_timeadd]
    for kind in set(kinds):
        sel_ = [k for k, d in enumerate(kinds) if d == kind]
        w = torch.exp(-33.27 * torch.tensor([lag_timeadd[k] for k in sel_], dtype=kind))
        rows_ = [lag_rows[k] for k in sel_]
        steps["tw_a"][rows_] = (1 - w).numpy().astype(F32)
        steps["tw_b"][rows_] = w.numpy().astype(F32)
    _lcyl_tables(patch, lcyl_rows, ta4_v, ewall_t, sbc_t)
    _kside_tables(patch, kside_rows, diff_vals, params.albedo_b, azimuth, altitude)
    sun = sun_rows if n_dr else np.zeros(0, N.SUN_STEP_DTYPE)
    table = tables[0] if n_dr else np.zeros(0, N.STEP_DTYPE)
    final = {"CI": float(CI), "firstdaytime": float(firstdaytime), "timeadd": float(timeadd)}
    return Series(steps, sun, table, patch, T.gvf_table(int(second_f)), final, class_idx)
