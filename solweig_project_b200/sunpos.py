"""Sun geometry of a forcing table: the Solar Position Algorithm (Reda and
Andreas 2004, Solar Energy 76(5):577-589) and the per-row geometry the
chain takes (altitude, azimuth, zenith, day of year, decimal time and the
day's maximum altitude).

Follows the reference's ``Solweig_2015a_metdata_noload`` and its
``sun_position`` (solweig_gpu/sun_position.py:26-117, 119-887, 905-1010)
operation for operation in float64 numpy, so the angles agree to the last
bit (checked against the reference's own outputs for 65 sites in
tests/test_sunpos.py): the float32 march tables built from them decide
which pixels a sun march shades.  Host-side: a day is a few dozen calls.
The periodic-term tables are the algorithm's published constants
(``data/spa_terms.json``).
"""
from __future__ import annotations

import datetime
import functools
import json
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "spa_terms.json")


@functools.lru_cache(maxsize=1)
def _terms():
    with open(_DATA) as fh:
        raw = json.load(fh)
    return {k: np.array(v, np.float64) for k, v in raw.items() if k != "source"}


def _wrap(x, period=360.0):
    """x reduced into [0, period) (sun_position.py:887-903)."""
    x = x - period * np.floor(x / period)
    if x < 0.0:
        x = x + period
    return x


def _series(name, jme, summed=True):
    """sum A cos(B + C * JME) over a term table (one row tables: the array)."""
    t = _terms()[name]
    v = t[:, 0] * np.cos(t[:, 1] + (t[:, 2] * jme))
    return np.sum(v) if summed else v


def _cubic(p, x):
    """p0 x^3 + p1 x^2 + p2 x + p3, written out as the reference does."""
    return p[0] * np.power(x, 3) + p[1] * np.power(x, 2) + p[2] * x + p[3]


def _julian(year, month, day, hour, minute, sec, utc):
    """Julian day and ephemeris century / millennium (delta T = 0;
    sun_position.py:119-186)."""
    if month == 1 or month == 2:
        y, m = year - 1, month + 12
    else:
        y, m = year, month
    ut = ((hour - utc) / 24) + (minute / (60 * 24)) + (sec / (60 * 60 * 24))
    d = day + ut
    if year < 1582 or (year == 1582 and (month < 10 or (month == 10 and day < 15))):
        b = 0   # Julian calendar (days 5-14 of October 1582 never existed; taken as the 4th)
    else:
        a = np.floor(y / 100)
        b = 2 - a + np.floor(a / 4)
    jd = d + b + np.floor(365.25 * (y + 4716)) + np.floor(30.6001 * (m + 1)) - 1524.5
    jde = jd + (0 / 86400)
    jc = (jd - 2451545) / 36525
    jce = (jde - 2451545) / 36525
    return jd, jc, jce, jce / 10


def sun_position(year, month, day, hour, minute, utc, latitude, longitude, altitude_m, sec=0):
    """(zenith, azimuth) in degrees of the sun seen from a site at the given
    local time (UTC offset in hours), with the reference's refraction
    correction.  Steps 1-14 of the algorithm."""
    jd, jc, jce, jme = _julian(year, month, day, hour, minute, sec, utc)
    # 2. heliocentric longitude, latitude (degrees) and radius (AU)
    lon_h = (_series("L0_terms", jme) + (_series("L1_terms", jme) * jme) +
             (_series("L2_terms", jme) * np.power(jme, 2)) + (_series("L3_terms", jme) * np.power(jme, 3)) +
             (_series("L4_terms", jme) * np.power(jme, 4)) +
             (_series("L5_terms", jme, summed=False) * np.power(jme, 5))) / 1e8
    lon_h = _wrap(lon_h * 180 / np.pi)
    lat_h = (_series("B0_terms", jme) + (_series("B1_terms", jme) * jme)) / 1e8
    lat_h = _wrap(lat_h * 180 / np.pi)
    radius = (_series("R0_terms", jme) + (_series("R1_terms", jme) * jme) +
              (_series("R2_terms", jme) * np.power(jme, 2)) + (_series("R3_terms", jme) * np.power(jme, 3)) +
              (_series("R4_terms", jme, summed=False) * np.power(jme, 4))) / 1e8
    # 3. geocentric longitude / latitude
    theta = _wrap(lon_h + 180)
    beta = _wrap(-lat_h)
    # 4. nutation in longitude and obliquity (degrees)
    xs = np.array([_cubic(((1 / 189474), -0.0019142, 445267.11148, 297.85036), jce),
                   _cubic((-(1 / 300000), -0.0001603, 35999.05034, 357.52772), jce),
                   _cubic(((1 / 56250), 0.0086972, 477198.867398, 134.96298), jce),
                   _cubic(((1 / 327270), -0.0036825, 483202.017538, 93.27191), jce),
                   _cubic(((1 / 450000), 0.0020708, -1934.136261, 125.04452), jce)])
    t = _terms()
    arg = t["Y_terms"].dot(np.transpose(xs)) * (np.pi / 180)
    nt = t["nutation_terms"]
    dpsi = np.sum((nt[:, 0] + (nt[:, 1] * jce)) * np.sin(arg)) / 36000000
    deps = np.sum((nt[:, 2] + (nt[:, 3] * jce)) * np.cos(arg)) / 36000000
    # 5. true obliquity of the ecliptic (degrees)
    u = jme / 10
    p = (2.45, 5.79, 27.87, 7.12, -39.05, -249.67, -51.38, 1999.25, -1.55, -4680.93, 84381.448)
    eps0 = p[0] * np.power(u, 10) + p[1] * np.power(u, 9) + \
        p[2] * np.power(u, 8) + p[3] * np.power(u, 7) + \
        p[4] * np.power(u, 6) + p[5] * np.power(u, 5) + \
        p[6] * np.power(u, 4) + p[7] * np.power(u, 3) + \
        p[8] * np.power(u, 2) + p[9] * u + p[10]
    eps = (eps0 / 3600) + deps
    # 6.-7. aberration and apparent sun longitude
    lam = theta + dpsi + (-20.4898 / (3600 * radius))
    # 8. apparent sidereal time at Greenwich
    nu0 = 280.46061837 + (360.98564736629 * (jd - 2451545)) + \
        (0.000387933 * np.power(jc, 2)) - \
        (np.power(jc, 3) / 38710000)
    nu = _wrap(nu0) + (dpsi * np.cos(eps * np.pi / 180))
    # 9.-10. geocentric right ascension and declination
    num = (np.sin(lam * np.pi / 180) * np.cos(eps * np.pi / 180)) - \
        (np.tan(beta * np.pi / 180) * np.sin(eps * np.pi / 180))
    alpha = _wrap(np.arctan2(num, np.cos(lam * np.pi / 180)) * 180 / np.pi)
    delta = np.arcsin((np.sin(beta * np.pi / 180) * np.cos(eps * np.pi / 180)) +
                      (np.cos(beta * np.pi / 180) * np.sin(eps * np.pi / 180) *
                       np.sin(lam * np.pi / 180))) * 180 / np.pi
    # 11. observer local hour angle
    h = _wrap(nu + longitude - alpha)
    # 12. topocentric right ascension parallax and declination
    xi = 8.794 / (3600 * radius)
    uu = np.arctan(0.99664719 * np.tan(latitude * np.pi / 180))
    x = np.cos(uu) + ((altitude_m / 6378140) * np.cos(latitude * np.pi / 180))
    y = (0.99664719 * np.sin(uu)) + ((altitude_m / 6378140) * np.sin(latitude * np.pi / 180))
    dalpha = np.arctan2(-x * np.sin(xi * np.pi / 180) * np.sin(h * np.pi / 180),
                        np.cos(delta * np.pi / 180) - (x * np.sin(xi * np.pi / 180) * np.cos(h * np.pi / 180)))
    delta_t = np.arctan2((np.sin(delta * np.pi / 180) - (y * np.sin(xi * np.pi / 180))) * np.cos(dalpha),
                         np.cos(delta * np.pi / 180) - (y * np.sin(xi * np.pi / 180)) *
                         np.cos(h * np.pi / 180)) * 180 / np.pi
    # 13. topocentric local hour angle
    hp = h - dalpha * 180 / np.pi
    # 14. zenith (with refraction) and azimuth
    e0 = np.arcsin((np.sin(latitude * np.pi / 180) * np.sin(delta_t * np.pi / 180)) +
                   (np.cos(latitude * np.pi / 180) * np.cos(delta_t * np.pi / 180) *
                    np.cos(hp * np.pi / 180))) * 180 / np.pi
    refr = 1.02 / (60 * np.tan((e0 + (10.3 / (e0 + 5.11))) * np.pi / 180))
    zenith = 90 - (e0 + refr)
    az = (np.arctan2(np.sin(hp * np.pi / 180),
                     (np.cos(hp * np.pi / 180) * np.sin(latitude * np.pi / 180)) -
                     (np.tan(delta_t * np.pi / 180) * np.cos(latitude * np.pi / 180))) * 180 / np.pi) + 180
    return float(np.asarray(zenith).squeeze()), float(np.asarray(_wrap(az)).squeeze())


def _at(stamp, utc, loc):
    return sun_position(stamp.year, stamp.month, stamp.day, stamp.hour, stamp.minute, utc, loc["latitude"],
                        loc["longitude"], loc["altitude"])


def metdata_noload(met, location, utc):
    """Sun geometry of every row of a forcing table in the reference's met
    layout (columns 0 year, 1 day of year, 2 hour, 3 minute), as
    ``Solweig_2015a_metdata_noload`` returns it (sun_position.py:905-1010):
    ``(YYYY, altitude, azimuth, zen, jday, leafon, dectime, altmax)`` --
    (1, T) float64 arrays except ``dectime`` (T,).  The sun of a row is taken
    half a time step before its stamp; zenith angles in (89, 90] are clamped
    to 89; ``altmax`` is the day's largest altitude found in 15-minute steps
    from 10:15."""
    met = np.asarray(met)
    n = met.shape[0]
    dectime = met[:, 1] + met[:, 2] / 24 + met[:, 3] / (60 * 24.)
    half = 0 if n == 1 else (dectime[1] - dectime[0]) / 2.
    out = {k: np.empty((1, n)) for k in ("YYYY", "altitude", "azimuth", "zen", "jday", "leafon", "altmax")}
    sunmaximum = 0.
    for i in range(n):
        ymd = datetime.datetime(int(met[i, 0]), 1, 1) + datetime.timedelta(int(met[i, 1]) - 1)
        if i == 0 or np.mod(dectime[i], np.floor(dectime[i])) == 0:
            fifteen = 0.
            sunmaximum = -90.
            zen_max = 90.
            while sunmaximum <= 90. - zen_max:
                sunmaximum = 90. - zen_max
                fifteen = fifteen + 15. / 1440.
                zen_max, _ = _at(ymd + datetime.timedelta(days=(60 * 10) / 1440.0 + fifteen), utc, location)
        out["altmax"][0, i] = float(sunmaximum)
        stamp = ymd + datetime.timedelta(hours=met[i, 2]) + datetime.timedelta(minutes=met[i, 3]) - \
            datetime.timedelta(days=half)
        zenith, azimuth = _at(stamp, utc, location)
        if 89.0 < zenith <= 90.0:
            zenith = 89.0
        out["altitude"][0, i] = 90. - zenith
        out["zen"][0, i] = zenith * (np.pi / 180.)
        out["azimuth"][0, i] = azimuth
        out["YYYY"][0, i] = met[i, 0]
        doy = ymd.timetuple().tm_yday
        out["jday"][0, i] = doy
        out["leafon"][0, i] = 1 if (doy > 97) | (doy < 300) else 0
    return (out["YYYY"], out["altitude"], out["azimuth"], out["zen"], out["jday"], out["leafon"], dectime,
            out["altmax"])
