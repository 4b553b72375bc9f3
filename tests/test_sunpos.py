"""The sun geometry of a forcing table (sunpos.metdata_noload) equals, bit
for bit, what the reference's Solweig_2015a_metdata_noload returned for the
same forcing and site (tests/golden/sun_geometry.npz, written by
tests/golden/make_sun_geometry.py from the unmodified reference): the
single-site workloads and the 64 sites of the batched workload (latitudes
0-60 N)."""
import numpy as np
import pytest

from solweig_project_b200 import sunpos, synthetic

KEYS = ("altitude", "azimuth", "zen", "jday", "dectime", "altmax")


def _check(prefix, met, loc):
    want = synthetic.load_sun_geometry(prefix)
    _, alt, azi, zen, jday, _, dectime, altmax = sunpos.metdata_noload(met, loc, synthetic.DEFAULT_UTC)
    got = dict(altitude=alt, azimuth=azi, zen=zen, jday=jday, dectime=dectime, altmax=altmax)
    for k in KEYS:
        g, w = np.asarray(got[k], np.float64), np.asarray(want[k], np.float64)
        assert g.shape == w.shape, (prefix, k)
        assert np.array_equal(g.view(np.uint64), w.view(np.uint64)), (prefix, k, np.abs(g - w).max())


def test_single_site_geometry_is_the_references():
    _check("single", synthetic.make_met(1234), dict(synthetic.DEFAULT_LOCATION))


@pytest.mark.parametrize("i", range(0, 64, 1))
def test_batched_site_geometry_is_the_references(i):
    s = synthetic.multi_site_specs()[i]
    _check(f"multi{i}", synthetic.make_met(s["seed"]),
           {"latitude": s["latitude"], "longitude": s["longitude"], "altitude": 3.0})


def test_sun_position_known_values():
    """Reda and Andreas (2004) example, 2003-10-17 12:30:30 UT-7 at
    39.742476 N, 105.1786 W, 1830.14 m: zenith 50.111622, azimuth
    194.340241 (their Table A5.1, with delta T and refraction inputs of the
    paper; this variant uses delta T = 0 and the standard refraction, so
    the match is to ~0.01 degree)."""
    z, a = sunpos.sun_position(2003, 10, 17, 12, 30, -7, 39.742476, -105.1786, 1830.14, sec=30)
    assert abs(z - 50.111622) < 0.02 and abs(a - 194.340241) < 0.02
