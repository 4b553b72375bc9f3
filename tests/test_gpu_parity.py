"""CUDA path (through the C ABI) against the reference-generated golden
fixtures and the CPU oracle.

Bars (the target tolerances):
* SVF planes, the three patch cubes, the sun-march planes and the shadow
  output: bit-exact;
* Tmrt within 1e-3 K, UTCI within 1e-3 C, the flux outputs within 1e-3 of
  their own scale (W/m2) on the same inputs.
"""
import numpy as np
import pytest

from conftest import FULL_CASES, SVF_CASES, golden_location, load_golden
from golden_util import assert_bits_equal, max_abs

pytestmark = pytest.mark.gpu

TMRT_TOL = 1e-3    # K
UTCI_TOL = 1e-3    # C
FLUX_TOL = 1e-3    # W m-2 (Kup, Kdown, Lup, Ldown)

SVF_ORDER = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS", "svfSaveg",
             "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg")


def make_site(d, cuda):
    from solweig_project_b200.engine import DeviceSite
    lc_class = d.get("lc_class")
    return DeviceSite(d["dsm"], d["trees"], d["dem"], d["walls_ref"], d["aspect_ref"], float(d["scale"]),
                      landcover=d["landcover"] if lc_class is not None else None, lc_class=lc_class,
                      amaxvalue=d["amaxvalue"])


@pytest.mark.parametrize("case", SVF_CASES)
def test_svf_sweep_bit_exact(case, cuda):
    d = load_golden(case)
    site = make_site(d, cuda)
    res = site.run_svf()
    planes = res.planes.cpu().numpy()
    for k, name in enumerate(SVF_ORDER):
        assert_bits_equal(planes[k], d["svf_" + name], f"{case} {name}")
    assert_bits_equal(planes[15], d["svf_svftotal"], f"{case} svftotal")
    sh, veg, vb = (x.cpu().numpy() for x in res.cubes())
    assert_bits_equal(sh, d["svf_shmat"].astype(np.float32), f"{case} shmat")
    assert_bits_equal(veg, d["svf_vegshmat"].astype(np.float32), f"{case} vegshmat")
    assert_bits_equal(vb, d["svf_vbshvegshmat"].astype(np.float32), f"{case} vbshvegshmat")


def _series(site, d):
    return site.build_series(d["met"], d["altitude"], d["azimuth"], d["zen"], d["jday"], d["dectime"], d["altmax"],
                             golden_location(d))


@pytest.mark.parametrize("case", FULL_CASES)
def test_sun_march_bit_exact(case, cuda):
    d = load_golden(case)
    site = make_site(d, cuda)
    site.run_svf()
    ser = _series(site, d)
    _, dbg = site.run_sun_march(ser)
    dbg = dbg.cpu().numpy()
    names = ("vegsh", "sh", "vbshvegsh", "wallsh", "wallsun", "wallshve", "facesh", "facesun")
    assert dbg.shape[0] == len(d["march_steps"])
    for k, name in enumerate(names):
        assert_bits_equal(dbg[:, k], d["march_" + name], f"{case} {name}")


@pytest.mark.parametrize("case", FULL_CASES)
def test_time_loop_against_reference(case, cuda):
    d = load_golden(case)
    site = make_site(d, cuda)
    site.run_svf()
    ser = _series(site, d)
    out = site.run_time_loop(ser, requested=("utci", "tmrt", "kup", "kdown", "lup", "ldown", "shadow"))
    out = {k: v.cpu().numpy() for k, v in out.items()}
    assert_bits_equal(out["shadow"], d["out_shadow"], f"{case} shadow")
    assert max_abs(out["tmrt"], d["out_tmrt"]) <= TMRT_TOL
    assert max_abs(out["utci"], d["out_utci"]) <= UTCI_TOL
    for k in ("kup", "kdown", "lup", "ldown"):
        assert max_abs(out[k], d["out_" + k]) <= FLUX_TOL, k
    state = site.state_dict()
    for k in ("Tgmap1", "Tgmap1E", "Tgmap1S", "Tgmap1W", "Tgmap1N", "TgOut1"):
        assert max_abs(state[k].cpu().numpy(), d["final_" + k]) <= FLUX_TOL, k
