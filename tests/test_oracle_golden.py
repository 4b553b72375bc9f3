"""The CPU oracle against the golden fixtures produced by running the
reference (tests/golden/make_golden.py).  Every comparison is on raw float32
bits: the oracle restates the reference's operation order exactly."""
import numpy as np
import pytest

from conftest import FULL_CASES, SVF_CASES, golden_location, load_golden
from golden_util import assert_bits_equal

from oracle import march as om
from oracle import svf as osvf
from oracle import window as ow


@pytest.mark.parametrize("case", SVF_CASES)
def test_oracle_svf_bit_exact(case):
    d = load_golden(case)
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(d["dsm"], d["trees"], d["dem"])
    assert amax == d["amaxvalue"]
    out = osvf.svf_calculator(2, amax, d["dsm"], vegdsm, vegdsm2, bush, float(d["scale"]))
    for name, v in zip(osvf.SVF_ORDER, out):
        assert_bits_equal(v, d["svf_" + name].astype(np.float32), f"{case} {name}")


def test_oracle_svf_march_pool_bit_exact():
    """The CPU timing's form of the sweep: the patch marches in a spawn pool
    of two processes, the sums in this process in patch order."""
    case = "bush24" if "bush24" in SVF_CASES else SVF_CASES[0]
    d = load_golden(case)
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(d["dsm"], d["trees"], d["dem"])
    pool, one = osvf.march_pool(2, amax, d["dsm"], vegdsm, vegdsm2, bush, float(d["scale"]))
    try:
        out = osvf.svf_calculator(2, amax, d["dsm"], vegdsm, vegdsm2, bush, float(d["scale"]),
                                  march_map=lambda tasks: pool.imap(one, tasks))
    finally:
        pool.close()
        pool.join()
    for name, v in zip(osvf.SVF_ORDER, out):
        assert_bits_equal(v, d["svf_" + name].astype(np.float32), f"{case} {name}")
    acc = osvf.SvfAccumulator(2, *d["dsm"].shape, vegdsm2)
    with pytest.raises(ValueError, match="out of order"):
        acc.add(osvf.patch_tasks(2)[1], *out[15:18], 0)


@pytest.mark.parametrize("case", FULL_CASES)
def test_oracle_sun_march_bit_exact(case):
    d = load_golden(case)
    import torch
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(d["dsm"], d["trees"], d["dem"])
    asp = om.aspect_radians(d["aspect_ref"])
    names = ("vegsh", "sh", "vbshvegsh", "wallsh", "wallsun", "wallshve", "facesh", "facesun")
    for j, i in enumerate(d["march_steps"]):
        az = torch.tensor(d["azimuth"][0][i]).item()
        alt = torch.tensor(d["altitude"][0][i]).item()
        out = om.wallheight_23(d["dsm"], vegdsm, vegdsm2, az, alt, float(d["scale"]), float(amax), bush,
                               d["walls_ref"], asp)
        for name, v in zip(names, out):
            assert_bits_equal(v, d["march_" + name][j], f"{case} step {i} {name}")


@pytest.mark.parametrize("case", FULL_CASES)
def test_oracle_time_loop_bit_exact(case):
    d = load_golden(case)
    bundle = tuple(d["svf_" + k].astype(np.float32) for k in osvf.SVF_ORDER)
    outs, final = ow.run_utci_window(
        a=d["dsm"], temp1=d["trees"], temp2=d["dem"], walls=d["walls_ref"], dirwalls=d["aspect_ref"],
        svf_bundle=bundle, met_file=d["met"], altitude=d["altitude"], azimuth=d["azimuth"], zen=d["zen"],
        jday=d["jday"], dectime=d["dectime"], altmax=d["altmax"], location=golden_location(d),
        scale=float(d["scale"]), amaxvalue=d["amaxvalue"], landcover_grid=d["landcover"], lc_class=d["lc_class"],
        requested_variables=ow.VARIABLES, return_final_state=True)
    for k in ow.VARIABLES:
        assert_bits_equal(outs[k], d["out_" + k], f"{case} {k}")
    for k in ow.STATE_PLANES:
        assert_bits_equal(final[k], d["final_" + k], f"{case} final {k}")
    assert final["CI"] == pytest.approx(float(d["final_CI"]), abs=0)
    assert final["timeadd"] == float(d["final_timeadd"])
    assert final["Twater"] == float(d["final_Twater"])


def test_oracle_rejects_unknown_variable():
    d = load_golden("city36")
    bundle = tuple(d["svf_" + k].astype(np.float32) for k in osvf.SVF_ORDER)
    with pytest.raises(ValueError):
        ow.run_utci_window(a=d["dsm"], temp1=d["trees"], temp2=d["dem"], walls=d["walls_ref"],
                           dirwalls=d["aspect_ref"], svf_bundle=bundle, met_file=d["met"], altitude=d["altitude"],
                           azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"], dectime=d["dectime"],
                           altmax=d["altmax"], location=golden_location(d), scale=1.0,
                           requested_variables=("utci", "bogus"))
    with pytest.raises(ValueError):
        ow.run_utci_window(a=d["dsm"], temp1=d["trees"], temp2=d["dem"], walls=d["walls_ref"],
                           dirwalls=d["aspect_ref"], svf_bundle=bundle, met_file=d["met"], altitude=d["altitude"],
                           azimuth=d["azimuth"], zen=d["zen"], jday=d["jday"], dectime=d["dectime"],
                           altmax=d["altmax"], location=golden_location(d), scale=1.0, time_start=5, time_stop=3)
