"""The CPU timing legs of bench.py (``cpu_baseline`` and ``--impl
reference``): one pass of the oracle cut into timed pieces, the sweep's
patch marches in a spawn pool or in process, must give the oracle's single
call bit for bit, whatever the cut."""
import numpy as np
import pytest

import bench
from oracle import svf as osvf
from oracle import window as ow
from solweig_project_b200.synthetic import DEFAULT_LOCATION


@pytest.fixture(scope="module")
def site():
    city, met, geo, lc_class = bench.make_workload("exact500", 0, 32)
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(city.dsm, city.trees, city.dem)
    bundle = osvf.svf_calculator(2, amax, city.dsm, vegdsm, vegdsm2, bush, city.scale)
    want = ow.run_utci_window(a=city.dsm, temp1=city.trees, temp2=city.dem, walls=city.walls,
                              dirwalls=city.aspect, svf_bundle=bundle, met_file=met, location=dict(DEFAULT_LOCATION),
                              scale=city.scale, landcover_grid=city.landcover, lc_class=lc_class,
                              requested_variables=("utci", "tmrt"), **geo)
    return city, met, geo, lc_class, want


# one piece; the sweep + the window in 4 pieces; the sweep cut into patch
# groups as well (more pieces than window steps)
@pytest.mark.parametrize("n_pieces,processes", [(1, 1), (5, 2), (30, 1)])
def test_pass_in_pieces_is_the_single_call(site, n_pieces, processes):
    city, met, geo, lc_class, want = site
    march_map, close = bench._march_map(city, processes)
    try:
        times, out = bench.oracle_pass(city, met, geo, lc_class, n_pieces, march_map)
    finally:
        close()
    assert len(times) == n_pieces and all(t >= 0 for t in times)
    for k in ("utci", "tmrt"):
        assert np.array_equal(out[k].view(np.uint32), want[k].view(np.uint32)), k


def test_crop_keeps_every_raster_aligned(site):
    city = site[0]
    sub = bench._crop(city, 20)
    for k in ("dsm", "trees", "dem", "walls", "aspect", "landcover"):
        assert np.array_equal(getattr(sub, k), getattr(city, k)[:20, :20]), k
    assert sub.scale == city.scale
