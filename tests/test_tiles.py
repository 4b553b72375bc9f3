"""Tile orchestration (preprocessor.py:341-385 tiling, run_utci_tiles /
compute_utci outputs): windows on CPU, a whole tiled run as one batch
against single-tile runs on the GPU."""
import numpy as np
import pytest

from solweig_project_b200 import formats as FM
from solweig_project_b200 import tiles as TL


def _reference_windows(width, height, tilesize, overlap):
    """The reference's loop, restated (x = column offset i, y = row offset j)."""
    if tilesize >= width and tilesize >= height:
        return {"0_0": (0, 0, width, height)}
    out = {}
    for i in range(0, width, tilesize):
        for j in range(0, height, tilesize):
            out[f"{i}_{j}"] = (i, j, min(tilesize + overlap, width - i), min(tilesize + overlap, height - j))
    return out


@pytest.mark.parametrize("rows,cols,ts,ov", [(150, 130, 64, 10), (64, 64, 64, 5), (200, 90, 100, 0), (33, 500, 40, 39)])
def test_windows_follow_the_reference_tiling(rows, cols, ts, ov):
    want = _reference_windows(cols, rows, ts, ov)
    got = TL.tile_windows(rows, cols, ts, ov)
    assert [k for k, *_ in got] == list(want)
    for key, r0, r1, c0, c1 in got:
        i, j, w, h = want[key]
        assert (c0, r0, c1 - c0, r1 - r0) == (i, j, w, h)


def test_bad_overlap_is_refused():
    with pytest.raises(ValueError, match="overlap"):
        TL.tile_windows(100, 100, 50, 50)


def test_multiband_tiff_carries_time_metadata():
    a = np.random.default_rng(0).random((4, 6, 5)).astype(np.float32)
    md = [{"Time": f"2025-07-01T{h:02d}:00:00"} for h in range(4)]
    b, gt, md2 = FM.read_tiff(FM.tiff_bytes(a, (10.0, 1.0, 0.0, 20.0, 0.0, -1.0), md), with_metadata=True)
    assert np.array_equal(a, b) and md2 == md and gt == (10.0, 1.0, 0.0, 20.0, 0.0, -1.0)


@pytest.mark.gpu
def test_tiled_batch_equals_single_tile_runs(cuda, tmp_path, monkeypatch):
    from solweig_project_b200 import api, synthetic
    from solweig_project_b200 import engine as E
    # the in-loop patch sums (the reference's float32 order) in the batch
    # kernels and in the single-tile runs alike; the tensor-core form is
    # checked batch against single site in tests/test_batch.py
    monkeypatch.setattr(E, "TENSOR_SUMS", False)
    city = synthetic.make_city(150, 130, seed=9, n_buildings=20, n_trees=16, side_range=(5, 14))
    met = synthetic.make_met(9)
    geo = synthetic.load_sun_geometry("single")
    loc = dict(synthetic.DEFAULT_LOCATION)
    lc = synthetic.default_lc_class()
    gt = (500000.0, 1.0, 0.0, 3300000.0, 0.0, -1.0)
    res = TL.run_tiles(dsm=city.dsm, trees=city.trees, dem=city.dem, walls=city.walls, aspect=city.aspect,
                       scale=city.scale, met_file=met, location=loc, tile_size=64, overlap=10,
                       landcover=city.landcover, lc_class=lc, requested=("utci", "tmrt"), output_dir=str(tmp_path),
                       selected_date="2025-07-01", geotransform=gt, graph=True, **geo)
    assert len(res) == 9
    for key, r0, r1, c0, c1 in TL.tile_windows(150, 130, 64, 10):
        sl = (slice(r0, r1), slice(c0, c1))
        one = api.run_exact_chain(dsm=city.dsm[sl], trees=city.trees[sl], dem=city.dem[sl], walls=city.walls[sl],
                                  aspect=city.aspect[sl], scale=city.scale, met_file=met, location=loc,
                                  landcover=city.landcover[sl], lc_class=lc, requested=("utci", "tmrt"), **geo)
        for k in ("utci", "tmrt"):
            assert np.array_equal(res[key][k].view(np.uint32), one[k].view(np.uint32)), (key, k)
        arr, tgt, md = FM.read_tiff(open(tmp_path / key / f"UTCI_{key}.tif", "rb").read(), with_metadata=True)
        assert np.array_equal(arr.view(np.uint32), res[key]["utci"].view(np.uint32))
        assert tgt == (gt[0] + c0, 1.0, 0.0, gt[3] - r0, 0.0, -1.0)
        assert md[13]["Time"].startswith("2025-07-01T13:")
    # one tile against the CPU oracle (the reference's chain restated) run on
    # that tile's own window, as the reference runs each tile
    from golden_util import max_abs
    from oracle import svf as osvf
    from oracle import window as ow
    key, r0, r1, c0, c1 = TL.tile_windows(150, 130, 64, 10)[4]
    sl = (slice(r0, r1), slice(c0, c1))
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(city.dsm[sl], city.trees[sl], city.dem[sl])
    bundle = osvf.svf_calculator(2, amax, city.dsm[sl], vegdsm, vegdsm2, bush, city.scale)
    want = ow.run_utci_window(a=city.dsm[sl], temp1=city.trees[sl], temp2=city.dem[sl], walls=city.walls[sl],
                              dirwalls=city.aspect[sl], svf_bundle=bundle, met_file=met, location=loc,
                              scale=city.scale, landcover_grid=city.landcover[sl], lc_class=lc,
                              requested_variables=("utci", "tmrt"), **geo)
    assert max_abs(res[key]["tmrt"], want["tmrt"]) <= 1e-3
    assert max_abs(res[key]["utci"], want["utci"]) <= 1e-3
