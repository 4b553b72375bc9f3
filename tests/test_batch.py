"""Batched launches (one launch per stage for many sites): descriptor
layout, tile lists and validation on CPU; results against the single-site
path on the GPU, plain, graph-replayed and autotuned."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import REPO

from solweig_project_b200 import _native as N
from solweig_project_b200 import batch as B
from solweig_project_b200 import build


def test_descriptor_layout_matches_the_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include "solweig_b200.h"\nint main(void){'
                   'printf("%zu %zu\\n", sizeof(sw100_batch_site), sizeof(sw100_tile)); return 0;}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    site, tile = (int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split())
    assert site == ctypes.sizeof(B.BatchSite)
    assert tile == B.TILE_DTYPE.itemsize == 16


@pytest.mark.parametrize("shape", B.SHAPES)
def test_tile_lists_cover_every_pixel_once(shape):
    rng = np.random.default_rng(1)
    dims = [(int(rng.integers(1, 90)), int(rng.integers(1, 140)), int(rng.integers(1, 4))) for _ in range(6)]
    order = [3, 0, 5, 1, 4]          # site 2 left out
    tiles = B.build_tiles(dims, shape, order)
    bx, by = shape
    for i, (rows, cols, n_day) in enumerate(dims):
        cover = np.zeros((n_day, rows, cols), np.int32)
        for t in tiles[tiles["site"] == i]:
            cover[t["day"], t["ty"] * by:(t["ty"] + 1) * by, t["tx"] * bx:(t["tx"] + 1) * bx] += 1
        assert (cover == (0 if i == 2 else 1)).all()
    # launch order follows `order`
    firsts = [int(np.flatnonzero(tiles["site"] == i)[0]) for i in order]
    assert firsts == sorted(firsts)


def test_size_bucket_is_the_pixel_weighted_median():
    assert B.size_bucket([128] * 10 + [1024]) == "side<=1536"
    assert B.size_bucket([128] * 100 + [300]) == "side<=192"
    assert B.size_bucket([500, 500, 200]) == "side<=768"


@pytest.fixture(scope="module")
def lib():
    build.build()
    return N.load()


def test_validate_refuses_bad_descriptors(lib):
    host = (B.BatchSite * 1)()
    rc = lib.sw100_batch_validate(ctypes.cast(host, ctypes.c_void_p), 1)
    assert rc != 0 and b"grid" in lib.sw100_last_error()
    host[0].rows, host[0].cols = 8, 8
    assert lib.sw100_batch_validate(ctypes.cast(host, ctypes.c_void_p), 1) != 0
    assert b"dsm" in lib.sw100_last_error()
    assert lib.sw100_batch_validate(None, 0) == 0


def test_launch_refuses_block_shapes_other_than_128_threads(lib):
    fake = ctypes.c_void_p(256)
    rc = lib.sw100_batch_svf(fake, fake, 4, 32, 8, 4, None)
    assert rc != 0 and b"128 threads" in lib.sw100_last_error()
    assert lib.sw100_batch_svf(None, None, 0, 32, 4, 1, None) == 0   # nothing to do


# ------------------------------------------------------------------- GPU
def _sites(cuda):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    met = synthetic.make_met(7)
    geo = synthetic.load_sun_geometry("single")
    loc = dict(synthetic.DEFAULT_LOCATION)
    lc_class = synthetic.default_lc_class()
    out = []
    for seed, (rows, cols) in ((3, (48, 64)), (4, (70, 55)), (5, (33, 90))):
        c = synthetic.make_city(rows, cols, seed=seed, n_buildings=6, n_trees=6, side_range=(4, 12))
        mk = lambda c=c: DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, landcover=c.landcover,  # noqa
                                    lc_class=lc_class)
        out.append((mk, lambda s: s.build_series(met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"],
                                                 geo["dectime"], geo["altmax"], loc)))
    # a site with bush: ground lowered to -0.25 x canopy under the trees of
    # the left half makes vegdem2 == 0 != vegdem there (the whole-grid bush
    # step flags run)
    c = synthetic.make_city(40, 50, seed=6, n_buildings=4, n_trees=10, side_range=(4, 10))
    dem = c.dem.copy()
    sel = (c.trees > 0) & (np.arange(50)[None, :] < 25)
    dem[sel] = np.float32(-0.25) * c.trees[sel]
    dsm = np.maximum(c.dsm, dem).astype(np.float32)
    mk = lambda: DeviceSite(dsm, c.trees, dem, c.walls, c.aspect, c.scale, landcover=c.landcover,  # noqa
                            lc_class=lc_class)
    out.append((mk, lambda s: s.build_series(met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"],
                                             geo["dectime"], geo["altmax"], loc)))
    return out


REQ = ("utci", "tmrt", "kup", "kdown", "lup", "ldown", "shadow")


@pytest.mark.gpu
def test_batch_equals_single_site_runs(cuda, tmp_path):
    import torch
    specs = _sites(cuda)
    singles = []
    for mk, ser in specs:
        s = mk()
        res = s.run_svf()
        # the batch takes the dense patch sums from the tensor cores, as the
        # single-site run does (the in-loop form: tests/test_tiles.py)
        out = s.run_time_loop(ser(s), requested=REQ, tensor_sums=True)
        singles.append((res.planes.cpu().numpy(), res.bits.cpu().numpy(),
                        {k: v.cpu().numpy() for k, v in out.items()}))
    sites = [mk() for mk, _ in specs]
    series = [ser(s) for s, (_, ser) in zip(sites, specs)]
    assert sites[-1].bush_any
    tuner = B.Autotuner(str(tmp_path / "tune.json"))
    batch = B.SiteBatch(sites, series, requested=REQ, tuner=tuner)

    def check(what):
        torch.cuda.synchronize()
        for i, (planes, bits, outs) in enumerate(singles):
            p, b = batch.svf(i)
            assert np.array_equal(p.cpu().numpy().view(np.uint32), planes.view(np.uint32)), (what, i, "planes")
            assert np.array_equal(b.cpu().numpy(), bits), (what, i, "bits")
            got = batch.outputs(i)
            for k in REQ:
                g, w = got[k].cpu().numpy(), outs[k]
                assert np.array_equal(g.view(np.uint32), w.view(np.uint32)), (what, i, k)

    batch.run()
    check("plain")
    # the first site against the CPU oracle (the reference's chain restated)
    from golden_util import max_abs
    from oracle import svf as osvf
    from oracle import window as ow
    from solweig_project_b200 import synthetic
    c = synthetic.make_city(48, 64, seed=3, n_buildings=6, n_trees=6, side_range=(4, 12))
    geo = synthetic.load_sun_geometry("single")
    vegdsm, vegdsm2, bush, amax = osvf.scene_from_rasters(c.dsm, c.trees, c.dem)
    bundle = osvf.svf_calculator(2, amax, c.dsm, vegdsm, vegdsm2, bush, c.scale)
    p0, _ = batch.svf(0)
    p0 = p0.cpu().numpy()
    for k in range(15):
        assert np.array_equal(p0[k].view(np.uint32), np.asarray(bundle[k], np.float32).view(np.uint32)), k
    want = ow.run_utci_window(a=c.dsm, temp1=c.trees, temp2=c.dem, walls=c.walls, dirwalls=c.aspect,
                              svf_bundle=bundle, met_file=synthetic.make_met(7),
                              location=dict(synthetic.DEFAULT_LOCATION), scale=c.scale, landcover_grid=c.landcover,
                              lc_class=synthetic.default_lc_class(), requested_variables=("utci", "tmrt", "shadow"),
                              **geo)
    got = {k: v.cpu().numpy() for k, v in batch.outputs(0).items()}
    assert np.array_equal(got["shadow"].view(np.uint32), want["shadow"].view(np.uint32))
    assert max_abs(got["tmrt"], want["tmrt"]) <= 1e-3
    assert max_abs(got["utci"], want["utci"]) <= 1e-3
    for p, b in (batch.svf(i) for i in range(len(sites))):
        p.zero_()
    batch.replay()
    batch.replay()
    check("graph")
    chosen = tuner.tune(batch)
    assert set(chosen) == {"pack", "bush", "svf", "sun", "flux"}
    assert os.path.exists(tmp_path / "tune.json")
    batch.run()
    check("tuned")
    again = B.SiteBatch(sites, series, requested=REQ, tuner=B.Autotuner(str(tmp_path / "tune.json")))
    assert again.shapes["svf"] == (tuple(chosen["svf"][0]), chosen["svf"][1])
