"""The time / flux loops' patch order (sw100_site_planes.patch_order): the
per-patch ground-view walk work of sw100_walk_work against a numpy
restatement of its definition, the order built from it, and the loops'
results with the order equal to those without it, bit for bit."""
import ctypes as C

import numpy as np
import pytest

REQ = ("utci", "tmrt", "kup", "kdown", "lup", "ldown", "shadow")


def _site(rows=72, cols=61, seed=43):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    c = synthetic.make_city(rows, cols, seed=seed, n_buildings=9, n_trees=10)
    return c, DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, landcover=c.landcover,
                         lc_class=synthetic.default_lc_class())


def walk_work_numpy(buildings, gvf, second):
    """Per 8 x 4 patch: sum over the 18 azimuths of the longest walk of its
    pixels to the first in-grid building sample (buildings == 0), at most
    `second` steps, 0 for a building pixel or a pixel outside the grid."""
    rows, cols = buildings.shape
    pr, pc = -(-rows // 4), -(-cols // 8)
    n0 = np.zeros((18, pr * 4, pc * 8), np.int64)
    rr, cc = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    for az in range(18):
        res = np.full((rows, cols), second, np.int64)
        done = np.zeros((rows, cols), bool)
        for n in range(second):
            sr, sc = rr + int(gvf["dx"][az, n]), cc + int(gvf["dy"][az, n])
            ok = (sr >= 0) & (sr < rows) & (sc >= 0) & (sc < cols)
            hit = ok & ~done & (buildings[np.clip(sr, 0, rows - 1), np.clip(sc, 0, cols - 1)] == 0)
            res[hit] = n
            done |= hit
        res[buildings == 0] = 0
        n0[az, :rows, :cols] = res
    return n0.reshape(18, pr, 4, pc, 8).max(axis=(2, 4)).sum(0).reshape(-1)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(72, 61), (33, 17), (4, 8)])
def test_walk_work_matches_definition(cuda, shape):
    import torch
    from solweig_project_b200 import engine as E, tables as T, timeseries as TS
    _, site = _site(*shape)
    second = int(TS.walk_steps(site.params, site.scale)[1])
    order = site.walk_order()
    _, work, _ = site._cache["walk_order"]
    torch.cuda.synchronize()
    bld = site.t["buildings"].cpu().numpy().reshape(shape)
    want = walk_work_numpy(bld, T.gvf_table(second), second)
    got = work.cpu().numpy()
    assert np.array_equal(got, want)
    o = order.cpu().numpy()
    assert np.array_equal(np.sort(o), np.arange(len(want)))             # a permutation of the patches
    level = got // max(1, (18 * second) // E.WALK_LEVELS)
    assert np.all(np.diff(level[o]) <= 0)                                # heaviest level first
    ties = [o[level[o] == v] for v in np.unique(level)]
    assert all(np.all(np.diff(t) > 0) for t in ties)                     # grid order within a level


@pytest.mark.gpu
@pytest.mark.parametrize("tensor_sums", [True, False])
def test_loops_with_patch_order_equal_grid_order(cuda, monkeypatch, tensor_sums):
    from solweig_project_b200 import engine as E, synthetic
    geo = synthetic.load_sun_geometry("single")
    met = synthetic.make_met(12)
    args = (met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"], geo["dectime"], geo["altmax"],
            dict(synthetic.DEFAULT_LOCATION))
    outs, states = [], []
    for ordered in (False, True):
        monkeypatch.setattr(E, "WALK_ORDER", ordered)
        _, s = _site()
        s.run_svf()
        ser = s.build_series(*args)
        got = s.run_time_loop(ser, requested=REQ, tensor_sums=tensor_sums)
        outs.append({k: v.cpu().numpy() for k, v in got.items()})
        states.append(s.state.cpu().numpy())
        assert ("walk_order" in s._cache) == ordered
    for k in REQ:
        assert np.array_equal(outs[0][k].view(np.uint32), outs[1][k].view(np.uint32)), k
    assert np.array_equal(states[0].view(np.uint32), states[1].view(np.uint32))


@pytest.mark.gpu
def test_patch_order_count_is_checked(cuda):
    import torch
    from solweig_project_b200 import _native as N, synthetic
    _, s = _site()
    s.run_svf()
    geo = synthetic.load_sun_geometry("single")
    ser = s.build_series(synthetic.make_met(12), geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"],
                         geo["dectime"], geo["altmax"], dict(synthetic.DEFAULT_LOCATION))
    sd, keep = s.upload_series(ser)
    site = s.loop_site_struct()
    site.n_patch_order -= 1
    out = torch.empty((1, len(ser.steps), s.rows, s.cols), dtype=torch.float32, device="cuda")
    gsrc = torch.zeros((max(1, sd.n_day), s.rows, s.cols, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(N.NativeError, match="n_patch_order"):
        N.call("sw100_flux_loop", C.byref(site), s.rows, s.cols, C.byref(sd), gsrc.data_ptr(), s.state.data_ptr(),
               N.OUT_BITS["tmrt"], out.data_ptr(), torch.cuda.current_stream().cuda_stream)


@pytest.mark.gpu
def test_large_sites_keep_grid_order(cuda, monkeypatch):
    """Above WALK_ORDER_MAX_PIXELS the loops run in grid order (the sorted
    blocks would gather from all over a grid whose records miss L2)."""
    from solweig_project_b200 import engine as E
    _, s = _site()
    monkeypatch.setattr(E, "WALK_ORDER_MAX_PIXELS", s.rows * s.cols - 1)
    site = s.loop_site_struct()
    assert not site.patch_order and site.n_patch_order == 0
    monkeypatch.setattr(E, "WALK_ORDER_MAX_PIXELS", s.rows * s.cols)
    site = s.loop_site_struct()
    assert site.patch_order and site.n_patch_order == ((s.rows + 3) // 4) * ((s.cols + 7) // 8)
