"""Windowed exact SVF recompute after an edit (the corridor closure of
solweig_core/sparse_work.py:633-781): host-side corridor descriptors and
windows on CPU; the device result against a full sweep on the GPU."""
import numpy as np
import pytest

from solweig_project_b200 import _native as N
from solweig_project_b200 import tables as T

F32 = np.float32


def _patch_steps(plan, steps, q):
    off, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
    return steps["dx"][off:off + n].astype(np.int64), steps["dy"][off:off + n].astype(np.int64)


def _brute(dx, dy, t, rect):
    r0, r1, c0, c1 = rect
    if r0 <= t[0] <= r1 and c0 <= t[1] <= c1:
        return True
    rr, cc = t[0] + dx, t[1] + dy
    return bool(np.any((rr >= r0) & (rr <= r1) & (cc >= c0) & (cc <= c1)))


@pytest.mark.parametrize("rows,cols,scale,amax", [(60, 45, 1.0, 20.0), (37, 80, 0.5, 33.0), (90, 90, 2.0, 12.0)])
def test_corridor_descriptors_have_the_major_minor_form(rows, cols, scale, amax):
    plan, steps, _ = T.svf_plan(rows, cols, scale, F32(amax), False)
    desc = T.svf_corridor(plan, steps, 40.0)
    assert not np.any(desc == N.CORRIDOR_ALWAYS)
    # only the zenith patch (last, altitude band 90) is height-blind
    local = np.flatnonzero(desc == N.CORRIDOR_LOCAL)
    assert list(local) == [int(plan["n_patches"][0]) - 1]


@pytest.mark.parametrize("rows,cols,scale,amax", [(60, 45, 1.0, 20.0), (37, 80, 0.5, 33.0)])
def test_corridor_test_equals_brute_force(rows, cols, scale, amax):
    plan, steps, _ = T.svf_plan(rows, cols, scale, F32(amax), False)
    desc = T.svf_corridor(plan, steps, 40.0)
    rng = np.random.default_rng(11)
    n_p = int(plan["n_patches"][0])
    for _ in range(12):
        r0, c0 = int(rng.integers(0, rows)), int(rng.integers(0, cols))
        rect = (r0, min(rows - 1, r0 + int(rng.integers(0, 8))), c0, min(cols - 1, c0 + int(rng.integers(0, 8))))
        window = T.edit_window(rect, plan, steps, desc, rows, cols)
        for q in range(n_p):
            dx, dy = _patch_steps(plan, steps, q)
            for _ in range(25):
                t = (int(rng.integers(0, rows)), int(rng.integers(0, cols)))
                got = T.in_corridor(int(desc[q]), dx, dy, t, rect)
                want = _brute(dx, dy, t, rect)
                if desc[q] == N.CORRIDOR_LOCAL:
                    assert got == (rect[0] <= t[0] <= rect[1] and rect[2] <= t[1] <= rect[3])
                else:
                    assert got == want, (q, t, rect)
                if want and desc[q] != N.CORRIDOR_LOCAL:
                    assert window[0] <= t[0] <= window[1] and window[2] <= t[1] <= window[3]


def test_window_is_clipped_and_contains_the_rectangle():
    plan, steps, _ = T.svf_plan(200, 150, 1.0, F32(30.0), False)
    desc = T.svf_corridor(plan, steps, 40.0)
    rect = (5, 9, 140, 149)
    w = T.edit_window(rect, plan, steps, desc, 200, 150)
    assert w[0] == 0 and w[3] == 149 and w[1] <= 199 and w[2] >= 0
    assert w[0] <= rect[0] and w[1] >= rect[1] and w[2] <= rect[2] and w[3] >= rect[3]


# ------------------------------------------------------------------- GPU
def _scene(seed, rows, cols):
    from solweig_project_b200 import synthetic
    city = synthetic.make_city(rows, cols, seed=seed, n_buildings=14, n_trees=10)
    return city


def _edits(city, rng):
    rows, cols = city.shape
    dsm, trees, dem = city.dsm.copy(), city.trees.copy(), city.dem.copy()
    out = []
    d = dsm.copy()                                    # add a building
    d[40:52, 60:69] = dem[40:52, 60:69] + F32(25.0)
    out.append(("add building", d, trees.copy(), dem))
    d = dsm.copy()                                    # remove buildings in a box
    box = (slice(10, 60), slice(10, 70))
    d[box] = dem[box]
    out.append(("remove", d, trees.copy(), dem))
    d = dsm.copy()                                    # raise whatever stands in a box
    d[80:110, 30:60] = np.where(d[80:110, 30:60] > dem[80:110, 30:60] + 1, d[80:110, 30:60] + F32(7.5),
                                d[80:110, 30:60])
    out.append(("raise", d, trees.copy(), dem))
    t = trees.copy()                                  # plant a tree
    yy, xx = np.mgrid[0:rows, 0:cols]
    canopy = (F32(9.0) * np.exp(-((yy - 70) ** 2 + (xx - 20) ** 2) / F32(2 * 3.0 ** 2))).astype(F32)
    canopy[canopy < 0.5] = 0
    t = np.maximum(t, canopy).astype(F32)
    out.append(("tree", dsm.copy(), t, dem))
    d = dsm.copy()                                    # edit touching the border
    d[rows - 6:rows, cols - 9:cols] = dem[rows - 6:rows, cols - 9:cols] + F32(18.0)
    out.append(("border", d, trees.copy(), dem))
    return out


@pytest.mark.gpu
def test_windowed_recompute_equals_full_sweep(cuda):
    from golden_util import assert_bits_equal
    from solweig_project_b200.engine import DeviceSite
    city = _scene(21, 130, 150)
    rng = np.random.default_rng(5)
    amax = 48.0
    site = DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale, amaxvalue=amax)
    site.run_svf()
    modes = []
    for name, dsm, trees, dem in _edits(city, rng):
        info = site.edit_svf(dsm, trees, dem)
        modes.append(info["mode"])
        ref = DeviceSite(dsm, trees, dem, city.walls, city.aspect, city.scale, amaxvalue=amax)
        full = ref.run_svf()
        got = site.svf_result
        assert_bits_equal(got.planes.cpu().numpy(), full.planes.cpu().numpy(), f"{name}: planes")
        assert np.array_equal(got.bits.cpu().numpy(), full.bits.cpu().numpy()), f"{name}: bits"
    assert modes == ["window"] * 5
    # an edit that changes nothing
    assert site.edit_svf(dsm, trees, dem)["mode"] == "none"


@pytest.mark.gpu
def test_windowed_recompute_against_the_oracle(cuda):
    """One edit checked against the CPU oracle (the reference's
    svf_calculator restated) run on the edited rasters: the window update's
    planes and patch cubes are bit-exact."""
    from golden_util import assert_bits_equal
    from oracle import svf as osvf
    from solweig_project_b200.engine import DeviceSite
    city = _scene(23, 72, 80)
    amax = F32(48.0)
    site = DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale, amaxvalue=amax)
    site.run_svf()
    dsm = city.dsm.copy()
    dsm[30:41, 35:44] = city.dem[30:41, 35:44] + F32(25.0)
    assert site.edit_svf(dsm, city.trees, city.dem)["mode"] == "window"
    vegdsm, vegdsm2, bush, _ = osvf.scene_from_rasters(dsm, city.trees, city.dem)
    want = osvf.svf_calculator(2, amax, dsm, vegdsm, vegdsm2, bush, city.scale)
    got = site.svf_result
    planes = got.planes.cpu().numpy()
    for k, name in enumerate(osvf.SVF_ORDER[:15]):
        assert_bits_equal(planes[k], want[k], name)
    assert_bits_equal(planes[15], want[18], "svftotal")
    sh, veg, vb = (x.cpu().numpy() for x in got.cubes())
    assert_bits_equal(veg, np.asarray(want[15], F32), "vegshmat")
    assert_bits_equal(vb, np.asarray(want[16], F32), "vbshvegshmat")
    assert_bits_equal(sh, np.asarray(want[17], F32), "shmat")


@pytest.mark.gpu
def test_windowed_recompute_falls_back_to_a_full_sweep(cuda):
    from solweig_project_b200.engine import DeviceSite
    city = _scene(4, 64, 64)
    site = DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale)
    site.run_svf()
    d = city.dsm.copy()
    d[20:30, 20:30] = F32(d.max() + 20.0)   # raises amaxvalue: new step tables
    info = site.edit_svf(d, city.trees, city.dem)
    assert info["mode"] == "full"
    ref = DeviceSite(d, city.trees, city.dem, city.walls, city.aspect, city.scale)
    assert np.array_equal(site.svf_result.planes.cpu().numpy().view(np.uint32),
                          ref.run_svf().planes.cpu().numpy().view(np.uint32))


@pytest.mark.gpu
def test_block_edits_equal_full_sweeps(cuda):
    from solweig_project_b200.engine import DeviceSite
    city = _scene(8, 120, 140)
    site = DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale)
    site.run_svf()
    rng = np.random.default_rng(3)
    dsm, trees = city.dsm.copy(), city.trees.copy()
    for k in range(4):
        r0, c0 = int(rng.integers(0, 100)), int(rng.integers(0, 120))
        h, w = int(rng.integers(3, 20)), int(rng.integers(3, 20))
        blk = dsm[r0:r0 + h, c0:c0 + w].copy()
        blk[:] = F32(rng.uniform(2, 30)) if k % 2 == 0 else city.dem[r0:r0 + h, c0:c0 + w]
        dsm[r0:r0 + h, c0:c0 + w] = blk
        info = site.edit_svf_block(r0, c0, dsm=blk)
        assert info["mode"] in ("window", "full")
        ref = DeviceSite(dsm, trees, city.dem, city.walls, city.aspect, city.scale, amaxvalue=float(site.amax))
        full = ref.run_svf()
        assert np.array_equal(site.svf_result.planes.cpu().numpy().view(np.uint32),
                              full.planes.cpu().numpy().view(np.uint32)), k
        assert np.array_equal(site.svf_result.bits.cpu().numpy(), full.bits.cpu().numpy()), k


@pytest.mark.gpu
def test_box_recompute_is_exact_inside_the_box(cuda):
    from solweig_project_b200.engine import DeviceSite
    city = _scene(12, 100, 110)
    site = DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale, amaxvalue=45.0)
    before = site.run_svf()
    planes0, bits0 = before.planes.clone(), before.bits.clone()
    dsm = city.dsm.copy()
    blk = np.full((14, 9), F32(22.0))
    dsm[40:54, 50:59] = blk
    site.update_rasters_block(40, 50, dsm=blk)
    site.exact_svf_box(40, 50, 14, 9)
    ref = DeviceSite(dsm, city.trees, city.dem, city.walls, city.aspect, city.scale, amaxvalue=45.0).run_svf()
    box = (slice(None), slice(40, 54), slice(50, 59))
    got_p, got_b = site.svf_result.planes.cpu().numpy(), site.svf_result.bits.cpu().numpy()
    assert np.array_equal(got_p[box].view(np.uint32), ref.planes.cpu().numpy()[box].view(np.uint32))
    assert np.array_equal(got_b[(slice(None),) + box], ref.bits.cpu().numpy()[(slice(None),) + box])
    # pixels outside the box keep what they held
    mask = np.ones((100, 110), bool)
    mask[40:54, 50:59] = False
    assert np.array_equal(got_p[:, mask].view(np.uint32), planes0.cpu().numpy()[:, mask].view(np.uint32))
