"""Early exits of the SVF sweep and the sun march.

Host side: the SW100_STEP_SKIP8 flags certify, per step, that the next 8
steps move at most one cell per axis each and that dz does not decrease
(checked against a direct restatement on random and real tables).  Device
side, on a city with tall buildings, one with NaN sources and one with
negative heights: a sweep with the flags cleared (every step marched)
equals the sweep with the 8-step shortcut bit for bit, and the sun march
(which stops at settled building shadow and when nothing can reach the
pixel any more) equals the oracle's full march bit for bit.
"""
import numpy as np
import pytest

from solweig_project_b200 import _native as N
from solweig_project_b200 import tables as T


def _flags_direct(dx, dy, dz):
    n = len(dz)
    out = np.zeros(n, np.int32)
    for k in range(1, n):
        ok = True
        for j in range(k, min(k + 8, n)):
            if not (dz[j] >= dz[j - 1]):
                ok = False
            if j > k and (abs(int(dx[j]) - int(dx[j - 1])) > 1 or abs(int(dy[j]) - int(dy[j - 1])) > 1):
                ok = False
        out[k] = N.STEP_SKIP8 if ok else 0
    return out


def test_skip_flags_match_direct_definition():
    rng = np.random.default_rng(5)
    for trial in range(200):
        n = int(rng.integers(0, 40))
        dx = np.cumsum(rng.choice([-1, 0, 1, 2], n, p=[0.2, 0.4, 0.35, 0.05])).astype(np.int32)
        dy = np.cumsum(rng.choice([-2, -1, 0, 1], n, p=[0.05, 0.35, 0.4, 0.2])).astype(np.int32)
        dz = np.cumsum(rng.choice([-0.5, 0.0, 1.0, 2.0], n, p=[0.05, 0.1, 0.6, 0.25])).astype(np.float32)
        if n > 3 and trial % 7 == 0:
            dz[n // 2] = np.nan
        np.testing.assert_array_equal(T.step_skip_flags(dx, dy, dz), _flags_direct(dx, dy, dz))


def test_real_tables_are_mostly_skippable():
    plan, steps, _ = T.svf_plan(300, 300, 1.0, 60.0, False, 2)
    for q in range(0, 153, 17):
        o, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
        t = steps[o:o + n]
        np.testing.assert_array_equal(t["flags"], _flags_direct(t["dx"], t["dy"], t["dz"]))
    assert (steps["flags"] != 0).mean() > 0.9
    for az, alt in ((95.0, 20.0), (180.0, 60.0), (272.5, 8.0), (45.0, 35.0)):
        dx, dy, dz, _ = T.sun_table(az, alt, 1.0, 60.0, 300, 300)
        f = T.step_skip_flags(dx, dy, dz)
        np.testing.assert_array_equal(f, _flags_direct(dx, dy, dz))
        assert f[0] == 0 and (len(f) < 2 or f[1:].mean() > 0.9)


# ------------------------------------------------------------------- GPU
def _city(kind):
    from solweig_project_b200 import synthetic
    c = synthetic.make_city(160, 144, seed=31, h_max=90.0, n_buildings=30, n_trees=40)
    dsm, trees, dem = c.dsm.copy(), c.trees.copy(), c.dem.copy()
    if kind == "nan":
        dsm[40:43, 50:52] = np.nan
        trees[100, 20] = np.nan
    elif kind == "negative":
        dem = dem - np.float32(3.0)
        dsm = dsm - np.float32(3.0)
    return c, dsm, trees, dem


def _clear_flags(table_dev):
    """Zero the flags word of every step of an uploaded step table."""
    import torch
    table_dev.view(torch.int32).view(-1, 4)[:, 3] = 0


def _site(kind):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    c, dsm, trees, dem = _city(kind)
    # a fixed amaxvalue: with NaN sources the derived one is NaN and no
    # march runs at all
    return c, DeviceSite(dsm, trees, dem, c.walls, c.aspect, c.scale, landcover=c.landcover,
                         lc_class=synthetic.default_lc_class(), amaxvalue=90.0)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["plain", "nan", "negative"])
def test_svf_shortcut_is_exact(cuda, kind):
    import torch

    def run(clear):
        _, s = _site(kind)
        if clear:
            _clear_flags(s.svf_tables()[1])
        res = s.run_svf()
        torch.cuda.synchronize()
        return res.planes.cpu().numpy().view(np.uint32), res.bits.cpu().numpy()

    fast, slow = run(False), run(True)
    for name, a, b in zip(("planes", "bits"), fast, slow):
        assert np.array_equal(a, b), (kind, name, int((a != b).sum()))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["plain", "nan", "negative"])
def test_sun_march_exits_are_exact(cuda, kind):
    import torch
    from oracle import march as om
    from solweig_project_b200 import synthetic
    c, s = _site(kind)
    s.run_svf()
    geo = synthetic.load_sun_geometry("single")
    ser = s.build_series(synthetic.make_met(7), geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"],
                         geo["dectime"], geo["altmax"], dict(synthetic.DEFAULT_LOCATION))
    _, dbg = s.run_sun_march(ser)
    dbg = dbg.cpu().numpy()
    assert dbg.shape[0] >= 4
    h = s.host
    vegdsm, vegdsm2 = (s.t[k].cpu().numpy() for k in ("vegdsm", "vegdsm2"))
    bush = s.t["bush"].cpu().numpy() if s.t["bush"] is not None else np.zeros_like(vegdsm)
    asp = om.aspect_radians(c.aspect)
    names = ("vegsh", "sh", "vbshvegsh", "wallsh", "wallsun", "wallshve", "facesh", "facesun")
    for d in range(0, dbg.shape[0], 3):
        i = int(ser.sun["t"][d])
        az = torch.tensor(geo["azimuth"][0][i]).item()
        alt = torch.tensor(geo["altitude"][0][i]).item()
        want = om.wallheight_23(h["dsm"], vegdsm, vegdsm2, az, alt, float(c.scale), 90.0, bush, c.walls, asp)
        for k, name in enumerate(names):
            got, ref = dbg[d, k], np.asarray(want[k], np.float32)
            # bit-equal, NaN payloads aside (the GPU's NaN is canonical, the
            # host's keeps the operand's payload)
            same = (got.view(np.uint32) == ref.view(np.uint32)) | (np.isnan(got) & np.isnan(ref))
            assert same.all(), (kind, d, name, int((~same).sum()))


@pytest.mark.parametrize("rows,cols,scale,amax", [(36, 36, 1.0, 12.5), (24, 40, 0.5, 9.0), (1, 16, 1.0, 3.0),
                                                   (300, 120, 2.0, 88.6), (64, 64, 1.0, 0.0), (64, 64, 1.0, -1.0),
                                                   (50, 50, 1.0, float("nan"))])
def test_plan_equals_per_patch_tables(rows, cols, scale, amax):
    """svf_plan builds every patch's steps at once; each patch's rows equal
    svf_patch_table's, and its flags the direct definition."""
    plan, steps, single = T.svf_plan(rows, cols, scale, np.float32(amax), False, 2)
    _, altint, _, nband = T.PATCH_LAYOUT[2]
    azs = T.sweep_azimuths(2)
    ring = np.repeat(np.arange(len(altint)), nband)
    for q in range(153):
        dx, dy, dz = T.svf_patch_table(azs[q], altint[ring[q]], scale, np.float32(amax), rows, cols)
        o, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
        assert n == len(dz)
        t = steps[o:o + n]
        assert np.array_equal(t["dx"], dx) and np.array_equal(t["dy"], dy)
        assert np.array_equal(t["dz"].view(np.uint32), dz.view(np.uint32))
        assert np.array_equal(t["flags"], _flags_direct(dx, dy, dz))
        assert bool((int(single[q >> 5]) >> (q & 31)) & 1) == (n <= 1)


def _monotone(d):
    """Shifts along one axis keep one sign and never shrink in magnitude."""
    d = np.asarray(d, np.int64)
    return bool(((d >= 0).all() or (d <= 0).all()) and (np.diff(np.abs(d)) >= 0).all())


@pytest.mark.parametrize("rows,cols,scale,amax", [(300, 300, 1.0, 60.0), (24, 40, 0.5, 9.0), (500, 80, 2.0, 120.0)])
def test_tables_grow_monotonically(rows, cols, scale, amax):
    """Both marches skip per-step bounds tests when a table's last cell is in
    the grid; that is exact only if every intermediate cell lies between the
    pixel and the last cell, i.e. each axis' shifts keep one sign and grow."""
    plan, steps, _ = T.svf_plan(rows, cols, scale, np.float32(amax), False, 2)
    for q in range(153):
        o, n = int(plan["step_offset"][0, q]), int(plan["step_count"][0, q])
        assert _monotone(steps["dx"][o:o + n]) and _monotone(steps["dy"][o:o + n]), q
    rng = np.random.default_rng(11)
    az = rng.uniform(0, 360, 300).tolist() + [0.0, 45.0, 90.0, 135.0, 180.0, 225.0, 270.0, 315.0, 359.999]
    alt = rng.uniform(0.3, 89.5, len(az)).tolist()
    for k, v in enumerate(T.sun_tables(az, alt, scale, np.float32(amax), rows, cols)):
        assert _monotone(v[0]) and _monotone(v[1]), (az[k], alt[k])


def _numpy_tables(consts, first_index, amax, rows, cols):
    """The step tables by the numpy one-step form (_march_steps, _executed,
    step_skip_flags) for each march record."""
    idx = np.arange(first_index, max(rows, cols) + 3)
    out = []
    with np.errstate(all="ignore"):
        for c in consts:
            dx, dy, dz = T._march_steps(bool(c["branch_y"]), c["ssin"], c["scos"], c["tan_a"], c["ds"],
                                        c["tanalt"], idx)
            n = T._executed(dx, dy, dz, amax, rows, cols)
            t = np.zeros(n, N.STEP_DTYPE)
            t["dx"], t["dy"], t["dz"] = dx[:n].astype(np.int32), dy[:n].astype(np.int32), dz[:n]
            t["flags"] = T.step_skip_flags(t["dx"], t["dy"], t["dz"])
            out.append(t)
    return out


@pytest.mark.parametrize("amax", [40.0, 0.0, -1.0, float("nan"), float("inf"), 3.0e38])
@pytest.mark.parametrize("first_index,rows,cols", [(1, 300, 120), (0, 37, 64), (0, 1, 1), (1, 2, 700)])
def test_native_march_tables_equal_numpy_form(amax, first_index, rows, cols):
    """sw100_march_tables (host C, one float32 rounding per operation) gives
    the numpy form's steps bit for bit, counts and flags included, over
    random directions and the edge values of the constants."""
    rng = np.random.default_rng(17)
    n = 64
    consts = np.zeros(n, N.MARCH_CONST_DTYPE)
    consts["branch_y"] = rng.integers(0, 2, n)
    consts["ssin"] = rng.choice([-1.0, 0.0, 1.0], n)
    consts["scos"] = rng.choice([-1.0, 0.0, 1.0], n)
    consts["tan_a"] = rng.uniform(-3, 3, n).astype(np.float32)
    consts["ds"] = rng.uniform(1, 1.42, n).astype(np.float32)
    consts["tanalt"] = np.float32(10.0) ** rng.uniform(-2, 2, n).astype(np.float32)
    consts["tan_a"][:6] = [0.0, -0.0, 1e-30, np.nan, np.inf, -2.3e7]
    consts["tanalt"][6:12] = [0.0, -2.3e7, np.nan, np.inf, 1e-30, -1.0]
    consts["ds"][12] = np.nan
    want = _numpy_tables(consts, first_index, np.float32(amax), rows, cols)
    steps, counts = N.march_tables(consts, first_index, np.float32(amax), rows, cols)
    assert list(counts) == [len(t) for t in want]
    ref = np.concatenate(want) if want else np.zeros(0, N.STEP_DTYPE)
    assert steps.tobytes() == ref.tobytes()


@pytest.mark.parametrize("amax", [40.0, 3.0])
def test_native_march_tables_exact_capacity_equals_full_capacity(amax):
    """A buffer of exactly the total step count (the count-then-fill path)
    and one with room for every march at full length (the one-pass path)
    give the same table and counts."""
    import ctypes
    rng = np.random.default_rng(5)
    consts = np.zeros(40, N.MARCH_CONST_DTYPE)
    consts["branch_y"] = rng.integers(0, 2, 40)
    consts["ssin"] = rng.choice([-1.0, 1.0], 40)
    consts["scos"] = rng.choice([-1.0, 1.0], 40)
    consts["tan_a"] = rng.uniform(-3, 3, 40).astype(np.float32)
    consts["ds"] = np.float32(1.0)
    consts["tanalt"] = np.float32(10.0) ** rng.uniform(-1, 1, 40).astype(np.float32)
    full, counts = N.march_tables(consts, 1, np.float32(amax), 90, 70)
    lib = N.load()
    exact = np.zeros(len(full), N.STEP_DTYPE)
    c2 = np.zeros(40, np.int32)
    total = ctypes.c_int64(0)
    rc = lib.sw100_march_tables(consts.ctypes.data, 40, 1, ctypes.c_float(amax), 90, 70, exact.ctypes.data,
                                len(exact), c2.ctypes.data, ctypes.byref(total))
    assert rc == 0 and total.value == len(full) < 40 * (90 + 2)
    assert exact.tobytes() == full.tobytes() and list(c2) == list(counts)


def test_native_march_tables_refuse_small_capacity():
    import ctypes
    consts = np.zeros(2, N.MARCH_CONST_DTYPE)
    consts["ds"], consts["tanalt"], consts["scos"] = 1.0, 0.1, 1.0
    steps, counts = N.march_tables(consts, 1, np.float32(5.0), 50, 50)
    assert len(steps) == counts.sum() > 2
    lib = N.load()
    small = np.zeros(2, N.STEP_DTYPE)
    total = ctypes.c_int64(0)
    rc = lib.sw100_march_tables(consts.ctypes.data, 2, 1, ctypes.c_float(5.0), 50, 50, small.ctypes.data, 2,
                                counts.astype(np.int32).ctypes.data, ctypes.byref(total))
    assert rc == 1003 and total.value == counts.sum()  # SW100_E_WORKSPACE
