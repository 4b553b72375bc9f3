"""The time loop's dense patch sums on the tensor cores (sw100_patch_sums):
the four sums of every step against a float64 evaluation of the same
increments from the series table and the patch-bit cubes, the time loop
fed by them against the loop that computes them itself, and the bounded
waits' timeout path."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _site(seed=11, rows=70, cols=90):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    c = synthetic.make_city(rows, cols, seed=seed, n_buildings=10, n_trees=12, side_range=(4, 14))
    s = DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, landcover=c.landcover,
                   lc_class=synthetic.default_lc_class())
    s.run_svf()
    geo = synthetic.load_sun_geometry("single")
    ser = s.build_series(synthetic.make_met(seed), geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"],
                         geo["dectime"], geo["altmax"], dict(synthetic.DEFAULT_LOCATION))
    return s, ser


def test_sums_match_a_float64_evaluation(cuda):
    import torch
    site, ser = _site()
    s, dev = site.upload_series(ser)
    sums = site.launch_patch_sums(s).cpu().numpy().astype(np.float64)      # (n_t, 4, rows, cols)
    torch.cuda.synchronize()
    site.check_tensor_error()
    bits = site.svf_result.bits.cpu().numpy().view(np.uint32)            # (3, 5, rows, cols)
    P = ser.patch.shape[1]
    q = np.arange(P)
    sh = (bits[0][q // 32] >> (q % 32)[:, None, None]) & 1               # (P, rows, cols)
    veg = (bits[1][q // 32] >> (q % 32)[:, None, None]) & 1
    code = (sh * 2 + veg).astype(np.int64)
    qi = q[:, None, None]
    for t in range(len(ser.steps)):
        pt = ser.patch[t]
        day = bool(ser.steps[t]["is_day"])
        kd = pt["kside_d"].astype(np.float64)[qi, code].sum(axis=0) if day else 0.0
        al = pt["anilum"].astype(np.float64)[qi, code].sum(axis=0) if day else 0.0
        sky = code == 3
        ld = (pt["ld_sky"].astype(np.float64)[:, None, None] * sky).sum(axis=0)
        ls = (pt["ls_sky"].astype(np.float64)[:, None, None] * sky).sum(axis=0)
        for j, want in enumerate((kd, al, ld, ls)):
            want = np.broadcast_to(want, sums.shape[2:])
            scale = max(1.0, float(np.abs(want).max()))
            assert np.abs(sums[t, j] - want).max() <= 2e-6 * scale, (t, j)


def test_loop_with_tensor_sums_matches_the_loop_alone(cuda):
    from golden_util import max_abs
    req = ("utci", "tmrt", "kdown", "ldown", "shadow", "lup")
    a, ser = _site(seed=12)
    b, _ = _site(seed=12)
    ta = {k: v.cpu().numpy() for k, v in a.run_time_loop(ser, requested=req, tensor_sums=True).items()}
    tb = {k: v.cpu().numpy() for k, v in b.run_time_loop(ser, requested=req, tensor_sums=False).items()}
    a.check_tensor_error()
    # the loop alone sums in patch order in float32 (the reference's order);
    # the tensor-core sums are nearer the exact sums (previous test): the two
    # differ by that float32 rounding, well inside the parity bars
    assert np.array_equal(ta["shadow"].view(np.uint32), tb["shadow"].view(np.uint32))
    assert max_abs(ta["tmrt"], tb["tmrt"]) <= 1e-3
    assert max_abs(ta["utci"], tb["utci"]) <= 1e-3
    for k in ("kdown", "ldown"):
        assert max_abs(ta[k], tb[k]) <= 1e-5 * max(1.0, float(np.abs(tb[k]).max())), k


def test_wait_timeout_is_reported(cuda):
    import torch
    from solweig_project_b200 import _native as N
    lib = N.load()
    site, ser = _site(seed=13, rows=40, cols=40)
    s, dev = site.upload_series(ser)
    prev = lib.sw100_set_wait_limit(0)
    try:
        site.launch_patch_sums(s)
        torch.cuda.synchronize()
    finally:
        lib.sw100_set_wait_limit(-1)
    assert prev == 1 << 22
    with pytest.raises(N.NativeError, match="bounded wait"):
        site.check_tensor_error()
    sums = site.launch_patch_sums(s)
    torch.cuda.synchronize()
    site.check_tensor_error()                      # the context is usable and the flag clear
    assert np.isfinite(sums.cpu().numpy()).all()
