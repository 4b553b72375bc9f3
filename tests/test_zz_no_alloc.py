"""The allocation-free SVF sweep (sw100_svf_sweep_noalloc) against the
workspace entry point (sw100_svf_sweep), both called through the C ABI.

sw100_svf_sweep_noalloc exists for callers that cannot allocate device
memory themselves (a host framework that owns all device allocations, or a
latency-bound loop that cannot afford cudaMalloc / cudaFree): its scratch is
a static device array inside the library.  Its results must be the same as
the workspace entry point's, bit for bit (the SVF tolerance of the parity
tests), on every call -- the array keeps the previous call's contents, so
two calls in a row are compared.  This file is collected last so that a run
stopping at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _site(seed, side, dem_level=0.0):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    city = synthetic.make_city(side, side, seed=seed, n_buildings=max(2, side // 12), n_trees=max(2, side // 12),
                               side_range=(3, max(4, side // 6)), dem_level=dem_level)
    return DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale,
                      landcover=city.landcover, lc_class=synthetic.default_lc_class())


def _sweep_pair(site):
    from solweig_project_b200 import _native as N
    from solweig_project_b200.engine import _ptr, _stream
    plan_d, steps_d, n_steps, _, ws = site.svf_tables(2)
    rows, cols = site.rows, site.cols

    def buffers():
        return (torch.full((N.SVF_PLANES, rows, cols), float("nan"), device="cuda"),
                torch.full((3, N.CUBE_WORDS, rows, cols), -1, dtype=torch.int32, device="cuda"))

    planes_ref, bits_ref = buffers()
    s = site.site_struct()
    N.call("sw100_svf_sweep", C.byref(s), rows, cols, _ptr(plan_d), _ptr(steps_d), n_steps, _ptr(planes_ref),
           _ptr(bits_ref), _ptr(ws), ws.numel(), _stream())
    results = []
    for _ in range(2):
        planes, bits = buffers()
        N.call("sw100_svf_sweep_noalloc", C.byref(s), rows, cols, _ptr(plan_d), _ptr(steps_d), n_steps,
               _ptr(planes), _ptr(bits), _stream())
        results.append((planes, bits))
    torch.cuda.synchronize()
    return (planes_ref.cpu().numpy(), bits_ref.cpu().numpy()), [(p.cpu().numpy(), b.cpu().numpy())
                                                                for p, b in results]


@pytest.mark.parametrize("seed,side,dem_level", [(21, 64, 0.0), (22, 48, 2.0)])
def test_noalloc_sweep_matches_workspace_sweep(cuda, seed, side, dem_level):
    site = _site(seed, side, dem_level)
    (want_p, want_b), got = _sweep_pair(site)
    for planes, bits in got:
        assert np.array_equal(planes.view(np.uint32), want_p.view(np.uint32))
        assert np.array_equal(bits, want_b)


def test_noalloc_sweep_with_bush_after_other_grids(cuda):
    """A grid with bush (its step flags live in the shared array and are
    cleared on every call) swept between calls on a larger grid without bush:
    every call equals the workspace sweep of its own grid."""
    from conftest import load_golden
    from solweig_project_b200.engine import DeviceSite
    d = load_golden("bush24")
    bush = DeviceSite(d["dsm"], d["trees"], d["dem"], d["walls_ref"], d["aspect_ref"], float(d["scale"]),
                      landcover=d["landcover"], lc_class=d["lc_class"], amaxvalue=d["amaxvalue"])
    assert bush.bush_any
    other = _site(24, 80)
    for site in (bush, other, bush):
        (want_p, want_b), got = _sweep_pair(site)
        for planes, bits in got:
            assert np.array_equal(planes.view(np.uint32), want_p.view(np.uint32))
            assert np.array_equal(bits, want_b)


def test_noalloc_sweep_refuses_grids_beyond_its_scratch(cuda):
    from solweig_project_b200 import _native as N
    lib = N.load()
    site = _site(23, 32)
    plan_d, steps_d, n_steps, _, _ = site.svf_tables(2)
    s = site.site_struct()
    before = lib.sw100_launch_count()
    rc = lib.sw100_svf_sweep_noalloc(C.byref(s), 1100, 1100, C.c_void_p(plan_d.data_ptr()),
                                     C.c_void_p(steps_d.data_ptr()), n_steps, C.c_void_p(1), C.c_void_p(1), None)
    assert rc == 1002  # SW100_E_SIZE
    assert b"allocation-free" in lib.sw100_last_error()
    assert lib.sw100_launch_count() == before
