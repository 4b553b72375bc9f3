"""Spatial split of one site with a static halo (partition.py): two gloo
ranks each run the CPU oracle (the reference's chain restated) on their
window, rank 0 stitches the cores, and the result equals the oracle on the
whole site bit for bit; on the GPU, the parts run through the CUDA path
equal the whole-site run bit for bit."""
import os
import socket

import numpy as np
import pytest

from solweig_project_b200 import partition as PT
from solweig_project_b200 import synthetic

REQ = ("utci", "tmrt", "shadow", "kup", "lup", "ldown")


def _site(rows=180, cols=36, seed=71, scale=0.5, h_max=6.0):
    city = synthetic.make_city(rows, cols, seed=seed, n_buildings=10, n_trees=8, side_range=(3, 8),
                               tree_peak=(1.0, 2.5), h_max=h_max, scale=scale)
    return city, synthetic.make_met(seed), synthetic.load_sun_geometry("single"), synthetic.default_lc_class()


def test_split_rows_covers_and_clips():
    parts = PT.split_rows(100, 3, 12)
    assert [(p.r0, p.r1) for p in parts] == [(0, 33), (33, 67), (67, 100)]
    assert [(p.w0, p.w1) for p in parts] == [(0, 45), (21, 79), (55, 100)]


def test_halo_is_below_the_site_and_refuses_bush():
    city, met, geo, _ = _site()
    parts, amax, halo = PT.plan(city.dsm, city.trees, city.dem, city.scale, met, geo, 2)
    assert 10 < halo < 75 and len(parts) == 2 and amax == np.float32(max(city.dsm.max(), city.trees.max()))
    dem = city.dem.copy()
    sel = city.trees > 0
    dem[sel] = np.float32(-0.25) * city.trees[sel]
    with pytest.raises(ValueError, match="bush"):
        PT.plan(np.maximum(city.dsm, dem), city.trees, dem, city.scale, met, geo, 2)


def _oracle(city, met, geo, lc, rows, amax):
    from oracle import svf as osvf
    from oracle import window as ow
    sl = slice(*rows)
    dsm, trees, dem = city.dsm[sl], city.trees[sl], city.dem[sl]
    vegdsm, vegdsm2, bush, _ = osvf.scene_from_rasters(dsm, trees, dem)
    bundle = osvf.svf_calculator(2, amax, dsm, vegdsm, vegdsm2, bush, city.scale)
    return ow.run_utci_window(a=dsm, temp1=trees, temp2=dem, walls=city.walls[sl], dirwalls=city.aspect[sl],
                              svf_bundle=bundle, met_file=met, location=dict(synthetic.DEFAULT_LOCATION),
                              scale=city.scale, amaxvalue=amax, landcover_grid=city.landcover[sl], lc_class=lc,
                              requested_variables=REQ, **geo)


def _rank(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        city, met, geo, lc = _site()
        parts, amax, _ = PT.plan(city.dsm, city.trees, city.dem, city.scale, met, geo, world)
        p = parts[rank]
        res = _oracle(city, met, geo, lc, (p.w0, p.w1), amax)
        core = {k: v[:, p.core_in_window] for k, v in res.items()}
        got = [None] * world if rank == 0 else None
        dist.gather_object(core, got, dst=0)
        if rank == 0:
            np.savez(out_path, **PT.stitch(parts, got, city.shape[0]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_stitch_to_the_whole_site(tmp_path):
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "stitched.npz")
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    city, met, geo, lc = _site()
    whole = _oracle(city, met, geo, lc, (0, city.shape[0]), np.float32(max(city.dsm.max(), city.trees.max())))
    with np.load(out) as z:
        for k in REQ:
            assert np.array_equal(z[k].view(np.uint32), whole[k].view(np.uint32)), k


@pytest.mark.gpu
def test_parts_on_the_gpu_equal_the_whole_site(cuda):
    from solweig_project_b200.engine import DeviceSite
    city, met, geo, lc = _site(rows=420, cols=96, seed=72, scale=1.0, h_max=12.0)
    parts, amax, halo = PT.plan(city.dsm, city.trees, city.dem, city.scale, met, geo, 3)
    assert all(p.w1 - p.w0 < city.shape[0] for p in parts)
    loc = dict(synthetic.DEFAULT_LOCATION)
    args = (met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"], geo["dectime"], geo["altmax"], loc)

    def run(rows):
        sl = slice(*rows)
        s = DeviceSite(city.dsm[sl], city.trees[sl], city.dem[sl], city.walls[sl], city.aspect[sl], city.scale,
                       landcover=city.landcover[sl], lc_class=lc, amaxvalue=amax)
        s.run_svf()
        out = s.run_time_loop(s.build_series(*args), requested=REQ)
        return {k: v.cpu().numpy() for k, v in out.items()}

    whole = run((0, city.shape[0]))
    cores = []
    for p in parts:
        r = run((p.w0, p.w1))
        cores.append({k: v[:, p.core_in_window] for k, v in r.items()})
    got = PT.stitch(parts, cores, city.shape[0])
    for k in REQ:
        assert np.array_equal(got[k].view(np.uint32), whole[k].view(np.uint32)), k
