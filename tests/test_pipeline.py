"""The chunked time loop (host tables of later steps built while the GPU
runs earlier ones) equals one launch over all steps bit for bit: every
output, the thermal state after the last step and the carried scalars."""
import numpy as np
import pytest

REQ = ("utci", "tmrt", "kup", "kdown", "lup", "ldown", "shadow")


def _site():
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    c = synthetic.make_city(72, 60, seed=41, n_buildings=8, n_trees=12)
    return c, DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, landcover=c.landcover,
                         lc_class=synthetic.default_lc_class())


def test_chunk_bounds():
    from solweig_project_b200.engine import chunk_bounds
    assert chunk_bounds(0, 24, 8) == [(0, 8), (8, 16), (16, 24)]
    assert chunk_bounds(3, 20, 5) == [(3, 8), (8, 13), (13, 18), (18, 20)]
    assert chunk_bounds(0, 24, (12, 8, 4)) == [(0, 12), (12, 20), (20, 24)]
    assert chunk_bounds(0, 30, (12, 8, 4)) == [(0, 12), (12, 20), (20, 24), (24, 28), (28, 30)]
    assert chunk_bounds(0, 10, (12, 8)) == [(0, 10)]
    assert chunk_bounds(5, 5, 8) == []
    for bad in (0, (4, 0), ()):
        with pytest.raises(ValueError):
            chunk_bounds(0, 24, bad)


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [1, 5, 24, (12, 8, 4), (3, 9)])
def test_chunked_time_loop_equals_single_launch(cuda, chunk):
    import torch
    from solweig_project_b200 import synthetic
    geo = synthetic.load_sun_geometry("single")
    met = synthetic.make_met(11)
    loc = dict(synthetic.DEFAULT_LOCATION)
    args = (met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"], geo["dectime"], geo["altmax"], loc)

    _, a = _site()
    a.run_svf()
    ser = a.build_series(*args)
    ref = {k: v.cpu().numpy() for k, v in a.run_time_loop(ser, requested=REQ).items()}
    ref_state = a.state.cpu().numpy()

    _, b = _site()
    b.run_svf()
    got, final = b.run_chain_chunked(*args, requested=REQ, chunk_steps=chunk)
    torch.cuda.synchronize()
    for k in REQ:
        assert np.array_equal(got[k].view(np.uint32), ref[k].view(np.uint32)), (chunk, k)
    assert np.array_equal(b.state.cpu().numpy().view(np.uint32), ref_state.view(np.uint32))
    assert final == ser.final


@pytest.mark.gpu
def test_chunked_time_loop_device_memory_does_not_grow_with_steps(cuda):
    """Three days of forcing hold no more device memory than one: only a
    bounded ring of chunks keeps its device buffers."""
    import torch
    from solweig_project_b200 import synthetic
    geo = synthetic.load_sun_geometry("single")
    met1 = synthetic.make_met(11)
    loc = dict(synthetic.DEFAULT_LOCATION)

    def days(n):
        met = np.concatenate([met1] * n)
        met[:, 1] = np.repeat(met1[0, 1] + np.arange(n), 24)
        g = {k: np.concatenate([geo[k] + (d if k in ("dectime", "jday") else 0) for d in range(n)], axis=-1)
             for k in geo}
        return (met, g["altitude"], g["azimuth"], g["zen"], g["jday"], g["dectime"], g["altmax"], loc)

    peaks = []
    for n in (1, 3):
        _, s = _site()
        s.run_svf()
        torch.cuda.synchronize()
        base = torch.cuda.memory_allocated()
        torch.cuda.reset_peak_memory_stats()
        out, _ = s.run_chain_chunked(*days(n), requested=("utci", "tmrt"), chunk_steps=4)
        assert out["tmrt"].shape[0] == 24 * n and np.isfinite(out["tmrt"]).all()
        peaks.append(torch.cuda.max_memory_allocated() - base)
        del s
    assert peaks[1] <= peaks[0] * 1.05 + (1 << 20), peaks
