"""Learned SVF preview on the GPU: training by the library's own kernels
reduces the loss, the shipped weights beat keeping the stale SVF on seeded
edits, and a net whose error check fails falls back to the exact windowed
recompute."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_training_reduces_the_loss(cuda):
    from solweig_project_b200 import preview as PV
    data = PV.training_sites(2, 128, seed=5)
    net = PV.UNet(seed=1)
    rep = PV.train(net, [s for s, _ in data], [p for _, p in data], steps=120, batch=4, size=64, margin=16,
                   lr=2e-3)
    assert rep.loss_last < 0.35 * rep.loss_first, rep


def _site(seed, side):
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    c = synthetic.make_city(side, side, seed=seed, density=0.3, canopy_cover=0.15)
    s = DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale, landcover=c.landcover,
                   lc_class=synthetic.default_lc_class(), amaxvalue=48.0)
    s.run_svf()
    met = synthetic.make_met(1234)
    geo = synthetic.load_sun_geometry("single")
    ser = s.build_series(met, geo["altitude"], geo["azimuth"], geo["zen"], geo["jday"], geo["dectime"],
                         geo["altmax"], dict(synthetic.DEFAULT_LOCATION))
    return s, ser


def test_trained_preview_beats_the_stale_svf(cuda):
    """What the network gains: over the edited window, SVF and Tmrt come
    closer to the exact chain than leaving the SVF as it was."""
    from solweig_project_b200 import preview as PV
    net = PV.load_pretrained()
    site, ser = _site(9090, 512)
    rows = PV.evaluate_edits(net, site, ser, n_edits=12, seed=3)
    mean = lambda k: float(np.mean([r[k] for r in rows]))  # noqa: E731
    assert all(r["mode"] == "preview" for r in rows)
    assert mean("svf_mae_preview") < 0.8 * mean("svf_mae_stale")
    assert mean("tmrt_rmse_preview") < 0.8 * mean("tmrt_rmse_stale")
    assert mean("tmrt_rmse_preview") <= 0.5


def test_failed_error_check_falls_back_to_the_exact_recompute(cuda):
    from solweig_project_b200 import preview as PV
    from solweig_project_b200.engine import DeviceSite
    site, _ = _site(77, 320)
    prev = PV.SvfPreview(PV.UNet(seed=2), threshold=1e-6)     # untrained: always above the threshold
    blk = np.full((20, 16), np.float32(25.0))
    info = prev.edit(site, 150, 140, dsm=blk)
    assert info["mode"] == "exact"
    ref = DeviceSite(site.host["dsm"], site.host["trees"], site.host["dem"], site.host["dsm"] * 0,
                     site.host["dsm"] * 0, 1.0, amaxvalue=48.0).run_svf()
    assert np.array_equal(site.svf_result.planes.cpu().numpy().view(np.uint32),
                          ref.planes.cpu().numpy().view(np.uint32))
