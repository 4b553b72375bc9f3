"""The counting SVF sweep (sw100_svf_sweep_count, used by bench.py for the
sweep's algorithmic bytes; one block per 8 x 16 tile) returns the plain,
persistent sweep's planes and bits bit for bit, and counts no more source
gathers than the step tables hold."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["city36", "bush24", "large"])
def test_counting_sweep_matches_and_bounds(case, cuda):
    import torch
    from solweig_project_b200 import _native as N
    from solweig_project_b200 import synthetic
    from solweig_project_b200.engine import DeviceSite
    if case == "large":
        c = synthetic.make_city(160, 144, seed=5, h_max=60.0)
        site = DeviceSite(c.dsm, c.trees, c.dem, c.walls, c.aspect, c.scale)
    else:
        d = load_golden(case)
        site = DeviceSite(d["dsm"], d["trees"], d["dem"], d["walls_ref"], d["aspect_ref"], float(d["scale"]),
                          amaxvalue=d["amaxvalue"])
    ref = site.run_svf()
    planes = torch.empty_like(ref.planes)
    bits = torch.empty_like(ref.bits)
    n = site.count_svf_gathers(planes, bits)
    assert torch.equal(planes.view(torch.int32), ref.planes.view(torch.int32))
    assert torch.equal(bits, ref.bits)
    table_steps = int(site.svf_tables(2)[2])
    assert 0 < n <= table_steps * site.rows * site.cols
    # a second call restarts the count
    assert site.count_svf_gathers(planes, bits) == n
    # the persistent sweep resets its patch counter: another sweep into
    # fresh buffers writes the same result again
    planes2 = torch.full_like(ref.planes, float("nan"))
    bits2 = torch.full_like(ref.bits, -1)
    site.launch_svf(planes2, bits2)
    assert torch.equal(planes2.view(torch.int32), ref.planes.view(torch.int32))
    assert torch.equal(bits2, ref.bits)
