"""The host tables of the chunked time loop built in the helper process
(hostwork.TableBuilder): the same bytes as building them in this process,
chunk by chunk; an abandoned job's tables never reach the next job; a
failing build raises here."""
import numpy as np
import pytest

from solweig_project_b200 import hostwork, synthetic
from solweig_project_b200 import timeseries as TS


def _kw(seed=3, rows=40, cols=50):
    city = synthetic.make_city(rows, cols, seed=seed, with_walls=False)
    lc = np.array(city.landcover, np.float32)
    lc[(lc < 1) | (lc > 7)] = 6
    lc[(lc == 3) | (lc == 4)] = 5
    codes = 0
    for v in np.unique(lc):
        codes |= 1 << int(v)
    geo = synthetic.load_sun_geometry("single")
    return dict(met_file=synthetic.make_met(seed), location=dict(synthetic.DEFAULT_LOCATION), scale=1.0,
                amax=float(city.dsm.max()), rows=rows, cols=cols,
                props=TS.device_props(synthetic.default_lc_class(), codes), params=TS.ModelParams(), **geo)


def _same(a, b):
    for k in ("steps", "sun", "sun_table", "patch", "gvf"):
        x, y = (np.ascontiguousarray(getattr(s, k)).view(np.uint8) for s in (a, b))
        assert np.array_equal(x, y), k
    assert a.final == b.final


@pytest.fixture(scope="module")
def builder():
    return hostwork.builder()


@pytest.mark.parametrize("span", [(0, 24, 8), (3, 20, 5), (0, 24, 24)])
def test_helper_tables_equal_local(builder, span):
    kw = _kw()
    job = builder.submit(kw, *span)
    local = hostwork.LocalTables(kw, *span)
    n = len(range(span[0], span[1], span[2]))
    for _ in range(n):
        _same(job.next(), local.next())
    with pytest.raises(StopIteration):
        job.next()


def test_abandoned_job_does_not_leak(builder):
    a, b = _kw(seed=3), _kw(seed=8)
    job = builder.submit(a, 0, 24, 8)
    job.next()
    job.finish()                       # two chunks of `a` still to come from the helper
    job = builder.submit(b, 0, 24, 8)
    local = hostwork.LocalTables(b, 0, 24, 8)
    for _ in range(3):
        _same(job.next(), local.next())


def test_helper_error_raises(builder):
    kw = _kw()
    kw["params"] = TS.ModelParams(anisotropic_sky=0)     # refused by build_series
    job = builder.submit(kw, 0, 24, 8)
    with pytest.raises(RuntimeError, match="anisotropic"):
        job.next()
    # the builder takes the next job
    kw = _kw()
    job = builder.submit(kw, 0, 8, 8)
    _same(job.next(), hostwork.LocalTables(kw, 0, 8, 8).next())


def test_dead_helper_raises_and_is_replaced():
    b = hostwork.TableBuilder()
    b._proc.kill()
    b._proc.wait()
    with pytest.raises((RuntimeError, BrokenPipeError)):
        b.submit(_kw(), 0, 8, 8).next()
    saved = hostwork._BUILDER
    try:
        hostwork._BUILDER = b
        fresh = hostwork.builder()
        assert fresh is not b and fresh.alive()
        kw = _kw()
        _same(fresh.submit(kw, 0, 8, 8).next(), hostwork.LocalTables(kw, 0, 8, 8).next())
        fresh.close()
    finally:
        b.close()
        hostwork._BUILDER = saved
