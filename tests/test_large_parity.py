"""Parity at the benchmark sizes: the seeded 200 x 200 and 500 x 500 cities
(the latter is the city bench.py times), 24 hourly steps, against pins that
the unmodified reference produced on the host CPU
(tests/golden/make_golden_large.py).

* inputs: the repository's generator reproduces the rasters the reference
  ran on (sha256 of the raw float32 bytes, the reference's own wall height
  and aspect included);
* SVF: the 15 planes, SVFtotal and the three packed patch cubes, bit-exact
  (sha256);
* sun march: the 8 planes of every daytime step, bit-exact (sha256);
* shadow output of every step, bit-exact (sha256);
* Tmrt within 1e-3 K and UTCI within 1e-3 C of the reference at 4352 seeded
  pixels (4096 ground, 256 building) of every step, and the per-step means
  over all pixels within the same bounds;
* the error of this path and of the reference against an FP64
  re-evaluation of the same chain (same geometry) at those pixels, printed
  and bounded: this path may not be further from FP64 than the reference
  plus the parity tolerance.

Both the device-resident path (one launch per stage, what bench.py times)
and the drop-in host call ``api.run_exact_chain`` are checked.
"""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN

TMRT_TOL = 1e-3    # K
UTCI_TOL = 1e-3    # C
# 200 x 200 and 500 x 500 (the benchmarked city), three sites of the 64-site
# batched workload and a 512 x 512 city of the 4096 x 4096 tile's generator
# (buildings up to 120 m)
LARGE_CASES = ("c1_200", "c2_500", "c3_site37", "c3_site47", "c3_site17", "c4_proxy512")
SVF_ORDER = ("svf", "svfaveg", "svfE", "svfEaveg", "svfEveg", "svfN", "svfNaveg", "svfNveg", "svfS", "svfSaveg",
             "svfSveg", "svfveg", "svfW", "svfWaveg", "svfWveg")
LOCATION = {"latitude": 30.3, "longitude": -97.7, "altitude": 3.0}


def load_large(case):
    path = os.path.join(GOLDEN, f"large_{case}.npz")
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def digest(a, dtype=np.float32):
    a = np.ascontiguousarray(np.asarray(a, dtype))
    return hashlib.sha256(a.tobytes()).hexdigest()


def _multi_index(d):
    spec = [str(x) for x in d["spec"]] if "spec" in d else []
    return int(spec[1]) if spec and spec[0] == "multi" else None


def make_inputs(d):
    from solweig_project_b200 import synthetic
    i = _multi_index(d)
    if i is not None:
        sp = synthetic.multi_site_specs()[i]
        city = synthetic.make_city(sp["side"], sp["side"], seed=sp["seed"], density=sp["density"],
                                   canopy_cover=sp["canopy"])
    else:
        side = int(d["side"])
        city = synthetic.make_city(side, side, seed=int(d["seed"]), h_max=float(d["h_max"]))
    return city, synthetic.default_lc_class()


def location(d):
    if "latitude" in d:
        return {"latitude": float(d["latitude"]), "longitude": float(d["longitude"]),
                "altitude": float(d["site_altitude"])}
    return dict(LOCATION)


def error_stats(got, want):
    diff = np.asarray(got, np.float64) - np.asarray(want, np.float64)
    ok = ~np.isnan(diff)
    return float(np.abs(diff[ok]).max()), float(np.sqrt(np.mean(diff[ok] ** 2)))


@pytest.mark.parametrize("case", LARGE_CASES)
def test_generator_reproduces_reference_inputs(case):
    d = load_large(case)
    city, _ = make_inputs(d)
    for k, v in (("dsm", city.dsm), ("trees", city.trees), ("dem", city.dem), ("landcover", city.landcover),
                 ("walls", city.walls), ("aspect", city.aspect)):
        assert digest(v) == str(d["digest_in_" + k]), k


@pytest.mark.parametrize("case", LARGE_CASES)
def test_sun_geometry_of_fixture_is_the_workloads(case):
    from solweig_project_b200 import synthetic
    d = load_large(case)
    i = _multi_index(d)
    geo = synthetic.load_sun_geometry("single" if i is None else f"multi{i}")
    for k, v in geo.items():
        assert np.array_equal(v, d[k]), k
    assert np.array_equal(synthetic.make_met(int(d["seed"])), d["met"])


class _Run:
    """One device-resident run of a case, shared by the tests below."""
    cache = {}

    @classmethod
    def get(cls, case):
        if case not in cls.cache:
            cls.cache.clear()
            cls.cache[case] = cls(case)
        return cls.cache[case]

    def __init__(self, case):
        from solweig_project_b200.engine import DeviceSite
        d = load_large(case)
        city, lc_class = make_inputs(d)
        self.d, self.city, self.lc_class = d, city, lc_class
        site = DeviceSite(city.dsm, city.trees, city.dem, city.walls, city.aspect, city.scale,
                          landcover=city.landcover, lc_class=lc_class)
        self.res = site.run_svf()
        self.ser = site.build_series(d["met"], d["altitude"], d["azimuth"], d["zen"], d["jday"], d["dectime"],
                                     d["altmax"], location(d))
        _, dbg = site.run_sun_march(self.ser)
        self.march = dbg.cpu().numpy()
        out = site.run_time_loop(self.ser, requested=("utci", "tmrt", "shadow"))
        self.out = {k: v.cpu().numpy() for k, v in out.items()}
        self.planes = self.res.planes.cpu().numpy()
        self.words = self.res.bits.cpu().numpy()
        self.single = np.asarray(self.res.single_step)


@pytest.mark.gpu
@pytest.mark.parametrize("case", LARGE_CASES)
def test_large_svf_bit_exact(case, cuda):
    r = _Run.get(case)
    d = r.d
    for k, name in enumerate(SVF_ORDER):
        if digest(r.planes[k]) != str(d["digest_svf_" + name]):
            diff = np.abs(r.planes[k].reshape(-1)[d["samples"]] - d["sample_svf_" + name])
            pytest.fail(f"{case} {name}: digest differs (max |diff| at the sample pixels {diff.max():.3g})")
    assert digest(r.planes[15]) == str(d["digest_svf_svftotal"]), "svftotal"
    assert not r.single.any()          # no one-step patches on these grids: the cubes are 0/1
    rows, cols = r.planes.shape[1:]
    for c, name in enumerate(("shmat", "vegshmat", "vbshvegshmat")):
        # word-planar 32-bit words -> per pixel little-endian bytes = packbits(little) along the patch axis
        packed = np.ascontiguousarray(r.words[c].transpose(1, 2, 0)).view(np.uint8).reshape(rows, cols, 20)
        assert digest(packed, np.uint8) == str(d["digest_svf_" + name]), name


@pytest.mark.gpu
@pytest.mark.parametrize("case", LARGE_CASES)
def test_large_sun_march_bit_exact(case, cuda):
    r = _Run.get(case)
    want = r.d["digest_march"]
    assert r.march.shape[0] == want.shape[0] == len(r.d["march_steps"])
    names = ("vegsh", "sh", "vbshvegsh", "wallsh", "wallsun", "wallshve", "facesh", "facesun")
    bad = [(int(r.d["march_steps"][s]), names[k]) for s in range(want.shape[0]) for k in range(8)
           if digest(r.march[s, k]) != str(want[s, k])]
    assert not bad, f"{case}: sun-march planes differ at (step, plane) {bad[:8]}"


def _check_outputs(case, d, tmrt, utci, shadow, what):
    T = d["met"].shape[0]
    if shadow is not None:
        bad = [t for t in range(T) if digest(shadow[t]) != str(d["digest_shadow"][t])]
        assert not bad, f"{case} {what}: shadow differs at steps {bad}"
    s = d["samples"]
    tm = tmrt.reshape(T, -1)
    ut = utci.reshape(T, -1)
    assert np.array_equal(np.isnan(ut[:, s]), np.isnan(d["sample_utci"])), "UTCI NaN placement"
    e_tm = error_stats(tm[:, s], d["sample_tmrt"])
    e_ut = error_stats(ut[:, s], d["sample_utci"])
    assert e_tm[0] <= TMRT_TOL, f"{case} {what}: Tmrt max {e_tm[0]:.3g} K at the sample pixels"
    assert e_ut[0] <= UTCI_TOL, f"{case} {what}: UTCI max {e_ut[0]:.3g} C at the sample pixels"
    npix = tm.shape[1]
    mean_tm = np.abs(tm.astype(np.float64).sum(axis=1) - d["sum_tmrt"]) / npix
    assert mean_tm.max() <= TMRT_TOL, f"{case} {what}: per-step Tmrt mean off by {mean_tm.max():.3g} K"
    valid = np.sum(~np.isnan(ut), axis=1)
    assert np.array_equal(valid, d["n_utci_valid"])
    mean_ut = np.abs(np.nansum(ut.astype(np.float64), axis=1) - d["sum_utci"]) / np.maximum(valid, 1)
    assert mean_ut.max() <= UTCI_TOL, f"{case} {what}: per-step UTCI mean off by {mean_ut.max():.3g} C"
    # FP64 re-evaluation of the same chain at the sample pixels
    tm64 = d["sample_tmrt"].astype(np.float64) + d["sample_tmrt64_delta"]
    ut64 = d["sample_utci"].astype(np.float64) + d["sample_utci64_delta"]
    ours = error_stats(tm[:, s], tm64) + error_stats(ut[:, s], ut64)
    ref = error_stats(d["sample_tmrt"], tm64) + error_stats(d["sample_utci"], ut64)
    print(f"\n{case} {what} vs FP64 at {s.size} px x {T} steps: Tmrt max/rms {ours[0]:.3g}/{ours[1]:.3g} K "
          f"(reference {ref[0]:.3g}/{ref[1]:.3g}), UTCI max/rms {ours[2]:.3g}/{ours[3]:.3g} C "
          f"(reference {ref[2]:.3g}/{ref[3]:.3g})")
    assert ours[0] <= ref[0] + TMRT_TOL and ours[1] <= ref[1] + TMRT_TOL
    assert ours[2] <= ref[2] + UTCI_TOL and ours[3] <= ref[3] + UTCI_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("case", LARGE_CASES)
def test_large_chain_device_resident(case, cuda):
    r = _Run.get(case)
    _check_outputs(case, r.d, r.out["tmrt"], r.out["utci"], r.out["shadow"], "device-resident")


@pytest.mark.gpu
@pytest.mark.parametrize("case", LARGE_CASES)
def test_large_chain_drop_in_call(case, cuda):
    from solweig_project_b200 import api, synthetic
    d = load_large(case)
    city, lc_class = make_inputs(d)
    geo = {k: d[k] for k in ("altitude", "azimuth", "zen", "jday", "dectime", "altmax")}
    out = api.run_exact_chain(dsm=city.dsm, trees=city.trees, dem=city.dem, walls=city.walls, aspect=city.aspect,
                              scale=city.scale, met_file=d["met"], location=location(d),
                              landcover=city.landcover, lc_class=lc_class,
                              requested=("utci", "tmrt", "shadow"), **geo)
    _check_outputs(case, d, out["tmrt"], out["utci"], out.get("shadow"), "run_exact_chain")
