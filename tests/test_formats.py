"""SVF cache formats (shadow.py:100-164, utci_process.py:260-313) and the
packed per-patch bit layout (solweig_core/bitplanes.py)."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from golden_util import assert_bits_equal

from solweig_project_b200 import formats as FM

GT = (500000.0, 1.0, 0.0, 3300000.0, 0.0, -1.0)


def test_tiff_roundtrip_keeps_values_and_geotransform():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((37, 53)).astype(np.float32)
    a[3, 4] = np.nan
    back, gt = FM.read_tiff(FM.tiff_bytes(a, GT))
    assert_bits_equal(back, a, "tiff")
    assert gt == GT
    back, gt = FM.read_tiff(FM.tiff_bytes(a))
    assert gt is None and back.shape == a.shape


def test_truncated_tiff_is_refused():
    buf = FM.tiff_bytes(np.zeros((8, 8), np.float32))
    with pytest.raises(ValueError):
        FM.read_tiff(buf[:-10])


def _random_bits(rows, cols, n_patches, rng):
    bits = rng.integers(0, 2 ** 31, (3, 5, rows, cols), dtype=np.int64).astype(np.int32)
    tail = n_patches - 128
    bits[:, 4] &= np.int32((1 << tail) - 1)
    return torch.from_numpy(bits)


def test_packed_bits_match_numpy_packbits_little_order():
    rng = np.random.default_rng(1)
    bits = _random_bits(6, 7, 153, rng)
    packed = FM.to_packed_bits(bits, 153, np.zeros(5, np.uint32))
    w = bits.numpy().astype(np.int64) & 0xFFFFFFFF
    for i, name in enumerate(("shmat", "vegshmat", "vbshvegshmat")):
        dense = np.stack([(w[i, q >> 5] >> (q & 31)) & 1 for q in range(153)], axis=-1).astype(np.uint8)
        want = np.packbits(dense, axis=-1, bitorder="little")
        assert packed[name].shape == (6, 7, FM.bytes_per_patch(153)) == want.shape
        assert np.array_equal(packed[name], want), name
    back = FM.from_packed_bits(packed, device="cpu")
    assert torch.equal(back, bits)


def test_one_step_regime_is_refused():
    rng = np.random.default_rng(2)
    bits = _random_bits(4, 4, 153, rng)
    single = np.zeros(5, np.uint32)
    single[4] = 1 << (152 - 128)
    bits[2, 4] &= ~np.int32(1 << (152 - 128))      # vbshvegsh == 2 on the one-step patch
    with pytest.raises(ValueError, match="one-step"):
        FM.to_packed_bits(bits, 153, single)


def test_cache_roundtrip_and_extent_check(tmp_path):
    rng = np.random.default_rng(3)
    planes = torch.from_numpy(rng.random((19, 12, 9)).astype(np.float32))
    cubes = [rng.integers(0, 2, (12, 9, 153)).astype(np.float32) for _ in range(3)]
    FM.write_svf_cache(str(tmp_path), planes, cubes, GT, number=7)
    got, cubes2 = FM.read_svf_cache(str(tmp_path), number=7)
    for name in FM.SVF_TIFS + ("svftotal",):
        assert_bits_equal(got[name], planes[FM._PLANE[name]].numpy(), name)
    for a, b in zip(cubes, cubes2):
        assert np.array_equal(a, b)
    assert FM.svf_cache_extent_matches((12, 9), GT, str(tmp_path), 7)
    assert not FM.svf_cache_extent_matches((12, 10), GT, str(tmp_path), 7)
    assert not FM.svf_cache_extent_matches((12, 9), (0.0, 1.0, 0.0, 0.0, 0.0, -1.0), str(tmp_path), 7)
    assert not FM.svf_cache_extent_matches((12, 9), GT, str(tmp_path), 8)      # missing
    zip_path, _, _ = FM.cache_paths(str(tmp_path), 7)
    with open(zip_path, "r+b") as fh:                                          # damaged zip
        fh.truncate(40)
    assert not FM.svf_cache_extent_matches((12, 9), GT, str(tmp_path), 7)


@pytest.mark.gpu
def test_cache_of_a_device_sweep_matches_the_reference(cuda, tmp_path):
    from oracle.svf import scene_from_rasters
    from solweig_project_b200.engine import DeviceSite
    d = load_golden("city36")
    vegdsm, vegdsm2, bush, amax = scene_from_rasters(d["dsm"], d["trees"], d["dem"])
    site = DeviceSite.from_march_rasters(d["dsm"], vegdsm, vegdsm2, bush, amax, 1.0)
    res = site.run_svf()
    FM.write_svf_cache(str(tmp_path), res.planes, res.cubes(), GT, number=1)
    got, (sh, veg, vb) = FM.read_svf_cache(str(tmp_path), number=1)
    for name in FM.SVF_TIFS + ("svftotal",):
        assert_bits_equal(got[name], d["svf_" + name].astype(np.float32), name)
    assert_bits_equal(sh, d["svf_shmat"].astype(np.float32), "shadowmat")
    assert_bits_equal(veg, d["svf_vegshmat"].astype(np.float32), "vegshadowmat")
    assert_bits_equal(vb, d["svf_vbshvegshmat"].astype(np.float32), "vbshmat")
    packed = FM.to_packed_bits(res.bits, 153, res.single_step)
    dense = np.packbits(d["svf_shmat"].astype(np.uint8), axis=-1, bitorder="little")
    assert np.array_equal(packed["shmat"], dense)
