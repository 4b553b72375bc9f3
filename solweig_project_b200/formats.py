"""SVF cache formats of the reference, written and read without GDAL.

* ``svfs_<k>.zip`` -- 15 single-band float32 GeoTIFFs (svf.tif, svfE.tif,
  ... svfNaveg.tif), ``SkyViewFactor_<k>.tif`` (SVFtotal) and
  ``shadowmats_<k>.npz`` (shadowmat / vegshadowmat / vbshmat, float32
  (rows, cols, P) cubes): ``solweig_gpu/shadow.py:100-164``
  save_svf_zip_npz_outputs.
* The extent check of a cache against its tile
  (``solweig_gpu/utci_process.py:260-313``): raster size and geotransform
  equal within a tolerance, unreadable files meaning "cache unusable".
* The packed per-patch bit layout of ``solweig_core/bitplanes.py``: uint8
  (rows, cols, ceil(P / 8)), little bit order, zero tail, values exactly
  {0, 1} (the one-step regime's vbshvegsh == 2 is refused).

The TIFF writer emits baseline, uncompressed, one-strip float32 images with
the three GeoTIFF tags a reader needs for the geotransform
(ModelPixelScale, ModelTiepoint, a minimal GeoKeyDirectory); the reader
accepts exactly what the writer produces.  Device results are converted on
the GPU (bit cubes <-> packed bytes are a byte-level transpose of the
word-planar cubes) and copied to the host once.
"""
from __future__ import annotations

import os
import struct
import zipfile

import numpy as np
import torch

F32 = np.float32
SVF_TIFS = ("svf", "svfE", "svfS", "svfW", "svfN", "svfveg", "svfEveg", "svfSveg", "svfWveg", "svfNveg",
            "svfaveg", "svfEaveg", "svfSaveg", "svfWaveg", "svfNaveg")
# plane index of each name in the library's SVF plane order
_PLANE = {"svf": 0, "svfaveg": 1, "svfE": 2, "svfEaveg": 3, "svfEveg": 4, "svfN": 5, "svfNaveg": 6, "svfNveg": 7,
          "svfS": 8, "svfSaveg": 9, "svfSveg": 10, "svfveg": 11, "svfW": 12, "svfWaveg": 13, "svfWveg": 14,
          "svftotal": 15}


# ----------------------------------------------------------------- TIFF
def _geotransform_tags(gt):
    x0, sx, _, y0, _, sy = gt
    return [(33550, 12, 3, struct.pack("<3d", sx, -sy, 0.0)),
            (33922, 12, 6, struct.pack("<6d", 0.0, 0.0, 0.0, x0, y0, 0.0)),
            (34735, 3, 4, struct.pack("<4H", 1, 1, 0, 0))]


def tiff_bytes(data: np.ndarray, geotransform=None, band_metadata=None) -> bytes:
    """Baseline float32 TIFF, one strip per band (bands stored as separate
    planes), with GeoTIFF geotransform tags when ``geotransform`` (GDAL
    order: x0, dx, 0, y0, 0, dy) is given and per-band metadata
    (``band_metadata[b] = {"Time": ...}``, written as GDAL's metadata tag)."""
    a = np.asarray(data, F32)
    if a.ndim == 2:
        a = a[None]
    bands, rows, cols = a.shape
    a = np.ascontiguousarray(a)
    band_bytes = rows * cols * 4
    pixels = a.astype("<f4").tobytes()
    entries = [(256, 4, 1, struct.pack("<I", cols)), (257, 4, 1, struct.pack("<I", rows)),
               (258, 3, bands, struct.pack(f"<{bands}H", *([32] * bands))), (259, 3, 1, struct.pack("<H", 1)),
               (262, 3, 1, struct.pack("<H", 1)), (273, 4, bands, None),
               (277, 3, 1, struct.pack("<H", bands)), (278, 4, 1, struct.pack("<I", rows)),
               (279, 4, bands, struct.pack(f"<{bands}I", *([band_bytes] * bands))),
               (284, 3, 1, struct.pack("<H", 2 if bands > 1 else 1)),
               (339, 3, bands, struct.pack(f"<{bands}H", *([3] * bands)))]
    if bands > 1:
        entries.append((338, 3, bands - 1, struct.pack(f"<{bands - 1}H", *([0] * (bands - 1)))))
    if geotransform is not None:
        entries += _geotransform_tags(geotransform)
    if band_metadata:
        items = "".join(f'<Item name="{k}" sample="{b}">{v}</Item>' for b, md in enumerate(band_metadata)
                        for k, v in (md or {}).items())
        xml = f"<GDALMetadata>{items}</GDALMetadata>".encode() + b"\0"
        entries.append((42112, 2, len(xml), xml))
    entries.sort(key=lambda e: e[0])
    ifd_off = 8
    ifd_len = 2 + 12 * len(entries) + 4
    extra = bytearray()
    extra_off = ifd_off + ifd_len
    placed = []
    strip_slot = None
    for tag, typ, count, payload in entries:
        if payload is None:                                  # StripOffsets: filled below
            payload = bytes(4 * count)
            if len(payload) > 4:
                strip_slot = extra_off + len(extra)
        if len(payload) > 4:
            placed.append((tag, typ, count, struct.pack("<I", extra_off + len(extra))))
            extra += payload
            if len(extra) % 2:
                extra += b"\0"
        else:
            placed.append((tag, typ, count, payload))
    data_off = extra_off + len(extra)
    offsets = struct.pack(f"<{bands}I", *[data_off + b * band_bytes for b in range(bands)])
    if strip_slot is not None:
        extra[strip_slot - extra_off:strip_slot - extra_off + len(offsets)] = offsets
    out = bytearray(b"II*\0" + struct.pack("<I", ifd_off))
    out += struct.pack("<H", len(placed))
    for tag, typ, count, payload in placed:
        if tag == 273 and strip_slot is None:
            payload = offsets
        out += struct.pack("<HHI", tag, typ, count) + payload.ljust(4, b"\0")
    out += struct.pack("<I", 0)
    out += extra
    out += pixels
    return bytes(out)


def read_tiff(buf: bytes, with_metadata: bool = False):
    """(array, geotransform or None[, band metadata]) of a TIFF written by
    :func:`tiff_bytes`; the array is (rows, cols) for one band, else
    (bands, rows, cols)."""
    import re
    if buf[:4] != b"II*\0":
        raise ValueError("not a little-endian TIFF")
    (ifd,) = struct.unpack_from("<I", buf, 4)
    (n,) = struct.unpack_from("<H", buf, ifd)
    tags = {}
    for k in range(n):
        tag, typ, count, val = struct.unpack_from("<HHI4s", buf, ifd + 2 + 12 * k)
        size = {2: 1, 3: 2, 4: 4, 12: 8}[typ] * count
        if size <= 4:
            raw = val[:size]
        else:
            (off,) = struct.unpack("<I", val)
            raw = buf[off:off + size]
        tags[tag] = raw if typ == 2 else struct.unpack(f"<{count}{ {3: 'H', 4: 'I', 12: 'd'}[typ] }", raw)
    cols, rows = tags[256][0], tags[257][0]
    bands = tags.get(277, (1,))[0]
    if any(b != 32 for b in tags[258]) or any(f != 3 for f in tags[339]) or tags[259][0] != 1:
        raise ValueError("only uncompressed float32 images are read")
    planes = []
    for b in range(bands):
        off, nbytes = tags[273][b], tags[279][b]
        if nbytes != rows * cols * 4 or off + nbytes > len(buf):
            raise ValueError("truncated image data")
        planes.append(np.frombuffer(buf, "<f4", rows * cols, off).reshape(rows, cols).astype(F32))
    a = planes[0] if bands == 1 else np.stack(planes)
    gt = None
    if 33550 in tags and 33922 in tags:
        sx, sy, _ = tags[33550]
        x0, y0 = tags[33922][3], tags[33922][4]
        gt = (x0, sx, 0.0, y0, 0.0, -sy)
    if not with_metadata:
        return a, gt
    md = [dict() for _ in range(bands)]
    if 42112 in tags:
        xml = tags[42112].rstrip(b"\0").decode()
        for name, sample, value in re.findall(r'<Item name="([^"]+)" sample="(\d+)">([^<]*)</Item>', xml):
            md[int(sample)][name] = value
    return a, gt, md


# ------------------------------------------------------------ packed bits
def bytes_per_patch(n_patches: int) -> int:
    """ceil(P / 8) (solweig_core/bitplanes.py:107)."""
    if n_patches <= 0:
        raise ValueError("patch count must be positive")
    return (n_patches + 7) // 8


def to_packed_bits(bits: torch.Tensor, n_patches: int, single_step) -> dict:
    """Word-planar bit cubes (3, 5, rows, cols) int32 of the sweep -> the
    reference's packed layout, {"shmat", "vegshmat", "vbshvegshmat"} uint8
    (rows, cols, ceil(P / 8)).  The one-step regime's vbshvegsh == 2 cannot
    be packed and is refused with ValueError, as bitplanes.pack_bits does."""
    single = [(int(single_step[q >> 5]) >> (q & 31)) & 1 for q in range(n_patches)]
    if any(single):
        vb = bits[2]
        for q in np.flatnonzero(single):
            if bool(((vb[q >> 5] >> (q & 31)) & 1).eq(0).any()):
                raise ValueError(f"patch {q} holds vbshvegsh == 2 (one-step march): not representable as packed bits")
    nb = bytes_per_patch(n_patches)
    # little-endian words: byte 4w + i of a pixel holds patches 32w + 8i ..
    planar = bits.permute(0, 2, 3, 1).contiguous()                     # (3, rows, cols, words)
    packed = planar.view(torch.uint8)[..., :nb].cpu().numpy()
    return {"shmat": packed[0].copy(), "vegshmat": packed[1].copy(), "vbshvegshmat": packed[2].copy()}


def from_packed_bits(packed: dict, words: int = 5, device="cuda") -> torch.Tensor:
    """The inverse of :func:`to_packed_bits`: (3, words, rows, cols) int32."""
    cubes = [np.asarray(packed[k], np.uint8) for k in ("shmat", "vegshmat", "vbshvegshmat")]
    rows, cols, nb = cubes[0].shape
    full = np.zeros((3, rows, cols, words * 4), np.uint8)
    for i, c in enumerate(cubes):
        full[i, :, :, :nb] = c
    t = torch.from_numpy(full).to(device)
    return t.view(torch.int32).view(3, rows, cols, words).permute(0, 3, 1, 2).contiguous()


# -------------------------------------------------------------- caches
def cache_paths(output_dir: str, number=None):
    suffix = f"_{number}" if number is not None else ""
    return (os.path.join(output_dir, f"svfs{suffix}.zip"), os.path.join(output_dir, f"shadowmats{suffix}.npz"),
            os.path.join(output_dir, f"SkyViewFactor{suffix}.tif"))


def write_svf_cache(output_dir: str, planes: torch.Tensor, cubes, geotransform=None, number=None):
    """The reference's SVF cache (shadow.py:100-164) from the library's SVF
    planes (19, rows, cols) and the dense cubes (shmat, vegshmat,
    vbshvegshmat), (rows, cols, P) each (:meth:`SvfResult.cubes`)."""
    os.makedirs(output_dir, exist_ok=True)
    zip_path, npz_path, total_path = cache_paths(output_dir, number)
    host = planes.detach().cpu().numpy()
    if os.path.isfile(zip_path):
        os.remove(zip_path)
    with zipfile.ZipFile(zip_path, "w", compression=zipfile.ZIP_DEFLATED) as zf:
        for name in SVF_TIFS:
            zf.writestr(f"{name}.tif", tiff_bytes(host[_PLANE[name]], geotransform))
    with open(total_path, "wb") as fh:
        fh.write(tiff_bytes(host[_PLANE["svftotal"]], geotransform))
    sh, veg, vb = (c.detach().cpu().numpy().astype(F32) if isinstance(c, torch.Tensor) else np.asarray(c, F32)
                   for c in cubes)
    np.savez_compressed(npz_path, shadowmat=sh, vegshadowmat=veg, vbshmat=vb)
    return zip_path, npz_path, total_path


def read_svf_cache(output_dir: str, number=None):
    """({name: plane} for the 15 SVF planes and "svftotal", (shmat,
    vegshmat, vbshvegshmat)) of a cache written by :func:`write_svf_cache`."""
    zip_path, npz_path, total_path = cache_paths(output_dir, number)
    out = {}
    with zipfile.ZipFile(zip_path) as zf:
        for name in SVF_TIFS:
            out[name] = read_tiff(zf.read(f"{name}.tif"))[0]
    with open(total_path, "rb") as fh:
        out["svftotal"] = read_tiff(fh.read())[0]
    with np.load(npz_path) as z:
        cubes = (z["shadowmat"], z["vegshadowmat"], z["vbshmat"])
    return out, cubes


def _geotransforms_equal(a, b, tol=1e-9):
    return a is not None and b is not None and len(a) == 6 and len(b) == 6 and \
        all(abs(x - y) <= tol for x, y in zip(a, b))


def svf_cache_extent_matches(shape, geotransform, output_dir: str, number=None) -> bool:
    """Whether a cache shares the tile's size and geotransform
    (utci_process.py:260-296); unreadable or missing files mean False."""
    zip_path, npz_path, total_path = cache_paths(output_dir, number)
    try:
        with open(total_path, "rb") as fh:
            rasters = [read_tiff(fh.read())]
        with zipfile.ZipFile(zip_path) as zf:
            rasters.append(read_tiff(zf.read("svf.tif")))
        if not os.path.isfile(npz_path):
            return False
    except (OSError, ValueError, KeyError, struct.error, zipfile.BadZipFile):
        return False
    rows, cols = shape
    return all(a.shape == (rows, cols) and _geotransforms_equal(gt, geotransform) for a, gt in rasters)
