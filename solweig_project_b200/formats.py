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
takes the GeoTIFFs GDAL writes (strips or tiles; uncompressed, LZW,
Deflate or PackBits; predictors 2 and 3; integer or float samples).  Device results are converted on
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
def _geotransform_tags(gt, epsg=None):
    x0, sx, _, y0, _, sy = gt
    if epsg is None:
        keys = struct.pack("<4H", 1, 1, 0, 0)
    elif epsg == 4326 or 4000 <= epsg < 5000:
        keys = struct.pack("<12H", 1, 1, 0, 2, 1024, 0, 1, 2, 2048, 0, 1, epsg)     # geographic
    else:
        keys = struct.pack("<12H", 1, 1, 0, 2, 1024, 0, 1, 1, 3072, 0, 1, epsg)     # projected
    return [(33550, 12, 3, struct.pack("<3d", sx, -sy, 0.0)),
            (33922, 12, 6, struct.pack("<6d", 0.0, 0.0, 0.0, x0, y0, 0.0)),
            (34735, 3, len(keys) // 2, keys)]


def tiff_bytes(data: np.ndarray, geotransform=None, band_metadata=None, epsg=None) -> bytes:
    """Baseline float32 TIFF, one strip per band (bands stored as separate
    planes), with GeoTIFF geotransform tags when ``geotransform`` (GDAL
    order: x0, dx, 0, y0, 0, dy) is given (and the EPSG code of its
    coordinate system with ``epsg``) and per-band metadata
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
        entries += _geotransform_tags(geotransform, epsg)
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


_FIELD = {1: ("B", 1), 2: ("c", 1), 3: ("H", 2), 4: ("I", 4), 5: ("II", 8), 6: ("b", 1), 7: ("B", 1),
          8: ("h", 2), 9: ("i", 4), 10: ("ii", 8), 11: ("f", 4), 12: ("d", 8), 16: ("Q", 8), 17: ("q", 8),
          18: ("Q", 8)}


def _tiff_tags(buf: bytes):
    """({tag: values}, byte order) of the first image directory of a
    classic or BigTIFF file, either byte order."""
    bo = {b"II": "<", b"MM": ">"}.get(buf[:2])
    if bo is None:
        raise ValueError("not a TIFF file")
    (magic,) = struct.unpack_from(bo + "H", buf, 2)
    if magic == 42:
        (ifd,) = struct.unpack_from(bo + "I", buf, 4)
        (n,) = struct.unpack_from(bo + "H", buf, ifd)
        entry, head, inline, off_fmt = 12, 2, 4, "I"
    elif magic == 43:
        (ifd,) = struct.unpack_from(bo + "Q", buf, 8)
        (n,) = struct.unpack_from(bo + "Q", buf, ifd)
        entry, head, inline, off_fmt = 20, 8, 8, "Q"
    else:
        raise ValueError("not a TIFF file")
    tags = {}
    for k in range(n):
        pos = ifd + head + entry * k
        tag, typ = struct.unpack_from(bo + "HH", buf, pos)
        (count,) = struct.unpack_from(bo + ("I" if magic == 42 else "Q"), buf, pos + 4)
        if typ not in _FIELD:
            continue
        code, size = _FIELD[typ]
        nbytes = size * count
        vpos = pos + 4 + (4 if magic == 42 else 8)
        if nbytes <= inline:
            raw = buf[vpos:vpos + nbytes]
        else:
            (off,) = struct.unpack_from(bo + off_fmt, buf, vpos)
            raw = buf[off:off + nbytes]
        if typ == 2:
            tags[tag] = raw
        elif typ in (5, 10):
            v = struct.unpack(f"{bo}{2 * count}{code[0].upper() if typ == 5 else code[0]}", raw)
            tags[tag] = tuple(v[i] / v[i + 1] if v[i + 1] else 0.0 for i in range(0, len(v), 2))
        else:
            tags[tag] = struct.unpack(f"{bo}{count}{code}", raw)
    return tags, bo


def _lzw_decode(data: bytes) -> bytes:
    """TIFF LZW (most significant bit first, 9-12 bit codes, early change)."""
    out = bytearray()
    table = [bytes([i]) for i in range(256)] + [b"", b""]
    width, bitbuf, nbits, prev = 9, 0, 0, None
    for byte in data:
        bitbuf = (bitbuf << 8) | byte
        nbits += 8
        while nbits >= width:
            nbits -= width
            code = (bitbuf >> nbits) & ((1 << width) - 1)
            if code == 256:                       # clear
                table = table[:258]
                width, prev = 9, None
                continue
            if code == 257:                       # end of information
                return bytes(out)
            if code < len(table):
                entry = table[code]
                if prev is not None:
                    table.append(prev + entry[:1])
            elif prev is not None:
                entry = prev + prev[:1]
                table.append(entry)
            else:
                raise ValueError("corrupt LZW data")
            out += entry
            prev = entry
            if len(table) + 1 >= (1 << width) and width < 12:
                width += 1
        bitbuf &= (1 << nbits) - 1
    return bytes(out)


def _packbits_decode(data: bytes) -> bytes:
    out = bytearray()
    i, n = 0, len(data)
    while i < n:
        h = data[i]
        i += 1
        if h < 128:
            out += data[i:i + h + 1]
            i += h + 1
        elif h > 128:
            out += data[i:i + 1] * (257 - h)
            i += 1
    return bytes(out)


def _decompress(chunk: bytes, compression: int) -> bytes:
    import zlib
    if compression == 1:
        return chunk
    if compression in (8, 32946):
        return zlib.decompress(chunk)
    if compression == 5:
        return _lzw_decode(chunk)
    if compression == 32773:
        return _packbits_decode(chunk)
    raise ValueError(f"TIFF compression {compression} is not supported (none, LZW, Deflate, PackBits are)")


def _unpredict(a: np.ndarray, predictor: int) -> np.ndarray:
    """Undo the horizontal-differencing predictor on samples (h, w, spp)."""
    if predictor == 2:
        return np.cumsum(a, axis=1, dtype=a.dtype)
    return a


def _unpredict_float(raw: np.ndarray, h: int, w: int, spp: int, dtype: np.dtype) -> np.ndarray:
    """Undo the floating-point predictor: each row holds the byte planes of
    its samples (most significant first), byte-differenced along the row."""
    isz = dtype.itemsize
    b = np.cumsum(raw.reshape(h, w * spp * isz), axis=1, dtype=np.uint8)
    b = b.reshape(h, isz, w * spp).transpose(0, 2, 1).copy()      # -> big-endian sample bytes
    return b.view(np.dtype(dtype.str[1:]).newbyteorder(">")).reshape(h, w, spp).astype(dtype.newbyteorder("="))


def read_tiff(buf: bytes, with_metadata: bool = False):
    """(array, geotransform or None[, band metadata]) of a GeoTIFF: baseline
    strips or tiles, chunky or planar samples, 8-64 bit integer / float
    samples, uncompressed, LZW, Deflate or PackBits, horizontal or
    floating-point predictor, either byte order, classic or BigTIFF.  The
    array is (rows, cols) for one band, else (bands, rows, cols), in the
    file's sample type.  The geotransform (GDAL order) comes from
    ModelPixelScale + ModelTiepoint or ModelTransformation, shifted by half
    a pixel for PixelIsPoint rasters as GDAL does."""
    import re
    tags, bo = _tiff_tags(buf)
    cols, rows = int(tags[256][0]), int(tags[257][0])
    spp = int(tags.get(277, (1,))[0])
    bps = tags.get(258, (1,) * spp)
    fmt = int(tags.get(339, (1,))[0])
    if len(set(bps)) != 1 or bps[0] not in (8, 16, 32, 64):
        raise ValueError(f"TIFF bits per sample {bps} are not supported")
    kind = {1: "u", 2: "i", 3: "f"}.get(fmt)
    if kind is None:
        raise ValueError(f"TIFF sample format {fmt} is not supported")
    dtype = np.dtype(f"{kind}{bps[0] // 8}").newbyteorder(bo)
    compression = int(tags.get(259, (1,))[0])
    predictor = int(tags.get(317, (1,))[0])
    planar = int(tags.get(284, (1,))[0])
    nplanes, cspp = (spp, 1) if planar == 2 else (1, spp)
    if 322 in tags:
        tw, th = int(tags[322][0]), int(tags[323][0])
        offsets, counts = tags[324], tags[325]
        across, down = (cols + tw - 1) // tw, (rows + th - 1) // th
        chunks = [(b, (i // across) * th, (i % across) * tw, th, tw)
                  for b in range(nplanes) for i in range(across * down)]
    else:
        rps = min(int(tags.get(278, (rows,))[0]), rows)
        offsets, counts = tags[273], tags.get(279)
        per = (rows + rps - 1) // rps
        chunks = [(b, i * rps, 0, min(rps, rows - i * rps), cols) for b in range(nplanes) for i in range(per)]
        if counts is None:
            counts = [h * cols * cspp * dtype.itemsize for _, _, _, h, _ in chunks]
    out = np.zeros((nplanes, rows, cols, cspp), dtype.newbyteorder("="))
    for k, (b, r0, c0, h, w) in enumerate(chunks):
        raw = _decompress(bytes(buf[offsets[k]:offsets[k] + counts[k]]), compression)
        need = h * w * cspp * dtype.itemsize
        if len(raw) < need:
            raise ValueError("truncated image data")
        if predictor == 3:
            a = _unpredict_float(np.frombuffer(raw, np.uint8, need), h, w, cspp, dtype)
        else:
            a = np.frombuffer(raw, dtype, h * w * cspp).reshape(h, w, cspp)
            a = _unpredict(a.astype(dtype.newbyteorder("=")), predictor)
        hh, ww = min(h, rows - r0), min(w, cols - c0)
        out[b, r0:r0 + hh, c0:c0 + ww] = a[:hh, :ww]
    bands = out.transpose(0, 3, 1, 2).reshape(spp, rows, cols)
    arr = bands[0] if spp == 1 else bands
    arr = arr.astype(F32) if arr.dtype == np.float32 else arr
    gt = None
    if 33550 in tags and 33922 in tags:
        sx, sy = tags[33550][0], tags[33550][1]
        i0, j0, x, y = tags[33922][0], tags[33922][1], tags[33922][3], tags[33922][4]
        gt = (x - i0 * sx, sx, 0.0, y + j0 * sy, 0.0, -sy)
    elif 34264 in tags:
        m = tags[34264]
        gt = (m[3], m[0], m[1], m[7], m[4], m[5])
    keys = _geokeys(tags)
    if gt is not None and keys.get(1025) == 2:            # RasterPixelIsPoint
        gt = (gt[0] - 0.5 * gt[1] - 0.5 * gt[2], gt[1], gt[2], gt[3] - 0.5 * gt[4] - 0.5 * gt[5], gt[4], gt[5])
    if not with_metadata:
        return arr, gt
    md = [dict() for _ in range(spp)]
    if 42112 in tags:
        xml = tags[42112].rstrip(b"\0").decode()
        for name, sample, value in re.findall(r'<Item name="([^"]+)" sample="(\d+)">([^<]*)</Item>', xml):
            md[int(sample)][name] = value
    return arr, gt, md


def _geokeys(tags) -> dict:
    """{GeoKey id: value} of the GeoKeyDirectory (short values only)."""
    d = tags.get(34735)
    if not d or len(d) < 4:
        return {}
    out = {}
    for k in range(int(d[3])):
        key, loc, count, val = d[4 + 4 * k:8 + 4 * k]
        if loc == 0 and count == 1:
            out[int(key)] = int(val)
    return out


class Raster:
    """A raster read from disk: float32 (rows, cols) values, the GDAL-order
    geotransform (None for .npy), the EPSG code of its coordinate system
    (None when the file names none) and the nodata value."""

    def __init__(self, data, geotransform=None, epsg=None, nodata=None):
        self.data, self.geotransform, self.epsg, self.nodata = data, geotransform, epsg, nodata

    @property
    def shape(self):
        return self.data.shape


def read_raster(path: str) -> Raster:
    """First band of a GeoTIFF (:func:`read_tiff`) or a .npy array, as
    float32, with its georeferencing."""
    if path.lower().endswith(".npy"):
        return Raster(np.asarray(np.load(path), F32))
    with open(path, "rb") as fh:
        buf = fh.read()
    arr, gt = read_tiff(buf)
    if arr.ndim == 3:
        arr = arr[0]
    tags, _ = _tiff_tags(buf)
    keys = _geokeys(tags)
    epsg = keys.get(3072) or keys.get(2048)
    nodata = None
    if 42113 in tags:
        try:
            nodata = float(tags[42113].rstrip(b"\0").decode())
        except ValueError:
            nodata = None
    return Raster(np.asarray(arr, F32), gt, epsg, nodata)


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


def write_svf_cache(output_dir: str, planes: torch.Tensor, cubes, geotransform=None, number=None, epsg=None):
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
            zf.writestr(f"{name}.tif", tiff_bytes(host[_PLANE[name]], geotransform, epsg=epsg))
    with open(total_path, "wb") as fh:
        fh.write(tiff_bytes(host[_PLANE["svftotal"]], geotransform, epsg=epsg))
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
