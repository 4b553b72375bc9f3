"""The GeoTIFF reader (formats.read_tiff / read_raster) on the layouts GDAL
writes: libtiff-compressed strips written by PIL (LZW, Deflate, PackBits),
and tiled, predicted (horizontal and floating-point), big-endian and BigTIFF
files built here byte by byte from the TIFF 6.0 / GeoTIFF layouts."""
import io
import struct
import zlib

import numpy as np
import pytest

from solweig_project_b200 import formats as FM


@pytest.mark.parametrize("comp", [None, "tiff_lzw", "tiff_adobe_deflate", "packbits"])
def test_libtiff_strips(comp):
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(0)
    a = (rng.standard_normal((37, 53)) * 10).astype(np.float32)
    buf = io.BytesIO()
    Image.fromarray(a, mode="F").save(buf, format="TIFF", **({} if comp is None else {"compression": comp}))
    b, gt = FM.read_tiff(buf.getvalue())
    assert b.dtype == np.float32 and np.array_equal(a, b) and gt is None
    u = rng.integers(0, 255, (33, 41)).astype(np.uint8)
    buf = io.BytesIO()
    Image.fromarray(u, mode="L").save(buf, format="TIFF", **({} if comp is None else {"compression": comp}))
    assert np.array_equal(FM.read_tiff(buf.getvalue())[0], u)


def _tiff(a, *, bo="<", tile=None, predictor=1, compress=True, big=False, geo=None):
    """A single-band GeoTIFF of `a`, strips (8 rows) or tiles."""
    rows, cols = a.shape
    dt = a.dtype.newbyteorder(bo)
    fmt = {"f": 3, "i": 2, "u": 1}[a.dtype.kind]

    def encode(block):
        h, w = block.shape
        if predictor == 2:
            x = block.astype(dt)
            x = np.concatenate([x[:, :1], (x[:, 1:].astype(np.int64) - x[:, :-1].astype(np.int64)).astype(dt)], 1)
            raw = x.astype(dt).tobytes()
        elif predictor == 3:
            be = block.astype(block.dtype.newbyteorder(">")).view(np.uint8).reshape(h, w, -1)
            planes = be.transpose(0, 2, 1).reshape(h, -1)
            d = np.concatenate([planes[:, :1], np.diff(planes.astype(np.int16), axis=1).astype(np.uint8)], 1)
            raw = d.astype(np.uint8).tobytes()
        else:
            raw = block.astype(dt).tobytes()
        return zlib.compress(raw) if compress else raw

    chunks = []
    if tile:
        th, tw = tile
        for r in range(0, rows, th):
            for c in range(0, cols, tw):
                blk = np.zeros((th, tw), a.dtype)
                part = a[r:r + th, c:c + tw]
                blk[:part.shape[0], :part.shape[1]] = part
                chunks.append(encode(blk))
    else:
        for r in range(0, rows, 8):
            chunks.append(encode(a[r:r + 8]))
    n = len(chunks)
    off_t, cnt_t = (16, 16) if big else (4, 4)
    entries = [(256, 4, [cols]), (257, 4, [rows]), (258, 3, [a.dtype.itemsize * 8]),
               (259, 3, [8 if compress else 1]), (262, 3, [1]), (277, 3, [1]), (284, 3, [1]),
               (317, 3, [predictor]), (339, 3, [fmt])]
    if tile:
        entries += [(322, 3, [tile[1]]), (323, 3, [tile[0]]), (324, off_t, None), (325, cnt_t, [len(c) for c in chunks])]
    else:
        entries += [(273, off_t, None), (278, 3, [8]), (279, cnt_t, [len(c) for c in chunks])]
    if geo is not None:
        x0, px, y0, epsg = geo
        entries += [(33550, 12, [px, px, 0.0]), (33922, 12, [0.0, 0.0, 0.0, x0, y0, 0.0]),
                    (34735, 3, [1, 1, 0, 2, 1024, 0, 1, 1, 3072, 0, 1, epsg])]
    entries.sort()
    code = {3: "H", 4: "I", 12: "d", 16: "Q"}
    size = {3: 2, 4: 4, 12: 8, 16: 8}
    head = 16 if big else 8
    ent_len, cnt_len, inline = (20, 8, 8) if big else (12, 2, 4)
    ifd_len = cnt_len + ent_len * len(entries) + (8 if big else 4)
    extra_at = head + ifd_len
    data_at = extra_at + sum(size[t] * (n if v is None else len(v)) for _, t, v in entries
                             if size[t] * (n if v is None else len(v)) > inline)
    offsets, pos = [], data_at
    for c in chunks:
        offsets.append(pos)
        pos += len(c)
    out = bytearray(b"II" if bo == "<" else b"MM")
    out += struct.pack(bo + "HHHQ", 43, 8, 0, head) if big else struct.pack(bo + "HI", 42, head)
    out += struct.pack(bo + ("Q" if big else "H"), len(entries))
    extra = bytearray()
    for tag, typ, vals in entries:
        vals = offsets if vals is None else vals
        payload = struct.pack(f"{bo}{len(vals)}{code[typ]}", *vals)
        if len(payload) <= inline:
            field = payload.ljust(inline, b"\0")
        else:
            field = struct.pack(bo + ("Q" if big else "I"), extra_at + len(extra))
            extra += payload
        out += struct.pack(bo + "HH", tag, typ) + struct.pack(bo + ("Q" if big else "I"), len(vals)) + field
    out += bytes(8 if big else 4)
    out += extra
    assert len(out) == data_at
    for c in chunks:
        out += c
    return bytes(out)


@pytest.mark.parametrize("bo", ["<", ">"])
@pytest.mark.parametrize("tile", [None, (16, 16)])
@pytest.mark.parametrize("big", [False, True])
def test_float_predictor_tiles_and_byte_orders(bo, tile, big):
    rng = np.random.default_rng(1)
    a = (rng.standard_normal((45, 70)) * 30 + 100).astype(np.float32)
    for predictor in (1, 3):
        b, gt = FM.read_tiff(_tiff(a, bo=bo, tile=tile, predictor=predictor, big=big))
        assert b.dtype == np.float32 and np.array_equal(a, b), (predictor, bo, tile, big)


def test_integer_horizontal_predictor():
    rng = np.random.default_rng(2)
    a = rng.integers(-3000, 3000, (30, 50)).astype(np.int16)
    b, _ = FM.read_tiff(_tiff(a, predictor=2, tile=(16, 32)))
    assert np.array_equal(a, b)


def test_read_raster_georeference(tmp_path):
    a = np.arange(20 * 30, dtype=np.float32).reshape(20, 30)
    p = tmp_path / "dsm.tif"
    p.write_bytes(_tiff(a, geo=(621000.0, 2.0, 3350000.0, 32614)))
    r = FM.read_raster(str(p))
    assert np.array_equal(r.data, a) and r.epsg == 32614
    assert r.geotransform == (621000.0, 2.0, 0.0, 3350000.0, 0.0, -2.0)
    np.save(tmp_path / "dsm.npy", a)
    r2 = FM.read_raster(str(tmp_path / "dsm.npy"))
    assert np.array_equal(r2.data, a) and r2.geotransform is None and r2.epsg is None
