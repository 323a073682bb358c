"""Frame export (export/FrameExporter.java:51-80): the PNG writer the
library uses for RGBA8 display images, checked by decoding what it wrote."""
import os
import struct
import zlib

import numpy as np
import pytest

from retrocam_b200 import export


def test_png_round_trip_and_header(tmp_path):
    rng = np.random.default_rng(5)
    img = rng.integers(0, 256, (37, 53, 4), dtype=np.uint8)
    path = str(tmp_path / "a" / "b" / "frame.png")   # parent folders are created
    export.write_png(path, img)
    data = open(path, "rb").read()
    assert data[:8] == export.PNG_SIGNATURE
    n, kind = struct.unpack(">I4s", data[8:16])
    assert (n, kind) == (13, b"IHDR")
    assert struct.unpack(">IIBBBBB", data[16:29]) == (53, 37, 8, 6, 0, 0, 0)
    assert struct.unpack(">I", data[29:33])[0] == zlib.crc32(data[12:29]) & 0xFFFFFFFF
    assert np.array_equal(export.read_png(path), img)


def test_png_reader_undoes_every_filter_type(tmp_path):
    """A file with rows in each of the five PNG filter types decodes to the
    source image (the reader is also usable on other writers' files)."""
    rng = np.random.default_rng(6)
    img = rng.integers(0, 256, (5, 7, 4), dtype=np.uint8)
    prev = np.zeros(28, np.int32)
    rows = []
    for y in range(5):
        cur = img[y].reshape(-1).astype(np.int32)
        out = np.zeros(28, np.int32)
        for i in range(28):
            a = cur[i - 4] if i >= 4 else 0
            b, c = prev[i], (prev[i - 4] if i >= 4 else 0)
            pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
            paeth = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            out[i] = (cur[i] - (0, a, b, (a + b) >> 1, paeth)[y]) & 0xFF
        rows.append(bytes([y]) + out.astype(np.uint8).tobytes())
        prev = cur
    ihdr = struct.pack(">IIBBBBB", 7, 5, 8, 6, 0, 0, 0)
    data = (export.PNG_SIGNATURE + export._chunk(b"IHDR", ihdr)
            + export._chunk(b"IDAT", zlib.compress(b"".join(rows))) + export._chunk(b"IEND", b""))
    p = tmp_path / "f.png"
    p.write_bytes(data)
    assert np.array_equal(export.read_png(str(p)), img)


def test_bad_inputs(tmp_path):
    with pytest.raises(export.ExportError):
        export.write_png(str(tmp_path / "x.jpg"), np.zeros((2, 2, 4), np.uint8))
    with pytest.raises(export.ExportError):
        export.write_png(str(tmp_path / "x.png"), np.zeros((2, 2, 3), np.uint8))
    with pytest.raises(export.ExportError):
        export.write_png(str(tmp_path / "x.png"), np.zeros((2, 2, 4), np.float32))
    (tmp_path / "n.png").write_bytes(b"not a png")
    with pytest.raises(export.ExportError):
        export.read_png(str(tmp_path / "n.png"))
    assert not os.path.exists(str(tmp_path / "x.jpg"))
