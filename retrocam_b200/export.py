"""Frame export: export/FrameExporter.java:51-80 for the library's frames.

The reference reads its display framebuffer back as RGBA8 and hands it to
stb_image_write with a vertical flip.  Here `Context.display` already
returns the RGBA8 image with its rows top first, and `write_png` stores it
as an 8-bit RGBA PNG (filter type 0 on every row, zlib-deflated), creating
missing parent directories as `FrameExporter.ensureParentDirs` does.  JPEG
(the reference's other extension) is not written: no encoder is bundled,
and asking for one raises ExportError.
"""
from __future__ import annotations

import os
import struct
import zlib

import numpy as np

PNG_SIGNATURE = b"\x89PNG\r\n\x1a\n"


class ExportError(RuntimeError):
    """FrameExporter.ExportException."""


def _chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def encode_png(rgba8: np.ndarray, level: int = 6) -> bytes:
    """PNG bytes of an (H, W, 4) uint8 image, first row at the top."""
    a = np.ascontiguousarray(rgba8)
    if a.dtype != np.uint8 or a.ndim != 3 or a.shape[2] != 4:
        raise ExportError(f"expected an (H, W, 4) uint8 image, got {a.dtype} {a.shape}")
    h, w = a.shape[:2]
    rows = np.zeros((h, 1 + 4 * w), np.uint8)   # filter byte 0 (None) per row
    rows[:, 1:] = a.reshape(h, 4 * w)
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)   # 8-bit RGBA, deflate, no interlace
    return (PNG_SIGNATURE + _chunk(b"IHDR", ihdr) + _chunk(b"IDAT", zlib.compress(rows.tobytes(), level))
            + _chunk(b"IEND", b""))


def write_png(path: str, rgba8: np.ndarray) -> None:
    lower = path.lower()
    if lower.endswith((".jpg", ".jpeg")):
        raise ExportError(f"JPEG output is not provided (no encoder bundled): {path}")
    parent = os.path.dirname(os.path.abspath(path))
    os.makedirs(parent, exist_ok=True)
    data = encode_png(rgba8)
    try:
        with open(path, "wb") as f:
            f.write(data)
    except OSError as e:
        raise ExportError(f"failed to write frame: {path}") from e


def _unfilter(kind: int, line: np.ndarray, prev: np.ndarray, bpp: int) -> np.ndarray:
    out = line.astype(np.int32)
    p = prev.astype(np.int32)
    if kind == 0:
        return line
    if kind == 2:
        return ((out + p) & 0xFF).astype(np.uint8)
    res = np.zeros_like(out)
    for i in range(len(out)):
        a = res[i - bpp] if i >= bpp else 0
        b = p[i]
        c = p[i - bpp] if i >= bpp else 0
        if kind == 1:
            pred = a
        elif kind == 3:
            pred = (a + b) >> 1
        elif kind == 4:
            pa, pb, pc = abs(b - c), abs(a - c), abs(a + b - 2 * c)
            pred = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
        else:
            raise ExportError(f"bad PNG filter type {kind}")
        res[i] = (out[i] + pred) & 0xFF
    return res.astype(np.uint8)


def read_png(path: str) -> np.ndarray:
    """The (H, W, 4) uint8 image of an 8-bit RGBA, non-interlaced PNG (the
    files write_png makes; any filter types)."""
    with open(path, "rb") as f:
        data = f.read()
    if not data.startswith(PNG_SIGNATURE):
        raise ExportError(f"not a PNG file: {path}")
    pos, idat = len(PNG_SIGNATURE), []
    w = h = None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        pos += 12 + n
        if kind == b"IHDR":
            w, h, depth, ctype, _, _, interlace = struct.unpack(">IIBBBBB", body)
            if (depth, ctype, interlace) != (8, 6, 0):
                raise ExportError("only 8-bit RGBA non-interlaced PNGs are read")
        elif kind == b"IDAT":
            idat.append(body)
        elif kind == b"IEND":
            break
    if w is None:
        raise ExportError(f"PNG without IHDR: {path}")
    raw = np.frombuffer(zlib.decompress(b"".join(idat)), np.uint8).reshape(h, 1 + 4 * w)
    out = np.zeros((h, 4 * w), np.uint8)
    prev = np.zeros(4 * w, np.uint8)
    for y in range(h):
        out[y] = _unfilter(int(raw[y, 0]), raw[y, 1:], prev, 4)
        prev = out[y]
    return out.reshape(h, w, 4)


def export_frame(ctx, path: str, total_samples: int = 1, exposure: float = 1.0) -> np.ndarray:
    """FrameExporter.exportFrame for a context's last output (what
    RenderPipeline exports after its display pass): tonemap to RGBA8 on the
    GPU, read back, write `path`; returns the image."""
    img = ctx.display(total_samples, exposure)
    write_png(path, img)
    return img
