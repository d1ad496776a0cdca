"""Image output of the render command: linear EXR and display PNG.

``write_exr`` follows Image::write_exr (src/core/exr_io.cpp:36-110): three 32-bit float channels
named B, G, R (sorted by name, as OpenEXR requires), linear values, nonfinite values rejected. The
reference encodes with tinyexr using ZIP compression; this writer stores the scanlines
uncompressed (compression NONE), which every OpenEXR reader accepts and which carries the same
pixels. ``write_png`` follows Image::write_png (src/core/raster_io.cpp:115-138): 8-bit RGB, each
channel through linear_to_srgb and a rounded unorm8 encoding (src/core/image.cpp:26-47); the
reference encodes with stb_image_write, this writer with zlib (filter 0 per row).
"""

from __future__ import annotations

import struct
import zlib

import numpy as np

F32 = np.float32


def linear_to_srgb(linear: np.ndarray) -> np.ndarray:
    """linear_to_srgb (src/core/image.cpp:26-32) in float32: nonfinite -> 0, negative -> 0."""
    x = np.asarray(linear, F32)
    x = np.where(np.isfinite(x), np.maximum(x, F32(0)), F32(0)).astype(F32)
    powered = (F32(1.055) * np.power(x, F32(1.0) / F32(2.4)).astype(F32) - F32(0.055)).astype(F32)
    return np.where(x <= F32(0.0031308), F32(12.92) * x, powered).astype(F32)


def encode_unorm8(value: np.ndarray) -> np.ndarray:
    """encode_unorm8 (src/core/image.cpp:42-47): clamp to [0, 1], scale by 255, round half away
    from zero; nonfinite -> 0."""
    v = np.asarray(value, F32)
    v = np.where(np.isfinite(v), np.clip(v, F32(0), F32(1)), F32(0)).astype(F32) * F32(255)
    return np.floor(v.astype(np.float64) + 0.5).astype(np.uint8)  # values are >= 0


def _png_chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data))


def write_png(path: str, rgb: np.ndarray):
    """8-bit sRGB PNG of a linear (height, width, 3) image."""
    rgb = np.asarray(rgb, F32)
    height, width = rgb.shape[:2]
    if width > 16384 or height > 16384 or width == 0 or height == 0:
        raise ValueError("PNG dimensions exceed texture limits")
    pixels = encode_unorm8(linear_to_srgb(rgb)).reshape(height, width * 3)
    raw = b"".join(b"\x00" + row.tobytes() for row in pixels)
    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(_png_chunk(b"IHDR", struct.pack(">IIBBBBB", width, height, 8, 2, 0, 0, 0)))
        f.write(_png_chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(_png_chunk(b"IEND", b""))


def _attribute(name: str, kind: str, value: bytes) -> bytes:
    return name.encode() + b"\x00" + kind.encode() + b"\x00" + struct.pack("<i", len(value)) + value


def write_exr(path: str, rgb: np.ndarray):
    """Scanline OpenEXR of a linear (height, width, 3) image: FLOAT channels B, G, R, no
    compression, increasing-Y line order, one scanline per block."""
    rgb = np.asarray(rgb, F32)
    height, width = rgb.shape[:2]
    if width == 0 or height == 0 or width * height > 2 ** 31 - 1:
        raise ValueError("EXR dimensions exceed codec limits")
    if not np.all(np.isfinite(rgb)):
        raise ValueError("EXR output contains nonfinite radiance")
    channels = b"".join(name + b"\x00" + struct.pack("<iBBBBii", 2, 0, 0, 0, 0, 1, 1)
                        for name in (b"B", b"G", b"R")) + b"\x00"
    box = struct.pack("<iiii", 0, 0, width - 1, height - 1)
    header = (struct.pack("<ii", 20000630, 2)
              + _attribute("channels", "chlist", channels)
              + _attribute("compression", "compression", b"\x00")
              + _attribute("dataWindow", "box2i", box)
              + _attribute("displayWindow", "box2i", box)
              + _attribute("lineOrder", "lineOrder", b"\x00")
              + _attribute("pixelAspectRatio", "float", struct.pack("<f", 1.0))
              + _attribute("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
              + _attribute("screenWindowWidth", "float", struct.pack("<f", 1.0))
              + b"\x00")
    line_bytes = width * 3 * 4
    block = 8 + line_bytes
    first = len(header) + 8 * height
    offsets = struct.pack(f"<{height}Q", *(first + y * block for y in range(height)))
    planes = np.ascontiguousarray(rgb[:, :, ::-1].transpose(0, 2, 1), dtype="<f4")  # B, G, R
    with open(path, "wb") as f:
        f.write(header)
        f.write(offsets)
        for y in range(height):
            f.write(struct.pack("<ii", y, line_bytes))
            f.write(planes[y].tobytes())
