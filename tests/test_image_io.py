"""Image output: the EXR holds the linear floats in B, G, R channel planes and the PNG the
reference's sRGB unorm8 encoding (src/core/image.cpp:26-47), both read back here with minimal
parsers of the two formats."""

import os
import struct
import tempfile
import zlib

import numpy as np
import pytest

from minirender_b200 import image_io


def read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, width = 8, b"", 0
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        assert struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0] == zlib.crc32(kind + body)
        if kind == b"IHDR":
            width, height, depth, color = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and color == 2
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(height, 1 + 3 * width)
    assert np.all(raw[:, 0] == 0)
    return raw[:, 1:].reshape(height, width, 3)


def read_exr(path):
    data = open(path, "rb").read()
    magic, version = struct.unpack("<ii", data[:8])
    assert magic == 20000630 and version == 2
    pos, attrs = 8, {}
    while data[pos] != 0:
        end = data.index(b"\x00", pos)
        name = data[pos:end].decode()
        tend = data.index(b"\x00", end + 1)
        size = struct.unpack("<i", data[tend + 1:tend + 5])[0]
        attrs[name] = data[tend + 5:tend + 5 + size]
        pos = tend + 5 + size
    pos += 1
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"])
    width, height = x1 - x0 + 1, y1 - y0 + 1
    assert attrs["compression"] == b"\x00"
    names = [n for n in attrs["channels"].split(b"\x00") if n and len(n) == 1 and n in b"BGR"]
    offsets = struct.unpack(f"<{height}Q", data[pos:pos + 8 * height])
    image = np.zeros((height, width, 3), np.float32)
    for y, off in enumerate(offsets):
        line, size = struct.unpack("<ii", data[off:off + 8])
        planes = np.frombuffer(data[off + 8:off + 8 + size], "<f4").reshape(3, width)
        image[line] = planes[::-1].T  # B, G, R -> R, G, B
    return image, names


def test_exr_and_png_round_trip():
    rng = np.random.default_rng(3)
    linear = rng.uniform(0, 4, (7, 11, 3)).astype(np.float32)
    linear[0, 0] = [0.0, 0.0031308, 1.0]
    with tempfile.TemporaryDirectory() as d:
        image_io.write_exr(os.path.join(d, "a.exr"), linear)
        image_io.write_png(os.path.join(d, "a.png"), linear)
        back, names = read_exr(os.path.join(d, "a.exr"))
        png = read_png(os.path.join(d, "a.png"))
    assert np.array_equal(back, linear)
    assert png.shape == linear.shape
    assert np.array_equal(png, image_io.encode_unorm8(image_io.linear_to_srgb(linear)))
    assert png[0, 0].tolist() == [0, 10, 255]  # 12.92 * 0.0031308 * 255 = 10.3


def test_writers_reject_what_the_reference_rejects():
    with tempfile.TemporaryDirectory() as d:
        with pytest.raises(ValueError, match="nonfinite"):
            image_io.write_exr(os.path.join(d, "b.exr"), np.full((2, 2, 3), np.nan, np.float32))
        with pytest.raises(ValueError, match="limits"):
            image_io.write_png(os.path.join(d, "b.png"), np.zeros((1, 16385, 3), np.float32))
