"""Image output: the EXR holds the linear floats in B, G, R channel planes in ZIP blocks of 16
scanlines (the compression the reference asks tinyexr for, src/core/exr_io.cpp:72) and the PNG
the reference's sRGB unorm8 encoding (src/core/image.cpp:26-47), both read back here with minimal
parsers of the two formats; OpenCV's OpenEXR decoder, where present, reads the EXR bit for bit."""

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
    """A minimal reader of what write_exr writes: FLOAT channels B, G, R, ZIP blocks of 16
    scanlines (inflate, undo the delta predictor, re-interleave the two byte halves; a block no
    smaller than its raw size is stored raw)."""
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
    assert attrs["compression"] == b"\x03"  # ZIP, as the reference's tinyexr call writes
    names = [n for n in attrs["channels"].split(b"\x00") if n and len(n) == 1 and n in b"BGR"]
    blocks = (height + 15) // 16
    offsets = struct.unpack(f"<{blocks}Q", data[pos:pos + 8 * blocks])
    image = np.zeros((height, width, 3), np.float32)
    for k, off in enumerate(offsets):
        first, size = struct.unpack("<ii", data[off:off + 8])
        assert first == 16 * k
        lines = min(16, height - first)
        chunk = data[off + 8:off + 8 + size]
        if size < lines * width * 12:
            d = bytearray(zlib.decompress(chunk))
            for i in range(1, len(d)):
                d[i] = (d[i - 1] + d[i] - 128) & 0xFF
            half = (len(d) + 1) // 2
            chunk = bytes(b for pair in zip(d[:half], d[half:] + b"\x00") for b in pair)[:len(d)]
        planes = np.frombuffer(chunk, "<f4").reshape(lines, 3, width)
        image[first:first + lines] = planes[:, ::-1].transpose(0, 2, 1)  # B, G, R -> R, G, B
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


def exr_cases():
    rng = np.random.default_rng(5)
    ramp = np.tile(np.linspace(0, 1, 64, dtype=np.float32)[None, :, None], (37, 1, 3))
    return [rng.uniform(0, 4, (7, 11, 3)),      # incompressible: blocks stored raw
            ramp,                                 # compressible: deflated blocks, a partial last one
            np.zeros((16, 3, 3)),                 # one full block
            rng.uniform(0, 1e6, (1, 1, 3))]


def test_exr_zip_blocks_round_trip():
    with tempfile.TemporaryDirectory() as d:
        for k, image in enumerate(exr_cases()):
            image = image.astype(np.float32)
            path = os.path.join(d, f"{k}.exr")
            image_io.write_exr(path, image)
            back, names = read_exr(path)
            assert np.array_equal(back, image) and sorted(names) == [b"B", b"G", b"R"]
            assert np.array_equal(image_io.read_exr(path), image)
        raw_bytes = exr_cases()[1].size * 4
        assert os.path.getsize(os.path.join(d, "1.exr")) < raw_bytes / 4  # deflated


def test_exr_decodes_in_openexr():
    """OpenCV's OpenEXR decoder (when this image's OpenCV has it) reads the files bit for bit."""
    import subprocess
    import sys
    script = (
        "import os, sys, numpy as np\n"
        "import cv2\n"
        "ok = True\n"
        "for path, ref in zip(sys.argv[1::2], sys.argv[2::2]):\n"
        "    img = cv2.imread(path, cv2.IMREAD_UNCHANGED)\n"
        "    if img is None: sys.exit(3)\n"
        "    ok = ok and np.array_equal(img[..., ::-1], np.load(ref))\n"
        "sys.exit(0 if ok else 1)\n")
    with tempfile.TemporaryDirectory() as d:
        args = []
        for k, image in enumerate(exr_cases()):
            image = image.astype(np.float32)
            path, ref = os.path.join(d, f"{k}.exr"), os.path.join(d, f"{k}.npy")
            image_io.write_exr(path, image)
            np.save(ref, image)
            args += [path, ref]
        env = dict(os.environ, OPENCV_IO_ENABLE_OPENEXR="1")
        result = subprocess.run([sys.executable, "-c", script, *args], env=env,
                                capture_output=True, text=True, timeout=120)
    if result.returncode in (3,) or "No module named 'cv2'" in result.stderr:
        pytest.skip("no OpenEXR decoder in this image's OpenCV")
    assert result.returncode == 0, result.stderr
