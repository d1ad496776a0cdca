"""Image output of the render command: linear EXR and display PNG.

``write_exr`` follows Image::write_exr (src/core/exr_io.cpp:36-110): three 32-bit float channels
named B, G, R (sorted by name, as OpenEXR requires), linear values, nonfinite values rejected. The
reference encodes with tinyexr using ZIP compression (blocks of 16 scanlines, deflated after
OpenEXR's byte split and delta predictor), and so does this writer. ``write_png`` follows Image::write_png (src/core/raster_io.cpp:115-138): 8-bit RGB, each
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


def _zip_block(raw: bytes) -> bytes:
    """OpenEXR's ZIP coding of one block: the bytes split into even- and odd-indexed halves, each
    byte replaced by its difference from the previous one plus 128 (mod 256), then deflated. A
    block that does not shrink is stored as it is, as the format prescribes."""
    b = np.frombuffer(raw, np.uint8)
    t = np.concatenate([b[0::2], b[1::2]]).astype(np.int16)
    d = t.copy()
    d[1:] = (t[1:] - t[:-1] + 128) & 0xFF
    packed = zlib.compress(d.astype(np.uint8).tobytes(), 6)
    return packed if len(packed) < len(raw) else raw


def write_exr(path: str, rgb: np.ndarray):
    """Scanline OpenEXR of a linear (height, width, 3) image: FLOAT channels B, G, R, ZIP
    compression (blocks of 16 scanlines), increasing-Y line order."""
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
              + _attribute("compression", "compression", b"\x03")
              + _attribute("dataWindow", "box2i", box)
              + _attribute("displayWindow", "box2i", box)
              + _attribute("lineOrder", "lineOrder", b"\x00")
              + _attribute("pixelAspectRatio", "float", struct.pack("<f", 1.0))
              + _attribute("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
              + _attribute("screenWindowWidth", "float", struct.pack("<f", 1.0))
              + b"\x00")
    lines = 16
    planes = np.ascontiguousarray(rgb[:, :, ::-1].transpose(0, 2, 1), dtype="<f4")  # B, G, R
    blocks = [_zip_block(planes[y:y + lines].tobytes()) for y in range(0, height, lines)]
    offsets, at = [], len(header) + 8 * len(blocks)
    for block in blocks:
        offsets.append(at)
        at += 8 + len(block)
    with open(path, "wb") as f:
        f.write(header)
        f.write(struct.pack(f"<{len(blocks)}Q", *offsets))
        for k, block in enumerate(blocks):
            f.write(struct.pack("<ii", k * lines, len(block)))
            f.write(block)


# ---- texture input (Image::read, src/core/raster_io.cpp:40-113) ----

def srgb_to_linear(encoded: np.ndarray) -> np.ndarray:
    """srgb_to_linear (src/core/image.cpp:34-40) in float32: nonfinite -> 0, negative -> 0."""
    x = np.asarray(encoded, F32)
    x = np.where(np.isfinite(x), np.maximum(x, F32(0)), F32(0)).astype(F32)
    powered = np.power(((x + F32(0.055)) / F32(1.055)).astype(F32), F32(2.4)).astype(F32)
    return np.where(x <= F32(0.04045), (x / F32(12.92)).astype(F32), powered).astype(F32)


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))


def _unfilter(raw: bytes, height: int, stride: int, bpp: int) -> np.ndarray:
    """PNG scanline filters (types 0-4) undone; (height, stride) bytes."""
    data = np.frombuffer(raw, np.uint8)
    if data.size != height * (stride + 1):
        raise ValueError("PNG image data has the wrong size")
    rows = data.reshape(height, stride + 1)
    out = np.zeros((height, stride), np.int32)
    previous = np.zeros(stride, np.int32)
    for y in range(height):
        kind, line = rows[y, 0], rows[y, 1:].astype(np.int32)
        if kind == 0:
            cur = line
        elif kind == 2:
            cur = (line + previous) & 0xFF
        elif kind == 1:  # Sub: a running sum per byte of the pixel
            padded = np.zeros(((stride + bpp - 1) // bpp) * bpp, np.int32)
            padded[:stride] = line
            cur = (np.cumsum(padded.reshape(-1, bpp), axis=0).reshape(-1) & 0xFF)[:stride]
        elif kind in (3, 4):  # Average, Paeth: pixel by pixel, each pixel's bytes at once
            cur = np.zeros(stride, np.int32)
            left = np.zeros(bpp, np.int32)
            upleft = np.zeros(bpp, np.int32)
            for i in range(0, stride, bpp):
                up = previous[i:i + bpp]
                k = up.size
                if kind == 3:
                    pred = (left[:k] + up) >> 1
                else:
                    pred = _paeth(left[:k], up, upleft[:k])
                cur[i:i + k] = (line[i:i + k] + pred) & 0xFF
                left, upleft = cur[i:i + k], up
        else:
            raise ValueError("PNG uses an unknown filter type")
        out[y] = cur
        previous = cur
    return out


def read_png(path: str) -> np.ndarray:
    """RGB samples of a PNG scaled to [0, 1] as stb_image delivers three channels (grey
    replicated, alpha dropped, palette expanded; 1/2/4-bit grey scaled to 8 bits): (height,
    width, 3) float32. Interlaced (Adam7) files are rejected."""
    data = open(path, "rb").read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("Unsupported or corrupt texture image")
    pos, idat, palette, header = 8, [], None, None
    while pos + 8 <= len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if kind == b"IHDR":
            header = struct.unpack(">IIBBBBB", body[:13])
        elif kind == b"PLTE":
            palette = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif kind == b"IDAT":
            idat.append(body)
        elif kind == b"IEND":
            break
        pos += 12 + n
    if header is None:
        raise ValueError("Unsupported or corrupt texture image")
    width, height, depth, color, _, _, interlace = header
    if width == 0 or height == 0 or width > 16384 or height > 16384 or width * height > 64 * 1024 * 1024:
        raise ValueError("Texture exceeds the 64-megapixel budget")
    if interlace:
        raise ValueError("Interlaced PNG textures are not supported")
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}.get(color)
    if channels is None or depth not in (1, 2, 4, 8, 16):
        raise ValueError("Unsupported or corrupt texture image")
    bits = channels * depth
    stride = (width * bits + 7) // 8
    rows = _unfilter(zlib.decompress(b"".join(idat)), height, stride, max(1, bits // 8))
    if depth == 16:
        samples = (rows[:, 0::2] << 8 | rows[:, 1::2]).reshape(height, width, channels)
        scale = F32(65535)
    elif depth == 8:
        samples = rows.reshape(height, width, channels)
        scale = F32(255)
    else:
        per = 8 // depth
        shifts = np.arange(per - 1, -1, -1) * depth
        unpacked = ((rows[:, :, None] >> shifts) & ((1 << depth) - 1)).reshape(height, -1)[:, :width]
        samples = unpacked.reshape(height, width, 1)
        if color == 0:  # grey scaled to 8 bits
            samples = samples * (255 // ((1 << depth) - 1))
        scale = F32(255)
    if color == 3:
        if palette is None:
            raise ValueError("Unsupported or corrupt texture image")
        rgb = palette[np.minimum(samples[..., 0], len(palette) - 1)].astype(np.int32)
    elif color in (0, 4):
        rgb = np.repeat(samples[..., :1], 3, axis=2)
    else:
        rgb = samples[..., :3]
    return (rgb.astype(F32) / scale).astype(F32)


def _half_to_float(h: np.ndarray) -> np.ndarray:
    return h.astype("<u2").view("<f2").astype(F32)


def read_exr(path: str) -> np.ndarray:
    """(height, width, 3) float32 RGB of a scanline OpenEXR file: HALF or FLOAT channels R, G, B
    (or Y, replicated), compression NONE, ZIPS or ZIP."""
    data = open(path, "rb").read()
    magic, version = struct.unpack("<ii", data[:8])
    if magic != 20000630 or (version & 0xFF) != 2 or version & 0x200:
        raise ValueError("Only scanline OpenEXR files are supported")
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
    compression = attrs["compression"][0]
    lines = {0: 1, 2: 1, 3: 16}.get(compression)
    if lines is None:
        raise ValueError("EXR compression must be NONE, ZIPS or ZIP")
    chlist, channels, k = attrs["channels"], [], 0
    while chlist[k] != 0:
        end = chlist.index(b"\x00", k)
        name = chlist[k:end].decode()
        kind = struct.unpack("<i", chlist[end + 1:end + 5])[0]
        channels.append((name, kind))
        k = end + 17
    sizes = {1: 2, 2: 4}
    if any(kind not in sizes for _, kind in channels):
        raise ValueError("EXR channels must be HALF or FLOAT")
    blocks = (height + lines - 1) // lines
    offsets = struct.unpack(f"<{blocks}Q", data[pos:pos + 8 * blocks])
    planes = {name: np.zeros((height, width), F32) for name, _ in channels}
    for off in offsets:
        y, size = struct.unpack("<ii", data[off:off + 8])
        chunk = data[off + 8:off + 8 + size]
        n = min(lines, y1 + 1 - y)
        expected = n * width * sum(sizes[kind] for _, kind in channels)
        if compression and size < expected:
            raw = np.frombuffer(zlib.decompress(chunk), np.uint8).astype(np.int32)
            raw = np.cumsum(np.concatenate([raw[:1], raw[1:] - 128])) & 0xFF  # predictor
            half = (raw.size + 1) // 2
            interleaved = np.empty(raw.size, np.uint8)
            interleaved[0::2], interleaved[1::2] = raw[:half], raw[half:]
            chunk = interleaved.tobytes()
        at = 0
        for line in range(n):
            for name, kind in channels:
                count = width * sizes[kind]
                values = np.frombuffer(chunk[at:at + count], "<u2" if kind == 1 else "<f4")
                planes[name][y - y0 + line] = _half_to_float(values) if kind == 1 else values
                at += count
    if all(c in planes for c in "RGB"):
        return np.stack([planes["R"], planes["G"], planes["B"]], axis=2)
    if "Y" in planes:
        return np.repeat(planes["Y"][..., None], 3, axis=2)
    raise ValueError("EXR texture needs R, G and B or Y channels")


def read_hdr(path: str) -> np.ndarray:
    """(height, width, 3) float32 RGB of a Radiance RGBE file (flat or run-length scanlines),
    converted as stb_image converts it (mantissa x 2^(exponent - 136))."""
    data = open(path, "rb").read()
    pos = data.index(b"\n\n") + 2
    end = data.index(b"\n", pos)
    parts = data[pos:end].split()
    if len(parts) != 4 or parts[0] != b"-Y" or parts[2] != b"+X":
        raise ValueError("Unsupported or corrupt texture image")
    height, width = int(parts[1]), int(parts[3])
    pos = end + 1
    rgbe = np.zeros((height, width, 4), np.uint8)
    for y in range(height):
        if width >= 8 and width < 32768 and data[pos] == 2 and data[pos + 1] == 2 and not data[pos + 2] & 0x80:
            pos += 4
            for c in range(4):
                x = 0
                while x < width:
                    count = data[pos]
                    pos += 1
                    if count > 128:
                        rgbe[y, x:x + count - 128, c] = data[pos]
                        pos += 1
                        x += count - 128
                    else:
                        rgbe[y, x:x + count, c] = np.frombuffer(data[pos:pos + count], np.uint8)
                        pos += count
                        x += count
        else:
            rgbe[y] = np.frombuffer(data[pos:pos + 4 * width], np.uint8).reshape(width, 4)
            pos += 4 * width
    exponent = rgbe[..., 3].astype(np.int32)
    scale = np.where(exponent > 0, np.ldexp(np.float32(1), exponent - 136), 0).astype(F32)
    return (rgbe[..., :3].astype(F32) * scale[..., None]).astype(F32)


def read_texture(path: str, linear: bool) -> np.ndarray:
    """Image::read (src/core/raster_io.cpp:40-113): (height, width, 3) float32 linear RGB. EXR and
    HDR files must be declared linear; 8- and 16-bit images are converted from sRGB unless
    declared linear."""
    extension = path.lower().rsplit(".", 1)[-1]
    if extension in ("exr", "hdr"):
        if not linear:
            raise ValueError(f"{extension.upper()} textures require linear encoding")
        image = read_exr(path) if extension == "exr" else read_hdr(path)
    else:
        image = read_png(path)
        if not linear:
            image = srgb_to_linear(image)
    if not np.all(np.isfinite(image)):
        raise ValueError("Texture contains nonfinite samples")
    return image
