"""HDR film files: PFM and OpenEXR, from planar float32 buffers (the FrameBuffer
layout: plane after plane, rows top to bottom).

`write_pfm` / `read_pfm` restate Rendering/PfmImage.cs: a "PF" (3 channels)
or "Pf" (1 channel) header, the scale -1.0 for little-endian, then the rows
bottom to top, channels interleaved.

`write_exr` restates Rendering/ExrImage.cs: a single-part scanline OpenEXR
file with ZIP compression in 16-line blocks, channels stored in ordinal name
order. Each block goes through the ImfZip transform (even/odd byte split and
delta predictor), and then zlib; a block that zlib does not shrink is stored
raw. Half channels clamp to +-65504 first. The header carries the attributes
the reference writes, in the same order: channels, chromaticities (Rec.709,
D65), compression, dataWindow, displayWindow, lineOrder, pixelAspectRatio,
screenWindowCenter, screenWindowWidth. zlib output is not byte-identical
across implementations, so the files decode to the same pixels but need not
match byte for byte. `read_exr` decodes the files `write_exr` writes (and
other uncompressed or ZIP scanline files).
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

HALF = 1
FLOAT = 2
LINES_PER_BLOCK = 16      # ZIP block height
HALF_MAX = 65504.0        # largest finite half


# --- PFM ----------------------------------------------------------------------
def write_pfm(path: str, planes: np.ndarray, width: int, height: int, channels: int):
    """PfmImage.Write (PfmImage.cs:27-66)."""
    if channels not in (1, 3):
        raise ValueError(f"PFM supports 1 or 3 channels, got {channels}.")
    planes = np.asarray(planes, np.float32).reshape(-1)
    if planes.size < width * height * channels:
        raise ValueError("Plane buffer smaller than width*height*channels.")
    img = planes[:width * height * channels].reshape(channels, height, width)
    rows = np.ascontiguousarray(img.transpose(1, 2, 0)[::-1]).astype("<f4")   # bottom to top, interleaved
    with open(path, "wb") as f:
        f.write(f"{'PF' if channels == 3 else 'Pf'}\n{width} {height}\n-1.0\n".encode("ascii"))
        f.write(rows.tobytes())


def read_pfm(path: str):
    """PfmImage.Read (PfmImage.cs:72-120): (planes [C, H, W], width, height, channels)."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0

    def token():
        nonlocal pos
        while pos < len(data) and data[pos] in b" \n\r\t":
            pos += 1
        if pos >= len(data):
            raise ValueError("Truncated PFM header.")
        start = pos
        while pos < len(data) and data[pos] not in b" \n\r\t":
            pos += 1
        tok = data[start:pos].decode("ascii")
        pos += 1   # the single terminating whitespace byte
        return tok

    magic = token()
    if magic not in ("PF", "Pf"):
        raise ValueError(f"Not a PFM file (magic '{magic}').")
    channels = 3 if magic == "PF" else 1
    width, height = int(token()), int(token())
    if width <= 0 or height <= 0:
        raise ValueError("Invalid PFM dimensions.")
    scale = float(token())
    if scale == 0.0:
        raise ValueError("Invalid PFM scale.")
    dt = "<f4" if scale < 0 else ">f4"
    n = width * height * channels
    rows = np.frombuffer(data, dt, n, pos).reshape(height, width, channels)[::-1]
    return np.ascontiguousarray(rows.transpose(2, 0, 1)).astype(np.float32), width, height, channels


# --- OpenEXR ------------------------------------------------------------------
def zip_deconstruct(raw: bytes) -> bytes:
    """ExrImage.ZipDeconstruct (ImfZip's predictor): even bytes then odd
    bytes, then each byte minus its predecessor plus 128."""
    a = np.frombuffer(raw, np.uint8)
    t = np.concatenate([a[0::2], a[1::2]])
    if t.size > 1:
        d = t.astype(np.int16)
        d[1:] = (t[1:].astype(np.int16) - t[:-1].astype(np.int16) + 128)
        t = (d & 0xFF).astype(np.uint8)
    return t.tobytes()


def zip_reconstruct(enc: bytes) -> bytes:
    """ExrImage.ZipReconstruct: the inverse of zip_deconstruct."""
    t = np.frombuffer(enc, np.uint8).astype(np.int64)
    if t.size > 1:
        t = (np.cumsum(t - 128) + 128) & 0xFF   # t[i] = t[i-1] + t[i] - 128, mod 256
    t = t.astype(np.uint8)
    half = (t.size + 1) // 2
    raw = np.empty_like(t)
    raw[0::2] = t[:half]
    raw[1::2] = t[half:]
    return raw.tobytes()


def _attribute(name: str, typ: str, payload: bytes) -> bytes:
    return name.encode("ascii") + b"\0" + typ.encode("ascii") + b"\0" + struct.pack("<i", len(payload)) + payload


def _header(width: int, height: int, chans) -> bytes:
    """ExrImage.BuildHeader (ExrImage.cs:158-212)."""
    chl = b"".join(n.encode("ascii") + b"\0" + struct.pack("<iB3xii", t, 0, 1, 1) for n, t, _ in chans) + b"\0"
    chroma = struct.pack("<8f", 0.6400, 0.3300, 0.3000, 0.6000, 0.1500, 0.0600, 0.3127, 0.3290)
    box = struct.pack("<4i", 0, 0, width - 1, height - 1)
    return b"".join([
        _attribute("channels", "chlist", chl),
        _attribute("chromaticities", "chromaticities", chroma),
        _attribute("compression", "compression", bytes([3])),        # ZIP
        _attribute("dataWindow", "box2i", box),
        _attribute("displayWindow", "box2i", box),
        _attribute("lineOrder", "lineOrder", bytes([0])),             # INCREASING_Y
        _attribute("pixelAspectRatio", "float", struct.pack("<f", 1.0)),
        _attribute("screenWindowCenter", "v2f", bytes(8)),
        _attribute("screenWindowWidth", "float", struct.pack("<f", 1.0)),
    ]) + b"\0"


def _half(plane: np.ndarray) -> np.ndarray:
    """ToHalfBits: Math.Clamp to +-65504 (NaN passes), then round to half."""
    p = np.asarray(plane, np.float32)
    c = np.where(np.isnan(p), p, np.clip(p, -HALF_MAX, HALF_MAX))
    return c.astype("<f2")


def write_exr(path: str, width: int, height: int, channels, level: int = 9):
    """ExrImage.Write (ExrImage.cs:52-137). `channels` is a list of (name,
    HALF or FLOAT, plane of width*height floats, rows top to bottom)."""
    if width <= 0 or height <= 0:
        raise ValueError(f"Invalid EXR dimensions {width}x{height}.")
    if not channels:
        raise ValueError("EXR requires at least one channel.")
    seen = set()
    chans = []
    for name, typ, plane in channels:
        if not name or len(name) > 31 or any(c <= " " or c > "~" for c in name):
            raise ValueError(f"Invalid EXR channel name '{name}'.")
        if name in seen:
            raise ValueError(f"Duplicate EXR channel name '{name}'.")
        seen.add(name)
        plane = np.asarray(plane, np.float32).reshape(-1)
        if plane.size != width * height:
            raise ValueError(f"Channel '{name}' plane has {plane.size} floats, expected {width * height}.")
        chans.append((name, int(typ), plane.reshape(height, width)))
    chans.sort(key=lambda c: c[0].encode("ascii"))   # ordinal order
    enc = [(_half(p) if t == HALF else p.astype("<f4")) for _, t, p in chans]
    chunks = []
    for y0 in range(0, height, LINES_PER_BLOCK):
        y1 = min(y0 + LINES_PER_BLOCK, height)
        raw = b"".join(e[y].tobytes() for y in range(y0, y1) for e in enc)   # per line, channels in order
        z = zlib.compress(zip_deconstruct(raw), level)
        payload = z if len(z) < len(raw) else raw
        chunks.append(struct.pack("<ii", y0, len(payload)) + payload)
    header = _header(width, height, chans)
    with open(path, "wb") as f:
        f.write(struct.pack("<Ii", 0x01312F76, 2))
        f.write(header)
        off = 8 + len(header) + 8 * len(chunks)
        for c in chunks:
            f.write(struct.pack("<q", off))
            off += len(c)
        for c in chunks:
            f.write(c)


def write_exr_rgb(path: str, rgb: np.ndarray):
    """ExrImage.WriteRgb: a [3, H, W] buffer as half R, G, B."""
    rgb = np.asarray(rgb, np.float32)
    _, h, w = rgb.shape
    write_exr(path, w, h, [("R", HALF, rgb[0]), ("G", HALF, rgb[1]), ("B", HALF, rgb[2])])


def read_exr(path: str) -> dict:
    """Decodes a single-part scanline EXR with no or ZIP compression: dict of
    channel name -> [H, W] float32."""
    with open(path, "rb") as f:
        data = f.read()
    magic, version = struct.unpack_from("<Ii", data, 0)
    if magic != 0x01312F76:
        raise ValueError("Not an OpenEXR file.")
    pos = 8
    attrs = {}

    def cstr():
        nonlocal pos
        end = data.index(b"\0", pos)
        s = data[pos:end].decode("ascii")
        pos = end + 1
        return s

    while data[pos] != 0:
        name, typ = cstr(), cstr()
        (size,) = struct.unpack_from("<i", data, pos)
        pos += 4
        attrs[name] = (typ, data[pos:pos + size])
        pos += size
    pos += 1
    chl = attrs["channels"][1]
    chans, q = [], 0
    while chl[q] != 0:
        end = chl.index(b"\0", q)
        name = chl[q:end].decode("ascii")
        t = struct.unpack_from("<i", chl, end + 1)[0]
        chans.append((name, t))
        q = end + 1 + 16
    comp = attrs["compression"][1][0]
    if comp not in (0, 3):
        raise ValueError(f"EXR compression {comp} is not supported here.")
    x0, y0, x1, y1 = struct.unpack("<4i", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    lines = LINES_PER_BLOCK if comp == 3 else 1
    nblocks = (h + lines - 1) // lines
    offsets = struct.unpack_from(f"<{nblocks}q", data, pos)
    out = {n: np.zeros((h, w), np.float32) for n, _ in chans}
    bpp = [2 if t == HALF else 4 for _, t in chans]
    for off in offsets:
        ys, size = struct.unpack_from("<ii", data, off)
        payload = data[off + 8:off + 8 + size]
        nl = min(lines, y1 + 1 - ys)
        rawlen = nl * w * sum(bpp)
        raw = payload if len(payload) == rawlen else zip_reconstruct(zlib.decompress(payload))
        p = 0
        for ly in range(nl):
            for (n, t), b in zip(chans, bpp):
                seg = raw[p:p + w * b]
                out[n][ys - y0 + ly] = np.frombuffer(seg, "<f2" if t == HALF else "<f4").astype(np.float32)
                p += w * b
    return out
