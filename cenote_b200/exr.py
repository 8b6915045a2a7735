"""Minimal OpenEXR scanline writer/reader: the writer stores FLOAT or HALF
channels uncompressed, one scanline per block — enough for the renderer's
linear output (crates/cenote/src/output.rs writes the same channel set:
R, G, B, A, albedo.*, normal.*, Z); the reader also takes RLE, ZIPS and ZIP
(16-line) blocks and single-level tiles, enough for the reference's goldens
and the corpus's sky images. Written from the OpenEXR file-layout document.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

MAGIC = 20000630
HALF = 1
FLOAT = 2


def _attr(name: str, typ: str, data: bytes) -> bytes:
    return name.encode() + b"\0" + typ.encode() + b"\0" + struct.pack("<i", len(data)) + data


def write_exr(path, layers: dict[str, np.ndarray], compression: int = 0) -> None:
    """layers: channel name -> (H, W) array, float16 (stored HALF) or
    anything else (stored FLOAT). Channels are stored in sorted-name order,
    as the format requires. compression 0 = none."""
    names = sorted(layers)
    h, w = next(iter(layers.values())).shape
    kinds = {n: HALF if np.asarray(layers[n]).dtype == np.float16 else FLOAT for n in names}
    chlist = b"".join(n.encode() + b"\0" + struct.pack("<iB3xii", kinds[n], 0, 1, 1) for n in names) + b"\0"
    header = struct.pack("<ii", MAGIC, 2)
    header += _attr("channels", "chlist", chlist)
    header += _attr("compression", "compression", bytes([compression]))
    header += _attr("dataWindow", "box2i", struct.pack("<iiii", 0, 0, w - 1, h - 1))
    header += _attr("displayWindow", "box2i", struct.pack("<iiii", 0, 0, w - 1, h - 1))
    header += _attr("lineOrder", "lineOrder", bytes([0]))
    header += _attr("pixelAspectRatio", "float", struct.pack("<f", 1.0))
    header += _attr("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0))
    header += _attr("screenWindowWidth", "float", struct.pack("<f", 1.0))
    # ACEScg (AP1) chromaticities: red, green, blue, white (D60).
    header += _attr("chromaticities", "chromaticities",
                    struct.pack("<8f", 0.713, 0.293, 0.165, 0.830, 0.128, 0.044, 0.32168, 0.33767))
    header += b"\0"
    data = [np.ascontiguousarray(layers[n], np.float16 if kinds[n] == HALF else np.float32) for n in names]
    offsets_pos = len(header)
    first = offsets_pos + 8 * h
    blocks, offsets = [], []
    pos = first
    for y in range(h):
        payload = b"".join(d[y].tobytes() for d in data)
        block = struct.pack("<ii", y, len(payload)) + payload
        offsets.append(pos)
        blocks.append(block)
        pos += len(block)
    with open(path, "wb") as f:
        f.write(header)
        f.write(struct.pack(f"<{h}Q", *offsets))
        for b in blocks:
            f.write(b)


def write_aov_exr(path, beauty, albedo, normal, depth) -> None:
    """The CLI's multi-layer output (crates/cenote/src/output.rs:61-135):
    beauty as bare R/G/B/A, the guides as albedo.R/G/B and normal.X/Y/Z, all
    in f16, and depth as the bare f32 Z (+inf marks the sky)."""
    layers = {c: beauty[..., k].astype(np.float16) for k, c in enumerate("RGBA")}
    layers.update({f"albedo.{c}": albedo[..., k].astype(np.float16) for k, c in enumerate("RGB")})
    layers.update({f"normal.{c}": normal[..., k].astype(np.float16) for k, c in enumerate("XYZ")})
    layers["Z"] = np.asarray(depth, np.float32)
    write_exr(path, layers)


def _rle_decode(src: bytes, n: int) -> bytes:
    out = bytearray()
    i = 0
    while i < len(src) and len(out) < n:
        c = struct.unpack("<b", src[i:i + 1])[0]
        i += 1
        if c < 0:
            out += src[i:i - c]
            i += -c
        else:
            out += src[i:i + 1] * (c + 1)
            i += 1
    return _unpredict(bytes(out))


def _unpredict(data: bytes) -> bytes:
    """Reverse OpenEXR's RLE/ZIP pre-processing: the byte-delta predictor,
    then the split of even and odd bytes into two halves."""
    t = np.frombuffer(data, np.uint8).astype(np.int64)
    if len(t) == 0:
        return b""
    d = t - 128
    d[0] = t[0]
    buf = (np.cumsum(d) & 0xFF).astype(np.uint8)
    half = (len(buf) + 1) // 2
    res = np.empty(len(buf), np.uint8)
    res[0::2] = buf[:half]
    res[1::2] = buf[half:]
    return res.tobytes()


def _zip_decode(src: bytes) -> bytes:
    return _unpredict(zlib.decompress(src))


def read_exr(path) -> dict[str, np.ndarray]:
    """Scanline or single-level tiled images of HALF, FLOAT or UINT channels,
    compression none, RLE, ZIPS or ZIP."""
    raw = open(path, "rb").read()
    assert struct.unpack("<i", raw[:4])[0] == MAGIC
    pos = 8
    attrs = {}
    while raw[pos] != 0:
        e = raw.index(b"\0", pos)
        name = raw[pos:e].decode()
        e2 = raw.index(b"\0", e + 1)
        typ = raw[e + 1:e2].decode()
        size = struct.unpack("<i", raw[e2 + 1:e2 + 5])[0]
        attrs[name] = (typ, raw[e2 + 5:e2 + 5 + size])
        pos = e2 + 5 + size
    pos += 1
    chans = []
    cl = attrs["channels"][1]
    i = 0
    while cl[i] != 0:
        e = cl.index(b"\0", i)
        name = cl[i:e].decode()
        ptype = struct.unpack("<i", cl[e + 1:e + 5])[0]
        chans.append((name, ptype))
        i = e + 17
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"][1])
    w, h = x1 - x0 + 1, y1 - y0 + 1
    comp = attrs["compression"][1][0]
    sizes = {2: 4, 1: 2, 0: 4}
    out = {n: np.zeros((h, w), np.float32) for n, _ in chans}

    def unpack(payload, n, rows, cols, y_at, x_at):
        expect = sum(sizes[t] for _, t in chans) * rows * cols
        if comp == 1 and n < expect:
            payload = _rle_decode(payload, expect)
        elif comp in (2, 3) and n < expect:
            payload = _zip_decode(payload)
        elif comp not in (0, 1, 2, 3):
            raise ValueError(f"{path}: EXR compression {comp} is not read")
        p = 0
        for r in range(rows):
            for name, t in chans:
                if t == 2:
                    v = np.frombuffer(payload[p:p + 4 * cols], "<f4")
                elif t == 1:
                    v = np.frombuffer(payload[p:p + 2 * cols], "<f2").astype(np.float32)
                else:
                    v = np.frombuffer(payload[p:p + 4 * cols], "<u4").astype(np.float32)
                out[name][y_at + r, x_at:x_at + cols] = v
                p += sizes[t] * cols

    if "tiles" in attrs:  # single-level tiled image
        tx, ty = struct.unpack("<II", attrs["tiles"][1][:8])
        ntx, nty = (w + tx - 1) // tx, (h + ty - 1) // ty
        offsets = struct.unpack(f"<{ntx * nty}Q", raw[pos:pos + 8 * ntx * nty])
        for off in offsets:
            cx, cy, _, _, n = struct.unpack("<iiiii", raw[off:off + 20])
            cols, rows = min(tx, w - cx * tx), min(ty, h - cy * ty)
            unpack(raw[off + 20:off + 20 + n], n, rows, cols, cy * ty, cx * tx)
        return out
    lines = 16 if comp == 3 else 1  # scanlines per block
    blocks = (h + lines - 1) // lines
    offsets = struct.unpack(f"<{blocks}Q", raw[pos:pos + 8 * blocks])
    for off in offsets:
        y, n = struct.unpack("<ii", raw[off:off + 8])
        unpack(raw[off + 8:off + 8 + n], n, min(lines, h - (y - y0)), w, y - y0, 0)
    return out
