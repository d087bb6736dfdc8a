"""Render passes as one multi-layer OpenEXR file, written without
OpenImageIO.

`write_multilayer_exr` is io::write_multilayer_exr
(include/psycles/io/image.h:77-84, src/io/openexr.cpp:150-349): every pass
in one scanline, full-float OpenEXR part, channels named
`<view layer>.<pass name>.<component>` (Cycles' convention), ZIP
compression, the same argument checks and error messages.  The reference
hands the interleaved rows to OpenImageIO; this module writes the OpenEXR
2.0 single-part scanline file itself:

  magic 20000630, version 2 (the long-name flag when a channel name exceeds
  31 bytes); header attributes channels (chlist, FLOAT channels sorted by
  name), compression (ZIP), dataWindow / displayWindow (0, 0, w-1, h-1),
  lineOrder (increasing y), pixelAspectRatio 1, screenWindowCenter (0, 0),
  screenWindowWidth 1, Software; a line-offset table; then one chunk per 16
  scanlines: y, packed size, data.

A chunk's raw data holds, per scanline, each channel's row of little-endian
float32 values in channel-list order.  ZIP compression (the OpenEXR file
format's zip scheme) splits the raw bytes into the even- then odd-indexed
bytes, replaces each byte after the first by its difference to the previous
one plus 128 (mod 256), and deflates the result as a zlib stream; a chunk
whose deflated size is not smaller than its raw size is stored raw.

OpenImageIO's colour-space hint (`oiio:ColorSpace` = lin_rec709_scene in the
reference) is an OpenImageIO attribute, not part of the file format, and is
not written; the values are the passes' scene-linear Rec.709 floats
unchanged."""

from __future__ import annotations

import os
import pathlib
import struct
import zlib
from typing import Sequence

import numpy as np

from . import _abi

_PASS_KIND_DEPTH = 1  # contract::PassKind::depth
_FLOAT = 2            # OpenEXR pixel type FLOAT
_ZIP = 3              # OpenEXR ZIP_COMPRESSION
_ZIP_LINES = 16       # scanlines per ZIP chunk
_LONG_NAMES = 0x400   # version flag: names up to 255 bytes


def component_name(kind: int, channels: int, component: int) -> str:
    """Channel suffix of component `component` of a pass
    (openexr.cpp:33-55): X / Y / Z for a normal pass, Z for the first
    component of a depth pass, X / Y for passes of one or two channels,
    R / G / B / A up to four, C<n> beyond."""
    rgba, xyz = "RGBA", "XYZ"
    if kind == _abi.PASS_NORMAL and component < 3:
        return xyz[component]
    if kind == _PASS_KIND_DEPTH and component == 0:
        return "Z"
    if channels <= 4:
        if channels <= 2:
            return xyz[component]
        return rgba[component]
    return f"C{component}"


def _attribute(name: str, type_: str, value: bytes) -> bytes:
    return name.encode() + b"\0" + type_.encode() + b"\0" + struct.pack("<i", len(value)) + value


def zip_compress(raw: bytes) -> bytes:
    """The OpenEXR ZIP scheme's reorder + delta predictor, then zlib."""
    b = np.frombuffer(raw, np.uint8)
    if b.size == 0:
        return zlib.compress(raw)
    half = (b.size + 1) // 2
    t = np.empty_like(b)
    t[:half] = b[0::2]
    t[half:] = b[1::2]
    d = t.copy()
    d[1:] = (t[1:].astype(np.int32) - t[:-1].astype(np.int32) + 128) & 0xFF
    return zlib.compress(d.tobytes())


def zip_decompress(packed: bytes, raw_size: int) -> bytes:
    """Inverse of zip_compress (a chunk stored raw has packed size = raw size)."""
    if len(packed) == raw_size:
        return packed
    d = np.frombuffer(zlib.decompress(packed), np.uint8).astype(np.int64)
    t = ((np.cumsum(d - 128) + 128) & 0xFF).astype(np.uint8)
    t[0] = d[0]
    half = (t.size + 1) // 2
    b = np.empty_like(t)
    b[0::2] = t[:half]
    b[1::2] = t[half:]
    return b.tobytes()


def write_exr(path, width: int, height: int, channels: Sequence[tuple[str, np.ndarray]],
              software: str = "Psycles (B200 CUDA)") -> None:
    """One scanline, full-float, ZIP-compressed OpenEXR part with the named
    channels (each a [height, width] float array, top row first)."""
    named = sorted(channels, key=lambda c: c[0].encode())
    long_names = any(len(n.encode()) > 31 for n, _ in named)
    chlist = b"".join(n.encode() + b"\0" + struct.pack("<iB3xii", _FLOAT, 0, 1, 1) for n, _ in named) + b"\0"
    window = struct.pack("<iiii", 0, 0, width - 1, height - 1)
    header = (struct.pack("<ii", 20000630, 2 | (_LONG_NAMES if long_names else 0)) +
              _attribute("channels", "chlist", chlist) +
              _attribute("compression", "compression", struct.pack("<B", _ZIP)) +
              _attribute("dataWindow", "box2i", window) +
              _attribute("displayWindow", "box2i", window) +
              _attribute("lineOrder", "lineOrder", struct.pack("<B", 0)) +
              _attribute("pixelAspectRatio", "float", struct.pack("<f", 1.0)) +
              _attribute("screenWindowCenter", "v2f", struct.pack("<ff", 0.0, 0.0)) +
              _attribute("screenWindowWidth", "float", struct.pack("<f", 1.0)) +
              _attribute("Software", "string", software.encode()) + b"\0")
    # [height, channel, width] little-endian float32: scanline-major, channel rows within a line
    planes = np.stack([np.asarray(a, dtype="<f4").reshape(height, width) for _, a in named], axis=1)
    chunks = []
    for y0 in range(0, height, _ZIP_LINES):
        raw = np.ascontiguousarray(planes[y0:y0 + _ZIP_LINES]).tobytes()
        packed = zip_compress(raw)
        if len(packed) >= len(raw):
            packed = raw
        chunks.append(struct.pack("<ii", y0, len(packed)) + packed)
    offsets, at = [], len(header) + 8 * len(chunks)
    for c in chunks:
        offsets.append(at)
        at += len(c)
    with open(path, "wb") as f:
        f.write(header)
        f.write(struct.pack(f"<{len(offsets)}Q", *offsets))
        for c in chunks:
            f.write(c)


def write_multilayer_exr(images: Sequence, path, view_layer: str = "ViewLayer") -> None:
    """io::write_multilayer_exr (src/io/openexr.cpp:150-349).  `images` are
    pass images with `.pass_` (kind, name) and `.pixels` [height, width,
    channels] (PassTile, or MemoryOutputSink.tiles' values); raises
    ValueError with the reference's message where it returns false."""
    if not images:
        raise ValueError("no render passes were supplied")
    if not view_layer:
        raise ValueError("the OpenEXR view-layer name is empty")
    if pathlib.Path(os.fspath(path)).suffix not in (".exr", ".EXR"):
        raise ValueError("the output path does not have an .exr extension")
    first = np.asarray(images[0].pixels)
    height, width = (int(first.shape[0]), int(first.shape[1])) if first.ndim >= 2 else (0, 0)
    if width == 0 or height == 0 or width > 2**31 - 1 or height > 2**31 - 1:
        raise ValueError("the render extent is invalid for OpenEXR")
    channels, seen = [], set()
    for image in images:
        px = np.asarray(image.pixels, dtype=np.float32)
        if px.ndim == 2:
            px = px[..., None]
        if px.shape[0] != height or px.shape[1] != width:
            raise ValueError("all OpenEXR passes must have the same extent")
        if px.shape[2] == 0:
            raise ValueError("an OpenEXR pass has no channels")
        name = image.pass_.name
        if not name:
            raise ValueError("an OpenEXR pass has an empty name")
        n = int(px.shape[2])
        for component in range(n):
            channel = f"{view_layer}.{name}.{component_name(image.pass_.kind, n, component)}"
            if channel in seen:
                raise ValueError(f"duplicate OpenEXR channel name: {channel}")
            seen.add(channel)
            channels.append((channel, px[..., component]))
    if any(len(c.encode()) > 255 for c, _ in channels):
        raise ValueError("an OpenEXR channel name exceeds 255 bytes")
    write_exr(path, width, height, channels)


def read_exr(path) -> dict[str, np.ndarray]:
    """Channels of a file write_exr wrote (the inverse of its layout: one
    scanline part of FLOAT channels, uncompressed or ZIP), name -> [height,
    width] float32."""
    data = pathlib.Path(path).read_bytes()
    magic, version = struct.unpack_from("<ii", data, 0)
    if magic != 20000630 or (version & 0xFF) != 2:
        raise ValueError("not a single-part OpenEXR 2 file")
    at, attrs = 8, {}
    while data[at] != 0:
        name_end = data.index(b"\0", at)
        type_end = data.index(b"\0", name_end + 1)
        (size,) = struct.unpack_from("<i", data, type_end + 1)
        attrs[data[at:name_end].decode()] = data[type_end + 5:type_end + 5 + size]
        at = type_end + 5 + size
    at += 1
    names, c = [], attrs["channels"]
    k = 0
    while c[k] != 0:
        e = c.index(b"\0", k)
        ptype = struct.unpack_from("<i", c, e + 1)[0]
        if ptype != _FLOAT:
            raise ValueError("only FLOAT channels are read")
        names.append(c[k:e].decode())
        k = e + 17
    compression = attrs["compression"][0]
    x0, y0, x1, y1 = struct.unpack("<iiii", attrs["dataWindow"])
    width, height = x1 - x0 + 1, y1 - y0 + 1
    lines = {0: 1, 3: _ZIP_LINES}[compression]
    chunks = (height + lines - 1) // lines
    offsets = struct.unpack_from(f"<{chunks}Q", data, at)
    out = np.empty((height, len(names), width), np.float32)
    for off in offsets:
        y, size = struct.unpack_from("<ii", data, off)
        n = min(lines, height - (y - y0))
        raw_size = n * len(names) * width * 4
        raw = zip_decompress(data[off + 8:off + 8 + size], raw_size) if compression == _ZIP \
            else data[off + 8:off + 8 + size]
        out[y - y0:y - y0 + n] = np.frombuffer(raw, "<f4").reshape(n, len(names), width)
    return {name: out[:, i, :] for i, name in enumerate(names)}
