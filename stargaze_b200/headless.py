"""Headless capture: `stargaze render` (src/headless.rs:115-221) without a
graphics API. Renders a frame to a sample count through a PathTracer,
resolves the display into an 8-bit sRGB image with sg_display and writes it
as a PNG with an sRGB chunk, returning the reference's `Capture` record
(src/headless.rs:47-63) for the fields that exist here.
"""
from __future__ import annotations

import struct
import time
import zlib
from pathlib import Path

import numpy as np

from .pathtracer import PathTracer
from .scene import Frame


def write_png(path, rgba: np.ndarray) -> None:
    """8-bit RGBA PNG with an sRGB chunk, perceptual intent (as
    png::Encoder::set_source_srgb, src/headless.rs:196)."""
    rgba = np.ascontiguousarray(rgba, dtype=np.uint8)
    h, w, c = rgba.shape
    if c != 4:
        raise ValueError("rgba must be (height, width, 4)")

    def chunk(kind: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)

    raw = b"".join(b"\x00" + rgba[y].tobytes() for y in range(h))
    png = b"\x89PNG\r\n\x1a\n"
    png += chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0))
    png += chunk(b"sRGB", b"\x00")
    png += chunk(b"IDAT", zlib.compress(raw, 6))
    png += chunk(b"IEND", b"")
    Path(path).write_bytes(png)


def read_png_rgba(path) -> np.ndarray:
    """Reads back a PNG written by write_png (filter type 0 rows only)."""
    data = Path(path).read_bytes()
    pos, idat, w, h = 8, b"", 0, 0
    while pos < len(data):
        (length,) = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + length]
        if kind == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
        elif kind == b"IDAT":
            idat += body
        pos += 12 + length
    raw = np.frombuffer(zlib.decompress(idat), dtype=np.uint8).reshape(h, 1 + 4 * w)
    return raw[:, 1:].reshape(h, w, 4).copy()


def capture(tracer: PathTracer, frame: Frame, samples: int, output, size: tuple[int, int] | None = None) -> dict:
    """Encode `frame` until the accumulation holds `samples` samples (the
    tracer's sample limit caps it, as the reference's request does), resolve
    the display at `size` (default the trace size) and write `output`."""
    if not 1 <= samples <= 4096:
        raise ValueError("samples must be 1-4096")
    start = time.perf_counter()
    while tracer.samples() < samples:
        before = tracer.samples()
        tracer.encode(frame)
        if tracer.samples() == before:
            break
    rgba = tracer.display(size)
    render_ms = (time.perf_counter() - start) * 1e3
    write_png(output, rgba)
    trace_w, trace_h = tracer.size()
    return {"version": 1, "width": int(rgba.shape[1]), "height": int(rgba.shape[0]), "trace_width": trace_w,
            "trace_height": trace_h, "samples": tracer.samples(), "exposure": tracer.exposure(),
            "render_ms": render_ms}


__all__ = ["write_png", "read_png_rgba", "capture"]
