"""Rendered images: multi-frame accumulation, tonemapping and PNG output.

Mirrors the output side of the reference's headless renderers:

* ``render_frames`` -- HeadlessGpuRenderer.render (gfxlab/playground/HeadlessGpuRenderer.java:
  58-161): frame i is rendered with frameSeed = mix64(seed ^ i * 0x9E3779B97F4A7C15) and
  added into double sums as frame * samplesPerFrame after the warm-up frames.
* ``RenderedImage`` -- HeadlessCpuRenderer.RenderedImage (gfxlab/playground/
  HeadlessCpuRenderer.java:113-175): the mean radiance is scaled per pixel by the
  luminance tonemap 1 - 1 / (1 + (L * pre)^power) divided by L, then by a post factor that
  maps the brightest channel to 1, converted to bytes with the sRGB curve of
  Color.gamma / valueToByteClamp (gfxlab/Color.java:307-329), and written as 8-bit RGBA
  PNG (the reference writes TYPE_INT_ARGB through ImageIO).

The PNG encoder is this module's own (zlib-compressed scanlines with filter type 0); no
image library is needed.
"""
import dataclasses
import struct
import zlib
from pathlib import Path
from typing import Optional

import numpy as np

from .synth import mix64

DEFAULT_TONEMAP_PRE_FACTOR = 2.0 ** -4   # HeadlessCpuRenderer.java:20
DEFAULT_TONEMAP_POWER = 1.0              # HeadlessCpuRenderer.java:21
LUMINANCE = (0.212655, 0.715158, 0.072187)
_GOLDEN = 0x9E3779B97F4A7C15


def frame_seed(seed: int, frame_index: int) -> int:
    """HeadlessGpuRenderer.java:99: mix64(seed ^ frameIndex * 0x9E3779B97F4A7C15)."""
    z = (seed ^ (frame_index * _GOLDEN)) & 0xFFFFFFFFFFFFFFFF
    return int(mix64(np.uint64(z)))


def srgb_gamma(v):
    """Color.gamma: the sRGB transfer curve on linear values (double)."""
    v = np.asarray(v, dtype=np.float64)
    return np.where(v <= 0.0031308, v * 12.92, 1.055 * np.power(np.maximum(v, 0.0031308), 1.0 / 2.4) - 0.055)


def value_to_byte_clamp(v):
    """Color.valueToByteClamp: min((int)(gamma(v) * 255 + 0.5), 255); int truncates
    toward zero as Java's cast does."""
    b = np.trunc(srgb_gamma(v) * 255.0 + 0.5)
    return np.minimum(b, 255.0).astype(np.int64)


def _luminance_scale(r, g, b, pre, power):
    lum = LUMINANCE[0] * r + LUMINANCE[1] * g + LUMINANCE[2] * b
    with np.errstate(divide="ignore", invalid="ignore"):
        p = lum * pre
        mapped = 1.0 - 1.0 / (1.0 + np.power(p, power))
        s = mapped / lum
    return np.where(lum <= 0.0, 0.0, s)


@dataclasses.dataclass
class RenderedImage:
    """Accumulated radiance sums of ``samples`` samples per pixel (3 doubles per pixel)."""
    width: int
    height: int
    samples: int
    sums: np.ndarray

    def mean(self) -> np.ndarray:
        return np.asarray(self.sums, np.float64).reshape(self.height, self.width, 3) / self.samples

    def tonemap_post_factor(self, pre: float = DEFAULT_TONEMAP_PRE_FACTOR,
                            power: float = DEFAULT_TONEMAP_POWER) -> float:
        m = self.mean()
        s = _luminance_scale(m[..., 0], m[..., 1], m[..., 2], pre, power)
        mx = float(np.max(np.max(m, axis=-1) * s)) if m.size else 0.0
        return 1.0 / mx if mx > 0.0 else 1.0

    def to_rgba8(self, pre: float = DEFAULT_TONEMAP_PRE_FACTOR, power: float = DEFAULT_TONEMAP_POWER,
                 post: Optional[float] = None) -> np.ndarray:
        """(height, width, 4) uint8: toBufferedImage's tonemapped pixels, opaque."""
        if post is None:
            post = self.tonemap_post_factor(pre, power)
        m = self.mean()
        scale = _luminance_scale(m[..., 0], m[..., 1], m[..., 2], pre, power) * post
        out = np.empty((self.height, self.width, 4), np.uint8)
        for c in range(3):
            out[..., c] = value_to_byte_clamp(m[..., c] * scale).astype(np.uint8)
        out[..., 3] = 255
        return out

    def write_png(self, path, post: Optional[float] = None) -> Path:
        """writePng: the tonemapped image as an 8-bit RGBA PNG (parent folders created)."""
        p = Path(path)
        p.parent.mkdir(parents=True, exist_ok=True)
        p.write_bytes(encode_png(self.to_rgba8(post=post)))
        return p


def encode_png(rgba: np.ndarray) -> bytes:
    """8-bit RGBA (or RGB) PNG of an (H, W, 4|3) uint8 array."""
    a = np.ascontiguousarray(rgba, np.uint8)
    h, w, ch = a.shape
    if ch not in (3, 4):
        raise ValueError("expected 3 or 4 channels")
    color_type = 6 if ch == 4 else 2

    def chunk(tag, data):
        body = tag + data
        return struct.pack(">I", len(data)) + body + struct.pack(">I", zlib.crc32(body) & 0xFFFFFFFF)

    raw = np.zeros((h, 1 + w * ch), np.uint8)  # filter byte 0 per scanline
    raw[:, 1:] = a.reshape(h, w * ch)
    return (b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, color_type, 0, 0, 0))
            + chunk(b"IDAT", zlib.compress(raw.tobytes(), 6)) + chunk(b"IEND", b""))


def decode_png(data: bytes) -> np.ndarray:
    """Decoder for the PNGs encode_png writes (filter type 0 only)."""
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError("not a PNG")
    pos, idat, w = 8, b"", None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        tag = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            w, h, depth, color, _, _, _ = struct.unpack(">IIBBBBB", body)
            ch = 4 if color == 6 else 3
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + w * ch)
    if np.any(raw[:, 0] != 0):
        raise ValueError("only filter type 0 is supported")
    return raw[:, 1:].reshape(h, w, ch)


def render_frames(tracer, scene, camera, max_depth: int, frames: int, warmup_frames: int = 0,
                  seed: int = 1) -> RenderedImage:
    """HeadlessGpuRenderer.render: frames of ``tracer.render_sample`` (each the mean of the
    tracer's samples per frame) accumulated as frame * samplesPerFrame into double sums."""
    w, h, spf = tracer.width, tracer.height, tracer.samples_per_frame
    sums = np.zeros(w * h * 3, np.float64)
    frame = np.zeros(w * h * 3, np.float32)
    for i in range(max(0, warmup_frames) + max(0, frames)):
        tracer.render_sample(frame, scene, camera, max_depth, i, frame_seed(seed, i))
        if i >= warmup_frames:
            sums += frame.astype(np.float64) * spf
    return RenderedImage(w, h, max(1, frames * spf), sums)
