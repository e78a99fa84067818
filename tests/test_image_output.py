"""Output side of the headless renderers (rtb200.image): frame seeds and accumulation of
HeadlessGpuRenderer.render, the tonemap and byte conversion of HeadlessCpuRenderer.
RenderedImage (checked against a scalar restatement with Java's casts), and the PNG
encoder; plus grid-material plane records and the oracle's material choice on them."""
import math

import numpy as np
import pytest

from oracle import oracle
from rtb200 import image as I
from rtb200 import synth
from rtb200.scene import BvhBuildConfig, BvhBuildMode, GpuScene, MaterialData

M64 = 0xFFFFFFFFFFFFFFFF


def _mix64_py(z):
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def test_frame_seeds_follow_java_long_arithmetic():
    for seed in (1, 42, -7):
        for i in (0, 1, 5, 1000):
            want = _mix64_py((seed ^ (i * 0x9E3779B97F4A7C15)) & M64)
            assert I.frame_seed(seed, i) == want


def _java_pixel(r, g, b, pre, power, post):
    lum = 0.212655 * r + 0.715158 * g + 0.072187 * b
    scale = 0.0 if lum <= 0.0 else (1.0 - 1.0 / (1.0 + math.pow(lum * pre, power))) / lum
    scale *= post

    def byte(x):
        v = x * 12.92 if x <= 0.0031308 else 1.055 * math.pow(x, 1.0 / 2.4) - 0.055
        return min(int(v * 255 + 0.5), 255)
    return byte(r * scale), byte(g * scale), byte(b * scale)


def test_tonemap_matches_a_scalar_restatement():
    rng = np.random.default_rng(3)
    w, h, n = 7, 5, 16
    sums = (rng.exponential(2.0, (h * w * 3)) * n)
    sums[:6] = 0.0                      # black pixels
    sums[6:9] = [900.0, 10.0, 0.5]      # a bright one sets the post factor
    img = I.RenderedImage(w, h, n, sums)
    post = img.tonemap_post_factor()
    mean = sums.reshape(-1, 3) / n
    mx = 0.0
    for r, g, b in mean:
        lum = 0.212655 * r + 0.715158 * g + 0.072187 * b
        s = 0.0 if lum <= 0 else (1.0 - 1.0 / (1.0 + lum * I.DEFAULT_TONEMAP_PRE_FACTOR)) / lum
        mx = max(mx, max(r, g, b) * s)
    assert post == pytest.approx(1.0 / mx, rel=1e-15)
    rgba = img.to_rgba8()
    for k, (r, g, b) in enumerate(mean):
        y, x = divmod(k, w)
        assert tuple(rgba[y, x, :3]) == _java_pixel(r, g, b, I.DEFAULT_TONEMAP_PRE_FACTOR, 1.0, post)
    assert np.all(rgba[..., 3] == 255)


def test_png_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    a = rng.integers(0, 256, (9, 13, 4), dtype=np.uint8)
    data = I.encode_png(a)
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    np.testing.assert_array_equal(I.decode_png(data), a)
    img = I.RenderedImage(4, 3, 1, np.linspace(0.0, 2.0, 36))
    p = img.write_png(tmp_path / "out" / "img.png")
    np.testing.assert_array_equal(I.decode_png(p.read_bytes()), img.to_rgba8())


class _FakeTracer:
    width, height, samples_per_frame = 3, 2, 4

    def __init__(self):
        self.calls = []

    def render_sample(self, rgb, scene, camera, max_depth, frame_index, seed):
        self.calls.append((frame_index, seed))
        rgb[:] = np.float32(frame_index + 0.25)
        return rgb


def test_render_frames_accumulates_like_the_headless_renderer():
    t = _FakeTracer()
    img = I.render_frames(t, None, None, 4, frames=3, warmup_frames=2, seed=9)
    assert [c[0] for c in t.calls] == [0, 1, 2, 3, 4]
    assert [c[1] for c in t.calls] == [I.frame_seed(9, i) for i in range(5)]
    assert img.samples == 12
    np.testing.assert_allclose(img.sums, (2.25 + 3.25 + 4.25) * 4)


def grid_scene():
    """A floor with a 0.5-unit grid under a sphere, inside two walls."""
    s = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 4))
    s.add_sphere((0.0, 0.3, 0.0), 0.3, MaterialData.matte((0.8, 0.8, 0.8)))
    s.add_grid_plane((0.0, -0.2, 0.0), (0.0, 1.0, 0.0), (1.0, 0.0, 0.0), (0.3, 0.0, 1.0),
                     (0.5, 0.5), (0.05, 0.08), MaterialData.matte((0.2, 0.2, 0.2)),
                     MaterialData.matte((0.9, 0.9, 0.9)), MaterialData.matte((0.1, 0.1, 0.6)))
    s.add_plane((0.0, 0.0, 4.0), (0.0, 0.0, -1.0), MaterialData.light((1.0, 1.0, 1.0)))
    return s


def grid_rays(n=4000):
    rng = np.random.default_rng(11)
    o = np.zeros((n, 3))
    o[:, 1] = 1.5
    d = np.stack([rng.uniform(-1.5, 1.5, n), -np.ones(n), rng.uniform(-1.5, 1.5, n)], axis=1)
    return np.concatenate([o, d], axis=1).astype(np.float32)


def test_grid_plane_record_and_oracle_materials():
    s = grid_scene()
    rec = s.plane_data().reshape(-1, 26)[0]
    assert rec[18] == 1.0 and tuple(rec[19:23]) == (0.5, 0.5, 0.05, 0.08)
    e, f = np.array([1.0, 0, 0]), np.array([0.3, 0, 1.0])
    assert rec[13] == np.float32(e @ e) and rec[14] == np.float32(f @ f)
    hits = oracle.trace(s, grid_rays(), oracle.build_bvh(s))
    mats = hits["material"]
    floor = (hits["order"] == s.bounded_primitive_count())  # plane 0 follows the bounded primitives
    cell_id, line_id = int(rec[24]), int(rec[25])
    got = set(mats[floor].tolist())
    assert got == {cell_id, line_id}
    # coordinates of each floor hit in the (e, f) basis decide its material
    t = hits["t"][floor].astype(np.float64)
    r = grid_rays()[floor].astype(np.float64)
    p = r[:, :3] + r[:, 3:] * t[:, None]
    rel = p - np.array([0.0, -0.2, 0.0])
    u = rel[:, 0] - 0.3 * rel[:, 2]
    v = rel[:, 2]
    on_line = (np.mod(u + 0.025, 0.5) < 0.05) | (np.mod(v + 0.04, 0.5) < 0.08)
    agree = (mats[floor] == np.where(on_line, line_id, cell_id))
    assert agree.mean() > 0.995   # float rounding may move points that sit on a line edge


def test_grid_plane_validation():
    s = GpuScene()
    m = MaterialData.matte((0.5, 0.5, 0.5))
    with pytest.raises(ValueError):
        s.add_grid_plane((0, 0, 0), (0, 1, 0), (1, 0, 0), (2, 0, 0), (1, 1), (0.1, 0.1), m, m, m)
    with pytest.raises(ValueError):
        s.add_grid_plane((0, 0, 0), (0, 1, 0), (1, 0, 0), (0, 0, 1), (0, 1), (0.1, 0.1), m, m, m)
