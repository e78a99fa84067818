"""Seeded synthetic scenes for the five benchmark workloads and the reference's GI_TEST.

The reference measures on no public data set; its workloads here are synthetic scenes of
the stated shapes, generated from a counter-based splitmix64 stream
(``u = (mix64(key + i * golden) >> 11) * 2**-53``) keyed by (seed, workload, scene,
field).  Only IEEE + - * / and sqrt are used, never transcendental functions, so a scene is
bit-identical on every host that runs this numpy.

Workloads (sizes fixed by the benchmark description; "(chosen)" marks values it leaves open):
  * ``plain``      64 Lambertian spheres (centres U[-1,1]^3, r U[0.02,0.08], albedo
                   U[0.2,0.9]^3) + an emitter (r 0.3 at (0,2,0), emission 10) in a closed room
                   of six half-spaces at +-3 (albedo 0.7, chosen); camera at (0,0,-2.9) looking
                   +z with a 60 degree vertical field of view (chosen); 256x256, 16 spp, depth 4.
  * ``hetero``     10k primitives: 40 % spheres (r U[0.01,0.05], chosen), 30 % boxes (extents
                   U[0.01,0.1]), 15 % affine spheres + 15 % affine boxes (uniform random
                   rotation, per-axis scale U[0.5,2] x base half-size U[0.01,0.05], chosen);
                   same room and emitter; 1024x1024, 64 spp, depth 8.
  * ``scale``      1M primitives of the same mix, sizes scaled by 0.1 (chosen), centres from
                   64 clusters (centres U[0,1]^3, sigma 0.05 via a 12-uniform Irwin-Hall
                   approximation of the normal, chosen) clamped to the unit cube; room walls at
                   -0.5 and 1.5 (chosen); 1920x1080, 256 spp, depth 8.
  * ``batched``    64 scenes, N = floor(exp(U[ln 1e3, ln 2e5])) primitives of the mix,
                   resolution from {256^2, 512^2, 1024^2}, spp from {16, 64}, depth 6.
  * ``adjoint``    4096 primitives of the mix, 512x512, 32 spp, depth 6.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .scene import BvhBuildConfig, BvhBuildMode, GpuCamera, GpuScene, MaterialData

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def mix64(z):
    """splitmix64 finaliser on uint64 scalars or arrays (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = np.asarray(z, dtype=np.uint64) + _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


WORKLOAD_IDS = {"plain": 1, "hetero": 2, "scale": 3, "batched": 4, "adjoint": 5, "test": 9}


class Stream:
    """Uniform doubles in [0, 1) from a counter stream keyed by (seed, workload, scene, field)."""

    def __init__(self, seed: int, workload: int, scene: int, field: int):
        with np.errstate(over="ignore"):
            k = mix64(np.uint64(seed))
            k = mix64(k ^ np.uint64(workload))
            k = mix64(k ^ np.uint64((scene << 16) | field))
        self.key = k
        self.pos = 0

    def uniform(self, n: int) -> np.ndarray:
        with np.errstate(over="ignore"):
            i = np.arange(self.pos, self.pos + n, dtype=np.uint64)
            v = mix64(self.key + i * _GOLDEN)
        self.pos += n
        return (v >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)

    def range(self, n: int, lo: float, hi: float, shape=None) -> np.ndarray:
        u = self.uniform(n if shape is None else int(np.prod(shape)))
        u = lo + (hi - lo) * u
        return u if shape is None else u.reshape(shape)


def random_rotations(stream: Stream, n: int) -> np.ndarray:
    """Uniform random rotations: quaternions by rejection from the 4-cube, normalised."""
    out = np.empty((n, 4), dtype=np.float64)
    filled = 0
    while filled < n:
        m = max(2 * (n - filled), 16)
        q = stream.range(4 * m, -1.0, 1.0, (m, 4))
        l2 = ((q[:, 0] * q[:, 0] + q[:, 1] * q[:, 1]) + q[:, 2] * q[:, 2]) + q[:, 3] * q[:, 3]
        q = q[(l2 <= 1.0) & (l2 > 1e-6)]
        take = min(len(q), n - filled)
        out[filled:filled + take] = q[:take]
        filled += take
    norm = np.sqrt(((out[:, 0] * out[:, 0] + out[:, 1] * out[:, 1]) + out[:, 2] * out[:, 2])
                   + out[:, 3] * out[:, 3])
    out /= norm[:, None]
    w, x, y, z = out[:, 0], out[:, 1], out[:, 2], out[:, 3]
    r = np.empty((n, 3, 3))
    r[:, 0, 0] = 1 - 2 * (y * y + z * z)
    r[:, 0, 1] = 2 * (x * y - z * w)
    r[:, 0, 2] = 2 * (x * z + y * w)
    r[:, 1, 0] = 2 * (x * y + z * w)
    r[:, 1, 1] = 1 - 2 * (x * x + z * z)
    r[:, 1, 2] = 2 * (y * z - x * w)
    r[:, 2, 0] = 2 * (x * z - y * w)
    r[:, 2, 1] = 2 * (y * z + x * w)
    r[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return r


@dataclasses.dataclass
class Workload:
    name: str
    scene: GpuScene
    camera: GpuCamera
    width: int
    height: int
    spp: int
    max_depth: int
    frame_seed: int = 1
    frame_index: int = 0


def camera_looking_z(pos, aspect=1.0, vfov_deg=60.0) -> GpuCamera:
    """Pinhole camera looking along +z.  The kernel multiplies the horizontal sensor
    coordinate by the aspect ratio itself, so right and up share tan(vfov / 2)."""
    t = math.tan(math.radians(vfov_deg) * 0.5)
    return GpuCamera(tuple(pos), (0.0, 0.0, 1.0), (t, 0.0, 0.0), (0.0, t, 0.0))


def add_room(scene: GpuScene, lo: float, hi: float, albedo: float = 0.7) -> None:
    m = scene.register_material(MaterialData.matte((albedo, albedo, albedo)))
    pts = [(lo, 0, 0), (hi, 0, 0), (0, lo, 0), (0, hi, 0), (0, 0, lo), (0, 0, hi)]
    nrm = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    scene.add_planes(pts, nrm, [m] * 6)


def _lambert_ids(scene: GpuScene, albedo: np.ndarray) -> np.ndarray:
    rows = np.zeros((len(albedo), 13))
    rows[:, 0:3] = albedo
    rows[:, 12] = 1.5
    return scene.register_materials(rows)


def add_mix(scene: GpuScene, n: int, seed: int, workload: int, scene_id: int,
            centres_lo=-1.0, centres_hi=1.0, size_scale=1.0, clusters=0, sigma=0.05):
    """Adds n primitives in the 40/30/15/15 sphere/box/affine-sphere/affine-box mix."""
    ns = int(round(n * 0.4))
    nb = int(round(n * 0.3))
    nas = (n - ns - nb) // 2
    nab = n - ns - nb - nas

    def centres(field, k):
        st = Stream(seed, workload, scene_id, field)
        if clusters <= 0:
            return st.range(3 * k, centres_lo, centres_hi, (k, 3))
        cs = Stream(seed, workload, scene_id, 99).range(3 * clusters, centres_lo, centres_hi,
                                                          (clusters, 3))
        pick = np.minimum((st.uniform(k) * clusters).astype(np.int64), clusters - 1)
        u12 = st.uniform(12 * 3 * k).reshape(k, 3, 12)
        g = u12[:, :, 0].copy()
        for j in range(1, 12):  # sequential sum: identical on every host
            g = g + u12[:, :, j]
        g = g - 6.0
        return np.clip(cs[pick] + sigma * g, centres_lo, centres_hi)

    def albedo(field, k):
        return Stream(seed, workload, scene_id, field).range(3 * k, 0.2, 0.9, (k, 3))

    if ns:
        c = centres(1, ns)
        r = Stream(seed, workload, scene_id, 2).range(ns, 0.01, 0.05) * size_scale
        scene.add_spheres(c, r, _lambert_ids(scene, albedo(3, ns)))
    if nb:
        c = centres(4, nb)
        e = Stream(seed, workload, scene_id, 5).range(3 * nb, 0.01, 0.1, (nb, 3)) * size_scale
        scene.add_boxes(c - 0.5 * e, c + 0.5 * e, _lambert_ids(scene, albedo(6, nb)))
    for kind, k, f0 in (("sphere", nas, 10), ("box", nab, 20)):
        if not k:
            continue
        c = centres(f0, k)
        rot = random_rotations(Stream(seed, workload, scene_id, f0 + 1), k)
        base = Stream(seed, workload, scene_id, f0 + 2).range(k, 0.01, 0.05) * size_scale
        s = Stream(seed, workload, scene_id, f0 + 3).range(3 * k, 0.5, 2.0, (k, 3)) * base[:, None]
        t = np.zeros((k, 3, 4))
        t[:, :, :3] = rot * s[:, None, :]
        t[:, :, 3] = c
        ids = _lambert_ids(scene, albedo(f0 + 4, k))
        if kind == "sphere":
            scene.add_transformed_spheres(t, ids)
        else:
            scene.add_transformed_boxes(t, ids)


def plain_workload(seed: int = 1) -> Workload:
    cfg = BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 4)
    s = GpuScene(cfg)
    w = WORKLOAD_IDS["plain"]
    c = Stream(seed, w, 0, 1).range(64 * 3, -1.0, 1.0, (64, 3))
    r = Stream(seed, w, 0, 2).range(64, 0.02, 0.08)
    s.add_spheres(c, r, _lambert_ids(s, Stream(seed, w, 0, 3).range(64 * 3, 0.2, 0.9, (64, 3))))
    s.add_sphere((0.0, 2.0, 0.0), 0.3, MaterialData.light((10.0, 10.0, 10.0)))
    add_room(s, -3.0, 3.0)
    return Workload("plain", s, camera_looking_z((0.0, 0.0, -2.9)), 256, 256, 16, 4)


def hetero_scene(n: int, seed: int, workload: int, scene_id: int, leaf_size: int = 4,
                 mode=BvhBuildMode.WEIGHTED_SAH) -> GpuScene:
    s = GpuScene(BvhBuildConfig.weighted(leaf_size=leaf_size, mode=mode))
    add_mix(s, n, seed, workload, scene_id)
    s.add_sphere((0.0, 2.0, 0.0), 0.3, MaterialData.light((10.0, 10.0, 10.0)))
    add_room(s, -3.0, 3.0)
    return s


def hetero_workload(seed: int = 1, n: int = 10000, width: int = 1024, height: int = 1024,
                    spp: int = 64, depth: int = 8) -> Workload:
    s = hetero_scene(n, seed, WORKLOAD_IDS["hetero"], 0)
    return Workload("hetero", s, camera_looking_z((0.0, 0.0, -2.9), width / height),
                    width, height, spp, depth)


def scale_workload(seed: int = 1, n: int = 1_000_000, width: int = 1920, height: int = 1080,
                   spp: int = 256, depth: int = 8) -> Workload:
    s = GpuScene(BvhBuildConfig.weighted(leaf_size=4))
    add_mix(s, n, seed, WORKLOAD_IDS["scale"], 0, 0.0, 1.0, size_scale=0.1, clusters=64)
    s.add_sphere((0.5, 1.3, 0.5), 0.1, MaterialData.light((10.0, 10.0, 10.0)))
    add_room(s, -0.5, 1.5)
    return Workload("scale", s, camera_looking_z((0.5, 0.5, -0.45), width / height),
                    width, height, spp, depth)


def batched_workloads(seed: int = 1, count: int = 64):
    out = []
    w = WORKLOAD_IDS["batched"]
    for i in range(count):
        st = Stream(seed, w, i, 0)
        u = st.uniform(3)
        n = int(math.floor(math.exp(math.log(1e3) + (math.log(2e5) - math.log(1e3)) * u[0])))
        res = (256, 512, 1024)[min(int(u[1] * 3), 2)]
        spp = (16, 64)[min(int(u[2] * 2), 1)]
        s = hetero_scene(n, seed, w, i + 1)
        out.append(Workload("batched%02d" % i, s, camera_looking_z((0.0, 0.0, -2.9)),
                            res, res, spp, 6, frame_seed=int(mix64(np.uint64(seed + i)))))
    return out


def adjoint_workload(seed: int = 1) -> Workload:
    s = hetero_scene(4096, seed, WORKLOAD_IDS["adjoint"], 0)
    return Workload("adjoint", s, camera_looking_z((0.0, 0.0, -2.9)), 512, 512, 32, 6)


def gi_test_spheres() -> GpuScene:
    """The bounded part of the reference's GI_TEST scene (gfxlab/graphics3d/scene/v1/
    GITestPlain.java:34-44): four spheres with exact decimal centres and radii.  Its
    uniform-SAH topology hashes are published (benchmarks/results/main-bvh-study/
    leaf-size-time.csv:2-8)."""
    s = GpuScene(BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 8))
    glass = MaterialData(refractive=(0.95, 0.95, 0.95), reflective=(0.05, 0.05, 0.05),
                         refractive_index=1.4)
    s.add_sphere((-0.2, -0.5, 0.0), 0.3, glass)
    s.add_sphere((0.5, -0.5, -0.3), 0.3, MaterialData(refractive=(1.0, 1.0, 1.0),
                                                      refractive_index=1.5))
    s.add_sphere((0.0, 0.2, 0.0), 0.2, MaterialData.matte((0.7, 0.7, 0.7)))
    s.add_sphere((-0.4, 0.5, 0.1), 0.2, MaterialData(refractive=(0.9, 0.9, 0.9),
                                                     refractive_index=1.5))
    return s


def gi_test_scene() -> GpuScene:
    """GI_TEST with its five half-spaces (walls at +-1, emissive ceiling).  The wall
    colours of the reference come from Color.hsb in a closed library; equal-luminance
    stand-ins are used (chosen)."""
    s = gi_test_spheres()
    s.add_plane((-1.0, 0.0, 0.0), (1.0, 0.0, 0.0), MaterialData.matte((0.7, 0.35, 0.35)))
    s.add_plane((1.0, 0.0, 0.0), (-1.0, 0.0, 0.0), MaterialData.matte((0.35, 0.7, 0.35)))
    s.add_plane((0.0, -1.0, 0.0), (0.0, 1.0, 0.0), MaterialData.matte((0.7, 0.7, 0.7)))
    s.add_plane((0.0, 1.0, 0.0), (0.0, -1.0, 0.0), MaterialData.light((1.0, 1.0, 1.0)))
    s.add_plane((0.0, 0.0, 1.0), (0.0, 0.0, -1.0), MaterialData.matte((0.7, 0.7, 0.7)))
    return s


def primary_grid(camera: GpuCamera, width: int, height: int, phase_x=0.5, phase_y=0.5):
    """Deterministic camera-ray grid at pixel centres (BenchmarkRays.primaryGrid,
    gfxlab/benchmark/BenchmarkRays.java:14-26), using the pinhole camera's
    position/forward/right/up: origin.xyz then direction.xyz per ray, float32."""
    aspect = width / height
    xs = (np.arange(width) + phase_x)
    ys = (np.arange(height) + phase_y)
    sx = (-1.0 + 2.0 * xs / width) * aspect
    sy = 1.0 - 2.0 * ys / height
    X, Y = np.meshgrid(sx, sy)
    f = np.asarray(camera.forward)
    r = np.asarray(camera.right)
    u = np.asarray(camera.up)
    d = f[None, None, :] + r[None, None, :] * X[:, :, None] + u[None, None, :] * Y[:, :, None]
    o = np.broadcast_to(np.asarray(camera.position, dtype=np.float64), d.shape)
    return np.concatenate([o, d], axis=2).reshape(-1, 6).astype(np.float32)


def random_rays(n: int, seed: int, lo=-1.5, hi=1.5, origin_box=3.0) -> np.ndarray:
    """Rays from points in a cube towards random targets (test workload)."""
    st = Stream(seed, WORKLOAD_IDS["test"], 0, 1)
    o = st.range(3 * n, -origin_box, origin_box, (n, 3))
    t = st.range(3 * n, lo, hi, (n, 3))
    return np.concatenate([o, t - o], axis=1).astype(np.float32)
