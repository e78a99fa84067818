"""GpuRayTracer: the Python mirror of the reference's GPU render path over the C ABI.

Mirrors ``gfxlab/gpu/GpuRayTracer.java`` -- constructor (256-282), ``isAvailable`` (284-287),
``renderSample`` (317-432), ``traceReplay`` (593-716), ``lastFrameStats`` (298-306),
``lastPhysicalKernelLaunchCount`` (294-296), ``deviceInfo`` (308-310),
``validateFullPathDepth`` (470-476) and ``close`` (1223-1310) -- with the same argument
meaning and error behaviour: misuse raises ``ValueError`` (IllegalArgumentException),
an unavailable device or a failed/aborted kernel raises ``RuntimeError``
(IllegalStateException).
"""
from __future__ import annotations

import collections
import time
import ctypes as C
from typing import Optional

import numpy as np

from . import native as N
from .scene import BvhBuildConfig, GpuCamera, GpuScene

MIN_FULL_PATH_DEPTH = 0
MAX_FULL_PATH_DEPTH = 32

FrameStats = collections.namedtuple("FrameStats", [
    "total_nanos", "kernel_nanos", "maximum_physical_kernel_nanos", "copy_nanos",
    "upload_nanos", "rays", "aabb_tests", "primitive_tests", "sphere_tests", "box_tests",
    "plane_tests", "affine_sphere_tests", "affine_box_tests", "stack_overflows",
    "max_stack_size", "internal_node_visits", "leaf_node_visits",
    "homogeneous_leaf_node_visits", "mixed_leaf_node_visits"])

# GpuRayTracer.ConditioningStats (GpuRayTracer.java:434-452)
ConditioningStats = collections.namedtuple("ConditioningStats", [
    "physical_kernel_launch_count", "upload_nanos", "kernel_nanos",
    "maximum_physical_kernel_nanos", "total_nanos"])

TraceReplayResult = collections.namedtuple("TraceReplayResult", [
    "stats", "hit_flags", "hit_distances", "hit_primitive_orders", "hit_material_indices",
    "hit_normals"])

DeviceInfo = collections.namedtuple("DeviceInfo", ["name", "compute_capability", "sm_count"])

BvhStats = collections.namedtuple("BvhStats", [
    "node_count", "root_count", "leaf_count", "max_depth", "primitive_ref_count", "leaf_size",
    "build_mode", "generalized_sah_cost", "uniform_sah_cost", "weighted_sah_cost", "bytes",
    "min_leaf_occupancy", "max_leaf_occupancy", "mean_leaf_occupancy", "build_ms",
    "sequential_nodes", "rotation_count", "spatial_split_count", "duplicate_reference_count"])


def validate_full_path_depth(max_depth: int) -> None:
    if max_depth < MIN_FULL_PATH_DEPTH or max_depth > MAX_FULL_PATH_DEPTH:
        raise ValueError("GPU full-path depth must be in [%d, %d] but was %d"
                         % (MIN_FULL_PATH_DEPTH, MAX_FULL_PATH_DEPTH, max_depth))


class Context:
    """One rtb_context (device, stream, mutex)."""

    def __init__(self, device: int = 0):
        self.lib = N.lib()
        h = C.c_void_p()
        st = self.lib.rtb_context_create(device, C.byref(h))
        if st != N.RTB_OK:
            raise RuntimeError("CUDA path tracer is unavailable (%s)" % N.STATUS_NAMES.get(st, st))
        self.handle = h
        self.device = device

    def check(self, st: int) -> None:
        if st == N.RTB_OK:
            return
        msg = self.lib.rtb_last_error(self.handle).decode()
        if st == 1:
            raise ValueError(msg)
        raise N.RtbError(st, msg)

    def device_info(self) -> DeviceInfo:
        name = C.create_string_buffer(256)
        ma, mi, sm = C.c_int(), C.c_int(), C.c_int()
        self.check(self.lib.rtb_device_info(self.handle, name, 256, C.byref(ma), C.byref(mi),
                                            C.byref(sm)))
        return DeviceInfo(name.value.decode(), "compute_%d%d" % (ma.value, mi.value), sm.value)

    def close(self):
        if self.handle:
            self.lib.rtb_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scene_desc(scene: GpuScene):
    """Marshals a GpuScene into an rtb_scene_desc; returns (desc, keep-alive arrays)."""
    arrs, counts = scene.arrays()
    keep = [N.f32(a) if len(a) else np.zeros(1, np.float32) for a in arrs]
    ab = N.f32(scene.affine_sphere_bounds())
    bb = N.f32(scene.affine_box_bounds())
    keep += [ab if len(ab) else np.zeros(1, np.float32), bb if len(bb) else np.zeros(1, np.float32)]
    d = N.SceneDesc()
    d.spheres, d.sphere_count = N.fptr(keep[0]), counts[0]
    d.boxes, d.box_count = N.fptr(keep[1]), counts[1]
    d.planes, d.plane_count = N.fptr(keep[2]), counts[2]
    d.affine_spheres, d.affine_sphere_count = N.fptr(keep[3]), counts[3]
    d.affine_boxes, d.affine_box_count = N.fptr(keep[4]), counts[4]
    d.materials, d.material_count = N.fptr(keep[5]), counts[5]
    d.affine_sphere_bounds = N.fptr(keep[6])
    d.affine_box_bounds = N.fptr(keep[7])
    for k in range(3):
        d.background[k] = scene.background[k]
    return d, keep


def build_config(cfg: BvhBuildConfig) -> N.BuildConfig:
    return N.BuildConfig(int(cfg.mode), cfg.leaf_size, cfg.traversal_weight, cfg.sphere_weight,
                         cfg.box_weight, cfg.affine_sphere_weight, cfg.affine_box_weight, cfg.lam)


class ResidentScene:
    """A scene resident in device memory (rtb_scene)."""

    def __init__(self, ctx: Context, handle, stats: Optional[BvhStats] = None):
        self.ctx = ctx
        self.handle = handle
        self.stats = stats

    @staticmethod
    def upload(ctx: Context, scene: GpuScene, bvh=None) -> "ResidentScene":
        """Uploads the scene with a caller-built BVH in the reference's flattened layout
        (an object with node_bounds / node_data / refs / roots arrays), or none."""
        d, keep = scene_desc(scene)
        bd = None
        if bvh is not None:
            nb, nd = N.f32(bvh.node_bounds), N.i32(bvh.node_data)
            rf, rt = N.i32(bvh.refs), N.i32(bvh.roots)
            keep += [nb, nd, rf, rt]
            bd = N.BvhDesc(N.fptr(nb), N.iptr(nd), len(nd) // 4, N.iptr(rf), len(rf), N.iptr(rt),
                           len(rt))
        h = C.c_void_p()
        ctx.check(ctx.lib.rtb_scene_upload(ctx.handle, C.byref(d), C.byref(bd) if bd else None,
                                           C.byref(h)))
        return ResidentScene(ctx, h)

    @staticmethod
    def build(ctx: Context, scene: GpuScene, config: Optional[BvhBuildConfig] = None,
              bins: int = 0) -> "ResidentScene":
        """Builds the scene's BVH on the device (GpuScene.buildBvhData moved onto the GPU):
        the reference's full sweep, or with bins in 2..32 the binned object-SAH mode."""
        cfg = config if config is not None else scene.config
        d, keep = scene_desc(scene)
        bc = build_config(cfg)
        st = N.BvhStats()
        h = C.c_void_p()
        if bins:
            ctx.check(ctx.lib.rtb_scene_build_binned(ctx.handle, C.byref(d), C.byref(bc), int(bins),
                                                     C.byref(h), C.byref(st)))
        else:
            o = scene.options
            opts = N.BuildOptions(o.spatial_bins, o.max_reference_multiplier,
                                  o.max_splits_per_primitive, o.min_spatial_references,
                                  o.spatial_overlap_threshold, o.rotation_passes)
            ctx.check(ctx.lib.rtb_scene_build_with_options(ctx.handle, C.byref(d), C.byref(bc),
                                                           C.byref(opts), C.byref(h), C.byref(st)))
        mean = st.primitive_ref_count / st.leaf_count if st.leaf_count else 0.0
        stats = BvhStats(st.node_count, st.root_count, st.leaf_count, st.max_depth,
                         st.primitive_ref_count, st.leaf_size, cfg.mode.name,
                         st.generalized_sah_cost, st.uniform_sah_cost, st.weighted_sah_cost,
                         st.bytes, st.min_leaf_occupancy, st.max_leaf_occupancy, mean,
                         st.build_ms, st.sequential_nodes, st.rotation_count,
                         st.spatial_split_count, st.duplicate_reference_count)
        return ResidentScene(ctx, h, stats)

    def download_bvh(self):
        """The resident BVH in the reference's flattened layout:
        (node_bounds, node_data, refs, roots)."""
        n, r, k = C.c_int(), C.c_int(), C.c_int()
        self.ctx.check(self.ctx.lib.rtb_scene_bvh_sizes(self.ctx.handle, self.handle, C.byref(n),
                                                        C.byref(r), C.byref(k)))
        nb = np.zeros(max(1, 6 * n.value), np.float32)
        nd = np.zeros(max(1, 4 * n.value), np.int32)
        rf = np.zeros(max(1, r.value), np.int32)
        rt = np.zeros(max(1, k.value), np.int32)
        self.ctx.check(self.ctx.lib.rtb_scene_download_bvh(self.ctx.handle, self.handle,
                                                           N.fptr(nb), N.iptr(nd), N.iptr(rf),
                                                           N.iptr(rt)))
        return nb[:6 * n.value], nd[:4 * n.value], rf[:r.value], rt[:k.value]

    def close(self):
        if self.handle:
            self.ctx.lib.rtb_scene_destroy(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            if self.ctx.handle:
                self.close()
        except Exception:
            pass


def camera_struct(cam: GpuCamera) -> N.Camera:
    c = N.Camera()
    for k in range(3):
        c.position[k] = cam.position[k]
        c.forward[k] = cam.forward[k]
        c.right[k] = cam.right[k]
        c.up[k] = cam.up[k]
    return c


class GpuRayTracer:
    """Drop-in for gfxlab/gpu/GpuRayTracer.java over librtb200.so."""

    def __init__(self, width: int, height: int, samples_per_frame: int, bvh_traversal: bool = True,
                 collect_metrics: bool = False, device: int = 0):
        self.width = max(1, int(width))
        self.height = max(1, int(height))
        if self.width * self.height > (2 ** 31 - 1) // 3:
            raise ValueError("GPU image dimensions exceed array indexing")
        self.samples_per_frame = max(1, int(samples_per_frame))
        self.bvh_traversal = bool(bvh_traversal)
        self.collect_metrics = bool(collect_metrics)
        self.device = device
        self._ctx: Optional[Context] = None
        self._available = True
        self._resident = None
        self._resident_key = None
        self._last_launches = 0
        self._last_upload_ns = 0
        self._last_call_ns = 0

    # -- availability --
    def _init(self):
        if self._ctx is None and self._available:
            try:
                self._ctx = Context(self.device)
            except Exception:
                self._available = False
        return self._ctx

    def is_available(self) -> bool:
        return self._init() is not None

    def collects_metrics(self) -> bool:
        return self.collect_metrics

    def device_info(self) -> DeviceInfo:
        ctx = self._require()
        return ctx.device_info()

    def _require(self) -> Context:
        ctx = self._init()
        if ctx is None:
            raise RuntimeError("CUDA path tracer is unavailable")
        return ctx

    # -- residency (GpuRayTracer.ensureSceneResident, GpuRayTracer.java:934-948) --
    def ensure_scene_resident(self, scene: GpuScene, bvh=None) -> ResidentScene:
        if scene is None:
            raise ValueError("GPU scene must not be null")
        ctx = self._require()
        key = (id(scene), scene.revision, id(bvh))
        if self._resident is not None and self._resident_key == key:
            return self._resident
        if self._resident is not None:
            self._resident.close()
        if bvh is not None:
            self._resident = ResidentScene.upload(ctx, scene, bvh)
        elif self.bvh_traversal:
            self._resident = ResidentScene.build(ctx, scene)
        else:
            self._resident = ResidentScene.upload(ctx, scene, None)
        self._resident_key = key
        return self._resident

    # -- renderSample --
    def render_sample(self, rgb: Optional[np.ndarray], scene: GpuScene, camera: GpuCamera,
                      max_depth: int, frame_index: int, frame_seed: int, bvh=None) -> np.ndarray:
        validate_full_path_depth(max_depth)
        n = self.width * self.height * 3
        if rgb is None:
            rgb = np.zeros(n, np.float32)
        if rgb.dtype != np.float32 or not rgb.flags.c_contiguous or rgb.size < n:
            raise ValueError("RGB output must contain at least %d elements" % n)
        if scene is None or camera is None:
            raise ValueError("GPU scene and camera must not be null")
        ctx = self._require()
        t0 = time.perf_counter_ns()
        before = self._resident
        res = self.ensure_scene_resident(scene, bvh)
        # renderSample's lastUploadNanos: the scene upload this call made, 0 when resident
        upload_ns = time.perf_counter_ns() - t0 if res is not before else 0
        p = N.RenderParams(self.width, self.height, self.samples_per_frame, int(max_depth),
                           int(frame_index), int(frame_seed) & 0xFFFFFFFFFFFFFFFF,
                           1 if self.bvh_traversal else 0, 1 if self.collect_metrics else 0, 0)
        cam = camera_struct(camera)
        ctx.check(ctx.lib.rtb_render_sample(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                            N.fptr(rgb)))
        st = N.FrameStats()
        ctx.check(ctx.lib.rtb_last_frame_stats(ctx.handle, C.byref(st)))
        self._last_launches = st.physical_launches  # the frame kernel, plus the tail sum
        self._last_upload_ns = upload_ns
        self._last_call_ns = time.perf_counter_ns() - t0
        return rgb

    # -- steady-state samples (GpuRayTracer.java:434-467) --
    def condition_steady_state_sample(self, scene: GpuScene, camera: GpuCamera, max_depth: int,
                                      frame_index: int, frame_seed: int,
                                      bvh=None) -> ConditioningStats:
        """Renders one sample into an internal buffer (making the scene resident) and
        reports its launch count and times, as conditionSteadyStateSample does."""
        if getattr(self, "_conditioning", None) is None:
            self._conditioning = np.zeros(self.width * self.height * 3, np.float32)
        self.render_sample(self._conditioning, scene, camera, max_depth, frame_index, frame_seed, bvh)
        st = self.last_frame_stats()
        return ConditioningStats(self._last_launches, st.upload_nanos, st.kernel_nanos,
                                 st.maximum_physical_kernel_nanos, st.total_nanos)

    def render_steady_state_sample(self, rgb: np.ndarray, scene: GpuScene, camera: GpuCamera,
                                   max_depth: int, frame_index: int, frame_seed: int,
                                   bvh=None) -> np.ndarray:
        """renderSample that must not upload: raises RuntimeError (IllegalStateException)
        when the scene was not resident already."""
        out = self.render_sample(rgb, scene, camera, max_depth, frame_index, frame_seed, bvh)
        if self._last_upload_ns != 0:
            raise RuntimeError("A steady-state sample uploaded scene data")
        return out

    def compiled_ptx_sha256(self) -> str:
        """Identity of the device code (compiledPtxSha256, GpuRayTracer.java:313-315).  The
        reference hashes the PTX it JIT-compiles; this library ships its sm_100a code
        precompiled, so the hash is the SHA-256 of the loaded librtb200.so file."""
        import hashlib
        with open(N.LIB_PATH, "rb") as f:
            return hashlib.sha256(f.read()).hexdigest()

    # -- traceReplay --
    def trace_replay(self, scene: GpuScene, rays: np.ndarray, ray_count: Optional[int] = None,
                     collect_metrics: bool = False, bvh=None) -> TraceReplayResult:
        rays = N.f32(rays).reshape(-1)
        if ray_count is None:
            ray_count = rays.size // 6
        if ray_count <= 0 or rays.size < ray_count * 6:
            raise ValueError("Replay rays must contain origin.xyz and direction.xyz.")
        if scene is None:
            raise ValueError("GPU scene must not be null")
        ctx = self._require()
        res = self.ensure_scene_resident(scene, bvh)
        n = ray_count
        flags = np.zeros(n, np.int32)
        dist = np.zeros(n, np.float32)
        order = np.zeros(n, np.int32)
        mat = np.zeros(n, np.int32)
        nrm = np.zeros(3 * n, np.float32)
        ctx.check(ctx.lib.rtb_trace_replay(ctx.handle, res.handle, N.fptr(rays), n,
                                           1 if self.bvh_traversal else 0,
                                           1 if collect_metrics else 0, N.iptr(flags),
                                           N.fptr(dist), N.iptr(order), N.iptr(mat), N.fptr(nrm)))
        self._last_launches = 1
        self._last_call_ns = 0
        return TraceReplayResult(self.last_frame_stats(), flags, dist, order, mat, nrm)

    # -- stats --
    def last_frame_stats(self) -> FrameStats:
        ctx = self._require()
        st = N.FrameStats()
        ctx.check(ctx.lib.rtb_last_frame_stats(ctx.handle, C.byref(st)))
        c = list(st.counters)
        total, upload = st.total_ns, st.upload_ns
        if self._last_call_ns:  # the last call was render_sample: its own upload and span
            total, upload = max(total, self._last_call_ns), self._last_upload_ns
        return FrameStats(total, st.kernel_ns, st.max_physical_kernel_ns, st.copy_ns,
                          upload, c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8],
                          c[9], c[10], c[11], c[12], c[13])

    def last_physical_kernel_launch_count(self) -> int:
        return self._last_launches

    def close(self):
        if self._resident is not None:
            self._resident.close()
            self._resident = None
        if self._ctx is not None:
            self._ctx.close()
            self._ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
