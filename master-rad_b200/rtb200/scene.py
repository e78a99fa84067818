"""Host-side scene description: the Python mirror of the reference's GPU scene API.

Mirrors ``gfxlab/gpu/GpuScene.java`` (packing and validation), ``BvhBuildConfig.java``,
``BvhBuildMode.java``, ``BvhBuildOptions.java``, ``PrimitiveCostModel.java`` and
``GpuCamera.java`` (``gfxlab/`` = ``src/xyz/marsavic/gfxlab/`` of the reference).  The
packed float layouts produced here are exactly the reference's, because they are the
drop-in boundary: the C ABI (``include/rtb200.h``) accepts the arrays a Java caller gets
from ``GpuScene.sphereData()`` and friends.

Records are held column-wise in numpy arrays so that million-primitive scenes pack in
seconds; the single-record ``add_*`` methods are thin wrappers over the bulk ones.
"""
from __future__ import annotations

import dataclasses
import enum
import math
from typing import Optional, Sequence

import numpy as np

# GpuScene.java:19-29
MAX_AFFINE_SPECTRAL_CONDITION = 65536.0
MIN_PACKED_PRIMITIVE_EXTENT = np.float32(math.sqrt(np.finfo(np.float32).tiny))
AFFINE_CONDITION_ESTIMATE_RELATIVE_SLACK = 5.0e-4
FLOATS_PER_MATERIAL = 13
FLOATS_PER_SPHERE = 5
FLOATS_PER_BOX = 7
FLOATS_PER_PLANE = 26
FLOATS_PER_AFFINE = 22
FLOATS_PER_BVH_NODE = 6
INTS_PER_BVH_NODE = 4

REF_TYPE_SPHERE = 0x00000000
REF_TYPE_BOX = 0x40000000
REF_TYPE_AFFINE_SPHERE = -0x80000000
REF_TYPE_AFFINE_BOX = -0x40000000


class PrimitiveCostModel:
    """Sphere-normalised operation costs (PrimitiveCostModel.java:11-19)."""
    SPHERE = 1.000000000
    BOX = 1.288951704
    AFFINE_SPHERE = 2.552743938
    AFFINE_BOX = 2.728115282
    PLANE = 2.860319327
    NODE_AABB = 0.507189194
    INTERIOR_TRAVERSAL = 1.275576713


def traversal_work(aabb_tests, sphere_tests, box_tests, plane_tests, affine_sphere_tests,
                   affine_box_tests, model=PrimitiveCostModel) -> float:
    """TraversalWorkMetric.cost (TraversalWorkMetric.java:14-38): one cost term per
    measured AABB test and per primitive test, weighted by the cost model (any object with
    the PrimitiveCostModel attributes); shading, memory and divergence are left out."""
    return (model.NODE_AABB * aabb_tests + model.SPHERE * sphere_tests + model.BOX * box_tests
            + model.PLANE * plane_tests + model.AFFINE_SPHERE * affine_sphere_tests
            + model.AFFINE_BOX * affine_box_tests)


def frame_traversal_work(stats, model=PrimitiveCostModel) -> float:
    """traversal_work of a FrameStats (TraversalWorkMetric.cost(FrameStats))."""
    return traversal_work(stats.aabb_tests, stats.sphere_tests, stats.box_tests, stats.plane_tests,
                          stats.affine_sphere_tests, stats.affine_box_tests, model)


class BvhBuildMode(enum.IntEnum):
    """BvhBuildMode.java:4-44 (ordinals are part of the C ABI)."""
    UNIFORM_SAH = 0
    WEIGHTED_SAH = 1
    PER_TYPE_SAH = 2
    PER_TYPE_WEIGHTED_SAH = 3
    UNIFORM_SBVH = 4
    WEIGHTED_SBVH = 5
    SAH_ROTATIONS = 6
    WEIGHTED_SAH_ROTATIONS = 7

    def uses_primitive_weights(self) -> bool:
        return self in (BvhBuildMode.WEIGHTED_SAH, BvhBuildMode.PER_TYPE_WEIGHTED_SAH,
                        BvhBuildMode.WEIGHTED_SBVH, BvhBuildMode.WEIGHTED_SAH_ROTATIONS)

    def with_primitive_weights(self, weighted: bool) -> "BvhBuildMode":
        pairs = {
            BvhBuildMode.UNIFORM_SAH: (BvhBuildMode.UNIFORM_SAH, BvhBuildMode.WEIGHTED_SAH),
            BvhBuildMode.WEIGHTED_SAH: (BvhBuildMode.UNIFORM_SAH, BvhBuildMode.WEIGHTED_SAH),
            BvhBuildMode.PER_TYPE_SAH: (BvhBuildMode.PER_TYPE_SAH, BvhBuildMode.PER_TYPE_WEIGHTED_SAH),
            BvhBuildMode.PER_TYPE_WEIGHTED_SAH: (BvhBuildMode.PER_TYPE_SAH,
                                                 BvhBuildMode.PER_TYPE_WEIGHTED_SAH),
            BvhBuildMode.UNIFORM_SBVH: (BvhBuildMode.UNIFORM_SBVH, BvhBuildMode.WEIGHTED_SBVH),
            BvhBuildMode.WEIGHTED_SBVH: (BvhBuildMode.UNIFORM_SBVH, BvhBuildMode.WEIGHTED_SBVH),
            BvhBuildMode.SAH_ROTATIONS: (BvhBuildMode.SAH_ROTATIONS,
                                         BvhBuildMode.WEIGHTED_SAH_ROTATIONS),
            BvhBuildMode.WEIGHTED_SAH_ROTATIONS: (BvhBuildMode.SAH_ROTATIONS,
                                                  BvhBuildMode.WEIGHTED_SAH_ROTATIONS),
        }
        return pairs[self][1 if weighted else 0]

    def uses_per_type_trees(self) -> bool:
        return self in (BvhBuildMode.PER_TYPE_SAH, BvhBuildMode.PER_TYPE_WEIGHTED_SAH)

    def uses_spatial_splits(self) -> bool:
        return self in (BvhBuildMode.UNIFORM_SBVH, BvhBuildMode.WEIGHTED_SBVH)

    def uses_rotations(self) -> bool:
        return self in (BvhBuildMode.SAH_ROTATIONS, BvhBuildMode.WEIGHTED_SAH_ROTATIONS)


def _check_positive(label: str, w: float) -> None:
    if not (w > 0.0) or not math.isfinite(w):
        raise ValueError("Invalid %s weight: %r" % (label, w))


@dataclasses.dataclass(frozen=True)
class BvhBuildConfig:
    """Inputs to the uniform or cost-weighted SAH builder (BvhBuildConfig.java:6-50).

    ``construction_weight`` is q_i = 1 + lambda (c_i - 1) (BvhBuildConfig.java:66-69).
    The constructor canonicalises lambda exactly as the reference does.
    """
    mode: BvhBuildMode = BvhBuildMode.UNIFORM_SAH
    leaf_size: int = 8
    traversal_weight: float = PrimitiveCostModel.INTERIOR_TRAVERSAL
    sphere_weight: float = PrimitiveCostModel.SPHERE
    box_weight: float = PrimitiveCostModel.BOX
    affine_sphere_weight: float = PrimitiveCostModel.AFFINE_SPHERE
    affine_box_weight: float = PrimitiveCostModel.AFFINE_BOX
    lam: float = 0.0

    def __post_init__(self):
        mode = BvhBuildMode(self.mode)
        if self.leaf_size < 1:
            raise ValueError("BVH leaf size must be positive.")
        _check_positive("AABB traversal", self.traversal_weight)
        _check_positive("sphere", self.sphere_weight)
        _check_positive("box", self.box_weight)
        _check_positive("affine sphere", self.affine_sphere_weight)
        _check_positive("affine box", self.affine_box_weight)
        lam = self.lam
        if lam < 0.0 or not math.isfinite(lam):
            raise ValueError("Invalid SAH lambda: %r" % lam)
        if mode.uses_primitive_weights() and lam == 0.0:
            mode = mode.with_primitive_weights(False)
            lam = 0.0
        elif not mode.uses_primitive_weights() and lam != 0.0:
            raise ValueError(
                "An unweighted BVH mode requires the canonical lambda-zero configuration.")
        elif not mode.uses_primitive_weights():
            lam = 0.0
        if mode.uses_primitive_weights():
            for label, w in (("sphere", self.sphere_weight), ("box", self.box_weight),
                             ("affine sphere", self.affine_sphere_weight),
                             ("affine box", self.affine_box_weight)):
                _check_positive("generalized " + label, 1.0 + lam * (w - 1.0))
        object.__setattr__(self, "mode", mode)
        object.__setattr__(self, "lam", float(lam))

    @staticmethod
    def weighted(leaf_size=8, sphere=1.0, box=1.3, affine=2.1, lam=1.0,
                 traversal=PrimitiveCostModel.INTERIOR_TRAVERSAL,
                 mode=BvhBuildMode.WEIGHTED_SAH) -> "BvhBuildConfig":
        return BvhBuildConfig(mode, leaf_size, traversal, sphere, box, affine, affine, lam)

    def construction_weight(self, measured: float) -> float:
        return 1.0 + self.lam * (measured - 1.0) if self.mode.uses_primitive_weights() else 1.0


@dataclasses.dataclass(frozen=True)
class BvhBuildOptions:
    """SBVH / rotation tuning inputs (BvhBuildOptions.java:4-33)."""
    spatial_bins: int = 128
    max_reference_multiplier: float = 2.0
    max_splits_per_primitive: int = 8
    min_spatial_references: int = 16
    spatial_overlap_threshold: float = 1.0e-5
    rotation_passes: int = 4


@dataclasses.dataclass(frozen=True)
class MaterialData:
    """GpuScene.MaterialData (GpuScene.java:45-61): 13 packed floats per material."""
    diffuse: tuple = (0.0, 0.0, 0.0)
    reflective: tuple = (0.0, 0.0, 0.0)
    refractive: tuple = (0.0, 0.0, 0.0)
    refractive_index: float = 1.5
    emittance: tuple = (0.0, 0.0, 0.0)

    def packed(self) -> np.ndarray:
        return np.array(list(self.diffuse) + list(self.reflective) + list(self.refractive)
                        + list(self.emittance) + [self.refractive_index], dtype=np.float64)

    @staticmethod
    def matte(c) -> "MaterialData":
        return MaterialData(diffuse=tuple(float(v) for v in c))

    @staticmethod
    def light(c) -> "MaterialData":
        return MaterialData(emittance=tuple(float(v) for v in c))


@dataclasses.dataclass(frozen=True)
class GpuCamera:
    """Pinhole camera consumed by the kernels (GpuCamera.java): ray direction for sensor
    coordinates (u, v) is ``forward + right * u + up * v``."""
    position: tuple
    forward: tuple
    right: tuple
    up: tuple

    def packed(self) -> np.ndarray:
        return np.array(list(self.position) + list(self.forward) + list(self.right)
                        + list(self.up), dtype=np.float32)


def _f32(a):
    return np.asarray(a, dtype=np.float64).astype(np.float32)


def _require_finite_f32(values: np.ndarray, label: str) -> None:
    v = np.asarray(values, dtype=np.float64)
    if not np.all(np.isfinite(v)):
        raise ValueError(label + " must be finite.")
    with np.errstate(over="ignore"):
        if not np.all(np.isfinite(v.astype(np.float32))):
            raise ValueError(label + " must remain finite in the GPU float payload.")


def _require_nondegenerate(mn: np.ndarray, mx: np.ndarray, label: str) -> None:
    """requireNondegenerateFloatBounds (GpuScene.java:277-297), vectorised."""
    _require_finite_f32(mn, label + " minimum bound")
    _require_finite_f32(mx, label + " maximum bound")
    a = _f32(mn)
    b = _f32(mx)
    ok = np.all(a < b, axis=-1) & np.all((b - a) >= MIN_PACKED_PRIMITIVE_EXTENT, axis=-1)
    if not np.all(ok):
        raise ValueError(label + " bounds must retain a supported positive extent on every "
                         "axis after float packing.")


def _spectral_condition(m: np.ndarray) -> np.ndarray:
    """spectralConditionNumber (GpuScene.java:388-441) for (k, 9) float matrices."""
    m = m.astype(np.float64)
    scale = np.max(np.abs(m), axis=1)
    a = m / scale[:, None]
    s00 = a[:, 0] * a[:, 0] + a[:, 3] * a[:, 3] + a[:, 6] * a[:, 6]
    s01 = a[:, 0] * a[:, 1] + a[:, 3] * a[:, 4] + a[:, 6] * a[:, 7]
    s02 = a[:, 0] * a[:, 2] + a[:, 3] * a[:, 5] + a[:, 6] * a[:, 8]
    s11 = a[:, 1] * a[:, 1] + a[:, 4] * a[:, 4] + a[:, 7] * a[:, 7]
    s12 = a[:, 1] * a[:, 2] + a[:, 4] * a[:, 5] + a[:, 7] * a[:, 8]
    s22 = a[:, 2] * a[:, 2] + a[:, 5] * a[:, 5] + a[:, 8] * a[:, 8]
    off = s01 * s01 + s02 * s02 + s12 * s12
    mean = (s00 + s11 + s22) / 3.0
    var = (s00 - mean) ** 2 + (s11 - mean) ** 2 + (s22 - mean) ** 2 + 2.0 * off
    p = np.sqrt(np.maximum(var, 0.0) / 6.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        b00 = (s00 - mean) / p
        b01 = s01 / p
        b02 = s02 / p
        b11 = (s11 - mean) / p
        b12 = s12 / p
        b22 = (s22 - mean) / p
        det = (b00 * (b11 * b22 - b12 * b12) - b01 * (b01 * b22 - b12 * b02)
               + b02 * (b01 * b12 - b11 * b02))
        ang = np.arccos(np.clip(det / 2.0, -1.0, 1.0)) / 3.0
        largest = mean + 2.0 * p * np.cos(ang)
        smallest = mean + 2.0 * p * np.cos(ang + 2.0 * math.pi / 3.0)
    diag = off == 0.0
    dl = np.maximum(np.maximum(s00, s11), s22)
    ds = np.minimum(np.minimum(s00, s11), s22)
    largest = np.where(diag, dl, largest)
    smallest = np.where(diag, ds, smallest)
    with np.errstate(divide="ignore", invalid="ignore"):
        cond = np.sqrt(largest / smallest)
    return np.where((smallest > 0.0) & np.isfinite(largest), cond, np.inf)


def affine_inverse(m: np.ndarray) -> np.ndarray:
    """Affine.inverse for (k, 3, 4) double matrices, expression for expression
    (gfxlab/graphics3d/Affine.java:66-75 and its determinant)."""
    m00, m01, m02, m03 = m[:, 0, 0], m[:, 0, 1], m[:, 0, 2], m[:, 0, 3]
    m10, m11, m12, m13 = m[:, 1, 0], m[:, 1, 1], m[:, 1, 2], m[:, 1, 3]
    m20, m21, m22, m23 = m[:, 2, 0], m[:, 2, 1], m[:, 2, 2], m[:, 2, 3]
    det = (((((m00 * m11 * m22) + (m01 * m12 * m20)) + (m02 * m10 * m21))
            - (m02 * m11 * m20)) - (m01 * m10 * m22)) - (m00 * m12 * m21)
    out = np.empty_like(m)
    out[:, 0, 0] = (m11 * m22 - m12 * m21) / det
    out[:, 0, 1] = -(m01 * m22 - m02 * m21) / det
    out[:, 0, 2] = (m01 * m12 - m02 * m11) / det
    out[:, 0, 3] = -(m01 * m12 * m23 + m02 * m13 * m21 + m03 * m11 * m22 - m03 * m12 * m21
                     - m02 * m11 * m23 - m01 * m13 * m22) / det
    out[:, 1, 0] = -(m10 * m22 - m12 * m20) / det
    out[:, 1, 1] = (m00 * m22 - m02 * m20) / det
    out[:, 1, 2] = -(m00 * m12 - m02 * m10) / det
    out[:, 1, 3] = (m00 * m12 * m23 + m02 * m13 * m20 + m03 * m10 * m22 - m03 * m12 * m20
                    - m02 * m10 * m23 - m00 * m13 * m22) / det
    out[:, 2, 0] = (m10 * m21 - m11 * m20) / det
    out[:, 2, 1] = -(m00 * m21 - m01 * m20) / det
    out[:, 2, 2] = (m00 * m11 - m01 * m10) / det
    out[:, 2, 3] = -(m00 * m11 * m23 + m01 * m13 * m20 + m03 * m10 * m21 - m03 * m11 * m20
                     - m01 * m10 * m23 - m00 * m13 * m21) / det
    return out


def gpu_affine(transforms: np.ndarray, kind: str):
    """GpuSceneBuilder.gpuAffine + sphereBounds / boxBounds (GpuSceneBuilder.java:84-159).

    ``transforms`` are forward object-to-world (k, 3, 4) doubles mapping the unit sphere or
    the [-1, 1]^3 box.  Returns (inverse (k,3,3) float-quantised doubles, world centre
    (k,3) float-quantised doubles, bounds min (k,3), bounds max (k,3) doubles).
    """
    inv = affine_inverse(transforms)
    packed_inv = np.zeros_like(transforms)
    packed_inv[:, :, :3] = inv[:, :, :3].astype(np.float32).astype(np.float64)
    centre = transforms[:, :, 3].astype(np.float32).astype(np.float64)
    fwd = affine_inverse(packed_inv)[:, :, :3]
    if kind == "sphere":
        ext = np.sqrt(fwd[:, :, 0] * fwd[:, :, 0] + fwd[:, :, 1] * fwd[:, :, 1]
                      + fwd[:, :, 2] * fwd[:, :, 2])
    else:
        ext = (np.abs(fwd[:, :, 0] * 1.0) + np.abs(fwd[:, :, 1] * 1.0)) + np.abs(fwd[:, :, 2] * 1.0)
    return packed_inv[:, :, :3], centre, centre - ext, centre + ext


class GpuScene:
    """Compact scene description transferred to the tracer (GpuScene.java).

    Global primitive order (the tie-break of equal-distance hits) is spheres, boxes,
    affine spheres, affine boxes, planes, each in insertion order.
    """

    def __init__(self, config: Optional[BvhBuildConfig] = None,
                 options: Optional[BvhBuildOptions] = None):
        self.config = config if config is not None else BvhBuildConfig()
        self.options = options if options is not None else BvhBuildOptions()
        self.background = (0.0, 0.0, 0.0)
        self._mat_rows: list = []
        self._mat_index: dict = {}
        self._chunks = {k: [] for k in ("sphere", "box", "plane", "asphere", "abox")}
        self._plane_grids = {}
        self._cache: dict = {}
        self.revision = 0

    # -- materials (GpuScene.registerMaterial, GpuScene.java:850-859) --
    def register_materials(self, rows) -> np.ndarray:
        """Registers (k, 13) packed material rows (diffuse, reflective, refractive,
        emittance, ior), deduplicated by value in first-seen order; returns indices."""
        rows = np.asarray(rows, dtype=np.float64).reshape(-1, FLOATS_PER_MATERIAL)
        out = np.empty(len(rows), dtype=np.int64)
        for i, r in enumerate(map(tuple, rows.tolist())):
            idx = self._mat_index.get(r)
            if idx is None:
                idx = len(self._mat_rows)
                self._mat_rows.append(r)
                self._mat_index[r] = idx
            out[i] = idx
        if len(self._mat_rows) > (1 << 24):
            raise ValueError("material count exceeds the float-exact index range")
        return out

    def register_material(self, m: MaterialData) -> int:
        return int(self.register_materials(m.packed()[None, :])[0])

    def material_count(self) -> int:
        return len(self._mat_rows)

    def _invalidate(self):
        self.revision += 1
        self._cache.clear()

    def set_background(self, rgb) -> "GpuScene":
        self.background = tuple(float(v) for v in rgb)
        self._invalidate()
        return self

    # -- primitives --
    def add_spheres(self, centers, radii, material_ids) -> "GpuScene":
        """Bulk GpuScene.addSphere (GpuScene.java:205-221)."""
        c = np.asarray(centers, dtype=np.float64).reshape(-1, 3)
        r = np.asarray(radii, dtype=np.float64).reshape(-1)
        _require_finite_f32(c, "Sphere center")
        pr = r.astype(np.float32)
        if not (np.all(r > 0.0) and np.all(np.isfinite(r)) and np.all(pr >= MIN_PACKED_PRIMITIVE_EXTENT)
                and np.all(np.isfinite(pr))):
            raise ValueError("Sphere radius must remain finite and at least %g in the GPU "
                             "float payload." % MIN_PACKED_PRIMITIVE_EXTENT)
        cf = c.astype(np.float32)
        _require_nondegenerate((cf - pr[:, None]).astype(np.float64),
                               (cf + pr[:, None]).astype(np.float64), "Sphere")
        self._chunks["sphere"].append((c, r, np.asarray(material_ids, dtype=np.int64).reshape(-1)))
        self._invalidate()
        return self

    def add_sphere(self, center, radius, material: MaterialData) -> "GpuScene":
        return self.add_spheres([center], [radius], [self.register_material(material)])

    def add_boxes(self, mins, maxs, material_ids) -> "GpuScene":
        """Bulk GpuScene.addBox (GpuScene.java:223-233)."""
        a = np.asarray(mins, dtype=np.float64).reshape(-1, 3)
        b = np.asarray(maxs, dtype=np.float64).reshape(-1, 3)
        if not (np.all(np.isfinite(a)) and np.all(np.isfinite(b))):
            raise ValueError("Box endpoint must be finite.")
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        _require_nondegenerate(lo, hi, "Box")
        self._chunks["box"].append((lo, hi, np.asarray(material_ids, dtype=np.int64).reshape(-1)))
        self._invalidate()
        return self

    def add_box(self, mn, mx, material: MaterialData) -> "GpuScene":
        return self.add_boxes([mn], [mx], [self.register_material(material)])

    def add_planes(self, points, normals, material_ids) -> "GpuScene":
        """Bulk GpuScene.addPlane (GpuScene.java:235-254)."""
        p = np.asarray(points, dtype=np.float64).reshape(-1, 3)
        n = np.asarray(normals, dtype=np.float64).reshape(-1, 3)
        _require_finite_f32(p, "Plane point")
        _require_finite_f32(n, "Plane normal")
        l2 = n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1] + n[:, 2] * n[:, 2]
        if not (np.all(l2 > 0.0) and np.all(np.isfinite(l2))):
            raise ValueError("Plane normal must be non-zero.")
        length = np.sqrt(l2)
        unit = n / length[:, None]
        offset = -(unit[:, 0] * p[:, 0] + unit[:, 1] * p[:, 1] + unit[:, 2] * p[:, 2])
        if not np.all(np.isfinite(offset.astype(np.float32))):
            raise ValueError("Plane offset must remain finite in the GPU float payload.")
        self._chunks["plane"].append((unit, offset, np.asarray(material_ids, dtype=np.int64).reshape(-1)))
        self._invalidate()
        return self

    def add_plane(self, point, normal, material: MaterialData) -> "GpuScene":
        return self.add_planes([point], [normal], [self.register_material(material)])

    def add_grid_plane(self, point, normal, e, f, cell_size, line_width, surface: MaterialData,
                       cell: MaterialData, line: MaterialData) -> "GpuScene":
        """A plane carrying the kernel's grid material (GridData K:128-134, loadPlane
        K:233-249, choosePlaneMaterialIndex K:251-269): a hit point's coordinates (u, v) in
        the in-plane basis (e, f), measured from ``point``, select ``line`` within
        line_width of a cell edge (cells of cell_size) and ``cell`` elsewhere.  GpuScene
        itself writes no grid (GpuScene.java:548-569); the record layout is the kernel's."""
        index = self.plane_count
        self.add_plane(point, normal, surface)
        e = np.asarray(e, np.float64)
        f = np.asarray(f, np.float64)
        ee, ff, ef = float(e @ e), float(f @ f), float(e @ f)
        sin_sq = 1.0 - ef * ef / (ee * ff)
        if not (ee > 0.0 and ff > 0.0 and sin_sq > 0.0):
            raise ValueError("Grid basis vectors must be non-zero and not parallel.")
        cs = np.asarray(cell_size, np.float64).reshape(2)
        lw = np.asarray(line_width, np.float64).reshape(2)
        if not (np.all(cs > 0.0) and np.all(lw >= 0.0)):
            raise ValueError("Grid cell sizes must be positive and line widths non-negative.")
        rec = np.zeros(FLOATS_PER_PLANE - 4, np.float64)  # slots 4..25
        rec[0:3] = point
        rec[3:6] = e
        rec[6:9] = f
        rec[9], rec[10] = ee, ff
        # (u, v) solve rel = u e + v f: b_e = rel.e / |e|^2 = u + v ef/|e|^2 and
        # b_f = u ef/|f|^2 + v, so the kernel's e_f is ef/|f|^2 and f_e is ef/|e|^2
        rec[11], rec[12] = ef / ff, ef / ee
        rec[13] = sin_sq
        rec[14] = 1.0
        rec[15:17] = cs
        rec[17:19] = lw
        rec[20] = self.register_material(cell)
        rec[21] = self.register_material(line)
        _require_finite_f32(rec.reshape(1, -1), "Grid plane record")
        self._plane_grids[index] = rec
        self._invalidate()
        return self

    def _add_affine(self, kind, inverse, centre, bmin, bmax, material_ids, label):
        inv = np.asarray(inverse, dtype=np.float64).reshape(-1, 3, 3)
        c = np.asarray(centre, dtype=np.float64).reshape(-1, 3)
        lo = np.minimum(np.asarray(bmin, dtype=np.float64).reshape(-1, 3),
                        np.asarray(bmax, dtype=np.float64).reshape(-1, 3))
        hi = np.maximum(np.asarray(bmin, dtype=np.float64).reshape(-1, 3),
                        np.asarray(bmax, dtype=np.float64).reshape(-1, 3))
        _require_finite_f32(inv.reshape(-1, 9), label + " inverse matrix")
        _require_finite_f32(c, label + " world center")
        c = c.astype(np.float32).astype(np.float64)
        lin = inv.reshape(-1, 9).astype(np.float32).astype(np.float64)
        det = (lin[:, 0] * (lin[:, 4] * lin[:, 8] - lin[:, 5] * lin[:, 7])
               - lin[:, 1] * (lin[:, 3] * lin[:, 8] - lin[:, 5] * lin[:, 6])
               + lin[:, 2] * (lin[:, 3] * lin[:, 7] - lin[:, 4] * lin[:, 6]))
        if not np.all((det != 0.0) & np.isfinite(det)):
            raise ValueError(label + " inverse matrix must be nonsingular after float packing.")
        cond = _spectral_condition(lin)
        if np.any(~np.isfinite(cond)) or np.any(
                cond > MAX_AFFINE_SPECTRAL_CONDITION * (1.0 + AFFINE_CONDITION_ESTIMATE_RELATIVE_SLACK)):
            raise ValueError(label + " exceeds the empirically validated float conditioning "
                             "limit (kappa_2 <= 65536).")
        _require_nondegenerate(lo, hi, label)
        cf, lof, hif = _f32(c), _f32(lo), _f32(hi)
        if np.any(cf < lof) or np.any(cf > hif):
            raise ValueError(label + " bounds must enclose the packed world center.")
        self._chunks[kind].append((inv, c, lo, hi, np.asarray(material_ids, dtype=np.int64).reshape(-1)))
        self._invalidate()
        return self

    def add_affine_spheres(self, inverse, centre, bmin, bmax, material_ids) -> "GpuScene":
        """Bulk GpuScene.addAffineSphere (GpuScene.java:443-455)."""
        return self._add_affine("asphere", inverse, centre, bmin, bmax, material_ids, "Affine sphere")

    def add_affine_boxes(self, inverse, centre, bmin, bmax, material_ids) -> "GpuScene":
        """Bulk GpuScene.addAffineBox (GpuScene.java:457-469)."""
        return self._add_affine("abox", inverse, centre, bmin, bmax, material_ids, "Affine box")

    def add_transformed_spheres(self, transforms, material_ids) -> "GpuScene":
        """GpuSceneBuilder's path for affine spheres: forward (k,3,4) transforms of the
        unit sphere, quantised and bounded as GpuSceneBuilder.java:41-51, 84-159 does."""
        inv, c, lo, hi = gpu_affine(np.asarray(transforms, dtype=np.float64), "sphere")
        return self.add_affine_spheres(inv, c, lo, hi, material_ids)

    def add_transformed_boxes(self, transforms, material_ids) -> "GpuScene":
        inv, c, lo, hi = gpu_affine(np.asarray(transforms, dtype=np.float64), "box")
        return self.add_affine_boxes(inv, c, lo, hi, material_ids)

    # -- counts --
    def _count(self, kind):
        return int(sum(len(ch[-1]) for ch in self._chunks[kind]))

    @property
    def sphere_count(self):
        return self._count("sphere")

    @property
    def box_count(self):
        return self._count("box")

    @property
    def plane_count(self):
        return self._count("plane")

    @property
    def affine_sphere_count(self):
        return self._count("asphere")

    @property
    def affine_box_count(self):
        return self._count("abox")

    def primitive_count(self) -> int:
        return (self.sphere_count + self.box_count + self.plane_count
                + self.affine_sphere_count + self.affine_box_count)

    def bounded_primitive_count(self) -> int:
        return self.primitive_count() - self.plane_count

    # -- packers (GpuScene.java:507-601) --
    def _cat(self, kind, k):
        ch = self._chunks[kind]
        if not ch:
            return None
        return np.concatenate([c[k] for c in ch], axis=0)

    def material_data(self) -> np.ndarray:
        if "mat" not in self._cache:
            self._cache["mat"] = np.asarray(self._mat_rows, dtype=np.float64).astype(
                np.float32).reshape(-1)
        return self._cache["mat"]

    def sphere_data(self) -> np.ndarray:
        if "sphere" not in self._cache:
            n = self.sphere_count
            out = np.zeros((n, FLOATS_PER_SPHERE), dtype=np.float32)
            if n:
                out[:, 0:3] = self._cat("sphere", 0)
                out[:, 3] = self._cat("sphere", 1)
                out[:, 4] = self._cat("sphere", 2)
            self._cache["sphere"] = out.reshape(-1)
        return self._cache["sphere"]

    def box_data(self) -> np.ndarray:
        if "box" not in self._cache:
            n = self.box_count
            out = np.zeros((n, FLOATS_PER_BOX), dtype=np.float32)
            if n:
                out[:, 0:3] = self._cat("box", 0)
                out[:, 3:6] = self._cat("box", 1)
                out[:, 6] = self._cat("box", 2)
            self._cache["box"] = out.reshape(-1)
        return self._cache["box"]

    def plane_data(self) -> np.ndarray:
        if "plane" not in self._cache:
            n = self.plane_count
            out = np.zeros((n, FLOATS_PER_PLANE), dtype=np.float32)
            if n:
                out[:, 0:3] = self._cat("plane", 0)
                out[:, 3] = self._cat("plane", 1)
                out[:, 18 + 5] = self._cat("plane", 2)
                out[:, 18 + 6] = -1.0
                out[:, 18 + 7] = -1.0
                for i, rec in self._plane_grids.items():
                    surface = out[i, 18 + 5]
                    out[i, 4:] = rec
                    out[i, 18 + 5] = surface
            self._cache["plane"] = out.reshape(-1)
        return self._cache["plane"]

    def _affine_data(self, kind) -> np.ndarray:
        key = kind + "_data"
        if key not in self._cache:
            n = self._count(kind)
            out = np.zeros((n, FLOATS_PER_AFFINE), dtype=np.float32)
            if n:
                inv = self._cat(kind, 0)
                c = self._cat(kind, 1)
                # writeObjectRelativeAffine (GpuScene.java:924-937): rows of the inverse
                # linear map with the world centre in the translation slots.
                out[:, 0:3] = inv[:, 0, :]
                out[:, 3] = c[:, 0]
                out[:, 4:7] = inv[:, 1, :]
                out[:, 7] = c[:, 1]
                out[:, 8:11] = inv[:, 2, :]
                out[:, 11] = c[:, 2]
                # writeAffineLinear of the inverse transpose (GpuScene.java:939-949).
                out[:, 12:21] = np.transpose(inv, (0, 2, 1)).reshape(n, 9)
                out[:, 21] = self._cat(kind, 4)
            self._cache[key] = out.reshape(-1)
        return self._cache[key]

    def affine_sphere_data(self) -> np.ndarray:
        return self._affine_data("asphere")

    def affine_box_data(self) -> np.ndarray:
        return self._affine_data("abox")

    def _affine_bounds(self, kind) -> np.ndarray:
        key = kind + "_bounds"
        if key not in self._cache:
            n = self._count(kind)
            out = np.zeros((n, 6), dtype=np.float32)
            if n:
                out[:, 0:3] = self._cat(kind, 2)
                out[:, 3:6] = self._cat(kind, 3)
            self._cache[key] = out.reshape(-1)
        return self._cache[key]

    def affine_sphere_bounds(self) -> np.ndarray:
        """Float-cast world bounds of the affine spheres (the BVH build input,
        GpuScene.java:640-649)."""
        return self._affine_bounds("asphere")

    def affine_box_bounds(self) -> np.ndarray:
        return self._affine_bounds("abox")

    def arrays(self):
        """The six packed arrays in C-ABI order: spheres, boxes, planes, affine spheres,
        affine boxes, materials, with their record counts."""
        arrs = [self.sphere_data(), self.box_data(), self.plane_data(),
                self.affine_sphere_data(), self.affine_box_data(), self.material_data()]
        counts = [self.sphere_count, self.box_count, self.plane_count,
                  self.affine_sphere_count, self.affine_box_count, self.material_count()]
        return arrs, counts
