"""Host-side scene API (rtb200.scene), the mirror of gfxlab/gpu/GpuScene.java,
BvhBuildConfig.java and GpuSceneBuilder.java: packed layouts, material deduplication,
validation errors and configuration canonicalisation."""
import math

import numpy as np
import pytest

from rtb200 import synth
from rtb200.scene import (MIN_PACKED_PRIMITIVE_EXTENT, BvhBuildConfig, BvhBuildMode, GpuScene,
                          MaterialData, affine_inverse, gpu_affine)

M = MaterialData.matte((0.5, 0.25, 0.125))


def test_packed_layouts_match_the_reference():
    s = GpuScene()
    s.add_sphere((1.0, 2.0, 3.0), 0.5, M)
    s.add_box((1.0, 1.0, 1.0), (0.0, 2.0, -1.0), MaterialData.light((2.0, 2.0, 2.0)))
    s.add_plane((0.0, -1.0, 0.0), (0.0, 2.0, 0.0), M)
    # GpuScene.sphereData: centre, radius, material (GpuScene.java:518-531)
    np.testing.assert_array_equal(s.sphere_data(), np.float32([1, 2, 3, 0.5, 0]))
    # boxData: canonical min, max, material (addBox sorts the corners, GpuScene.java:223-233)
    np.testing.assert_array_equal(s.box_data(), np.float32([0, 1, -1, 1, 2, 1, 1]))
    # planeData: unit normal, offset -n.p, grid slots with surface material (GpuScene.java:548-569)
    p = s.plane_data()
    assert p.size == 26
    np.testing.assert_array_equal(p[:4], np.float32([0, 1, 0, 1]))
    assert p[18] == 0.0 and p[23] == 0.0 and p[24] == -1.0 and p[25] == -1.0
    # materialData: diffuse, reflective, refractive, emittance, ior (GpuScene.java:972-979)
    np.testing.assert_array_equal(s.material_data()[:13],
                                  np.float32([0.5, 0.25, 0.125, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1.5]))
    assert s.material_count() == 2


def test_materials_are_deduplicated_by_value_in_first_seen_order():
    s = GpuScene()
    a = s.register_material(M)
    b = s.register_material(MaterialData.matte((0.1, 0.1, 0.1)))
    c = s.register_material(MaterialData.matte((0.5, 0.25, 0.125)))
    assert (a, b, c) == (0, 1, 0)


def test_affine_records_are_object_relative():
    t = np.zeros((1, 3, 4))
    t[0, :, :3] = np.diag([2.0, 0.5, 1.0])
    t[0, :, 3] = (10.0, -3.0, 0.25)
    inv, centre, lo, hi = gpu_affine(t, "sphere")
    s = GpuScene()
    s.add_affine_spheres(inv, centre, lo, hi, [s.register_material(M)])
    d = s.affine_sphere_data()
    # rows of the inverse with the world centre in slots 3, 7, 11 (GpuScene.java:924-937)
    np.testing.assert_array_equal(d[[0, 5, 10]], np.float32([0.5, 2.0, 1.0]))
    np.testing.assert_array_equal(d[[3, 7, 11]], np.float32([10.0, -3.0, 0.25]))
    # then the inverse transpose (here diagonal) and the material
    np.testing.assert_array_equal(d[[12, 16, 20]], np.float32([0.5, 2.0, 1.0]))
    assert d[21] == 0.0
    # sphere bounds: centre +- row lengths of the forward map (GpuSceneBuilder.java:84-94)
    np.testing.assert_allclose(hi[0] - centre[0], [2.0, 0.5, 1.0])


def test_affine_inverse_is_exact_for_rotation_and_scale():
    rng_rot = synth.random_rotations(synth.Stream(3, 9, 0, 0), 5)
    t = np.zeros((5, 3, 4))
    t[:, :, :3] = rng_rot * np.array([0.5, 1.5, 2.0])[None, None, :]
    inv = affine_inverse(t)
    prod = np.einsum("kij,kjl->kil", inv[:, :, :3], t[:, :, :3])
    np.testing.assert_allclose(prod, np.broadcast_to(np.eye(3), prod.shape), atol=1e-12)


def test_validation_mirrors_the_reference():
    s = GpuScene()
    with pytest.raises(ValueError):
        s.add_sphere((0, 0, 0), 0.0, M)
    with pytest.raises(ValueError):
        s.add_sphere((0, 0, 0), float(MIN_PACKED_PRIMITIVE_EXTENT) / 4, M)
    with pytest.raises(ValueError):
        s.add_sphere((1e39, 0, 0), 1.0, M)  # not representable as float
    with pytest.raises(ValueError):
        s.add_box((0, 0, 0), (1, 1, 0), M)  # zero extent
    with pytest.raises(ValueError):
        s.add_plane((0, 0, 0), (0, 0, 0), M)
    t = np.zeros((1, 3, 4))
    t[0, :, :3] = np.diag([1e-3, 1.0, 1e3])  # condition number 1e6 > 65536
    inv, c, lo, hi = gpu_affine(t, "box")
    with pytest.raises(ValueError):
        s.add_affine_boxes(inv, c, lo, hi, [0])


def test_build_config_canonicalisation():
    c = BvhBuildConfig(BvhBuildMode.WEIGHTED_SAH, 4, lam=0.0)
    assert c.mode == BvhBuildMode.UNIFORM_SAH  # lambda zero is the ordinary objective
    with pytest.raises(ValueError):
        BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 4, lam=0.5)
    with pytest.raises(ValueError):
        BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 0)
    w = BvhBuildConfig.weighted(leaf_size=4)
    assert w.construction_weight(1.3) == 1.0 + 1.0 * (1.3 - 1.0)
    assert BvhBuildConfig().construction_weight(2.1) == 1.0


def test_synthetic_workloads_are_deterministic_and_sized():
    a, b = synth.plain_workload(), synth.plain_workload()
    for x, y in zip(a.scene.arrays()[0], b.scene.arrays()[0]):
        np.testing.assert_array_equal(x, y)
    assert a.scene.sphere_count == 65 and a.scene.plane_count == 6
    h = synth.hetero_workload()
    s = h.scene
    assert (s.sphere_count, s.box_count, s.affine_sphere_count, s.affine_box_count) == (4001, 3000, 1500, 1500)
    assert (h.width, h.height, h.spp, h.max_depth) == (1024, 1024, 64, 8)
    assert s.config.mode == BvhBuildMode.WEIGHTED_SAH and s.config.leaf_size == 4
    assert (s.config.box_weight, s.config.affine_sphere_weight) == (1.3, 2.1)


def test_primary_grid_matches_camera_convention():
    cam = synth.camera_looking_z((0.0, 0.0, -2.9))
    rays = synth.primary_grid(cam, 4, 2)
    t = math.tan(math.radians(30.0))
    # pixel (0, 0) centre: u = (-1 + 2 * 0.5 / 4) * 2, v = 1 - 2 * 0.5 / 2
    np.testing.assert_allclose(rays[0, 3:], np.float32([-1.5 * t, 0.5 * t, 1.0]), rtol=1e-6)
