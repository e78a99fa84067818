"""CPU checks of the primitive-cost calibration workload (rtb200.calibrate), a restatement of
gfxlab/gpu/PrimitiveCostBenchmark.java:488-697: the counter hash, table shapes, ray
normalisation, and one record recomputed from the generator's formulas."""
import math

import numpy as np

from rtb200 import calibrate as K


def _hash_py(x):
    x &= 0xFFFFFFFF
    for shift, mul in ((17, 0xED5AD4BB), (11, 0xAC4C1B51), (15, 0x31848BAB)):
        x ^= x >> shift
        x = (x * mul) & 0xFFFFFFFF
    return x ^ (x >> 14)


def _unit(v):
    return np.float32((v >> 8) * 2.0 ** -24)


def test_hash_matches_the_kernel_hash():
    vals = np.array([0, 1, 7, 0x9E3779B9, 0xFFFFFFFF], np.uint32)
    assert [int(v) for v in K._hash32(vals)] == [_hash_py(int(v)) for v in vals]


def test_workload_shapes_and_determinism():
    a, b = K.calibration_workload(), K.calibration_workload()
    assert a.rays.shape == (3, 4096, 6) and a.spheres.shape == (4096, 4)
    assert a.boxes.shape == (4096, 8) and a.affines.shape == (4096, 12)
    assert a.planes.shape == (4096, 4) and a.nodes.shape == (4096, 16)
    for f in ("rays", "spheres", "boxes", "affines", "planes", "nodes"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    d = a.rays[..., 3:].astype(np.float64)
    np.testing.assert_allclose(np.linalg.norm(d, axis=-1), 1.0, atol=1e-6)
    assert np.all(a.boxes[:, 0:3] < a.boxes[:, 4:7])
    assert np.all(a.nodes[:, 1] <= a.nodes[:, 5])  # left child's max x <= right child's max x


def test_record_zero_follows_the_generator():
    w = K.calibration_workload()
    s = _hash_py(0)  # record 0: hash32(0 * 0x9E3779B9)
    x = np.float32(2.0) * _unit(s) - np.float32(1.0)
    cx = np.float32(x * np.float32(0.28))
    r = np.float32(0.58) + np.float32(0.34) * _unit(_hash_py(s ^ 0x13198A2E))
    assert w.spheres[0, 0] == cx and w.spheres[0, 3] == np.float32(r)
    hx = np.float32(0.52) + np.float32(0.35) * _unit(_hash_py(s ^ 0x03707344))
    assert w.boxes[0, 0] == np.float32(cx - hx) and w.boxes[0, 4] == np.float32(cx + hx)
    ang = float(np.float32(2.0) * _unit(_hash_py(s ^ 0x452821E6)) - np.float32(1.0)) * 0.85
    sx = 0.62 + 0.78 * float(_unit(_hash_py(s ^ 0x38D01377)))
    assert abs(w.affines[0, 0] - math.cos(ang) / sx) < 1e-6
    # profile 0 ray of record 0: a narrow bundle from (0, 0, -3) along +z
    np.testing.assert_array_equal(w.rays[0, 0, :3], np.float32([0.0, 0.0, -3.0]))
    assert w.rays[0, 0, 5] > 0.999999


def test_build_config_from_weights():
    cal = K.CostCalibration("dev", {"sphere": 1.0, "box": 1.5, "affineSphere": 3.0, "affineBox": 3.5,
                                    "nodeAabb": 0.4, "interiorTraversal": 1.1, "plane": 2.0},
                            [], [], 0)
    c = cal.build_config(leaf_size=4)
    assert (c.box_weight, c.affine_sphere_weight, c.affine_box_weight, c.traversal_weight) == \
        (1.5, 3.0, 3.5, 1.1)
