"""Primitive-cost calibration on the current GPU (the counterpart of
gfxlab/gpu/PrimitiveCostBenchmark.java and of the constants it produced,
gfxlab/gpu/PrimitiveCostModel.java:11-19, measured on an RTX 3080).

``calibration_workload`` restates the benchmark's synthetic workload
(PrimitiveCostBenchmark.buildWorkload and its write*Record helpers, lines 488-697): 4096
records per table, three ray profiles (a narrow bundle straight at the records, a wide fan,
and origins spread over a disc), spheres, boxes, rotated-and-scaled affine records, tilted
planes and child-pair nodes around shared centres, all drawn from the counter hash.  The
trigonometry goes through numpy, so records can differ from the Java ones in the last bit;
the calibration needs the same distribution, not the same bits.

``calibrate`` runs rtb_calibrate_costs, the device protocol (paired setup / operation
launches, each operation paired with a local sphere measurement, medians over repeats, median
over profiles), and returns sphere-normalised weights for this library's own operations;
``CostCalibration.build_config`` turns them into a BvhBuildConfig for the weighted SAH.
"""
import ctypes as C
import dataclasses
from typing import Dict, List, Optional

import numpy as np

from . import native as N
from .scene import BvhBuildConfig, BvhBuildMode

LABELS = ("setup", "sphere", "box", "affineSphere", "affineBox", "nodeAabb", "interiorTraversal",
          "plane")
RECORDS = 4096
PROFILES = 3

# PrimitiveCostModel.java:11-19 (RTX 3080, compute_86), for comparison
RTX3080 = {"sphere": 1.0, "box": 1.288951704, "affineSphere": 2.552743938,
           "affineBox": 2.728115282, "plane": 2.860319327, "nodeAabb": 0.507189194,
           "interiorTraversal": 1.275576713}


def _hash32(v):
    """hash_u32 of the reference kernel (K:165-173) on uint32 arrays (wrapping)."""
    v = np.asarray(v, dtype=np.uint32).copy()
    v ^= v >> np.uint32(17)
    v *= np.uint32(0xED5AD4BB)
    v ^= v >> np.uint32(11)
    v *= np.uint32(0xAC4C1B51)
    v ^= v >> np.uint32(15)
    v *= np.uint32(0x31848BAB)
    v ^= v >> np.uint32(14)
    return v


def _unit(v):
    return (np.asarray(v, np.uint32) >> np.uint32(8)).astype(np.float32) * np.float32(2.0 ** -24)


def _signed_unit(v):
    return np.float32(2.0) * _unit(v) - np.float32(1.0)


def _u32(x):
    return np.uint32(x & 0xFFFFFFFF)


@dataclasses.dataclass
class CalibrationWorkload:
    rays: np.ndarray      # (profiles, records, 6) float32
    spheres: np.ndarray   # (records, 4): centre, radius
    boxes: np.ndarray     # (records, 8): min, pad, max, pad
    affines: np.ndarray   # (records, 12): inverse rows, centre in the 4th slot
    planes: np.ndarray    # (records, 4): unit normal, offset
    nodes: np.ndarray     # (records, 16) float32 view of child-pair nodes


def calibration_workload(records: int = RECORDS, profiles: int = PROFILES) -> CalibrationWorkload:
    """The calibration workload in this library's device layouts."""
    if records & (records - 1) or not 1 <= profiles <= 3:
        raise ValueError("records must be a power of two and profiles in 1..3")
    rec = np.arange(records, dtype=np.uint32)
    rays = np.zeros((profiles, records, 6), np.float32)
    for p in range(profiles):
        s = _hash32(rec ^ _u32(p * 0x6D2B79F5))
        x = _signed_unit(s).astype(np.float64)
        y = _signed_unit(_hash32(s ^ _u32(0x51ED270B))).astype(np.float64)
        z = _signed_unit(_hash32(s ^ _u32(0xA54FF53A))).astype(np.float64)
        ox = np.zeros(records)
        oy = np.zeros(records)
        oz = np.full(records, -3.0)
        dz = np.ones(records)
        if p == 0:    # narrow bundle
            dx, dy = x * 0.00075, y * 0.00075
        elif p == 1:  # wide fan
            dx, dy = x * 0.36, y * 0.24 - 0.12
        else:         # spread origins
            ox, oy, oz = x * 0.68, y * 0.68, oz + z * 0.20
            dx, dy = x * 0.055, y * 0.055
        il = 1.0 / np.sqrt(dx * dx + dy * dy + dz * dz)
        rays[p] = np.stack([ox, oy, oz, dx * il, dy * il, dz * il], axis=1).astype(np.float32)

    s = _hash32((rec * np.uint32(0x9E3779B9)).astype(np.uint32))
    x = _signed_unit(s)
    y = _signed_unit(_hash32(s ^ _u32(0x243F6A88)))
    z = _signed_unit(_hash32(s ^ _u32(0xB7E15162)))
    cx = x * np.float32(0.28)
    cy = y * np.float32(0.22)
    cz = z * np.float32(0.18) + np.float32(0.35)
    radius = np.float32(0.58) + np.float32(0.34) * _unit(_hash32(s ^ _u32(0x13198A2E)))
    spheres = np.stack([cx, cy, cz, radius], axis=1).astype(np.float32)
    hx = np.float32(0.52) + np.float32(0.35) * _unit(_hash32(s ^ _u32(0x03707344)))
    hy = np.float32(0.52) + np.float32(0.35) * _unit(_hash32(s ^ _u32(0xA4093822)))
    hz = np.float32(0.52) + np.float32(0.35) * _unit(_hash32(s ^ _u32(0x299F31D0)))
    zero = np.zeros(records, np.float32)
    boxes = np.stack([cx - hx, cy - hy, cz - hz, zero, cx + hx, cy + hy, cz + hz, zero],
                     axis=1).astype(np.float32)
    # affine records: rotation about z by up to 0.85 rad, anisotropic scale 0.62..1.40
    ang = _signed_unit(_hash32(s ^ _u32(0x452821E6))).astype(np.float64) * 0.85
    cs, sn = np.cos(ang), np.sin(ang)
    sx = 0.62 + 0.78 * _unit(_hash32(s ^ _u32(0x38D01377))).astype(np.float64)
    sy = 0.62 + 0.78 * _unit(_hash32(s ^ _u32(0xBE5466CF))).astype(np.float64)
    sz = 0.62 + 0.78 * _unit(_hash32(s ^ _u32(0x34E90C6C))).astype(np.float64)
    i00, i01 = (cs / sx).astype(np.float32), (sn / sx).astype(np.float32)
    i10, i11 = (-sn / sy).astype(np.float32), (cs / sy).astype(np.float32)
    i22 = (1.0 / sz).astype(np.float32)
    affines = np.stack([i00, i01, zero, cx, i10, i11, zero, cy, zero, zero, i22, cz],
                       axis=1).astype(np.float32)
    # planes: normals tilted up to 0.12 from -z through a point near the record
    nx = _signed_unit(_hash32(s ^ _u32(0xC0AC29B7))).astype(np.float64) * 0.12
    ny = _signed_unit(_hash32(s ^ _u32(0xC97C50DD))).astype(np.float64) * 0.12
    nz = -np.ones(records)
    il = 1.0 / np.sqrt(nx * nx + ny * ny + nz * nz)
    pnx, pny, pnz = (nx * il).astype(np.float32), (ny * il).astype(np.float32), (nz * il).astype(np.float32)
    pz = np.float32(0.15) * _signed_unit(_hash32(s ^ _u32(0x3F84D5B5)))
    off = -(pnx * cx + pny * cy + pnz * pz)
    planes = np.stack([pnx, pny, pnz, off], axis=1).astype(np.float32)
    # child-pair nodes: the box split at cx + spread along x
    spread = np.float32(0.04) * _signed_unit(_hash32(s ^ _u32(0x9216D5D9)))
    split = np.maximum(np.float32(-0.75) * hx, np.minimum(np.float32(0.75) * hx, spread))
    lx0, lx1 = cx - hx, cx + split
    rx0, rx1 = cx + split, cx + hx
    y0, y1, z0, z1 = cy - hy, cy + hy, cz - hz, cz + hz
    nodes = np.zeros((records, 16), np.float32)
    nodes[:, 0:4] = np.stack([lx0, lx1, y0, y1], axis=1)
    nodes[:, 4:8] = np.stack([rx0, rx1, y0, y1], axis=1)
    nodes[:, 8:12] = np.stack([z0, z1, z0, z1], axis=1)
    return CalibrationWorkload(rays, spheres, boxes, affines, planes, nodes)


@dataclasses.dataclass
class CostCalibration:
    """Sphere-normalised operation costs measured on one device."""
    device: str
    weights: Dict[str, float]
    per_profile: List[Dict[str, float]]
    sphere_ns: List[float]
    tests_per_observation: int

    def build_config(self, leaf_size: int = 4, lam: float = 1.0,
                     mode: BvhBuildMode = BvhBuildMode.WEIGHTED_SAH) -> BvhBuildConfig:
        """BvhBuildConfig with these weights (traversal weight = the interior traversal
        cost, as PrimitiveCostModel.INTERIOR_TRAVERSAL is the reference's default c_T)."""
        w = self.weights
        return BvhBuildConfig(mode, leaf_size, traversal_weight=w["interiorTraversal"],
                              sphere_weight=1.0, box_weight=w["box"],
                              affine_sphere_weight=w["affineSphere"],
                              affine_box_weight=w["affineBox"], lam=lam)


def default_params(sm_count: int, quick: bool = False) -> N.CalibrationParams:
    if quick:
        return N.CalibrationParams(sm_count * 2, 256, 16, 4, 4, 3, 1, 0, 250.0)
    return N.CalibrationParams(sm_count * 8, 256, 256, 8, 8, 6, 2, 0, 250.0)


def calibrate(ctx, params: Optional[N.CalibrationParams] = None,
              workload: Optional[CalibrationWorkload] = None) -> CostCalibration:
    """Runs the device calibration on the context's GPU."""
    w = workload if workload is not None else calibration_workload()
    info = ctx.device_info()
    p = params if params is not None else default_params(info.sm_count)
    arrs = [np.ascontiguousarray(a, np.float32) for a in
            (w.rays, w.spheres, w.boxes, w.affines, w.planes, w.nodes)]
    desc = N.CalibrationWorkload(N.fptr(arrs[0]), w.rays.shape[0], w.rays.shape[1],
                                 *[N.fptr(a) for a in arrs[1:]])
    res = N.CalibrationResult()
    ctx.check(ctx.lib.rtb_calibrate_costs(ctx.handle, C.byref(desc), C.byref(p), C.byref(res)))
    weights = {LABELS[t]: float(res.weight[t]) for t in range(1, 8)}
    per = [{LABELS[t]: float(res.ratio[k][t]) for t in range(1, 8)} for k in range(res.profiles)]
    return CostCalibration(info.name, weights, per,
                           [float(res.sphere_net_ns[k]) for k in range(res.profiles)],
                           int(res.tests_per_observation))


def _render_msamples(ctx, workload, config, frames: int = 5) -> Dict[str, float]:
    """Msamples/s of the workload's frame rendered over a tree built with ``config``
    (median of CUDA-event times, L2 flushed between frames)."""
    import torch

    from .tracer import ResidentScene, camera_struct
    w = workload
    res = ResidentScene.build(ctx, w.scene, config)
    pixels = w.width * w.height
    out = torch.empty(pixels * 3, dtype=torch.float32, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    sh = C.c_void_p(stream.cuda_stream)
    cam = camera_struct(w.camera)

    def render(frame):
        p = N.RenderParams(w.width, w.height, w.spp, w.max_depth, frame,
                           w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
        ctx.check(ctx.lib.rtb_render_device(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                            C.c_void_p(out.data_ptr()), sh))
    with torch.cuda.stream(stream):
        for i in range(2):
            render(i)
    stream.synchronize()
    ms = []
    for _ in range(frames):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            flush.zero_()
            s.record(stream)
            render(0)
            e.record(stream)
        stream.synchronize()
        ms.append(s.elapsed_time(e))
    st = res.stats
    res.close()
    m = sorted(ms)[len(ms) // 2]
    return {"ms": m, "msamples_per_s": pixels * w.spp / m / 1e3, "nodes": st.node_count,
            "generalized_sah": st.generalized_sah_cost}


def main(argv=None) -> None:
    """Prints the device's calibration as JSON; with --compare-render also the render speed
    of the heterogeneous 10k scene (1024x1024, 16 spp, depth 8) over trees built with the
    benchmark's weights, the RTX 3080 model, these weights and the uniform SAH."""
    import argparse
    import json

    from . import synth
    from .tracer import Context
    ap = argparse.ArgumentParser()
    ap.add_argument("--compare-render", action="store_true")
    ap.add_argument("--quick", action="store_true")
    a = ap.parse_args(argv)
    ctx = Context(0)
    cal = calibrate(ctx, default_params(ctx.device_info().sm_count, a.quick))
    out = {"device": cal.device, "weights": cal.weights, "rtx3080": RTX3080,
           "per_profile": cal.per_profile, "sphere_ns_per_test": cal.sphere_ns,
           "tests_per_observation": cal.tests_per_observation}
    if a.compare_render:
        w = synth.hetero_workload()
        w.spp = 16
        rtx = BvhBuildConfig(BvhBuildMode.WEIGHTED_SAH, 4, traversal_weight=RTX3080["interiorTraversal"],
                             box_weight=RTX3080["box"], affine_sphere_weight=RTX3080["affineSphere"],
                             affine_box_weight=RTX3080["affineBox"], lam=1.0)
        out["render_hetero10k_1024x1024x16spp"] = {
            "benchmark_weights": _render_msamples(ctx, w, w.scene.config),
            "rtx3080_model": _render_msamples(ctx, w, rtx),
            "this_calibration": _render_msamples(ctx, w, cal.build_config(leaf_size=4)),
            "uniform_sah": _render_msamples(ctx, w, BvhBuildConfig(BvhBuildMode.UNIFORM_SAH, 4)),
        }
    ctx.close()
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
