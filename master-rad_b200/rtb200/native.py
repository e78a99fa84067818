"""ctypes binding of librtb200.so (the C ABI declared in include/rtb200.h).

The library is loaded from this package directory; a missing or unloadable library raises
immediately -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librtb200.so")

RTB_OK = 0
STATUS_NAMES = {
    0: "RTB_OK", 1: "RTB_ERR_INVALID_ARGUMENT", 2: "RTB_ERR_UNAVAILABLE", 3: "RTB_ERR_CUDA",
    4: "RTB_ERR_OUT_OF_MEMORY", 5: "RTB_ERR_UNSUPPORTED", 6: "RTB_ERR_DEVICE_CHECK",
    7: "RTB_ERR_WATCHDOG", 8: "RTB_ERR_LIMIT",
}

FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int)


class SceneDesc(C.Structure):
    _fields_ = [("spheres", FP), ("sphere_count", C.c_int),
                ("boxes", FP), ("box_count", C.c_int),
                ("planes", FP), ("plane_count", C.c_int),
                ("affine_spheres", FP), ("affine_sphere_count", C.c_int),
                ("affine_boxes", FP), ("affine_box_count", C.c_int),
                ("materials", FP), ("material_count", C.c_int),
                ("affine_sphere_bounds", FP), ("affine_box_bounds", FP),
                ("background", C.c_float * 3)]


class BvhDesc(C.Structure):
    _fields_ = [("node_bounds", FP), ("node_data", IP), ("node_count", C.c_int),
                ("primitive_refs", IP), ("primitive_ref_count", C.c_int),
                ("root_indices", IP), ("root_count", C.c_int)]


class BuildConfig(C.Structure):
    _fields_ = [("mode", C.c_int), ("leaf_size", C.c_int), ("traversal_weight", C.c_double),
                ("sphere_weight", C.c_double), ("box_weight", C.c_double),
                ("affine_sphere_weight", C.c_double), ("affine_box_weight", C.c_double),
                ("lam", C.c_double)]


class BvhStats(C.Structure):
    _fields_ = [("node_count", C.c_int), ("root_count", C.c_int), ("leaf_count", C.c_int),
                ("max_depth", C.c_int), ("primitive_ref_count", C.c_int), ("leaf_size", C.c_int),
                ("min_leaf_occupancy", C.c_int), ("max_leaf_occupancy", C.c_int),
                ("generalized_sah_cost", C.c_double), ("uniform_sah_cost", C.c_double),
                ("weighted_sah_cost", C.c_double), ("bytes", C.c_longlong),
                ("build_ms", C.c_double), ("sequential_nodes", C.c_int),
                ("rotation_count", C.c_int), ("spatial_split_count", C.c_int),
                ("duplicate_reference_count", C.c_int)]


class BuildOptions(C.Structure):
    _fields_ = [("spatial_bins", C.c_int), ("max_reference_multiplier", C.c_double),
                ("max_splits_per_primitive", C.c_int), ("min_spatial_references", C.c_int),
                ("spatial_overlap_threshold", C.c_double), ("rotation_passes", C.c_int)]


class Camera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3),
                ("right", C.c_float * 3), ("up", C.c_float * 3)]


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("samples_per_frame", C.c_int),
                ("max_depth", C.c_int), ("frame_index", C.c_int),
                ("frame_seed", C.c_ulonglong), ("use_bvh", C.c_int),
                ("collect_metrics", C.c_int), ("shared_stack_entries", C.c_int)]


class FrameStats(C.Structure):
    _fields_ = [("total_ns", C.c_longlong), ("kernel_ns", C.c_longlong),
                ("max_physical_kernel_ns", C.c_longlong), ("copy_ns", C.c_longlong),
                ("upload_ns", C.c_longlong), ("counters", C.c_longlong * 14),
                ("physical_launches", C.c_int)]


class BatchJob(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", Camera), ("params", RenderParams),
                ("rgb_device", C.c_void_p)]


CALIBRATION_MAX_PROFILES = 3  # RTB_CALIBRATION_MAX_PROFILES


class CalibrationWorkload(C.Structure):
    _fields_ = [("rays", FP), ("profiles", C.c_int), ("records", C.c_int), ("spheres", FP),
                ("boxes", FP), ("affines", FP), ("planes", FP), ("nodes", FP)]


class CalibrationParams(C.Structure):
    _fields_ = [("blocks", C.c_int), ("threads", C.c_int), ("iterations", C.c_int),
                ("copies", C.c_int), ("sublaunches", C.c_int), ("repeats", C.c_int),
                ("warmups", C.c_int), ("order_offset", C.c_int), ("max_launch_ms", C.c_double)]


class CalibrationResult(C.Structure):
    _fields_ = [("profiles", C.c_int),
                ("net_ns", (C.c_double * 8) * CALIBRATION_MAX_PROFILES),
                ("sphere_ns", (C.c_double * 8) * CALIBRATION_MAX_PROFILES),
                ("ratio", (C.c_double * 8) * CALIBRATION_MAX_PROFILES),
                ("sphere_net_ns", C.c_double * CALIBRATION_MAX_PROFILES),
                ("weight", C.c_double * 8), ("tests_per_observation", C.c_longlong)]


class BatchTuning(C.Structure):
    _fields_ = [("threads_per_block", C.c_int), ("job_order", C.c_int), ("branches", C.c_int),
                ("shared_stack_entries", C.c_int), ("tail_pixels_per_thread", C.c_int)]


# Every symbol include/rtb200.h declares, with its ctypes signature.
SIGNATURES = {
    "rtb_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "rtb_context_destroy": (C.c_int, [C.c_void_p]),
    "rtb_status_string": (C.c_char_p, [C.c_int]),
    "rtb_last_error": (C.c_char_p, [C.c_void_p]),
    "rtb_device_info": (C.c_int, [C.c_void_p, C.c_char_p, C.c_int, IP, IP, IP]),
    "rtb_scene_upload": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(BvhDesc),
                                   C.POINTER(C.c_void_p)]),
    "rtb_scene_build": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(BuildConfig),
                                  C.POINTER(C.c_void_p), C.POINTER(BvhStats)]),
    "rtb_scene_build_with_options": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc),
                                               C.POINTER(BuildConfig), C.POINTER(BuildOptions),
                                               C.POINTER(C.c_void_p), C.POINTER(BvhStats)]),
    "rtb_scene_build_binned": (C.c_int, [C.c_void_p, C.POINTER(SceneDesc), C.POINTER(BuildConfig),
                                         C.c_int, C.POINTER(C.c_void_p), C.POINTER(BvhStats)]),
    "rtb_scene_bvh_sizes": (C.c_int, [C.c_void_p, C.c_void_p, IP, IP, IP]),
    "rtb_scene_download_bvh": (C.c_int, [C.c_void_p, C.c_void_p, FP, IP, IP, IP]),
    "rtb_scene_destroy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rtb_trace_replay": (C.c_int, [C.c_void_p, C.c_void_p, FP, C.c_int, C.c_int, C.c_int,
                                   IP, FP, IP, IP, FP]),
    "rtb_render_sample": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Camera),
                                    C.POINTER(RenderParams), FP]),
    "rtb_render_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Camera),
                                    C.POINTER(RenderParams), C.c_void_p, C.c_void_p]),
    "rtb_render_device_wavefront": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Camera),
                                              C.POINTER(RenderParams), C.c_void_p, C.c_void_p]),
    "rtb_render_rows_device": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Camera),
                                         C.POINTER(RenderParams), C.c_int, C.c_int, C.c_void_p,
                                         C.c_void_p]),
    "rtb_last_frame_stats": (C.c_int, [C.c_void_p, C.POINTER(FrameStats)]),
    "rtb_request_abort": (C.c_int, [C.c_void_p]),
    "rtb_calibrate_costs": (C.c_int, [C.c_void_p, C.POINTER(CalibrationWorkload),
                                      C.POINTER(CalibrationParams),
                                      C.POINTER(CalibrationResult)]),
    "rtb_trace_replay_static": (C.c_int, [C.c_void_p, FP, C.c_int, C.c_int, IP, FP, IP, IP, FP]),
    "rtb_batch_create": (C.c_int, [C.c_void_p, C.POINTER(BatchJob), C.c_int, C.POINTER(BatchTuning),
                                   C.POINTER(C.c_void_p)]),
    "rtb_batch_render": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "rtb_batch_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(BatchTuning),
                                     C.POINTER(C.c_double)]),
    "rtb_batch_destroy": (C.c_int, [C.c_void_p, C.c_void_p]),
    "rtb_scene_set_materials": (C.c_int, [C.c_void_p, C.c_void_p, FP, C.c_int]),
    "rtb_render_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Camera),
                                      C.POINTER(RenderParams), C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p]),
    "rtb_render_backward_sample": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Camera),
                                             C.POINTER(RenderParams), FP, FP, FP]),
}

STATIC_REPLAY_MAX_RAYS = 65536  # RTB_STATIC_REPLAY_MAX_RAYS in include/rtb200.h

_lib = None


def lib():
    """Loads librtb200.so (raises if it is missing: there is no other implementation)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("librtb200.so is not built (run master-rad_b200/build.py); "
                               "the renderer has no fallback implementation")
        l = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


class RtbError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


def fptr(a):
    return a.ctypes.data_as(FP) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(IP) if a is not None else None


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)
