"""ctypes bindings of the oracle (test infrastructure only).

The oracle is the checker, never the product: only tests/, ``__graft_entry__.smoke()`` and
bench.py's ``cpu_baseline`` / ``--impl reference`` legs import this module.

* ``build_bvh``  -- C++ restatement of the reference's Java GpuScene BVH builder
  (oracle_bvh.cpp), returning the reference's flattened arrays.
* ``trace``      -- FP32 restatement of the reference kernel's closest-hit query
  (oracle_trace.cpp), bit-exact against the reference kernel built with -fmad=false.
* ``render``     -- FP32 restatement of renderKernel's per-pixel sample loop.
* ``cpu_render`` -- FP64 restatement of the reference's CPU path tracer (oracle_cpu.cpp).
* ``ref_trace`` / ``ref_render`` -- the reference's own CUDA kernels, extracted and built
  for sm_100a (oracle/_ref/), launched with the reference's launch plan.
* ``topology_sha256`` -- MethodCatalog.topologySha256 (gfxlab/benchmark/MethodCatalog.java:
  164-172, 203-223): SHA-256 over big-endian int32 words, each array prefixed by its length.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run oracle/build_oracle.py)")
        _lib = C.CDLL(path)
        _lib.orc_build_bvh.restype = C.c_int
        _lib.orc_build_bvh_binned.restype = C.c_int
        _lib.orc_build_bvh_rotations.restype = C.c_int
        _lib.orc_trace.restype = None
        _lib.orc_render.restype = None
        _lib.orc_cpu_render.restype = C.c_int
        _lib.orc_adjoint.restype = None
        _lib.orc_primitive_distance.restype = None
    return _lib


def ref_lib(variant="fmad"):
    if variant not in _ref:
        path = os.path.join(HERE, "_ref", "libref_%s.so" % variant)
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        l = C.CDLL(path)
        l.ref_trace.restype = C.c_int
        l.ref_render.restype = C.c_int
        _ref[variant] = l
    return _ref[variant]


def ref_available(variant="fmad"):
    return os.path.exists(os.path.join(HERE, "_ref", "libref_%s.so" % variant))


class _Cfg(C.Structure):
    _fields_ = [("mode", C.c_int), ("leaf_size", C.c_int), ("traversal_weight", C.c_double),
                ("sphere_weight", C.c_double), ("box_weight", C.c_double),
                ("affine_sphere_weight", C.c_double), ("affine_box_weight", C.c_double),
                ("lam", C.c_double)]


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Bvh:
    """The reference's flattened BVH arrays (GpuScene.bvhNodeBoundsData / bvhNodeData /
    bvhPrimitiveRefs / bvhRootIndices) plus BvhStats fields."""

    def __init__(self, node_bounds, node_data, refs, roots, counts, sah):
        self.node_bounds = node_bounds
        self.node_data = node_data
        self.refs = refs
        self.roots = roots
        (self.node_count, self.root_count, self.leaf_count, self.max_depth,
         self.ref_count, self.min_leaf, self.max_leaf) = [int(v) for v in counts]
        self.generalized_sah, self.uniform_sah, self.weighted_sah = [float(v) for v in sah]

    def topology_sha256(self):
        return topology_sha256(self.node_bounds, self.node_data, self.refs, self.roots)


def build_bvh(scene, config=None, bins=0, rotation_passes=4):
    """Builds the reference BVH for a rtb200.scene.GpuScene (or config override); with
    bins in 2..32, the library's binned object-SAH mode instead of the full sweep.  The
    rotation modes apply BvhRotator with ``rotation_passes`` passes; the Bvh's
    ``rotations`` is the number of rotations made."""
    cfg = config if config is not None else scene.config
    c = _Cfg(int(cfg.mode), cfg.leaf_size, cfg.traversal_weight, cfg.sphere_weight,
             cfg.box_weight, cfg.affine_sphere_weight, cfg.affine_box_weight, cfg.lam)
    ns, nb = scene.sphere_count, scene.box_count
    nas, nab = scene.affine_sphere_count, scene.affine_box_count
    n = ns + nb + nas + nab
    sp, bx = _f32(scene.sphere_data()), _f32(scene.box_data())
    ab, bb = _f32(scene.affine_sphere_bounds()), _f32(scene.affine_box_bounds())
    nbounds = np.zeros(max(1, 2 * n) * 6, np.float32)
    ndata = np.zeros(max(1, 2 * n) * 4, np.int32)
    refs = np.zeros(max(1, n), np.int32)
    roots = np.zeros(4, np.int32)
    counts = np.zeros(7, np.int32)
    sah = np.zeros(3, np.float64)
    outs = (_fp(nbounds), _ip(ndata), _ip(refs), _ip(roots), _ip(counts),
            sah.ctypes.data_as(C.POINTER(C.c_double)))
    rot = C.c_int(0)
    if bins:
        rc = lib().orc_build_bvh_binned(_fp(sp), ns, _fp(bx), nb, _fp(ab), nas, _fp(bb), nab,
                                        C.byref(c), int(bins), *outs)
    elif int(cfg.mode) in (6, 7):
        rc = lib().orc_build_bvh_rotations(_fp(sp), ns, _fp(bx), nb, _fp(ab), nas, _fp(bb), nab,
                                           C.byref(c), int(rotation_passes), *outs, C.byref(rot))
    else:
        rc = lib().orc_build_bvh(_fp(sp), ns, _fp(bx), nb, _fp(ab), nas, _fp(bb), nab,
                                 C.byref(c), *outs)
    if rc != 0:
        raise RuntimeError("oracle BVH build failed: %d" % rc)
    nn, nr, nref = int(counts[0]), int(counts[1]), int(counts[4])
    out = Bvh(nbounds[:6 * nn].copy(), ndata[:4 * nn].copy(), refs[:nref].copy(),
              roots[:nr].copy(), counts, sah)
    out.rotations = rot.value
    return out


def build_bvh_sbvh(scene, config=None, options=None):
    """The SBVH modes (UNIFORM_SBVH / WEIGHTED_SBVH): the restatement of the reference's
    SpatialBuildState (oracle_bvh.cpp).  options: a BvhBuildOptions-like object (defaults
    128 bins, multiplier 2.0, 8 splits per primitive, 16 references, overlap 1e-5).  The
    Bvh's ``spatial_splits`` is BvhStats.spatialSplitCount."""
    cfg = config if config is not None else scene.config
    o = options if options is not None else scene.options
    c = _Cfg(int(cfg.mode), cfg.leaf_size, cfg.traversal_weight, cfg.sphere_weight,
             cfg.box_weight, cfg.affine_sphere_weight, cfg.affine_box_weight, cfg.lam)
    ns, nb = scene.sphere_count, scene.box_count
    nas, nab = scene.affine_sphere_count, scene.affine_box_count
    n = ns + nb + nas + nab
    cap = max(n, int(np.floor(n * o.max_reference_multiplier)), 1)
    sp, bx = _f32(scene.sphere_data()), _f32(scene.box_data())
    ab, bb = _f32(scene.affine_sphere_bounds()), _f32(scene.affine_box_bounds())
    nbounds = np.zeros(2 * cap * 6, np.float32)
    ndata = np.zeros(2 * cap * 4, np.int32)
    refs = np.zeros(cap, np.int32)
    roots = np.zeros(4, np.int32)
    counts = np.zeros(7, np.int32)
    sah = np.zeros(3, np.float64)
    splits = C.c_int(0)
    lib().orc_build_bvh_sbvh.restype = C.c_int
    rc = lib().orc_build_bvh_sbvh(
        _fp(sp), ns, _fp(bx), nb, _fp(ab), nas, _fp(bb), nab, C.byref(c), int(o.spatial_bins),
        C.c_double(o.max_reference_multiplier), int(o.max_splits_per_primitive),
        int(o.min_spatial_references), C.c_double(o.spatial_overlap_threshold), _fp(nbounds),
        _ip(ndata), _ip(refs), _ip(roots), _ip(counts), sah.ctypes.data_as(C.POINTER(C.c_double)),
        C.byref(splits))
    if rc != 0:
        raise RuntimeError("oracle SBVH build failed: %d" % rc)
    nn, nr, nref = int(counts[0]), int(counts[1]), int(counts[4])
    out = Bvh(nbounds[:6 * nn].copy(), ndata[:4 * nn].copy(), refs[:nref].copy(),
              roots[:nr].copy(), counts, sah)
    out.spatial_splits = splits.value
    out.rotations = 0
    return out


def topology_sha256(node_bounds, node_data, refs, roots):
    h = hashlib.sha256()
    for arr in (np.asarray(node_bounds, np.float32).view(np.int32), np.asarray(node_data, np.int32),
                np.asarray(refs, np.int32), np.asarray(roots, np.int32)):
        h.update(np.array([len(arr)], dtype=">i4").tobytes())
        h.update(arr.astype(">i4").tobytes())
    return h.hexdigest()


class _SceneArgs:
    """Keeps the marshalled arrays alive for one call."""

    def __init__(self, scene, bvh=None, use_bvh=True, stack_size=32):
        arrs, counts = scene.arrays()
        self.arrs = [_f32(a) if len(a) else np.zeros(1, np.float32) for a in arrs]
        self.ptrs = (C.POINTER(C.c_float) * 6)(*[_fp(a) for a in self.arrs])
        self.counts = _i32(counts)
        if bvh is None or not use_bvh:
            self.nb = np.zeros(6, np.float32)
            self.nd = np.zeros(4, np.int32)
            self.refs = np.zeros(1, np.int32)
            self.roots = np.zeros(1, np.int32)
            self.bvh_ints = _i32([0, 0, 0, 0, stack_size])
        else:
            self.nb = _f32(bvh.node_bounds)
            self.nd = _i32(bvh.node_data)
            self.refs = _i32(bvh.refs)
            self.roots = _i32(bvh.roots)
            self.bvh_ints = _i32([bvh.node_count, bvh.ref_count, bvh.root_count, 1, stack_size])

    def args(self):
        return (self.ptrs, _ip(self.counts), _ip(self.bvh_ints), _fp(self.nb), _ip(self.nd),
                _ip(self.refs), _ip(self.roots))


def _hit_arrays(n):
    return (np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros(n, np.int32),
            np.zeros(n, np.int32), np.zeros(3 * n, np.float32), np.zeros(14, np.uint64))


def _hits_dict(out):
    flags, t, order, mat, nrm, stats = out
    return {"hit": flags, "t": t, "order": order, "material": mat, "normal": nrm.reshape(-1, 3),
            "stats": stats}


def trace(scene, rays, bvh=None, use_bvh=True, stack_size=32):
    """FP32 restatement of traceReplayKernel over rays (n, 6) float32."""
    rays = _f32(rays).reshape(-1, 6)
    n = len(rays)
    sa = _SceneArgs(scene, bvh, use_bvh, stack_size)
    out = _hit_arrays(n)
    lib().orc_trace(*sa.args(), _fp(rays), n, _ip(out[0]), _fp(out[1]), _ip(out[2]), _ip(out[3]),
                    _fp(out[4]), out[5].ctypes.data_as(C.POINTER(C.c_ulonglong)))
    return _hits_dict(out)


def ref_trace(scene, rays, bvh=None, use_bvh=True, variant="fmad"):
    """The reference's traceReplayKernel (built for sm_100a) over rays; needs a GPU."""
    rays = _f32(rays).reshape(-1, 6)
    n = len(rays)
    sa = _SceneArgs(scene, bvh, use_bvh)
    out = _hit_arrays(n)
    rc = ref_lib(variant).ref_trace(*sa.args(), _fp(rays), n, _ip(out[0]), _fp(out[1]),
                                    _ip(out[2]), _ip(out[3]), _fp(out[4]),
                                    out[5].ctypes.data_as(C.POINTER(C.c_ulonglong)))
    if rc != 0:
        raise RuntimeError("reference trace failed: %d" % rc)
    return _hits_dict(out)


def primitive_distance(scene, rays, orders):
    """Distance of each ray to the primitive of the given global order (planes included),
    computed by that primitive's own test in the restatement's uncontracted FP32 arithmetic
    with no earlier hit; +inf where it misses."""
    rays = _f32(rays).reshape(-1, 6)
    orders = _i32(orders).reshape(-1)
    assert len(orders) == len(rays)
    arrs, counts = scene.arrays()
    arrs = [_f32(a) if len(a) else np.zeros(1, np.float32) for a in arrs]
    ptrs = (C.POINTER(C.c_float) * 6)(*[_fp(a) for a in arrs])
    out = np.zeros(len(rays), np.float32)
    lib().orc_primitive_distance(ptrs, _ip(_i32(counts)), _fp(rays), _ip(orders), len(rays),
                                 _fp(out))
    return out


def _render_params(w):
    return _i32([w.width, w.height, w.spp, w.max_depth, w.frame_index])


def render(workload, bvh=None, use_bvh=True, pixel_begin=0, pixel_end=None):
    """FP32 restatement of renderKernel for a pixel range of a synth.Workload."""
    w = workload
    pe = w.width * w.height if pixel_end is None else pixel_end
    sa = _SceneArgs(w.scene, bvh, use_bvh)
    cam = _f32(w.camera.packed())
    bg = _f32(w.scene.background)
    out = np.zeros(3 * (pe - pixel_begin), np.float32)
    lib().orc_render(*sa.args(), _fp(cam), _fp(bg), _ip(_render_params(w)),
                     C.c_ulonglong(w.frame_seed), pixel_begin, pe, _fp(out))
    return out.reshape(-1, 3)


def ref_render(workload, bvh=None, use_bvh=True, warmup=0, frames=1, variant="fmad",
               flush_bytes=0):
    """The reference's renderKernel with renderSample's launch plan; returns (image (H*W,3),
    summed CUDA-event milliseconds of the timed frames).  With ``flush_bytes`` > 0 every
    timed frame has its own events and a buffer of that size is written before it, outside
    the events (an L2 flush)."""
    w = workload
    sa = _SceneArgs(w.scene, bvh, use_bvh)
    cam = _f32(w.camera.packed())
    bg = _f32(w.scene.background)
    out = np.zeros(3 * w.width * w.height, np.float32)
    ms = C.c_double(0.0)
    lib_ = ref_lib(variant)
    if flush_bytes:
        lib_.ref_render_flushed.restype = C.c_int
        rc = lib_.ref_render_flushed(*sa.args(), _fp(cam), _fp(bg), _ip(_render_params(w)),
                                     C.c_ulonglong(w.frame_seed), warmup, frames,
                                     C.c_ulonglong(flush_bytes), _fp(out), C.byref(ms))
    else:
        rc = lib_.ref_render(*sa.args(), _fp(cam), _fp(bg), _ip(_render_params(w)),
                             C.c_ulonglong(w.frame_seed), warmup, frames, _fp(out), C.byref(ms))
    if rc != 0:
        raise RuntimeError("reference render failed: %d" % rc)
    return out.reshape(-1, 3), ms.value


def ref_render_stats(workload, bvh=None, use_bvh=True):
    """One frame of the reference's renderKernel from its metrics build (no contraction,
    GFXLAB_RENDER_METRICS): (image (H*W,3), the 14 frame counters of K:30-43)."""
    w = workload
    sa = _SceneArgs(w.scene, bvh, use_bvh)
    out = np.zeros(3 * w.width * w.height, np.float32)
    stats = np.zeros(14, np.uint64)
    rc = ref_lib("metrics").ref_render_stats(
        *sa.args(), _fp(_f32(w.camera.packed())), _fp(_f32(w.scene.background)),
        _ip(_render_params(w)), C.c_ulonglong(w.frame_seed), _fp(out),
        stats.ctypes.data_as(C.POINTER(C.c_ulonglong)))
    if rc != 0:
        raise RuntimeError("reference metrics render failed: %d" % rc)
    return out.reshape(-1, 3), stats


def cpu_render(workload, frames=None, rows=None, threads=0, seed=0x68EFD508E309A865):
    """FP64 restatement of the reference CPU renderer; returns (H_rows*W, 3) doubles."""
    w = workload
    arrs, counts = w.scene.arrays()
    arrs = [_f32(a) if len(a) else np.zeros(1, np.float32) for a in arrs]
    ptrs = (C.POINTER(C.c_float) * 6)(*[_fp(a) for a in arrs])
    cnt = _i32(counts)
    r0, r1 = (0, w.height) if rows is None else rows
    params = _i32([w.width, w.height, w.spp if frames is None else frames, w.max_depth])
    out = np.zeros(3 * (r1 - r0) * w.width, np.float64)
    lib().orc_cpu_render(ptrs, _ip(cnt), _fp(_f32(w.camera.packed())),
                         _fp(_f32(w.scene.background)), _ip(params), C.c_ulonglong(seed),
                         r0, r1, threads, out.ctypes.data_as(C.POINTER(C.c_double)))
    return out.reshape(-1, 3)


def adjoint(workload, adjoint_image, bvh=None, use_bvh=True, materials=None):
    """FP64 restatement of the path-replay adjoint (orc_adjoint): dLoss/d(albedo) and
    dLoss/d(emission) per material for dLoss/dI = adjoint_image (H*W*3)."""
    w = workload
    sa = _SceneArgs(w.scene, bvh, use_bvh)
    if materials is not None:
        sa.arrs[5] = _f32(materials).reshape(-1)
        sa.ptrs[5] = _fp(sa.arrs[5])
    cam = _f32(w.camera.packed())
    bg = _f32(w.scene.background)
    adj = _f32(adjoint_image).reshape(-1)
    m = int(sa.counts[5])
    ga = np.zeros(3 * m, np.float64)
    ge = np.zeros(3 * m, np.float64)
    lib().orc_adjoint(*sa.args(), _fp(cam), _fp(bg), _ip(_render_params(w)),
                      C.c_ulonglong(w.frame_seed), 0, w.width * w.height, _fp(adj),
                      ga.ctypes.data_as(C.POINTER(C.c_double)),
                      ge.ctypes.data_as(C.POINTER(C.c_double)))
    return ga.reshape(-1, 3), ge.reshape(-1, 3)
