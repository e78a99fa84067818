"""Benchmark: Msamples/s of the path tracer on the heterogeneous cost-weighted workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload hetero|plain|scale]

A step is one full frame of the workload: the 10k-primitive heterogeneous scene (40 %
spheres, 30 % boxes, 30 % affine spheres/boxes, per-type SAH weights 1.0/1.3/2.1, leaf <= 4)
at 1024x1024, 64 samples per pixel, path depth 8, FP32 radiance -- the configuration the
headline metric is quoted on.  Inputs are seeded synthetic scenes (the reference measures
on no public data set).

Arms and keys of the single JSON line printed by rank 0:
  value     frame samples / second with the scene resident in HBM, from CUDA events around
            each frame's render launch on the launching stream (L2 flushed between frames
            by writing a 256 MiB buffer outside the timed events), max over ranks.
  e2e       the same metric through the C ABI with host buffers: each step uploads the
            packed scene from pinned host memory, builds the BVH on the device, renders, and
            reads the image back into pinned host memory (rtb_scene_build +
            rtb_render_sample); wall-clock per step.
  roofline  the render kernel's algorithmic bytes (node + primitive + reference + material
            + plane bytes its traversal fetches, counted by the kernel's metrics build on
            the same frame) per launch / the launch's event time, against the measured HBM
            copy bandwidth.
  cpu_baseline  the FP64 restatement of the reference's CPU renderer on all host cores, on
            a bounded row band of the same frame (rank 0, N = 1).
  build_ms  device BVH build time of the workload's scene (tree identical to the reference
            Java builder's), median of 3; build.binned_ms the binned object-SAH mode (32 bins,
            16 for the plain scene) and its SAH cost relative to the full sweep's.
With --impl reference the line reports the reference CPU renderer (its FP64 restatement;
the Java original cannot run here) on bounded samples of the same frame.
With N > 1 (torchrun) every rank renders its own frames (distinct frame indices) of the same
workload: weak scaling with no data-path collective.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "master-rad_b200"))

import ctypes as C  # noqa: E402

import numpy as np  # noqa: E402

from rtb200 import native as N  # noqa: E402
from rtb200 import synth  # noqa: E402
from rtb200.tracer import Context, ResidentScene, build_config, camera_struct, scene_desc  # noqa: E402

PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
# dram__bytes_read.sum + dram__bytes_write.sum of k_render per sample, from one ncu capture
# of the same scene at a smaller frame: the 10k scene at 1024x768x4 spp
# (profiles/k_render_hetero10k_1024x768x4spp_full.md), the 1M scene at 480x270x4 spp
# (profiles/k_render_scale1M_480x270x4spp_full.md); workloads without a capture report
# null traffic.
CAPTURE_FRAME = {"hetero": "1024x768x4spp", "scale": "480x270x4spp"}
TRAFFIC_BYTES_PER_SAMPLE = {"hetero": (23.57e6 + 143.13e6) / 3145728,
                            "scale": (359.48e6 + 153.86e6) / 518400}
# smsp__inst_executed.sum of k_render per sample from the same captures (8.899 G warp
# instructions for 3,145,728 samples; 2.823 G for 518,400), for the issue bound: warp
# instructions per second against one instruction per cycle on each of the 4 schedulers of
# every SM.
INST_PER_SAMPLE = {"hetero": 8.8986e9 / 3145728, "scale": 2.8227e9 / 518400}
# smsp__thread_inst_executed_per_inst_executed of the same captures: active lanes per warp
# instruction, which scales the issue bound to lane-instructions doing useful work.
LANES_PER_INST = {"hetero": 9.30, "scale": 9.48}


def issue_roofline(workload, samples, launch_ms, sm_count, sm_mhz):
    """The issue bound of the render launch, or None without a capture of this workload."""
    if workload not in INST_PER_SAMPLE or not sm_mhz or not sm_count:
        return None
    inst = INST_PER_SAMPLE[workload] * samples
    achieved = inst / (launch_ms / 1e3)
    peak = sm_count * 4 * sm_mhz * 1e6
    lanes = LANES_PER_INST[workload]
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "warp-inst/s",
            "frac": achieved / peak, "inst_per_launch": inst,
            "active_lanes_per_inst": lanes, "useful_lane_frac": achieved / peak * lanes / 32.0,
            "note": "instructions per sample from the ncu capture of a " + CAPTURE_FRAME[workload] +
                    " frame of the same scene, scaled by samples; peak = SMs x 4 schedulers x the SM "
                    "clock sampled during the timed frames; useful_lane_frac also counts the "
                    "lanes a warp instruction leaves idle (divergent paths)"}


def parse_args(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hetero", choices=["hetero", "plain", "scale", "batched", "adjoint"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ref-kernel", action="store_true")
    ap.add_argument("--form", default="persistent", choices=["persistent", "wavefront"],
                    help="the timed frames' form: the persistent kernel (rtb_render_device) or "
                         "the wavefront kernels (rtb_render_device_wavefront), bit-identical")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the other configurations measured after the headline line's timing")
    ap.add_argument("--split", default="rows", choices=["rows", "frames"],
                    help="with N > 1 GPUs: rows -- every step is one frame whose rows are dealt "
                         "out across the ranks and all-gathered (strong scaling); frames -- "
                         "every rank renders its own frames (weak scaling)")
    ap.add_argument("--ref-frames", type=int, default=0,
                    help="timed frames of the reference kernel (0: 3, or 1 for the 1M scene)")
    # size overrides for small profiling captures of the same scene
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--spp", type=int, default=0)
    return ap.parse_args(argv)


def make_workload(name, args=None):
    if name == "plain":
        w, label = synth.plain_workload(), "plain-64-spheres"
    elif name == "scale":
        w, label = synth.scale_workload(), "scale-1M-clustered"
    else:
        w, label = synth.hetero_workload(), "hetero-10k"
    if args is not None:
        if args.width:
            w.width = args.width
            w.camera = synth.camera_looking_z(w.camera.position, w.width / w.height)
        if args.height:
            w.height = args.height
            w.camera = synth.camera_looking_z(w.camera.position, w.width / w.height)
        if args.spp:
            w.spp = args.spp
    return w, "%s %dx%d %dspp depth%d" % (label, w.width, w.height, w.spp, w.max_depth)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def algorithmic_bytes(counters, hits):
    """Bytes the render kernel's traversal fetches for the counted work: 64 B per interior
    node (both child boxes and links), 16 B per sphere test, 32 B per box test, 48 B per
    affine test, 4 B per leaf reference, 16 B per plane test, and per hit the 64 B material
    record (+36 B normal matrix for affine winners, bounded above by counting it always)."""
    (rays, aabb, prim, sph, box, plane, asph, abox, _ovf, _mx, internal, leaf, _h, _m) = counters
    bvh_prims = sph + box + asph + abox
    return (64 * internal + 16 * sph + 32 * box + 48 * (asph + abox) + 4 * bvh_prims
            + 16 * plane + (64 + 36) * hits)


def ref_kernel_leg(w, tree, frames, flush_bytes):
    """The reference's own renderKernel (extracted from GpuKernelSources.java and built for
    sm_100a by oracle/build_oracle.py) on the same frame, tree, seeds and camera, launched
    with renderSample's plan (one launch per (sample, tile), 16x16 blocks, tiles of at most
    262,144 pixels); CUDA events around each frame, the same L2 flush written before each
    frame outside the events.  Both builds: NVRTC's default (contraction on, the reference
    as shipped) and without contraction (the build this library's images equal bit for
    bit).  A checker leg outside the timed region: returns None when the reference kernel
    was not built."""
    from oracle import oracle
    if not oracle.ref_available("fmad"):
        return None
    samples = w.width * w.height * w.spp
    out = {"unit": "Msamples/s", "frames": frames,
           "launches_per_frame": w.spp * _ref_tiles(w.width, w.height),
           "launch_plan": "renderSample: one renderKernel launch per (sample, tile), 16x16 "
                          "blocks, tiles of <= 262144 pixels",
           "l2": "flushed before each frame outside the events"}
    for variant in ("fmad", "nofmad"):
        if not oracle.ref_available(variant):
            continue
        _, ms = oracle.ref_render(w, tree, warmup=1, frames=frames, variant=variant,
                                  flush_bytes=flush_bytes)
        out[variant] = {"value": samples * frames / (ms / 1e3) / 1e6,
                        "ms_per_frame": ms / frames}
    out["value"] = out["fmad"]["value"]
    out["variant"] = "fmad: NVRTC's default contraction, the reference as shipped"
    return out


def _ref_tiles(width, height, per_launch=262144):
    """GpuLaunchProvenance.renderTileLayout (GpuLaunchProvenance.java:44-60): tile count."""
    tw = min(width, per_launch)
    th = min(height, max(1, per_launch // tw))
    return (1 + (width - 1) // tw) * (1 + (height - 1) // th)


class _Tree:
    """A downloaded device tree in the reference's flattened layout, shaped for the oracle."""

    def __init__(self, arrays):
        self.node_bounds, self.node_data, self.refs, self.roots = arrays
        self.node_count = len(self.node_data) // 4
        self.ref_count = len(self.refs)
        self.root_count = len(self.roots)


def cpu_baseline(w, rows, threads=0):
    """The FP64 CPU renderer on the centre `rows` rows of the frame: (Msamples/s, seconds,
    samples, the rows' mean radiance (rows*width, 3), first row)."""
    from oracle import oracle
    r0 = w.height // 2 - rows // 2
    t0 = time.perf_counter()
    img = oracle.cpu_render(w, frames=w.spp, rows=(r0, r0 + rows), threads=threads)
    dt = time.perf_counter() - t0
    samples = rows * w.width * w.spp
    return samples / dt / 1e6, dt, samples, img, r0


def band_rmse(a, b):
    return float(np.sqrt(np.mean((np.asarray(a, np.float64) - np.asarray(b, np.float64)) ** 2)))


# Ranks render disjoint frame ranges of the same workload: rank r's frames start at
# r * FRAMES_PER_RANK (timed frames at 0, warm-up at 1000, end-to-end at 500, counters at 0).
FRAMES_PER_RANK = 100000


def frame_index(rank, step, offset=0):
    """Frame index of a rank's step; the render seeds every pixel sample from it."""
    return rank * FRAMES_PER_RANK + offset + step


def max_over_ranks(x, device="cuda"):
    """Max of a scalar over the process group (the identity without one)."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def scenes_of_rank(count, rank, world):
    """Scene indices a rank renders in the batched workload: round-robin over the ranks."""
    return list(range(rank, count, world))


def init_ranks(world, local):
    """Selects this rank's GPU and, with more than one rank, joins the NCCL process group."""
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1 and not dist.is_initialized():
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def finish_ranks(world):
    """Every rank leaves the process group together."""
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def whole_job_rate(world, steps, samples_per_frame, seconds):
    """Msamples/s of the whole job: every rank's frames over the slowest rank's time."""
    return world * steps * samples_per_frame / seconds / 1e6


def peak_hbm():
    try:
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def run_reference(args):
    """--impl reference: the reference's CPU renderer (FP64 restatement) on host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w, wname = make_workload(args.workload, args)
    rows = min(16, w.height)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_baseline(w, rows, threads)
    vals, times = [], []
    for _ in range(args.steps):
        v, dt, samples, _, _ = cpu_baseline(w, rows, threads)
        vals.append(v)
        times.append(dt)
    value = sum(rows * w.width * w.spp for _ in times) / sum(times) / 1e6
    sample = "%d centre rows x %d px x %d spp per step (%d samples)" % (rows, w.width, w.spp,
                                                                       rows * w.width * w.spp)
    line = {"metric": "Msamples/s", "value": value, "unit": "Msamples/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": wname, "renderer": "reference CPU path tracer (FP64 "
                       "restatement of PathTracer + BvhSolid; the Java original needs a JVM)"},
            "cpu_baseline": {"value": value, "unit": "Msamples/s", "cores": threads,
                             "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_measure(ctx, local, works, steps, warmup, world=1, autotune=True):
    """Per-scene frames launched back to back versus the batch replayed from its CUDA graph
    (after autotuning, or with the default tuning): CUDA-event milliseconds of each, the
    tuning, whether every image is identical, and the device build time of the scenes."""
    import torch
    from rtb200.batch import Batch
    lib = ctx.lib
    t0 = time.perf_counter()
    scenes = [ResidentScene.build(ctx, w.scene) for w in works]
    build_ms = sum(r.stats.build_ms for r in scenes)
    build_wall = time.perf_counter() - t0
    outs = [torch.zeros(w.width * w.height * 3, dtype=torch.float32, device="cuda") for w in works]
    stream = torch.cuda.Stream(device=local)
    sh = C.c_void_p(stream.cuda_stream)

    def sequential():
        for w, r, o in zip(works, scenes, outs):
            p = N.RenderParams(w.width, w.height, w.spp, w.max_depth, w.frame_index,
                               w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
            cam = camera_struct(w.camera)
            ctx.check(lib.rtb_render_device(ctx.handle, r.handle, C.byref(cam), C.byref(p),
                                            C.c_void_p(o.data_ptr()), sh))

    jobs = [(r, w.camera, w.width, w.height, w.spp, w.max_depth, w.frame_index, w.frame_seed,
             o.data_ptr()) for w, r, o in zip(works, scenes, outs)]
    batch = Batch(ctx, jobs)
    tuned = batch.autotune(repeats=1) if autotune else None

    def timed(fn):
        for _ in range(warmup):
            fn()
        stream.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        barrier(world)
        return e0.elapsed_time(e1) / steps

    seq_ms = max_over_ranks(timed(sequential))
    ref_imgs = [o.cpu().numpy().copy() for o in outs]
    bat_ms = max_over_ranks(timed(lambda: batch.render(stream.cuda_stream)))
    same = all(np.array_equal(o.cpu().numpy().view(np.int32), r.view(np.int32))
               for o, r in zip(outs, ref_imgs))
    differ = max_over_ranks(0.0 if same else 1.0)
    branches = tuned["branches"] if tuned else 4
    # each frame or shared-queue launch is followed by its single-sample tail sum
    launches = max_over_ranks(steps * 2 * (len(works) if branches > 0 else 1))
    batch.close()
    for r in scenes:
        r.close()
    return {"seq_ms": seq_ms, "bat_ms": bat_ms, "tuning": tuned, "identical": differ == 0.0,
            "build_ms": build_ms, "build_wall_s": build_wall, "launches": int(launches)}


def run_batched(args, rank=0, world=1, local=0):
    """The 64-scene batch (primitive counts log-uniform in [1k, 200k], resolutions from
    {256^2, 512^2, 1024^2}, 16 or 64 spp, depth 6): per-scene frames launched back to back
    versus the batch replayed from its CUDA graph after autotuning (one shared-queue kernel
    over all jobs, or the jobs' own frames spread over concurrent graph branches).  With
    several ranks the scenes are dealt round-robin, each rank batching its own on its GPU;
    the rate is all 64 scenes' samples over the slowest rank's time."""
    init_ranks(world, local)
    ctx = Context(local)
    all_works = synth.batched_workloads()
    total_samples = sum(w.width * w.height * w.spp for w in all_works)
    works = [all_works[i] for i in scenes_of_rank(len(all_works), rank, world)]
    m = batched_measure(ctx, local, works, args.steps, args.warmup, world)
    seq_ms, bat_ms = m["seq_ms"], m["bat_ms"]
    line = {"metric": "Msamples/s", "value": total_samples / (bat_ms / 1e3) / 1e6,
            "unit": "Msamples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": bat_ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batched-64-scenes", "scenes": len(all_works),
                       "samples": total_samples,
                       "primitives": sum(w.scene.bounded_primitive_count() for w in all_works),
                       "parallelism": ("scenes round-robin over ranks" if world > 1
                                       else "single GPU")},
            "sequential": {"value": total_samples / (seq_ms / 1e3) / 1e6, "ms_per_step": seq_ms},
            "batched_over_sequential": seq_ms / bat_ms, "tuning": m["tuning"],
            "images_identical": m["identical"], "device_build_ms_total": m["build_ms"],
            "build_wall_s": m["build_wall_s"], "gpu_launches": m["launches"] * world}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    finish_ranks(world)


def frames_measure(ctx, w, steps, warmup, flush, stream, ref_frames=0, sm_mhz=None):
    """Device build and frames of one configuration on one GPU: median build ms, Msamples/s
    over `steps` frames (CUDA events around each frame, L2 flushed before each outside the
    events), optionally the reference kernel on the same frame (ref_kernel_leg), and the
    issue bound and traffic where this workload has an ncu capture (sm_mhz: the SM clock
    sampled during the headline's timed frames)."""
    import torch
    builds = []
    for i in range(2):
        r = ResidentScene.build(ctx, w.scene)
        builds.append(r.stats.build_ms)
        if i == 0:
            r.close()
    res = r
    out = torch.empty(w.width * w.height * 3, dtype=torch.float32, device="cuda")
    cam = camera_struct(w.camera)
    sh = C.c_void_p(stream.cuda_stream)
    ms = []
    for i in range(warmup + steps):
        p = N.RenderParams(w.width, w.height, w.spp, w.max_depth, 2000 + i,
                           w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
        with torch.cuda.stream(stream):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.check(ctx.lib.rtb_render_device(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                                C.c_void_p(out.data_ptr()), sh))
            e1.record(stream)
        e1.synchronize()
        if i >= warmup:
            ms.append(e0.elapsed_time(e1))
    samples = w.width * w.height * w.spp
    d = {"value": samples / (statistics.mean(ms) / 1e3) / 1e6, "unit": "Msamples/s",
         "ms_per_frame": statistics.mean(ms), "frames": steps, "build_ms": builds[-1],
         "primitives": w.scene.bounded_primitive_count(),
         "frame": "%dx%d %dspp depth%d" % (w.width, w.height, w.spp, w.max_depth)}
    if w.name in INST_PER_SAMPLE:
        d["roofline_issue"] = issue_roofline(w.name, samples, statistics.mean(ms),
                                             ctx.device_info().sm_count, sm_mhz)
        d["traffic"] = {"bytes_per_frame": TRAFFIC_BYTES_PER_SAMPLE[w.name] * samples,
                        "gbs": TRAFFIC_BYTES_PER_SAMPLE[w.name] * samples
                               / (statistics.mean(ms) / 1e3) / 1e9,
                        "note": "dram bytes per sample of the ncu capture of a %s frame of the "
                                "same scene (cold caches), scaled by samples"
                                % CAPTURE_FRAME[w.name]}
    if ref_frames:
        rk = ref_kernel_leg(w, _Tree(res.download_bvh()), ref_frames, flush.numel() * 4)
        if rk is not None:
            d["ref_kernel"] = {"value": rk["value"], "ms_per_frame": rk["fmad"]["ms_per_frame"],
                               "variant": "fmad"}
            d["vs_ref_kernel"] = d["value"] / rk["value"]
    res.close()
    return d


def wavefront_measure(ctx, w, steps, warmup, flush, stream):
    """The same frames in both forms: the persistent kernel (rtb_render_device) and the
    wavefront kernels (rtb_render_device_wavefront); Msamples/s of each (CUDA events around
    each frame, L2 flushed before each outside the events) and whether the images agree
    bit for bit."""
    import torch
    res = ResidentScene.build(ctx, w.scene)
    cam = camera_struct(w.camera)
    sh = C.c_void_p(stream.cuda_stream)
    imgs, vals = {}, {}
    for form, fn in (("persistent", ctx.lib.rtb_render_device),
                     ("wavefront", ctx.lib.rtb_render_device_wavefront)):
        out = torch.empty(w.width * w.height * 3, dtype=torch.float32, device="cuda")
        ms = []
        for i in range(warmup + steps):
            p = N.RenderParams(w.width, w.height, w.spp, w.max_depth, 3000 + i,
                               w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, 0, 0)
            with torch.cuda.stream(stream):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.check(fn(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                             C.c_void_p(out.data_ptr()), sh))
                e1.record(stream)
            e1.synchronize()
            if i >= warmup:
                ms.append(e0.elapsed_time(e1))
        imgs[form] = out.cpu().numpy()
        vals[form] = w.width * w.height * w.spp / (statistics.mean(ms) / 1e3) / 1e6
    res.close()
    return {"value": vals["wavefront"], "unit": "Msamples/s", "persistent_value": vals["persistent"],
            "wavefront_over_persistent": vals["wavefront"] / vals["persistent"], "frames": steps,
            "images_identical": bool(np.array_equal(imgs["wavefront"].view(np.int32),
                                                    imgs["persistent"].view(np.int32))),
            "frame": "%dx%d %dspp depth%d" % (w.width, w.height, w.spp, w.max_depth),
            "form": "one wave per sample index; per bounce a trace and a shade kernel over the "
                    "compacted live paths; path state in HBM"}


def other_configs(ctx, local, flush, sm_mhz=None):
    """The benchmark's other configurations, measured once after the headline timing so that
    one default run shows them all: the plain 64-sphere frame (with the reference kernel
    beside it), the C2 frame in the wavefront form beside the persistent kernel, the
    1M-primitive scene (device build and frames), the 64-scene batch with
    the default tuning (versus its scenes' frames back to back) and the differentiable
    configuration (forward, backward and the finite-difference check)."""
    import torch
    stream = torch.cuda.Stream(device=local)
    out = {}
    out["C1_plain"] = frames_measure(ctx, synth.plain_workload(), 10, 3, flush, stream, ref_frames=3)
    out["C2_wavefront"] = wavefront_measure(ctx, synth.hetero_workload(), 2, 1, flush, stream)
    out["C3_scale"] = frames_measure(ctx, synth.scale_workload(), 2, 1, flush, stream,
                                     sm_mhz=sm_mhz)
    works = synth.batched_workloads()
    m = batched_measure(ctx, local, works, 1, 1, autotune=False)
    samples = sum(w.width * w.height * w.spp for w in works)
    out["C4_batched"] = {"value": samples / (m["bat_ms"] / 1e3) / 1e6, "unit": "Msamples/s",
                         "ms_per_batch": m["bat_ms"], "tuning": "default (per-job frames, 4 branches)",
                         "sequential_value": samples / (m["seq_ms"] / 1e3) / 1e6,
                         "batched_over_sequential": m["seq_ms"] / m["bat_ms"],
                         "images_identical": m["identical"], "scenes": len(works)}
    a = adjoint_measure(ctx, local, 3, 1)
    out["C5_adjoint"] = {"forward_ms": a["forward_ms"], "backward_ms": a["backward_ms"],
                         "backward_over_forward": a["backward_ms"] / a["forward_ms"],
                         "backward_value": a["samples"] / (a["backward_ms"] / 1e3) / 1e6,
                         "unit": "Msamples/s", "fd_check": a["fd_check"]}
    return out


FD_SMALL = 1e-2  # |FD| below this fraction of its group's typical gradient counts as small


def fd_check(g, n_albedo, loss, alb0, emi0, count, rng, h=1e-3):
    """Central finite differences (step h, common random numbers: every render uses the same
    frame seed) on ``count`` parameters drawn uniformly without replacement from all albedo
    and emission components, against the adjoint's gradient ``g`` (albedo components first).
    ``loss(albedo, emission)`` returns the FP64 image loss.

    The scale of a group (albedo, emission) is the median magnitude of its non-zero
    gradients (the largest ones -- room walls, the emitter -- are orders of magnitude above
    a primitive's).  Gradients below FD_SMALL x scale are reported apart: for those a
    relative error is dominated by the FP32 rounding of the image and of the gradient sums,
    so they are judged by their absolute error relative to the scale.

    Albedo components of materials whose albedo is zero in all three channels (emitters) are
    not drawn: there the path ends (the lobe weights sum to zero), and any positive albedo
    continues it, so the image has no derivative at that point."""
    dead = np.repeat(np.all(alb0.reshape(-1, 3) == 0.0, axis=1), 3)
    cand = np.concatenate([np.nonzero(~dead)[0], n_albedo + np.arange(len(g) - n_albedo)])
    idx = rng.choice(cand, size=min(count, len(cand)), replace=False)
    n_total = len(cand)
    def typical(x):
        nz = np.abs(x[x != 0.0])
        return float(np.median(nz)) if len(nz) else 0.0

    scale = np.array([typical(g[:n_albedo]), typical(g[n_albedo:])])
    rows = []
    for i in idx:
        alb, emi = alb0.copy(), emi0.copy()
        arr, k = (alb, i) if i < n_albedo else (emi, i - n_albedo)
        flat = arr.reshape(-1)
        v = flat[k]
        flat[k] = v + h
        lp = loss(alb, emi)
        flat[k] = v - h
        lm = loss(alb, emi)
        fd = (lp - lm) / (2 * h)
        grp = 0 if i < n_albedo else 1
        rows.append((int(i), grp, float(g[i]), fd, float(scale[grp])))
    large = [r for r in rows if abs(r[3]) >= FD_SMALL * r[4] and r[4] > 0]
    small = [r for r in rows if not (abs(r[3]) >= FD_SMALL * r[4] and r[4] > 0)]
    rel = np.array([abs(r[2] - r[3]) / abs(r[3]) for r in large])
    absn = np.array([abs(r[2] - r[3]) / r[4] if r[4] > 0 else abs(r[2] - r[3]) for r in small])
    return {"parameters": len(rows), "drawn_from": n_total, "h": h,
            "large": {"count": len(large),
                      "max_rel_err": float(rel.max()) if len(rel) else 0.0,
                      "median_rel_err": float(np.median(rel)) if len(rel) else 0.0},
            "small": {"count": len(small),
                      "threshold": "|FD| < %g x median non-zero |gradient| of the group" % FD_SMALL,
                      "max_abs_err_over_scale": float(absn.max()) if len(absn) else 0.0,
                      "exact_zero": int(sum(1 for r in small if r[2] == 0.0 and r[3] == 0.0))},
            "rows": rows}


def adjoint_measure(ctx, local, steps, warmup, world=1, fd_count=64):
    """The differentiable configuration: 4096-primitive mixed scene, 512x512, 32 spp, depth
    6; L2 image loss against a target rendered with albedos perturbed by N(0, 0.05)
    (12-uniform approximation, clamped to [0, 1]); forward frame vs path-replay backward
    time (CUDA events), and the error against central finite differences (h = 1e-3, common
    random numbers, FP64 loss) on ``fd_count`` parameters drawn uniformly from all albedo and
    emission components (fd_check)."""
    import torch
    from rtb200.diff import DifferentiableScene
    w = synth.adjoint_workload()
    ds = DifferentiableScene(ctx, w.scene, w.width, w.height, w.spp, w.max_depth, w.camera,
                             w.frame_index, w.frame_seed)
    alb0, emi0 = ds.albedo(), ds.emission()
    st = synth.Stream(1, synth.WORKLOAD_IDS["adjoint"], 1, 7)
    u12 = st.uniform(12 * alb0.size).reshape(-1, 3, 12)
    g12 = u12[:, :, 0].copy()
    for j in range(1, 12):
        g12 = g12 + u12[:, :, j]
    target_alb = np.clip(alb0 + 0.05 * (g12 - 6.0) * (alb0 > 0), 0.0, 1.0)
    n = w.width * w.height * 3
    img = torch.empty(n, dtype=torch.float32, device="cuda")
    ga = torch.empty(ds.count * 3, dtype=torch.float32, device="cuda")
    ge = torch.empty(ds.count * 3, dtype=torch.float32, device="cuda")
    sobj = torch.cuda.Stream(device=local)
    stream = sobj.cuda_stream

    def render(alb, emi):
        ds.set_parameters(alb, emi)
        ds.render_into(img.data_ptr(), stream)
        sobj.synchronize()
        return img.cpu().numpy().astype(np.float64)

    target = render(target_alb, emi0)
    base = render(alb0, emi0)
    adj = torch.from_numpy((2.0 * (base - target)).astype(np.float32)).cuda()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fwd, bwd = [], []
    torch.cuda.synchronize()
    barrier(world)
    for i in range(warmup + steps):
        e0.record(sobj)
        ds.render_into(img.data_ptr(), stream)
        e1.record(sobj)
        e1.synchronize()
        if i >= warmup:
            fwd.append(e0.elapsed_time(e1))
        e0.record(sobj)
        ds.backward_into(adj.data_ptr(), ga.data_ptr(), ge.data_ptr(), stream)
        e1.record(sobj)
        e1.synchronize()
        if i >= warmup:
            bwd.append(e0.elapsed_time(e1))
    sobj.synchronize()
    g = np.concatenate([ga.cpu().numpy(), ge.cpu().numpy()]).astype(np.float64)
    fd = fd_check(g, ga.numel(), lambda a, e: float(np.sum((render(a, e) - target) ** 2)),
                  alb0, emi0, fd_count, np.random.default_rng(1))
    fd.pop("rows")
    out = {"samples": w.width * w.height * w.spp, "materials": ds.count,
           "forward_ms": max_over_ranks(statistics.mean(fwd)),
           "backward_ms": max_over_ranks(statistics.mean(bwd)), "fd_check": fd}
    ds.close()
    return out


def run_adjoint(args, rank=0, world=1, local=0):
    """The differentiable workload (adjoint_measure).  One backward pass does not shard: with
    several ranks each runs an independent replica on its GPU, and the rate is all replicas'
    samples over the slowest rank's backward time."""
    init_ranks(world, local)
    ctx = Context(local)
    m = adjoint_measure(ctx, local, args.steps, args.warmup, world)
    f_ms, b_ms = m["forward_ms"], m["backward_ms"]
    line = {"metric": "Msamples/s", "value": world * m["samples"] / (b_ms / 1e3) / 1e6,
            "unit": "Msamples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": b_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "adjoint-4k 512x512 32spp depth6", "materials": m["materials"],
                       "parameters": 6 * m["materials"],
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "forward_ms": f_ms, "backward_ms": b_ms, "backward_over_forward": b_ms / f_ms,
            "fd_check": m["fd_check"],
            "gpu_launches": world * args.steps}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    finish_ranks(world)


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local)
        return
    if args.workload == "adjoint":
        run_adjoint(args, rank, world, local)
        return
    import torch
    import torch.distributed as dist
    init_ranks(world, local)
    w, wname = make_workload(args.workload, args)
    ctx = Context(local)
    lib = ctx.lib
    stream = torch.cuda.Stream(device=local)
    sh = C.c_void_p(stream.cuda_stream)

    # ---- device build (timed by the library with CUDA events) and residency
    res = ResidentScene.build(ctx, w.scene)
    build_ms = res.stats.build_ms
    # binned object-SAH builds of the same scene (16 bins for the plain scene, 32 otherwise):
    # the first build warms the allocation pool; the rest are timed by the library's events
    bins = 16 if args.workload == "plain" else 32
    binned_ms, binned_sah = [], None
    for i in range(4):
        rb = ResidentScene.build(ctx, w.scene, bins=bins)
        if i:
            binned_ms.append(rb.stats.build_ms)
        binned_sah = rb.stats.generalized_sah_cost
        rb.close()
    full_ms = []
    for i in range(3):
        rf = ResidentScene.build(ctx, w.scene)
        full_ms.append(rf.stats.build_ms)
        rf.close()
    build_ms = statistics.median(full_ms)
    pixels = w.width * w.height
    out = torch.empty(pixels * 3, dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    cam = camera_struct(w.camera)

    def params(frame, metrics=0):
        return N.RenderParams(w.width, w.height, w.spp, w.max_depth, frame,
                              w.frame_seed & 0xFFFFFFFFFFFFFFFF, 1, metrics, 0)

    render_fn = (lib.rtb_render_device_wavefront if args.form == "wavefront"
                 else lib.rtb_render_device)

    def render(frame, metrics=0):
        p = params(frame, metrics)
        ctx.check(render_fn(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                            C.c_void_p(out.data_ptr()), sh))

    # ---- counters for the roofline: the kernel's metrics build on this rank's first frame
    #      (untimed; a host-buffer render fills rtb_frame_stats with the counters)
    host_img = np.zeros(pixels * 3, np.float32)
    p = params(frame_index(rank, 0), 1)
    ctx.check(lib.rtb_render_sample(ctx.handle, res.handle, C.byref(cam), C.byref(p),
                                    N.fptr(host_img)))
    fs = N.FrameStats()
    ctx.check(lib.rtb_last_frame_stats(ctx.handle, C.byref(fs)))
    cnt = np.array(list(fs.counters), dtype=np.int64)
    samples_per_frame = pixels * w.spp
    # every segment ends in at most one material fetch: an upper bound for the hit bytes
    bytes_per_frame = algorithmic_bytes([int(v) for v in cnt], int(cnt[0]))

    # ---- a step: this rank's own frame, or (rows split) this rank's rows of one frame
    #      shared by all ranks followed by the all-gather of every rank's rows
    split_rows = world > 1 and args.split == "rows"
    if split_rows and args.form == "wavefront":
        raise SystemExit("--form wavefront renders whole frames: use --split frames")
    if split_rows:
        from rtb200 import split
        k_rows = split.band_rows(w.height, world)
        band = torch.zeros(k_rows * w.width * 3, dtype=torch.float32, device="cuda")
        gathered = torch.empty(world * band.numel(), dtype=torch.float32, device="cuda")

        def step(frame):
            p = params(frame)
            ctx.check(lib.rtb_render_rows_device(ctx.handle, res.handle, C.byref(cam),
                                                 C.byref(p), rank, world,
                                                 C.c_void_p(band.data_ptr()), sh))
            dist.all_gather_into_tensor(gathered, band)
            out.copy_(split.assemble(gathered, w.height, w.width, world).reshape(-1))

        def step_frame(i, offset=0):  # every rank renders the same frame
            return frame_index(0, i, offset)
    else:
        step = render

        def step_frame(i, offset=0):
            return frame_index(rank, i, offset)

    # ---- warm-up
    for i in range(args.warmup):
        with torch.cuda.stream(stream):
            step(step_frame(i, 1000))
    stream.synchronize()

    # ---- timed region: K steps, events around each step on its stream, L2 flushed between
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            starts[i].record(stream)
            step(step_frame(i))
            ends[i].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clock_info = clocks.stop()
    last_frame = out.cpu().numpy().reshape(-1, 3)  # an independent frame, for the noise floor
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = float(sum(step_ms))
    total_ms = max_over_ranks(total_ms)
    frames_per_step = 1 if split_rows else world
    value = whole_job_rate(frames_per_step, args.steps, samples_per_frame, total_ms / 1e3)
    launch_ms = statistics.mean(step_ms)
    # the roofline is one GPU's kernel: with the rows split each rank runs 1/N of the frame
    achieved = (bytes_per_frame / world if split_rows else bytes_per_frame) / (launch_ms / 1e3) / 1e9
    peak, peak_kind = peak_hbm()

    # ---- e2e through the C ABI with pinned host buffers: upload + device build + render +
    #      read-back, each step.
    d, keep = scene_desc(w.scene)
    pinned = []
    for name, arr in (("spheres", keep[0]), ("boxes", keep[1]), ("planes", keep[2]),
                      ("affine_spheres", keep[3]), ("affine_boxes", keep[4]),
                      ("materials", keep[5]), ("affine_sphere_bounds", keep[6]),
                      ("affine_box_bounds", keep[7])):
        t = torch.from_numpy(arr).pin_memory()
        pinned.append(t)
        setattr(d, name, C.cast(C.c_void_p(t.data_ptr()), N.FP))
    h2d = sum(t.numel() * 4 for t in pinned)
    img = torch.empty(pixels * 3, dtype=torch.float32).pin_memory()
    bc = build_config(w.scene.config)
    e2e_times = []
    for i in range(0 if args.no_e2e else args.warmup + args.steps):
        if split_rows:
            dist.barrier()
        t0 = time.perf_counter()
        h = C.c_void_p()
        st = N.BvhStats()
        ctx.check(lib.rtb_scene_build(ctx.handle, C.byref(d), C.byref(bc), C.byref(h), C.byref(st)))
        if split_rows:
            # this rank's rows, the all-gather, and the whole frame read back on rank 0
            p = params(frame_index(0, i, 500))
            with torch.cuda.stream(stream):
                ctx.check(lib.rtb_render_rows_device(ctx.handle, h, C.byref(cam), C.byref(p),
                                                     rank, world, C.c_void_p(band.data_ptr()),
                                                     sh))
                dist.all_gather_into_tensor(gathered, band)
                if rank == 0:
                    img.copy_(split.assemble(gathered, w.height, w.width, world).reshape(-1),
                              non_blocking=True)
            stream.synchronize()
        else:
            p = params(frame_index(rank, i, 500))
            ctx.check(lib.rtb_render_sample(ctx.handle, h, C.byref(cam), C.byref(p),
                                            C.cast(C.c_void_p(img.data_ptr()), N.FP)))
        lib.rtb_scene_destroy(ctx.handle, h)
        if i >= args.warmup:
            e2e_times.append(time.perf_counter() - t0)
    e2e_total = sum(e2e_times) if e2e_times else float("nan")
    e2e_total = max_over_ranks(e2e_total)
    e2e_value = whole_job_rate(frames_per_step, args.steps, samples_per_frame, e2e_total)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            rows = 80 if args.workload == "hetero" else 16
            rows = min(rows, w.height)
            v, dt, samples, cpu_img, r0 = cpu_baseline(w, rows)
            cpu = {"value": v, "unit": "Msamples/s", "cores": os.cpu_count(), "kind": "port",
                   "sample": "%d centre rows x %d px x %d spp of the same frame (%d samples, "
                             "%.1f s), FP64 restatement of the reference CPU renderer"
                             % (rows, w.width, w.spp, samples, dt)}
            # RMSE of the GPU frame against the FP64 CPU render on the same rows, beside the
            # RMSE between two GPU frames (the Monte Carlo noise floor at this spp)
            band = slice(r0 * w.width, (r0 + rows) * w.width)
            gpu_a = host_img.reshape(-1, 3)[band]
            gpu_b = last_frame[band]
            rm = band_rmse(gpu_a, cpu_img)
            floor = band_rmse(gpu_a, gpu_b)
            cpu["rmse_vs_gpu"] = {"rmse": rm, "gpu_noise_floor_rmse": floor,
                                  "ratio": rm / floor if floor > 0 else None,
                                  "mean_radiance_gpu": float(np.mean(gpu_a)),
                                  "mean_radiance_cpu": float(np.mean(cpu_img))}
        line = {
            "metric": "Msamples/s", "value": value, "unit": "Msamples/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong" if split_rows else "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": wname, "primitives": w.scene.bounded_primitive_count(),
                       "planes": w.scene.plane_count, "width": w.width, "height": w.height,
                       "spp": w.spp, "max_depth": w.max_depth, "bvh": "weighted SAH leaf<=4 "
                       "(sphere 1.0, box 1.3, affine 2.1), device-built",
                       "l2": "flushed between frames (256 MiB write outside the events)",
                       "form": args.form,
                       "parallelism": ("one frame per step, rows r, r+N, ... on rank r, "
                                       "NCCL all-gather of the rows" if split_rows else
                                       "frames per rank" if world > 1 else "single GPU")},
            "build_ms": build_ms,
            "build": {"full_sweep_ms": build_ms,
                      "full_sweep_note": "tree identical to the reference Java builder's",
                      "binned_ms": statistics.median(binned_ms), "bins": bins,
                      "binned_note": "binned object SAH, identical to its CPU restatement",
                      "binned_over_full_sah": binned_sah / res.stats.generalized_sah_cost},
            "e2e": {"value": e2e_value, "unit": "Msamples/s", "h2d_bytes_per_step": h2d * world,
                    "d2h_bytes_per_step": pixels * 12 * (1 if split_rows else world),
                    "includes": "scene upload from pinned memory + device BVH build + render "
                                "+ image read-back, per step"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (TRAFFIC_BYTES_PER_SAMPLE[args.workload] * samples_per_frame
                                     if args.workload in TRAFFIC_BYTES_PER_SAMPLE else None),
                         "traffic_note": ("ncu capture of a %s frame of the same scene, scaled "
                                          "by samples" % CAPTURE_FRAME.get(args.workload)
                                          if args.workload in TRAFFIC_BYTES_PER_SAMPLE
                                          else "no capture of this workload"),
                         "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)",
                         "algorithmic_bytes_per_launch": bytes_per_frame,
                         "launch_ms": launch_ms,
                         "note": "working set is L2-resident; the bytes are served mostly from "
                                 "L1/L2, so the kernel is latency/issue-bound, not HBM-bound"},
            "roofline_issue": issue_roofline(
                args.workload, samples_per_frame, launch_ms, ctx.device_info().sm_count,
                clock_info.get("sm_mhz") or clock_info.get("sm_max_mhz")),
            "counters_per_sample": {k: float(v) / samples_per_frame for k, v in zip(
                ["segments", "aabb_tests", "primitive_tests", "sphere", "box", "plane",
                 "affine_sphere", "affine_box", "overflows", "max_stack", "internal_nodes",
                 "leaves", "homogeneous_leaves", "mixed_leaves"], cnt)},
            "clocks": clock_info,
            "gpu_launches": args.steps * fs.physical_launches * world,
            "device": ctx.device_info().name,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        if world == 1 and args.workload == "hetero" and not args.no_other_configs:
            line["other_configs"] = other_configs(
                ctx, local, flush, clock_info.get("sm_mhz") or clock_info.get("sm_max_mhz"))
        if world == 1 and not args.no_ref_kernel:
            frames = args.ref_frames or (1 if args.workload == "scale" else 3)
            rk = ref_kernel_leg(w, _Tree(res.download_bvh()), frames, flush.numel() * 4)
            if rk is not None:
                line["ref_kernel"] = rk
                line["vs_ref_kernel"] = value / rk["value"]
                line["vs_ref_kernel_nofmad"] = value / rk["nofmad"]["value"] \
                    if "nofmad" in rk else None
        print(json.dumps(line), flush=True)
    res.close()
    ctx.close()
    finish_ranks(world)


if __name__ == "__main__":
    main()
