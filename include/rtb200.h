/* rtb200 -- B200-native path tracer over cost-weighted SAH BVHs of analytic primitives.
 *
 * C ABI of librtb200.so: the drop-in boundary for the reference's CUDA render path.
 * Reference paths are relative to the reference project; gfxlab/ stands for
 * src/xyz/marsavic/gfxlab/.
 *
 * Conventions (mirroring gfxlab/gpu/GpuRayTracer.java):
 *  - every call returns an rtb_status; nothing throws, traps or aborts;
 *  - host buffers are owned by the caller; device memory is owned by the library;
 *  - a context serialises its calls with its own mutex (the reference synchronises every
 *    public method on the tracer, GpuRayTracer.java:339,445,601) and may be used from
 *    any thread;
 *  - the packed float layouts are exactly those of gfxlab/gpu/GpuScene.java:23-31
 *    (sphere 5, box 7, plane 26, affine sphere / affine box 22, material 13 floats), so
 *    a Java caller passes GpuScene.sphereData() and friends unchanged.
 */
#ifndef RTB200_H
#define RTB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RTB_API __attribute__((visibility("default")))
#else
#define RTB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  RTB_OK = 0,
  RTB_ERR_INVALID_ARGUMENT = 1, /* IllegalArgumentException in the reference */
  RTB_ERR_UNAVAILABLE = 2,      /* no usable device (GpuRayTracer.isAvailable() false) */
  RTB_ERR_CUDA = 3,             /* a CUDA runtime call failed; see rtb_last_error */
  RTB_ERR_OUT_OF_MEMORY = 4,
  RTB_ERR_UNSUPPORTED = 5,      /* a mode this library does not implement */
  RTB_ERR_DEVICE_CHECK = 6,     /* a kernel's own bounds / input check failed */
  RTB_ERR_WATCHDOG = 7,         /* a kernel gave up at its work budget or was aborted
                                   (IllegalStateException in GpuRayTracer.java:572-580) */
  RTB_ERR_LIMIT = 8             /* a documented size limit was exceeded */
} rtb_status;

typedef struct rtb_context rtb_context;
typedef struct rtb_scene rtb_scene;

/* Scene payload in the reference's packed layouts (GpuScene.java:507-601).  The affine
 * bounds are the float-cast world bounds GpuScene keeps beside each affine record
 * (GpuScene.java:640-649); they are only read by rtb_scene_build. */
typedef struct {
  const float* spheres;        int sphere_count;        /* 5 floats: centre, radius, material */
  const float* boxes;          int box_count;           /* 7 floats: min, max, material */
  const float* planes;         int plane_count;         /* 26 floats (GpuScene.planeData) */
  const float* affine_spheres; int affine_sphere_count; /* 22 floats */
  const float* affine_boxes;   int affine_box_count;    /* 22 floats */
  const float* materials;      int material_count;      /* 13 floats */
  const float* affine_sphere_bounds;                    /* 6 floats: min.xyz, max.xyz */
  const float* affine_box_bounds;                       /* 6 floats */
  float background[3];
} rtb_scene_desc;

/* A flattened BVH as GpuScene.bvhNodeBoundsData / bvhNodeData / bvhPrimitiveRefs /
 * bvhRootIndices produce it (GpuScene.java:30-31, 772-808). */
typedef struct {
  const float* node_bounds;  /* 6 floats per node */
  const int* node_data;      /* 4 ints per node: left|kind, right, first ref, count */
  int node_count;
  const int* primitive_refs; /* type << 30 | index */
  int primitive_ref_count;
  const int* root_indices;   /* 1..4 roots */
  int root_count;
} rtb_bvh_desc;

/* BvhBuildConfig (gfxlab/gpu/BvhBuildConfig.java:6-15); mode is a BvhBuildMode ordinal
 * (0 UNIFORM_SAH, 1 WEIGHTED_SAH, 2 PER_TYPE_SAH, 3 PER_TYPE_WEIGHTED_SAH, 4 UNIFORM_SBVH,
 * 5 WEIGHTED_SBVH, 6 SAH_ROTATIONS, 7 WEIGHTED_SAH_ROTATIONS).  The SBVH modes build on the
 * host in depth-first order (their global reference budget makes every split depend on the
 * ones before it); the others build on the device.  The binned builder takes modes 0-3. */
typedef struct {
  int mode;
  int leaf_size;
  double traversal_weight;
  double sphere_weight, box_weight, affine_sphere_weight, affine_box_weight;
  double lambda;
} rtb_build_config;

/* BvhBuildOptions (gfxlab/gpu/BvhBuildOptions.java:4-33); defaults 128, 2.0, 8, 16, 1e-5, 4.
 * rotation_passes belongs to the rotation modes, the other fields to the SBVH modes. */
typedef struct {
  int spatial_bins;
  double max_reference_multiplier;
  int max_splits_per_primitive;
  int min_spatial_references;
  double spatial_overlap_threshold;
  int rotation_passes;
} rtb_build_options;

/* GpuScene.BvhStats (GpuScene.java:113-133) plus the device build time. */
typedef struct {
  int node_count, root_count, leaf_count, max_depth, primitive_ref_count, leaf_size;
  int min_leaf_occupancy, max_leaf_occupancy;
  double generalized_sah_cost, uniform_sah_cost, weighted_sah_cost;
  long long bytes;
  double build_ms;          /* build time: CUDA events for the device builders, host wall
                               time for the SBVH modes */
  int sequential_nodes;     /* nodes above 256 primitives whose split the count-based
                               weights could not certify, summed in the sequential order */
  int rotation_count;       /* BvhStats.rotationCount of the rotation modes */
  int spatial_split_count;  /* BvhStats.spatialSplitCount of the SBVH modes */
  int duplicate_reference_count; /* BvhStats.duplicateReferenceCount (references - primitives) */
} rtb_bvh_stats;

/* GpuCamera (gfxlab/gpu/GpuCamera.java): direction = forward + right u + up v. */
typedef struct {
  float position[3], forward[3], right[3], up[3];
} rtb_camera;

/* Arguments of GpuRayTracer.renderSample (GpuRayTracer.java:317-432). */
typedef struct {
  int width, height;
  int samples_per_frame;   /* >= 1 */
  int max_depth;           /* [0, 32], GpuRayTracer.validateFullPathDepth */
  int frame_index;
  unsigned long long frame_seed;
  int use_bvh;             /* 0: test every primitive (the reference's GPU_LINEAR) */
  int collect_metrics;     /* count traversal work into rtb_frame_stats.counters */
  int shared_stack_entries; /* traversal-stack entries per lane kept in shared memory (the
                              * rest in local memory): 0 picks by scene size (16 for scenes
                              * over 16 MB of nodes, references and records, else none),
                              * -1 none, 8 or 16; a tuning knob of the batch autotuner */
} rtb_render_params;

/* GpuRayTracer.FrameStats (GpuRayTracer.java:79-99).  counters follow the reference's
 * STAT_* order (GpuKernelSources.java:30-43): rays, aabb tests, primitive tests, sphere,
 * box, plane, affine sphere, affine box tests, stack overflows, max stack size, internal
 * node visits, leaf visits, homogeneous leaf visits, mixed leaf visits. */
typedef struct {
  long long total_ns, kernel_ns, max_physical_kernel_ns, copy_ns, upload_ns;
  long long counters[14];
  int physical_launches;
} rtb_frame_stats;

/* ---- context (GpuRayTracer constructor / isAvailable / close, GpuRayTracer.java:256-287,
 *      780-835, 1223-1310) ---- */
RTB_API rtb_status rtb_context_create(int device, rtb_context** out);
RTB_API rtb_status rtb_context_destroy(rtb_context* ctx);
RTB_API const char* rtb_status_string(rtb_status status);
/* Message of the last failed call on this context (empty when none). */
RTB_API const char* rtb_last_error(const rtb_context* ctx);
/* GpuRayTracer.deviceInfo (GpuRayTracer.java:308-310). */
RTB_API rtb_status rtb_device_info(rtb_context* ctx, char* name, int name_len, int* cc_major,
                           int* cc_minor, int* sm_count);

/* ---- scenes (GpuRayTracer.ensureSceneResident / uploadScene, GpuRayTracer.java:873-948) ----
 * rtb_scene_upload takes a caller-built BVH (or none: linear traversal only);
 * rtb_scene_build builds the BVH on the device from the packed primitives
 * (the GpuScene.buildBvhData step, GpuScene.java:614-700, moved onto the GPU). */
RTB_API rtb_status rtb_scene_upload(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_bvh_desc* bvh,
                            rtb_scene** out);
RTB_API rtb_status rtb_scene_build(rtb_context* ctx, const rtb_scene_desc* desc,
                           const rtb_build_config* config, rtb_scene** out, rtb_bvh_stats* stats);
/* rtb_scene_build with explicit BvhBuildOptions (GpuSceneBuilder.from(scene, config,
 * options), GpuSceneBuilder.java:19-35); options NULL means the defaults. */
RTB_API rtb_status rtb_scene_build_with_options(rtb_context* ctx, const rtb_scene_desc* desc,
                                        const rtb_build_config* config,
                                        const rtb_build_options* options, rtb_scene** out,
                                        rtb_bvh_stats* stats);
/* Binned object SAH on the device: 2..32 centroid bins per axis, the configuration's
 * per-type weights, counts accumulated by warp-aggregated atomics, FP64 split selection
 * from integer bin counts.  No counterpart in the reference (its builder is the full sweep
 * that rtb_scene_build reproduces node for node); the tree is deterministic and identical
 * to this library's CPU restatement of the binned rule, not to the Java builder's.
 * Other bin counts return RTB_ERR_INVALID_ARGUMENT. */
RTB_API rtb_status rtb_scene_build_binned(rtb_context* ctx, const rtb_scene_desc* desc,
                                  const rtb_build_config* config, int bins, rtb_scene** out,
                                  rtb_bvh_stats* stats);
/* Copies the scene's BVH back in the reference's flattened layout (for topology hashes).
 * Sizes come from rtb_scene_bvh_sizes. */
RTB_API rtb_status rtb_scene_bvh_sizes(rtb_context* ctx, const rtb_scene* scene, int* node_count,
                               int* ref_count, int* root_count);
RTB_API rtb_status rtb_scene_download_bvh(rtb_context* ctx, const rtb_scene* scene, float* node_bounds,
                                  int* node_data, int* refs, int* roots);
RTB_API rtb_status rtb_scene_destroy(rtb_context* ctx, rtb_scene* scene);

/* ---- queries ---- */
/* GpuRayTracer.traceReplay (GpuRayTracer.java:593-716): closest hit of caller rays
 * (origin.xyz, direction.xyz per ray, host memory).  Outputs are host arrays of
 * ray_count entries (hit_normals: 3 per ray); misses give flag 0, distance +inf,
 * order -1, material -1 and a zero normal. */
RTB_API rtb_status rtb_trace_replay(rtb_context* ctx, rtb_scene* scene, const float* rays, int ray_count,
                            int use_bvh, int collect_metrics, int* hit_flags,
                            float* hit_distances, int* hit_orders, int* hit_materials,
                            float* hit_normals);

/* GpuRayTracer.renderSample (GpuRayTracer.java:317-432): renders samples_per_frame
 * samples per pixel and writes the per-pixel mean (3 floats per pixel, row-major) to the
 * host buffer rgb. */
RTB_API rtb_status rtb_render_sample(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                             const rtb_render_params* params, float* rgb);

/* Same frame into a caller-owned DEVICE buffer on a caller stream (cudaStream_t, or NULL
 * for the context's stream); returns after the launch is queued. */
RTB_API rtb_status rtb_render_device(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                             const rtb_render_params* params, float* rgb_device, void* stream);

/* The same frame as rtb_render_device, bit for bit, computed in the wavefront form: one
 * wave per sample index over all pixels; per bounce, one kernel traces every live path of
 * the wave and one shades them (path state in device memory, held by the context and grown
 * to the largest frame).  The A/B counterpart of the persistent kernel behind
 * rtb_render_device, which is faster on the B200; no metrics build (RTB_ERR_UNSUPPORTED).
 * rtb_request_abort stops it at the start of the next wave (sample index), leaving the
 * frame unfinished.  No counterpart in the reference, whose renderKernel is one thread per
 * pixel (GpuKernelSources.java:1167-1315). */
RTB_API rtb_status rtb_render_device_wavefront(rtb_context* ctx, rtb_scene* scene,
                                               const rtb_camera* camera,
                                               const rtb_render_params* params,
                                               float* rgb_device, void* stream);

/* One frame's rows first_row, first_row + row_stride, ... (< height), packed densely into
 * rgb_device (3 floats per pixel, row k of the output = frame row first_row + k*row_stride).
 * Every pixel equals the same pixel of rtb_render_device's full frame bit for bit (its random
 * streams are keyed by the frame pixel).  This is the unit of a frame split across GPUs:
 * rank r of N renders first_row = r, row_stride = N and the rows are gathered (interleaved
 * rows balance the uneven cost of image regions).  No counterpart in the reference, which
 * renders a frame on one device (GpuRayTracer.java:796). */
RTB_API rtb_status rtb_render_rows_device(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                                          const rtb_render_params* params, int first_row,
                                          int row_stride, float* rgb_device, void* stream);

/* GpuRayTracer.lastFrameStats / lastPhysicalKernelLaunchCount (GpuRayTracer.java:294-306). */
RTB_API rtb_status rtb_last_frame_stats(rtb_context* ctx, rtb_frame_stats* out);

/* ---- differentiable rendering (no counterpart in the reference) ----
 * rtb_scene_set_materials replaces a resident scene's 13-float material records (same
 * count), e.g. with perturbed or optimised albedos and emissions; the next frames use them.
 * rtb_render_backward is the adjoint of rtb_render_device for the same scene, camera and
 * params: given dLoss/dImage (device, 3 floats per pixel) it re-traces every sample from its
 * random seed and writes dLoss/d(albedo) and dLoss/d(emission) per material record (device,
 * 3 floats per material each; zeroed first).  Albedo is the diffuse colour; the lobe choice
 * is not differentiated (exact for diffuse-only materials). */
RTB_API rtb_status rtb_scene_set_materials(rtb_context* ctx, rtb_scene* scene, const float* materials,
                                           int material_count);
RTB_API rtb_status rtb_render_backward(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                                       const rtb_render_params* params, const float* adjoint_device,
                                       float* grad_albedo_device, float* grad_emission_device,
                                       void* stream);
/* rtb_render_backward with host buffers (dLoss/dImage in, 3 floats per pixel; the two
 * gradient tables out, 3 floats per material each), staged through the context's device
 * buffers; returns when the gradients are written, or RTB_ERR_WATCHDOG after an abort.  The
 * entry a caller without CUDA memory of its own binds (the Java forward/backward Function). */
RTB_API rtb_status rtb_render_backward_sample(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                                              const rtb_render_params* params, const float* adjoint,
                                              float* grad_albedo, float* grad_emission);

/* ---- batched rendering (no counterpart in the reference, which renders one scene per
 *      renderSample call) ----
 * A batch renders many resident scenes -- each with its own camera, resolution, sample count
 * and depth -- in one persistent launch over a shared pixel queue, captured once into a CUDA
 * graph and replayed by rtb_batch_render.  Every job's image equals its rtb_render_device
 * frame bit for bit.  Output buffers are caller-owned device arrays (3 floats per pixel). */
typedef struct {
  rtb_scene* scene;
  rtb_camera camera;
  rtb_render_params params;   /* use_bvh is honoured; collect_metrics is ignored */
  float* rgb_device;
} rtb_batch_job;

typedef struct {
  int threads_per_block;      /* 64, 128 or 256 (shared-queue kernel) */
  int job_order;              /* 0: as given, 1: most expensive jobs first */
  int branches;               /* 0: one shared-queue kernel over all jobs; 1..4: each job
                                 its own persistent frame, the frames spread round-robin
                                 over this many concurrent graph branches */
  int shared_stack_entries;   /* traversal-stack depth kept in shared memory by the jobs'
                                 frames (branches > 0): 0 keeps each job's own
                                 rtb_render_params value, else -1, 8 or 16 for every job */
  int tail_pixels_per_thread; /* queue granularity at the end of a frame (or of the
                                 shared-queue batch): this many pixels per resident thread
                                 are queued one sample per item instead of one pixel per
                                 item; 0: the default (4 for frames, 2 for the shared
                                 queue), else 1..16 */
} rtb_batch_tuning;

typedef struct rtb_batch rtb_batch;

/* tuning may be NULL (per-job frames over 4 branches, most expensive first). */
RTB_API rtb_status rtb_batch_create(rtb_context* ctx, const rtb_batch_job* jobs, int job_count,
                                    const rtb_batch_tuning* tuning, rtb_batch** out);
/* Replays the batch's graph on `stream` (NULL: the context stream); returns once queued. */
RTB_API rtb_status rtb_batch_render(rtb_context* ctx, rtb_batch* batch, void* stream);
/* Times candidate tunings on the batch itself (`repeats` timed runs each after a warm-up
 * run) and keeps the fastest: first every kernel form (shared queue at 64/128/256 threads,
 * frames over 1/2/4 branches) in both job orders, then, around the best, the end-of-frame
 * queue granularity (1, 2, 4, 8 pixels per thread at one sample per item) and, for frames,
 * the shared-memory stack depth (none, 8, 16 entries, by scene size); re-captures the graph
 * and reports the choice. */
RTB_API rtb_status rtb_batch_autotune(rtb_context* ctx, rtb_batch* batch, int repeats,
                                      rtb_batch_tuning* best, double* best_ms);
RTB_API rtb_status rtb_batch_destroy(rtb_context* ctx, rtb_batch* batch);

/* Closest-hit replay that allocates nothing.  No counterpart in the reference.
 * For callers that cannot allocate device memory when they query (a host framework that
 * owns a fixed device-memory budget, a frame loop that forbids allocation after start-up):
 * same results as rtb_trace_replay on a resident scene, but rays and hit records are staged
 * in a fixed array of RTB_STATIC_REPLAY_MAX_RAYS rays inside the library, and the call makes
 * no cudaMalloc/cudaFree or other allocation.  Every GPU that loads the library holds that
 * array (about 3.4 MB) until exit.  The first call on a device looks up the array's address
 * (so make it before any stream capture) and keeps it for the process: after a
 * cudaDeviceReset of that device the address is stale, so do not call this entry point on a
 * device the process has reset.  Calls share the array: calls that overlap on the GPU race.  Returns RTB_ERR_LIMIT for ray_count > RTB_STATIC_REPLAY_MAX_RAYS.  Runs on the
 * scene's device on the calling thread's per-thread default stream and returns when the
 * host outputs are written. */
#define RTB_STATIC_REPLAY_MAX_RAYS 65536
RTB_API rtb_status rtb_trace_replay_static(const rtb_scene* scene, const float* rays, int ray_count,
                                           int use_bvh, int* hit_flags, float* hit_distances,
                                           int* hit_orders, int* hit_materials, float* hit_normals);

/* ---- primitive-cost calibration (the counterpart of gfxlab/gpu/PrimitiveCostBenchmark.java,
 * whose RTX 3080 results are the constants of PrimitiveCostModel.java:11-19) ----
 * Relative cost of this library's intersection operations on the current device,
 * normalised to the sphere test.  Operation index: 1 sphere, 2 box, 3 affine sphere,
 * 4 affine box, 5 node AABB, 6 interior traversal (both child boxes and their order),
 * 7 plane; 0 is the setup baseline. */
#define RTB_CALIBRATION_MAX_PROFILES 3
typedef struct {
  const float* rays;     /* profiles x records x 6: origin, direction */
  int profiles;          /* 1..3 */
  int records;           /* a power of two */
  const float* spheres;  /* 4 floats per record: centre, radius */
  const float* boxes;    /* 8 floats: min (+ pad), max (+ pad) */
  const float* affines;  /* 12 floats: inverse rows with the world centre in the 4th slot */
  const float* planes;   /* 4 floats: unit normal, offset */
  const float* nodes;    /* 16 floats: one child-pair node (x/y ranges of both children,
                            z ranges, links) */
} rtb_calibration_workload;

typedef struct {
  int blocks, threads;   /* launch shape of every timed launch (threads <= 256) */
  int iterations;        /* per thread per observation (a multiple of sublaunches) */
  int copies;            /* operations per iteration */
  int sublaunches;       /* timed launches per observation, alternated with the setup */
  int repeats, warmups;  /* paired observations per operation and profile */
  int order_offset;      /* rotation of the operation order */
  double max_launch_ms;  /* a longer launch aborts the calibration with RTB_ERR_LIMIT */
} rtb_calibration_params;

typedef struct {
  int profiles;
  double net_ns[RTB_CALIBRATION_MAX_PROFILES][8];     /* median net ns per operation */
  double sphere_ns[RTB_CALIBRATION_MAX_PROFILES][8];  /* its paired local sphere median */
  double ratio[RTB_CALIBRATION_MAX_PROFILES][8];      /* net / local sphere */
  double sphere_net_ns[RTB_CALIBRATION_MAX_PROFILES];
  double weight[8];                                   /* median ratio over the profiles */
  long long tests_per_observation;
} rtb_calibration_result;

RTB_API rtb_status rtb_calibrate_costs(rtb_context* ctx, const rtb_calibration_workload* workload,
                                       const rtb_calibration_params* params,
                                       rtb_calibration_result* result);

/* Host abort (no reference counterpart; the reference has only its launch watchdog).
 * Every render, batch and backward launch of this context submitted before this call
 * (running or still queued) stops at its next work fetch; work submitted after it is not
 * affected.  A stopped frame leaves the pixels it never fetched unwritten; rtb_render_sample
 * then returns RTB_ERR_WATCHDOG.  May be called from any thread while another thread holds
 * the context in a render call. */
RTB_API rtb_status rtb_request_abort(rtb_context* ctx);

#ifdef __cplusplus
}
#endif

#endif /* RTB200_H */
