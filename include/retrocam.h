/*
 * retrocam.h -- C ABI of the B200 render hot path of RetroCam.
 *
 * The library replaces the bodies of three Java classes of the reference:
 *   core/Renderer.java        (path-trace accumulation, pathtrace.comp)
 *   scene/SPPMManager.java    (photon trace + gather, photon_trace.comp /
 *                              photon_gather.comp, PhotonMap.java)
 *   post/AtrousDenoiser.java  (post/atrous_denoise.frag, p00_normalize.frag)
 * and offers the host-side scene logic those classes rely on
 * (scene/BVHBuilder.java, scene/SceneUploader.java, scene/Box.java,
 * scene/Sphere.java, scene/TransformedPrimitive.java,
 * camera/ThinLensCamera.java) so a caller can stay in Java and bind these
 * symbols with Panama FFM or JNI.
 *
 * Conventions:
 *   - Every function returns an int: RC_OK (0) or a negative RC_ERR_* code.
 *     rc_last_error() gives the text of the last failure on a context.
 *   - No exceptions cross the ABI; no torch or CUDA types in signatures.
 *   - Host arrays are owned by the caller and copied at call time; device
 *     buffers are owned by the context.
 *   - One rc_ctx owns one CUDA stream on one device.  Calls on one context
 *     must be serialised by the caller; different contexts may be driven
 *     from different threads.
 *   - Struct layouts are the std430 layouts of the reference SSBOs, so the
 *     Java side can pass its existing FloatBuffers unchanged.
 */
#ifndef RETROCAM_H
#define RETROCAM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RC_ABI_VERSION 1

/* ---- status codes ---- */
#define RC_OK 0
#define RC_ERR_INVALID_ARG (-1)   /* null pointer, bad size, bad enum       */
#define RC_ERR_CUDA (-2)          /* a CUDA runtime call failed             */
#define RC_ERR_OUT_OF_MEMORY (-3) /* device allocation failed               */
#define RC_ERR_NO_SCENE (-4)      /* render/trace before rc_scene_upload    */
#define RC_ERR_DEVICE_GUARD (-5)  /* a kernel hit an iteration cap or a bad
                                     index and stopped; see rc_counters     */
#define RC_ERR_CAPACITY (-6)      /* output array too small                 */
#define RC_ERR_BAD_SCENE (-7)     /* scene failed validation (e.g. a BVH
                                     child index out of range)              */

/* ---- std430 scene records (layouts of the reference SSBOs) ---- */

/* scene/GpuTriangle.java:68-78, 128 bytes. */
typedef struct rc_triangle {
    float v0[3]; float pad0;
    float v1[3]; float pad1;
    float v2[3]; float pad2;
    float n0[3]; float pad3;
    float n1[3]; float pad4;
    float n2[3]; float pad5;
    float uv0[2]; float uv1[2];
    float uv2[2]; int32_t mat_index; float pad6;
} rc_triangle;

/* scene/BVHNode.java:32-41, 48 bytes.  prim_count > 0 marks a leaf. */
typedef struct rc_bvh_node {
    float aabb_min[3]; float pad0;
    float aabb_max[3]; float pad1;
    int32_t left_child, right_child, prim_start, prim_count;
} rc_bvh_node;

/* scene/Material.java:61-69, 64 bytes. */
typedef struct rc_material {
    float albedo[3]; float metallic;
    float emission[3]; float emission_strength;
    float roughness; float ior; float transmission; int32_t albedo_tex;
    float pad[4];
} rc_material;

/* scene/SceneUploader.java:18-23, 80 bytes. */
typedef struct rc_light {
    float v0[3]; float area;
    float v1[3]; float pad1;
    float v2[3]; float pad2;
    float emission[3]; float power;
    float normal[3]; float cdf_weight;
} rc_light;

/* scene/PhotonMap.java:16-21, 48 bytes. */
typedef struct rc_photon {
    float position[3]; float pad0;
    float power[3]; float pad1;
    float dir[3]; float pad2;
} rc_photon;

/* Uniforms of pathtrace.comp:11-24 as set by camera/ThinLensCamera.java:27-58.
 * focal_dist is the caller's (for parity runs: RenderSettings.focusDistM). */
typedef struct rc_camera {
    float cam_pos[3];
    float cam_right[3];
    float cam_up[3];
    float cam_forward[3];
    float focal_dist;
    float lens_radius;
    float fov_tan_half;
    int32_t aperture_blades;
    float sa_strength;
    float lca_delta[3];
} rc_camera;

/* NEE uniforms of pathtrace.comp:32-35 (core/Renderer.java:93-96). */
typedef struct rc_settings {
    int32_t nee_enabled;
    float nee_firefly_clamp;
} rc_settings;

/* SPPM knobs (core/RenderSettings.java:35-38, scene/PhotonMap.java:33-36). */
typedef struct rc_sppm_params {
    int32_t photon_count;   /* photons emitted per iteration (<= capacity) */
    int32_t hash_size;      /* power of two */
    float alpha;            /* radius shrink parameter */
} rc_sppm_params;

/* À-trous knobs (core/RenderSettings.java:89-94, AtrousDenoiser.java:60-125). */
typedef struct rc_atrous_params {
    int32_t enabled;
    int32_t iterations;     /* clamped to [1,5] */
    float sigma_color;
    float sigma_normal;
    float sigma_depth;
    int32_t max_spp;        /* 0 = always active */
    float exposure;
} rc_atrous_params;

/* Device counters (replace the reference's console summaries and the BVH
 * heat-map shader with numbers). */
typedef struct rc_counters {
    uint64_t camera_paths;   /* traced paths (3 per sample with LCA) */
    uint64_t closest_rays;   /* closest-hit traversals (path tracer + g-buffer) */
    uint64_t shadow_rays;    /* any-hit traversals (NEE) */
    uint64_t photon_rays;    /* photon traversals */
    uint64_t gather_rays;    /* gather pinhole/specular traversals */
    uint64_t photons_stored; /* photons that reached the hash last trace */
    uint64_t node_tests;     /* ray-box tests of the path tracer */
    uint64_t tri_tests;      /* ray-triangle tests of the path tracer */
    uint64_t surface_hits;   /* path-tracer closest hits shaded (normal + material) */
    uint64_t light_samples;  /* NEE light records fetched */
    uint64_t photon_node_tests; /* ray-box tests of photon trace + gather */
    uint64_t photon_tri_tests;  /* ray-triangle tests of photon trace + gather */
    uint64_t kernel_launches;/* kernels this context launched */
    uint64_t h2d_bytes;      /* host -> device bytes copied by this context */
    uint64_t d2h_bytes;      /* device -> host bytes copied by this context */
    uint32_t error_word;     /* RC_GUARD_* bits raised by kernels */
    uint32_t bvh_depth;      /* levels below the root of the uploaded BVH (0: a
                                leaf root or no scene); past 28 the shadow walk,
                                past 60 every walk keeps the reference's own
                                stack policy (its stacks can overflow there) */
} rc_counters;

/* Kernel kinds for rc_get_kernel_times. */
#define RC_KERNEL_RENDER 0         /* megakernel path tracer */
#define RC_KERNEL_PHOTON_TRACE 1
#define RC_KERNEL_PHOTON_GATHER 2
#define RC_KERNEL_ATROUS 3
#define RC_KERNEL_NORMALIZE 4
#define RC_KERNEL_WF_GENERATE 5    /* wavefront: camera rays */
#define RC_KERNEL_WF_TRACE 6       /* wavefront: closest-hit + shadow traversal */
#define RC_KERNEL_WF_SHADE 7       /* wavefront: one bounce of shading + NEE sample */
#define RC_KERNEL_WF_ACCUMULATE 8  /* wavefront: in-order accumulation, G-buffer */
#define RC_KERNEL_PHOTON_LAYOUT 9  /* photon map: cell scan, scatter, heads/next */
#define RC_KERNEL_KPCNN 10         /* learned denoiser: features, 4 convolutions, filter */
#define RC_KERNEL_DISPLAY 11       /* ACES + sRGB to RGBA8 (rc_display) */
#define RC_KERNEL_VHS 12           /* the VHS chain's passes (rc_post_vhs) */
#define RC_KERNEL_WF_SORT 13       /* wavefront: misses finished, hits into material queues */
#define RC_KERNEL_KINDS 14

/* Path-tracer engines (rc_set_engine). */
#define RC_ENGINE_MEGAKERNEL 0  /* one thread per pixel runs whole paths */
#define RC_ENGINE_WAVEFRONT 1   /* per-bounce kernels over compacted path queues,
                                   traced with a persistent kernel that refills
                                   idle lanes with new rays (chunks of
                                   rc_tuning.refill_min_paths paths or more;
                                   smaller ones grid-stride); in exact math a
                                   ray keeps the reference's visiting order */
#define RC_ENGINE_WAVEFRONT_STATIC 2 /* as above, traced with a grid-stride loop */

/* rc_tuning.wide_bvh bits: which rays traverse the 4-wide copy of the BVH
 * (collapsed from the reference's binary tree at upload; fast math only --
 * exact math always walks the binary tree in the reference's order). */
#define RC_WIDE_PATHS 0x1    /* camera-path closest-hit and shadow rays */
#define RC_WIDE_PHOTONS 0x2  /* photon-trace and gather rays */

/* Launch-shape knobs of one context, picked by the autotuner
 * (retrocam_b200/autotune.py) or by hand.  No counterpart in the reference,
 * whose shaders have fixed local sizes.  Results do not depend on any knob in
 * exact math; in fast math the traversal width changes the order of float
 * operations of tied hits only.  Zero fields select the defaults. */
typedef struct rc_tuning {
    int32_t engine;        /* RC_ENGINE_*; default RC_ENGINE_WAVEFRONT */
    int32_t chunk_paths;   /* wavefront paths in flight (queue capacity), 0 = 16M */
    int32_t wide_bvh;      /* RC_WIDE_* bits; default 0 (the persistent trace of
                              RC_ENGINE_WAVEFRONT walks the binary tree always) */
    int32_t trace_block;   /* threads per block of the wavefront trace: 64, 128, 256 (0 = 128) */
    int32_t shade_block;   /* threads per block of the wavefront shade: 64, 128, 256 (0 = 128) */
    int32_t photon_block;  /* threads per block of the photon trace: 64, 128, 256 (0 = 128) */
    int32_t photon_full_first; /* fast math: 0 traces a photon's first segment against the
                                  specular triangles, then tests the others up to that hit
                                  (a diffuse first hit ends the photon unstored, so only
                                  the specular hit matters); 1 traces the whole scene */
    int32_t refill_lanes;  /* RC_ENGINE_WAVEFRONT trace: a warp fetches new rays when fewer
                              than this many lanes are busy, 1..32 (0 = 16) */
    int32_t leaf_quarters; /* RC_ENGINE_WAVEFRONT trace: a warp tests its parked leaves
                              once this many quarters of its busy lanes cannot step on
                              (or all have a leaf parked), 1..4 (0 = 2) */
    int32_t refill_min_paths; /* RC_ENGINE_WAVEFRONT: chunks of fewer paths are
                                 traced with the grid-stride loop, where a launch holds
                                 about one wave of rays (0 = 1048576; 1 = always refill) */
    int32_t material_queues;  /* wavefront engines: 1 sorts each bounce's hits into
                                 material queues (diffuse / metal or glass) before the
                                 shade, so a warp runs one BSDF branch; 0 shades the ray
                                 queue as it stands (default: in fast math the shade waits
                                 on path-state memory, not on divergence, and the sort costs
                                 more than the fuller warps save on the export frame; the
                                 exact build's heavier shade gains, and its tuned shape on
                                 the B200 sets it) */
    int32_t interior_steps;   /* RC_ENGINE_WAVEFRONT trace: moves through the tree a lane
                                 makes per scheduling round of its warp, 1..8 (0 = 6: the
                                 warp's ballots and phase choice are shared by up to six
                                 moves; export frame trace 65.0 -> 61.2 ms) */
} rc_tuning;

/* error_word bits. */
#define RC_GUARD_TRAVERSAL_CAP 0x1u  /* a traversal exceeded its node-visit cap */
#define RC_GUARD_BAD_INDEX 0x2u      /* a node/primitive/material index was out of range */
#define RC_GUARD_CHAIN_CAP 0x4u      /* reserved: gather chain cap (512) is a
                                        reference semantic, not an error */
#define RC_GUARD_MMA_WAIT 0x8u       /* a tensor-core kernel's bounded wait gave up */

/* Math modes of the kernels. */
#define RC_MATH_FAST 0   /* FMA contraction, CUDA intrinsics; checked by tolerance */
#define RC_MATH_EXACT 1  /* no contraction, rc_exact_math.h transcendentals;
                            bit-identical to the CPU oracle */

typedef struct rc_ctx rc_ctx;

/* ---------------------------------------------------------------------------
 * Context
 * ------------------------------------------------------------------------- */

/* Creates a context rendering width x height on a CUDA device; allocates the
 * accumulation (RGBA32F), G-buffer (RGBA16F), albedo (RGBA16F) and variance
 * (R32F) images of core/Renderer.java:152-193. */
int rc_ctx_create(int width, int height, int device, rc_ctx** out);
int rc_ctx_destroy(rc_ctx* ctx);
/* Copies the last error text of ctx (or of the last failed rc_ctx_create
 * when ctx is NULL) into buf, NUL-terminated. */
int rc_last_error(const rc_ctx* ctx, char* buf, size_t n);
int rc_set_math_mode(rc_ctx* ctx, int mode);
int rc_synchronize(rc_ctx* ctx);
/* Runs the context's work on a caller-owned cudaStream_t (passed as void*),
 * or on the context's own stream again when cuda_stream is NULL. */
int rc_ctx_set_stream(rc_ctx* ctx, void* cuda_stream);
/* When enabled, every kernel launch is bracketed by CUDA events on the
 * launching stream; rc_get_kernel_times synchronises and returns, per kernel
 * kind, the summed milliseconds and the launch count since the last call. */
int rc_set_kernel_timing(rc_ctx* ctx, int enable);
/* Measures the device's FP32 FMA throughput in TFLOP/s (16 independent FMA
 * chains per thread on every SM; best of 5, CUDA events).  No counterpart
 * in the reference; the denominator of the traversal kernels' FP32
 * roofline fraction. */
int rc_measure_fp32_peak(int device, double* tflops_out);
/* Selects the path-tracer engine; both give identical results in exact math.
 * chunk_paths bounds the wavefront's in-flight paths (path state is about
 * 200 bytes each); 0 picks the default. */
int rc_set_engine(rc_ctx* ctx, int engine, int chunk_paths);
/* Sets / reads all launch-shape knobs at once (rc_set_engine sets the first
 * two).  RC_ERR_INVALID_ARG for a value outside the documented ranges. */
int rc_set_tuning(rc_ctx* ctx, const rc_tuning* tuning);
int rc_get_tuning(rc_ctx* ctx, rc_tuning* out);
int rc_get_kernel_times(rc_ctx* ctx, double* ms_out, uint64_t* launches_out);
int rc_abi_version(void);

/* ---------------------------------------------------------------------------
 * Host scene logic (bit-exact restatements of the reference's Java)
 * ------------------------------------------------------------------------- */

/* scene/Box.java:25-76 plus scene/TransformedPrimitive.java:32-95 (applied
 * when any rotation is non-zero, as scene/SceneObject.java:80-88 does).
 * Writes 12 triangles. */
int rc_tessellate_box(float cx, float cy, float cz, float hx, float hy, float hz,
                      int mat_index, float rot_x_deg, float rot_y_deg, float rot_z_deg,
                      rc_triangle* out12);

/* scene/Sphere.java:34-101 (+ rotation as above).  Writes
 * 2*stacks*slices - 2*slices triangles (poles skipped). */
int rc_tessellate_sphere(float cx, float cy, float cz, float radius, int mat_index,
                         int stacks, int slices, float rot_x_deg, float rot_y_deg,
                         float rot_z_deg, rc_triangle* out, int capacity, int* count);

/* A flat-normal triangle list from vertex positions (9 floats each), as the
 * reference's Primitive.toTriangles extension point would produce with
 * GpuTriangle.withFlatNormal (scene/GpuTriangle.java:38-50). */
int rc_triangles_from_positions(const float* positions, int count, int mat_index,
                                rc_triangle* out);

/* scene/BVHBuilder.java:35-202: binned SAH (8 buckets, leaf <= 4,
 * C_trav 1, C_isect 1.5), depth-first node order, in-place partition.
 * Writes the reordered triangles and the nodes; node_capacity >= 2*count. */
int rc_build_bvh(const rc_triangle* in, int count, rc_triangle* out_tris,
                 rc_bvh_node* out_nodes, int node_capacity, int* node_count);

/* scene/SceneUploader.java:144-216: light list (BVH triangle order) with
 * power = luma601 * area * pi and a CDF whose last entry is 1.  With no
 * emissive triangle it writes one zeroed stub and *light_count = 0. */
int rc_build_lights(const rc_triangle* tris, int count, const rc_material* mats,
                    int material_count, rc_light* out, int capacity,
                    int* light_count, float* total_power);

/* camera/ThinLensCamera.java:27-68: lens radius f/(2N) and tan(fov/2) for a
 * 24 mm sensor height. */
int rc_thin_lens(float focal_length_mm, float f_stop, float* lens_radius,
                 float* fov_tan_half);

/* camera/OrbitCamera.java:155-171,274-291: eye, forward, right, up from
 * orbit angles about a target. out12 = eye[3], forward[3], right[3], up[3]. */
int rc_orbit_basis(float theta, float phi, float radius, float target_x,
                   float target_y, float target_z, float* out12);

/* scene/SPPMManager.java:170-173: r *= (float)sqrt((n+alpha)/(n+1.0)). */
float rc_sppm_next_radius(float radius, int iteration, float alpha);

/* keyframe/KeyframeTrack.java:102-178. interp[i]: 0 STEP, 1 LINEAR,
 * 2 BEZIER (Catmull-Rom Hermite).  times ascending. */
float rc_keyframe_evaluate(const float* times, const float* values,
                           const int32_t* interp, int count, float time,
                           float default_value);

/* ---------------------------------------------------------------------------
 * Device scene
 * ------------------------------------------------------------------------- */

/* scene/SceneUploader.java:54-99 after the BVH build: copies the four SSBO
 * arrays to the device (converting them to the kernels' internal layout)
 * and validates node and material indices (RC_ERR_BAD_SCENE on failure).
 * lights may be NULL when light_count == 0. */
int rc_scene_upload(rc_ctx* ctx, const rc_triangle* tris, int tri_count,
                    const rc_bvh_node* nodes, int node_count,
                    const rc_material* mats, int material_count,
                    const rc_light* lights, int light_count, float total_light_power);

/* ---------------------------------------------------------------------------
 * Path tracer (core/Renderer.java:72-130, pathtrace.comp)
 * ------------------------------------------------------------------------- */

/* Adds n_spp samples per pixel with frame indices first_frame ..
 * first_frame+n_spp-1 (u_frameIndex); frame 0 clears the accumulation and
 * writes the G-buffer and albedo images. */
int rc_render(rc_ctx* ctx, const rc_camera* cam, const rc_settings* settings,
              int first_frame, int n_spp);

/* Renderer.reset(): zeroes the images and the sample counter. */
int rc_reset(rc_ctx* ctx);
/* Samples accumulated since the last reset (Renderer.getTotalSamples). */
int rc_total_samples(const rc_ctx* ctx);

/* ---------------------------------------------------------------------------
 * SPPM (scene/SPPMManager.java, scene/PhotonMap.java)
 * ------------------------------------------------------------------------- */

/* SPPMManager.reset: radius = r0, iteration = 0.  The gathers of one SPPM
 * sequence share their pixel-centre rays (same camera, scene and settings:
 * traced by the first gather, reused by the next); a reset starts a new
 * sequence whose first gather traces them again. */
int rc_sppm_reset(rc_ctx* ctx, float initial_radius);
/* SPPMManager.tracePhotons: clears the hash (PhotonMap.clear) and traces
 * photon_count photons with seed iteration*7919+6271 at the current radius. */
int rc_sppm_trace(rc_ctx* ctx, const rc_sppm_params* params);
/* SPPMManager.gatherRadiance: adds weight * caustic radiance into the
 * accumulation image (weight 1 is the reference; the export loop uses
 * spp/iterations when iterations < spp). */
int rc_sppm_gather(rc_ctx* ctx, const rc_camera* cam, const rc_sppm_params* params,
                   float weight);
/* SPPMManager.updateRadius. */
int rc_sppm_update_radius(rc_ctx* ctx, float alpha);
int rc_sppm_state(const rc_ctx* ctx, float* radius, int* iteration);

/* ---------------------------------------------------------------------------
 * Denoiser (post/AtrousDenoiser.java:60-125, PostProcessStack.java:112-147)
 * ------------------------------------------------------------------------- */

/* p00 normalisation then 1..5 à-trous passes (or the normalised image alone
 * when disabled or over max_spp).  Result stays on the device; when
 * out_rgba is non-NULL it is also copied to that host array (W*H*4 floats). */
int rc_denoise_atrous(rc_ctx* ctx, const rc_atrous_params* params, float* out_rgba);

/* No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory -- hosts that own every device byte through their
 * own pool and budget, or loops that must not hit the synchronisation an
 * allocation can cause mid-frame.  Same p00 + à-trous chain as
 * rc_denoise_atrous, but every image is a caller-owned DEVICE pointer (accum
 * RGBA32F, gbuffer/albedo RGBA16F, variance R32F, out RGBA32F; out must not
 * share a byte with any input, else RC_ERR_INVALID_ARG) and the one
 * intermediate image lives in a static device array of RC_NOALLOC_MAX_PIXELS
 * RGBA32F pixels (16 MiB) that every GPU loading this library holds until the
 * process exits.  Larger images return RC_ERR_CAPACITY.  Every call looks up
 * that array's address in the caller's current CUDA context; the first call
 * on a device also loads the module there, so make it before any stream
 * capture.  Errors are read with rc_last_error(NULL, ...).  All calls on a
 * device share the array, so calls that overlap on the GPU race.
 * cuda_stream may be NULL (legacy stream). */
#define RC_NOALLOC_MAX_PIXELS 1048576
int rc_denoise_atrous_noalloc(const float* accum_rgba, const uint16_t* gbuffer_rgba16f,
                              const uint16_t* albedo_rgba16f, const float* variance,
                              float* out_rgba, int width, int height, int total_samples,
                              const rc_atrous_params* params, int math_mode, void* cuda_stream);

/* ---------------------------------------------------------------------------
 * Whole export frame (export/RenderPipeline.java:209-239)
 * ------------------------------------------------------------------------- */

/* renderer.reset; sppm.reset; for each block of spp/sppm_iterations samples:
 * trace photons -> render the block -> gather (weighted) -> shrink radius;
 * then p00 + à-trous.  sppm_iterations == spp reproduces the reference
 * order exactly; sppm_iterations == 0 disables SPPM.  out_rgba (nullable)
 * receives the denoised frame. */
int rc_render_frame(rc_ctx* ctx, const rc_camera* cam, const rc_settings* settings,
                    int spp, const rc_sppm_params* sppm, float sppm_initial_radius,
                    int sppm_iterations, const rc_atrous_params* atrous,
                    float* out_rgba);

/* ---------------------------------------------------------------------------
 * One export frame split across devices.  No counterpart in the reference
 * (one GL context, one GPU); the split keeps RenderPipeline.accumulateFrame's
 * work (export/RenderPipeline.java:209-239) and the shaders' seeds: frame
 * index f seeds pixel paths (pathtrace.comp:94-98, Renderer.java:99) and
 * iteration k seeds its photons (k*7919+6271, SPPMManager.java:88), so a
 * part renders exactly the samples and photon maps the whole frame would.
 * ------------------------------------------------------------------------- */

/* The part-th of `parts` contiguous shares of a frame: SPPM iterations
 * [k0, k1) with their sample blocks [s0, s1) (iteration k owns samples
 * [k*spp/it, (k+1)*spp/it), as in rc_render_frame), or, without SPPM,
 * samples [s0, s1) = [part*spp/parts, (part+1)*spp/parts) (k0 = k1 = 0).
 * Host arithmetic only. */
int rc_frame_part_range(int spp, int sppm_iterations, int part, int parts, int* k0, int* k1, int* s0,
                        int* s1);
/* Renders one part of rc_render_frame's work into this context's images:
 * rc_reset, then (SPPM) the radius and iteration counter advanced to
 * iteration k0 and, per iteration k < k1, trace -> render the block ->
 * gather -> shrink the radius; no denoise.  The images then hold this
 * part's sums (accum rgb and count, variance); the part holding sample 0
 * also writes the G-buffer and albedo.  The sum of all parts' accum and
 * variance images is the whole frame's, up to the order of the float
 * additions; after adding the other parts' images into one context, set
 * its sample count with rc_set_total_samples and denoise there.
 * rc_total_samples reports this part's sample count. */
int rc_render_frame_part(rc_ctx* ctx, const rc_camera* cam, const rc_settings* settings, int spp,
                         const rc_sppm_params* sppm, float sppm_initial_radius, int sppm_iterations, int part,
                         int parts);
/* The sample count rc_denoise_atrous and rc_denoise_learned divide by
 * (Renderer.getTotalSamples), for images merged from parts. */
int rc_set_total_samples(rc_ctx* ctx, int total_samples);
/* Device addresses of the context's images (accum RGBA32F, G-buffer and
 * albedo RGBA16F, variance R32F; W*H pixels each, row-major) and the
 * cudaStream_t its work runs on, for a caller that reduces parts with a
 * collective library in place.  Work queued on that stream must finish
 * (or be waited for on the caller's stream) before another stream reads or
 * writes the images. */
int rc_get_images(rc_ctx* ctx, void** accum, void** gbuffer, void** albedo, void** variance, void** stream);

/* ---------------------------------------------------------------------------
 * Batched export frames (export/RenderPipeline.java:149-239 per frame, the
 * video-export loop over keyframed cameras)
 * ------------------------------------------------------------------------- */

/* One frame of a batch: its camera (keyframes already evaluated), samples
 * per pixel and SPPM iterations (0 = no SPPM; <= spp). */
typedef struct rc_frame_desc {
    rc_camera camera;
    int32_t spp;
    int32_t sppm_iterations;
} rc_frame_desc;

/* Renders n_frames frames of uneven cost, each with the samples, gathers and
 * denoise rc_render_frame would give it (per frame: SPPM iteration k traces
 * a photon map, renders sample slice [k*spp/it, (k+1)*spp/it), gathers with
 * that slice's weight, shrinks the radius), and writes the finished frames to
 * out_frames (n_frames*W*H*4 floats, host; NULL keeps them on the device).
 *
 * With the wavefront engines the frames run together: iteration k traces
 * ONE photon map for all frames (it depends only on the scene, k and r_k),
 * then slice k of every frame is packed into shared wavefront chunks (each
 * chunk a list of (frame, sample range) segments, so frames of few samples
 * fill chunks with others) and gathered into each frame.  Per frame the
 * additions happen in rc_render_frame's order, so exact math gives its
 * bits up to the photon-hash insertion order that the gather sums in.
 * The megakernel engine renders the frames one after the other.
 *
 * Every buffer is sized before the first launch.  With use_graph != 0 the
 * whole batch is captured once into a CUDA graph and replayed on later
 * calls with the same frames, settings and launch shape, so the host issues
 * one launch per batch.  Several contexts on their own streams may render
 * disjoint batches concurrently. */
int rc_render_frames(rc_ctx* ctx, const rc_frame_desc* frames, int n_frames,
                     const rc_settings* settings, const rc_sppm_params* sppm,
                     float sppm_initial_radius, const rc_atrous_params* atrous,
                     float* out_frames, int use_graph);

/* ---------------------------------------------------------------------------
 * Learned denoiser (kernel-predicting CNN).  No counterpart in the
 * reference, which has only the à-trous filter; the entry point sits beside
 * rc_denoise_atrous (post/AtrousDenoiser.java:60) with the same inputs.
 *
 * Network: features (log1p radiance, albedo, normal, depth t/(1+t); 10
 * channels padded to 16) -> 3 x [conv3x3 32 ch + ReLU] -> conv3x3 head of 25
 * logits -> per-pixel softmax -> 5x5 filter (edge clamped) of the mean
 * radiance.  BF16 weights and activations, FP32 accumulation (tcgen05).
 *
 * Parameters are one FP32 vector of RC_KPCNN_PARAMS floats: for layers 1, 2,
 * 3 and the head in turn, W[tap][co][ci] (tap = 3*dy + dx over the 3x3
 * window, co < 32, ci < 16 for layer 1 and < 32 otherwise; head co >= 25 and
 * layer-1 ci >= 10 must be zero) followed by bias[32].
 * ------------------------------------------------------------------------- */
#define RC_KPCNN_PARAMS 32384

typedef struct rc_kpcnn {
    const float* params;   /* host, RC_KPCNN_PARAMS floats */
    int32_t param_count;   /* must equal RC_KPCNN_PARAMS */
} rc_kpcnn;

/* Denoises the context's current accumulation (accum / N with the G-buffer
 * and albedo as features) into the context's output frame; copies it to
 * out_rgba (W*H*4 floats) when non-NULL.  Uploads the parameters each call. */
int rc_denoise_learned(rc_ctx* ctx, const rc_kpcnn* weights, float* out_rgba);

/* Building blocks on caller-owned DEVICE buffers (training and tests), on
 * the given CUDA stream (NULL = legacy default).  Layouts as in kpcnn.cu:
 * NHWC bf16 activations (16 or 32 channels), packed bf16 weights
 * [tap][ci/8][co][8], float4 radiance.  `err` is a device word that
 * receives a nonzero bit when a kernel's bounded wait gave up. */
int rc_kp_conv3x3(const void* in, int cin, const void* wpk, const float* bias, void* out, int out_f32,
                  int relu, const void* mask, int n, int h, int w, unsigned int* err, void* stream);
int rc_kp_wgrad(const void* x, int cin, const void* dy, float* dw, float* db, int n, int h, int w,
                unsigned int* err, void* stream);
int rc_kp_head(const float* logits, const void* color, const void* target, void* out, void* dlogits,
               double* loss, float grad_scale, int n, int h, int w, void* stream);
/* packed7: w1, w2, w3, head (forward) and w2, w3, head (backward-data). */
int rc_kp_pack(const float* params, void* const* packed7, void* stream);
int rc_kp_adam(float* params, float* grads, float* m, float* v, int count, float lr, float beta1, float beta2,
               float eps, int step, void* stream);
int rc_kp_crop(const void* feat_all, const void* color_all, const void* target_all, const int* src,
               const int* tgt, const int* oy, const int* ox, int batch, int H, int W, int size, void* feat,
               void* color, void* target, void* stream);
/* The network input of the context's current images: feat (W*H*16 bf16)
 * and mean radiance (W*H float4), device buffers, on the context's stream. */
int rc_kp_features(rc_ctx* ctx, void* feat, void* color);

/* ---------------------------------------------------------------------------
 * Read-back and counters
 * ------------------------------------------------------------------------- */

/* Copies the images to host arrays (any may be NULL): accum W*H*4 floats,
 * gbuf/galb W*H*4 halves, variance W*H floats. */
int rc_read_buffers(rc_ctx* ctx, float* accum_rgba, uint16_t* gbuffer_rgba16f,
                    uint16_t* albedo_rgba16f, float* variance);
/* Copies the last denoised/normalised frame (W*H*4 floats). */
int rc_read_output(rc_ctx* ctx, float* out_rgba);
/* ---------------------------------------------------------------------------
 * The VHS chain (post/PostProcessStack.java:149-277, shaders post/p01..p16)
 * ------------------------------------------------------------------------- */

/* The chain's knobs, as core/RenderSettings.java names them (defaults
 * there, :49-191; rc_vhs_defaults fills them with every pass off), and the
 * per-frame values it reads: RenderSettings.frameIndex and TemporalState's
 * time (s) and AGC gain. */
typedef struct rc_vhs_params {
    int32_t enabled;                 /* bit k-1 enables pass pk (p01..p16; p05, p06 have no shader) */
    int32_t frame_index;
    float time_s;
    float agc_gain;
    float luma_blur_sigma;           /* p01 */
    float chroma_res_sigma;          /* p02 */
    float color_temp_bias, color_hue_rot, color_saturation, color_drift_speed;      /* p03 */
    float dr_black_lift, dr_shadow_crush, dr_highlight_knee, dr_highlight_clip;     /* p04 */
    float ccd_noise_luma_base, ccd_noise_chroma_scale;                            /* p07 */
    float ccd_smear_threshold, ccd_smear_intensity;                               /* p08 */
    int32_t ccd_smear_length;
    float chroma_bleed_factor;                                                    /* p09 */
    float timebase_amplitude_px, timebase_freq, timebase_speed;                   /* p10 */
    float dot_crawl_intensity, dot_crawl_subcarrier, dot_crawl_edge_thresh;       /* p11 */
    float tape_age, dropout_bright, dropout_burst_rate;                           /* p12 */
    int32_t head_switch_lines;                                                    /* p13 */
    float head_switch_jitter, head_switch_ripple, head_switch_chroma;
    float tracking_severity, tracking_max_displace_px, tracking_fringe_width_px;  /* p14 */
    float edge_enhance_amount, edge_enhance_core_threshold;                       /* p15 */
    float interlace_field_offset_px, interlace_comb_strength, interlace_comb_edge_thresh,
        interlace_line_weighting;                                                 /* p16 */
} rc_vhs_params;

#define RC_VHS_PASS(k) (1 << ((k) - 1))

/* RenderSettings' defaults, every pass disabled. */
void rc_vhs_defaults(rc_vhs_params* p);
/* PostProcessStack.runChain's passes p01..p16 (those enabled, in order) on
 * the last output (what rc_read_output returns, e.g. rc_denoise_atrous'
 * p00 + a-trous result), ping-ponging between RGBA32F images as the
 * reference's PingPongBuffer does; the result becomes the last output (for
 * rc_read_output and rc_display). */
int rc_post_vhs(rc_ctx* ctx, const rc_vhs_params* p);
/* One pass (1..16 except 5, 6) on device RGBA32F images of w x h, on
 * `stream` (NULL: the default stream); in and out must not overlap. */
int rc_vhs_pass(int pass, const void* in_rgba, void* out_rgba, int w, int h, const rc_vhs_params* p,
                void* stream);

/* display.frag:11-41 as the export path runs it (export/RenderPipeline.java:
 * 244-259, applyDisplayPass into a GL_RGBA8 framebuffer) and the read-back of
 * export/FrameExporter.java:51-80: the last output (what rc_read_output
 * returns) divided by max(total_samples, 1) and scaled by exposure -- the
 * shader's u_totalSamples and u_exposure; the export path passes 1 and 1.0
 * because the denoiser already normalised -- then the ACES fit and the sRGB
 * encode, stored as the RGBA8 framebuffer stores a fragment (each channel
 * round(clamp(v, 0, 1) * 255), NaN as 0, alpha 255), rows top to bottom as
 * FrameExporter writes them (stbi_flip_vertically_on_write).  out_rgba8:
 * W*H*4 bytes of host memory, or NULL to keep the image on the device. */
int rc_display(rc_ctx* ctx, int total_samples, float exposure, uint8_t* out_rgba8);
/* rc_display on frame `frame` (0-based) of the last rc_render_frames batch,
 * whose finished frames stay on the device: the export loop displays and
 * writes every frame it renders (RenderPipeline.tickVideoFrame,
 * export/RenderPipeline.java:150-185).  RC_ERR_INVALID_ARG outside the
 * batch. */
int rc_display_frame(rc_ctx* ctx, int frame, int total_samples, float exposure, uint8_t* out_rgba8);
/* Copies the photon map of the last trace (any may be NULL): photons
 * (capacity entries), heads (hash_size), next (capacity), counter. */
int rc_read_photon_map(rc_ctx* ctx, rc_photon* photons, int photon_capacity,
                       int32_t* heads, int hash_size, int32_t* next,
                       uint32_t* counter);
int rc_get_counters(rc_ctx* ctx, rc_counters* out);
int rc_reset_counters(rc_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* RETROCAM_H */
