/*
 * vkptc.h -- C ABI of libvkpt_cuda, the sm_100a render backend for vkPathTracer.
 *
 * This is the boundary a `src/gpu/cuda` IPathTracer adapter in the reference
 * binds.  Plain pointers and sizes only; every call
 * returns a vkptc_status_code (the numeric values of vkpt::core::StatusCode,
 * src/core/contracts/Result.h:13-23) and never throws.  Host buffers passed
 * in are read or written synchronously before the call returns; the context
 * owns all device memory (scene, BVH, film, path queues).
 *
 * Threading: one thread drives a context (the reference's contract for an
 * IPathTracer, src/render/RenderCoordinator.cpp:412); distinct contexts may
 * be driven concurrently.
 *
 * Record layouts follow the reference's standard GPU word maps
 * (src/pathtracer/PathTracer.h:778-786, src/gpu/VulkanGpuPathTracer.cpp:323-396):
 *   material[16] = albedo3, emissive3, roughness, model, metallic, ior,
 *                  transmission, clearcoat, sheen, anisotropy, alpha,
 *                  effect | (double_sided << 10)
 *   light[16]    = position3, color3, intensity, radius, direction3,
 *                  spot_inner_cos, spot_outer_cos, 0, 0, 0
 */
#ifndef VKPTC_H
#define VKPTC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Version of the struct layouts below.  2: vkptc_scene_view gained the camera lens fields,
 * vkptc_config.reserved[0] became triangle_test. */
#define VKPTC_ABI_VERSION 2u

typedef enum vkptc_status {
  VKPTC_OK = 0,
  VKPTC_UNSUPPORTED = 1,
  VKPTC_INVALID_ARGUMENT = 2,
  VKPTC_NOT_READY = 3,
  VKPTC_BUSY = 4,
  VKPTC_ALLOC_FAILED = 5,
  VKPTC_TIMEOUT = 6,
  VKPTC_CANCELLED = 7,
  VKPTC_INTERNAL_ERROR = 8
} vkptc_status_code;

/* Mirrors PathTracerLifecycle (src/pathtracer/PathTracer.h:485-491). */
typedef enum vkptc_lifecycle {
  VKPTC_UNINITIALIZED = 0,
  VKPTC_CONFIGURED = 1,
  VKPTC_SCENE_LOADED = 2,
  VKPTC_READY = 3,
  VKPTC_FAILED = 4
} vkptc_lifecycle;

typedef struct vkptc_ctx vkptc_ctx;

/* The VKPTC_ABI_VERSION the library was built with; a caller compiled against another version
 * must not pass its structs to it. */
uint32_t vkptc_abi_version(void);

typedef struct vkptc_config {
  int32_t device;            /* CUDA device ordinal */
  uint32_t block_size;       /* threads per block of the wavefront kernels; 0 = autotuned/default */
  uint32_t stack_depth;      /* traversal stack entries per thread kept in shared memory (the rest
                                spill to global memory); 0 = 16 */
  uint32_t math_mode;        /* 0 = parity (transcendentals in FP64, rounded once), 1 = fast FP32 */
  uint32_t collect_stats;    /* 1 = count node/leaf/triangle visits (device counters) */
  uint32_t wave_paths;       /* paths per wavefront wave (0 = 4 Mi) */
  uint32_t stage_timing;     /* 1 = CUDA-event timing of every stage launch */
  uint32_t steps;            /* traversal steps between warp refills in the low 16 bits (0 = 4); the
                                high 16 bits, when non-zero, refill a warp as soon as that many of its
                                lanes are idle (at most 32), checked after every step */
  uint32_t bvh_mode;         /* traversal tree: VKPTC_BVH_REFERENCE (the reference builder's tree,
                                flattened) or VKPTC_BVH_SAH (binned SAH); hit ids are the
                                reference's in both (ties/parallel rule use the reference tree) */
  uint32_t build_mode;       /* where vkptc_build_acceleration builds: VKPTC_BUILD_DEVICE (default;
                                the same reference tree, bit for bit, plus the traversal tree,
                                built by CUDA kernels) or VKPTC_BUILD_HOST (the host restatement of
                                ParallelBvhBuilder, kept as the parity mode) */
  uint32_t triangle_test;    /* VKPTC_TRIANGLE_MT (default): the reference's Moller-Trumbore test
                                (BvhTriangleIntersector.cpp:35-74), hit ids bit-exact against it;
                                VKPTC_TRIANGLE_WATERTIGHT: the watertight test of Woop, Benthin and
                                Wald (JCGT 2013) on the triangles' own vertices, so a ray through a
                                shared edge or vertex of a closed mesh never passes between its
                                triangles.  The watertight mode needs the device build; ray queries,
                                renders of a context and every batch driver honour it; the adjoint
                                does not take it (VKPTC_UNSUPPORTED). */
  uint32_t reserved[2];
} vkptc_config;

#define VKPTC_BVH_REFERENCE 0u
#define VKPTC_BVH_SAH 1u
#define VKPTC_BUILD_DEVICE 0u
#define VKPTC_BUILD_HOST 1u
#define VKPTC_TRIANGLE_MT 0u
#define VKPTC_TRIANGLE_WATERTIGHT 1u

/* Mirrors RenderSettings (src/pathtracer/PathTracer.h:134-178). */
typedef struct vkptc_render_settings {
  uint32_t width;
  uint32_t height;
  uint32_t spp;
  uint32_t max_depth;
  uint64_t seed;
  uint32_t enable_nee;
  uint32_t enable_mis;
  uint32_t deterministic;
  uint32_t rr_start_depth;
  float rr_min_survival;
  float rr_max_survival;
  float camera_aperture_radius;
  float camera_focus_distance;
  float firefly_clamp;       /* extension: per-channel clamp of each sample, 0 = off (reference) */
  uint32_t reserved;
} vkptc_render_settings;

/* POD view of PathTracerSceneSnapshot (src/pathtracer/PathTracer.h:358-409):
 * the triangle subset the render path consumes. */
typedef struct vkptc_scene_view {
  const float* vertices;       uint32_t vertex_count;     /* xyz per vertex */
  const uint32_t* indices;     uint32_t index_count;      /* 3 per triangle */
  const uint32_t* instances;   uint32_t instance_count;   /* first_triangle, triangle_count, material_index */
  const float* materials;      uint32_t material_count;   /* 16 floats each */
  const float* lights;         uint32_t light_count;      /* 16 floats each */
  float environment[3];
  float camera_position[3];
  float camera_target[3];
  float camera_up[3];
  float camera_fov_deg;
  float camera_aperture_radius;
  float camera_focus_distance;
  /* Optional equirectangular environment map (PathTracerSceneSnapshot's
   * environment_map, sampled as SampleSceneEnvironment does,
   * src/pathtracer/PathTracer.cpp:213-272): width*height rgb texels, row-major,
   * row 0 toward +y; scale multiplies the texels (all <= 1e-6: 1).  NULL or a
   * zero size: the constant environment above. */
  const float* environment_map;
  uint32_t environment_map_width;
  uint32_t environment_map_height;
  float environment_map_scale[3];
  /* Optional SDF primitives (PathTracerSceneSnapshot::sdf_primitives, the
   * RTSdfPrimitive records of src/pathtracer/PathTracer.h:330-339), tested
   * after the triangles for every extension and shadow ray with the nearest
   * surface kept, as ScalarCpuPathTracer::intersect_scene does
   * (src/pathtracer/ScalarCpuPathTracer.Intersect.cpp:91-129).  16 floats
   * each: shape (vkptc_sdf_shape), position xyz, scale xyz, rotation xyz
   * (Euler angles, radians), material index, radius, param_a, param_b, 0, 0.
   * Shapes outside vkptc_sdf_shape never hit (the reference's switch default). */
  const float* sdf_primitives;
  uint32_t sdf_count;
  /* Optional dynamic-transform instances (RTInstance, src/pathtracer/PathTracer.h:276-296),
   * flattened as CpuBvhAccelerator::build does (src/pathtracer/CpuBvhAccelerator.cpp:173-247):
   * instance_local holds 5 words per instance (flags, local_first_vertex, local_vertex_count,
   * local_first_index, local_index_count) and instance_transforms 10 floats per instance
   * (translation xyz, rotation quaternion xyzw, scale xyz).  An instance with flag bit 0
   * (kRTInstanceFlagDynamicTransform) and local vertices and indices takes each triangle from
   * local_vertices / local_indices, scaled, rotated and translated to world space, falling back
   * to the global arrays for a triangle whose local indices are out of range.  NULL arrays:
   * every instance uses the global arrays. */
  const uint32_t* instance_local;
  const float* instance_transforms;
  const float* local_vertices;
  uint32_t local_vertex_count;
  const uint32_t* local_indices;
  uint32_t local_index_count;
  /* Lens shape of the thin-lens camera (PathTracerSceneSnapshot camera_iris_blade_count,
   * camera_iris_rotation_degrees, camera_iris_roundness, camera_anamorphic_squeeze,
   * src/pathtracer/PathTracer.h:405-408), sampled as ScalarCpuPathTracer::camera_rays does
   * (src/pathtracer/ScalarCpuPathTracer.Render.cpp:88-116): 3..64 blades with roundness below
   * 0.999 give a polygonal aperture, the squeeze scales the lens offset along the camera's right
   * axis.  camera_lens_set = 0: the snapshot's defaults (no blades, rotation 0, roundness 1,
   * squeeze 1), whatever the four fields hold. */
  uint32_t camera_lens_set;
  uint32_t camera_iris_blade_count;
  float camera_iris_rotation_degrees;
  float camera_iris_roundness;
  float camera_anamorphic_squeeze;
} vkptc_scene_view;

/* SdfShape (src/pathtracer/PathTracer.h:232-240). */
typedef enum vkptc_sdf_shape {
  VKPTC_SDF_SPHERE = 0,
  VKPTC_SDF_BOX = 1,
  VKPTC_SDF_ROUNDED_BOX = 2,
  VKPTC_SDF_PLANE = 3,
  VKPTC_SDF_TORUS = 4,
  VKPTC_SDF_CAPSULE = 5
} vkptc_sdf_shape;

/* Binary BVH as ParallelBvhBuilder returns it (src/cpu/ParallelBvhBuilder.h:22-39):
 * per node min3, max3 (f32) then left, right, first_prim, prim_count (i32). */
typedef struct vkptc_bvh_view {
  const uint32_t* nodes;       /* 10 words per node */
  uint32_t node_count;
  const uint32_t* prim_indices;
  uint32_t prim_count;
} vkptc_bvh_view;

/* Mirrors RenderTile (src/pathtracer/PathTracer.h:914-922). */
typedef struct vkptc_tile {
  uint32_t x, y, width, height;
  uint32_t sample_index;
  uint32_t tile_id;
  uint32_t gpu_id;
} vkptc_tile;

/* Mirrors SampleCounters (src/pathtracer/PathTracer.h:218-230); the
 * traversal counters count this backend's wide-BVH work. */
typedef struct vkptc_counters {
  uint64_t samples;
  uint64_t rays;               /* bounce segments, the reference's definition */
  uint64_t triangle_tests;
  uint64_t sdf_tests;
  uint64_t sdf_steps;
  uint64_t triangle_hits;
  uint64_t sdf_hits;
  uint64_t sdf_misses;
  uint64_t bvh_node_visits;
  uint64_t bvh_leaf_visits;
  uint64_t shadow_tests;
} vkptc_counters;

/* Mirrors PathTracerStatus (src/pathtracer/PathTracer.h:854-865). */
typedef struct vkptc_tracer_status {
  uint32_t lifecycle;          /* vkptc_lifecycle */
  uint32_t scene_loaded;
  uint32_t accel_valid;
  uint32_t ready_to_render;
  uint32_t current_sample;
  uint32_t reserved;
  uint64_t last_sample_us;
  uint64_t total_samples;
  uint64_t accumulation_gen;
} vkptc_tracer_status;

typedef struct vkptc_accel_info {
  uint32_t primitive_count;
  uint32_t binary_node_count;
  uint32_t binary_leaf_count;
  uint32_t wide_node_count;
  uint32_t wide_depth;
  uint32_t stack_required;     /* traversal stack entries the BVH can need */
  double build_ms;
  uint64_t device_bytes;       /* BVH + triangle bytes resident in HBM */
} vkptc_accel_info;

#define VKPTC_QUERY_CLOSEST 0u
#define VKPTC_QUERY_ANY 1u

/* ---- lifecycle --------------------------------------------------------------
 * replaces: the IPathTracer object itself (src/pathtracer/PathTracer.h:1069-1184) */
int32_t vkptc_create(const vkptc_config* config, vkptc_ctx** out_ctx);
int32_t vkptc_destroy(vkptc_ctx* ctx);
/* replaces IPathTracer::configure (src/pathtracer/PathTracer.h:1074) */
int32_t vkptc_configure(vkptc_ctx* ctx, const vkptc_render_settings* settings);
/* replaces IPathTracer::load_scene_snapshot (src/pathtracer/PathTracer.h:1088) */
int32_t vkptc_load_scene(vkptc_ctx* ctx, const vkptc_scene_view* scene);
/* replaces IPathTracer::build_or_update_acceleration (src/pathtracer/PathTracer.h:1092):
 * builds the binary midpoint BVH exactly as ParallelBvhBuilder does
 * (deterministic mode), optionally a binned-SAH traversal tree, and flattens
 * the traversal tree into the wide HBM layout -- on the device by default
 * (VKPTC_BUILD_DEVICE), on the host with VKPTC_BUILD_HOST; the arrays are the
 * same either way. */
int32_t vkptc_build_acceleration(vkptc_ctx* ctx);
/* Same, from an externally built binary BVH (the reference's ParallelBvhBuilder
 * output over the accelerator's primitive order, CpuBvhAccelerator.cpp:247-256). */
int32_t vkptc_load_bvh(vkptc_ctx* ctx, const vkptc_bvh_view* bvh);
int32_t vkptc_get_accel_info(vkptc_ctx* ctx, vkptc_accel_info* out);

/* RTInstanceTransformUpdate (src/pathtracer/PathTracer.h:298-306), resolved to an instance index. */
typedef struct vkptc_instance_update {
  uint32_t instance_index;
  uint32_t flags;              /* OR-ed into the instance's flags */
  float translation[3];
  float rotation[4];           /* quaternion xyzw */
  float scale[3];
} vkptc_instance_update;
/* replaces IPathTracer::apply_instance_transform_update (src/pathtracer/PathTracer.h:1123-1135) as the
 * CPU accelerator implements it (src/pathtracer/CpuBvhAccelerator.cpp:265-358, 527-606): every updated
 * instance must be a dynamic-transform instance with local geometry (else VKPTC_UNSUPPORTED, the
 * reference's BlockedNeedsFullStaticAccelRebuild); its primitives are recomputed with the new
 * transform and both trees are refitted with their topology unchanged (no rebuild), on the device.
 * All updates are checked before any is applied.  The film is not reset (vkptc_reset does that). */
int32_t vkptc_update_instance_transforms(vkptc_ctx* ctx, const vkptc_instance_update* updates, uint32_t count);
/* replaces IPathTracer::plan_instance_transform_update (src/pathtracer/PathTracer.h:1115-1122): the
 * same checks and return codes as vkptc_update_instance_transforms, nothing applied. */
int32_t vkptc_check_instance_transforms(vkptc_ctx* ctx, const vkptc_instance_update* updates, uint32_t count);

/* The fields of RTCameraState (src/pathtracer/PathTracer.h:418-437) that the render reads; the
 * exposure fields (f-stop, shutter, ISO, compensation, white balance) only change the film resolve
 * settings, which the caller passes to vkptc_resolve_ldr. */
typedef struct vkptc_camera {
  float position[3];
  float target[3];
  float up[3];
  float fov_deg;
  float aperture_radius;       /* > 0: overrides vkptc_render_settings.camera_aperture_radius */
  float focus_distance;        /* > 0: overrides vkptc_render_settings.camera_focus_distance */
  uint32_t iris_blade_count;
  float iris_rotation_degrees;
  float iris_roundness;
  float anamorphic_squeeze;
} vkptc_camera;
/* replaces IPathTracer::update_camera_state (src/pathtracer/PathTracer.h:1105) as
 * ScalarCpuPathTracer implements it (src/pathtracer/ScalarCpuPathTracer.cpp:535-546, ApplyCameraState,
 * src/pathtracer/PathTracer.cpp:343-362): the camera of the loaded scene is replaced, the next render
 * uses it; no acceleration rebuild, the film is not reset (vkptc_reset does that).  VKPTC_NOT_READY
 * before a scene is loaded. */
int32_t vkptc_update_camera(vkptc_ctx* ctx, const vkptc_camera* camera);
/* The loaded scene's camera (ExtractCameraState, src/pathtracer/PathTracer.cpp:320-341), for a caller
 * that changes only some fields (IPathTracer::update_camera, src/pathtracer/PathTracer.h:1102). */
int32_t vkptc_get_camera(vkptc_ctx* ctx, vkptc_camera* out);

/* RTSceneDeltaUpdate (src/pathtracer/PathTracer.h:439-461) with its instance references resolved to
 * instance indices: replacement material records (16 floats each, the layout of
 * vkptc_scene_view.materials), replacement light records (16 floats each), new material indices of
 * instances, and optionally a new constant environment colour. */
typedef struct vkptc_scene_delta {
  const uint32_t* material_indices;
  const float* materials;
  uint32_t material_count;
  const uint32_t* light_indices;
  const float* lights;
  uint32_t light_count;
  const uint32_t* instance_indices;
  const uint32_t* instance_material_indices;
  uint32_t instance_material_count;
  uint32_t environment_changed;
  float environment[3];
} vkptc_scene_delta;
/* replaces IPathTracer::update_scene_delta (src/pathtracer/PathTracer.h:1141) with
 * ApplySceneDeltaUpdate's rules (src/pathtracer/PathTracer.cpp:427-483): every index is checked
 * before anything is applied (a material or light index past the scene's tables, an instance index
 * past its instances or an instance material past the materials: VKPTC_INVALID_ARGUMENT, nothing
 * changed); records are replaced in order, so the last of two updates of one index wins; a delta that
 * changes nothing (empty, or only instance materials already set) is VKPTC_INVALID_ARGUMENT as the
 * reference's false.  Instance material changes rewrite the material of the instance's primitives in
 * the built accelerator at once (as the GPU backends do, src/gpu/D3D12GpuPathTracer.Scene.cpp:614-624)
 * and are kept for later builds.  No acceleration rebuild; the film is not reset.  A context set up
 * for differentiable rendering must be set up again (vkptc_adjoint_setup) after a delta. */
int32_t vkptc_update_scene_delta(vkptc_ctx* ctx, const vkptc_scene_delta* delta);
/* Extension (no reference counterpart): copies one device array of the built
 * accelerator to host memory, for inspection and for checking the device
 * build against the host build.  what: VKPTC_ACCEL_WIDE_NODES (128 B each),
 * VKPTC_ACCEL_TRIANGLES (48 B each, leaf order), VKPTC_ACCEL_TIE_NODES (32 B
 * each, the reference binary tree), VKPTC_ACCEL_SHADING (16 B per primitive).
 * *bytes receives the array's size; out may be NULL to query it. */
int32_t vkptc_read_accel(vkptc_ctx* ctx, uint32_t what, void* out, uint64_t capacity, uint64_t* bytes);
#define VKPTC_ACCEL_WIDE_NODES 0u
#define VKPTC_ACCEL_TRIANGLES 1u
#define VKPTC_ACCEL_TIE_NODES 2u
#define VKPTC_ACCEL_SHADING 3u
/* Host-only (no device needed): the binary BVH vkptc_build_acceleration
 * builds, in ParallelBvhBuilder's layout, for callers that keep a CPU copy.
 * replaces ParallelBvhBuilder::build (src/cpu/ParallelBvhBuilder.cpp:165-257)
 * as CpuBvhAccelerator::build calls it (deterministic, leaf threshold 4).
 * nodes_out: capacity 2*prims-1 nodes of 10 words; prim_out: capacity prims.
 * *node_count and *prim_count receive the sizes. */
int32_t vkptc_build_binary_bvh(const vkptc_scene_view* scene, uint32_t* nodes_out, uint32_t* node_count,
                               uint32_t* prim_out, uint32_t* prim_count);
/* replaces IPathTracer::reset_accumulation (src/pathtracer/PathTracer.h:1096) */
int32_t vkptc_reset(vkptc_ctx* ctx);
/* replaces IPathTracer::shutdown (src/pathtracer/PathTracer.h:1182) */
int32_t vkptc_shutdown(vkptc_ctx* ctx);

/* ---- rendering --------------------------------------------------------------
 * replaces IPathTracer::render_tile / render_tile_cancellable / render_tiles
 * (src/pathtracer/PathTracer.h:1142-1170).  Each tile renders one sample
 * (tile.sample_index) of frame `frame` for every pixel it covers.  cancel_flag
 * (may be NULL) is polled before each tile; a set flag returns VKPTC_CANCELLED. */
int32_t vkptc_render(vkptc_ctx* ctx, const vkptc_tile* tiles, uint32_t tile_count, uint32_t frame,
                     const volatile int32_t* cancel_flag);
/* Renders samples [first_sample, first_sample + sample_count) of the full
 * frame; the samples are independent, so this is the batched form of
 * sample_count full-frame render_tile calls. */
int32_t vkptc_render_frame(vkptc_ctx* ctx, uint32_t first_sample, uint32_t sample_count, uint32_t frame);
/* Blocks until queued device work is done. */
int32_t vkptc_synchronize(vkptc_ctx* ctx);
/* Enqueues all further work of this context on `stream` (a cudaStream_t of
 * the caller, e.g. its framework's current stream); NULL restores the
 * context's own stream.  No synchronisation is implied. */
int32_t vkptc_set_stream(vkptc_ctx* ctx, void* stream);
/* Per-stage device time (CUDA events around every stage launch; enabled by
 * vkptc_config.reserved[1] = 1).  ms_out[0..4] = raygen, extend (closest-hit
 * traversal), shade, shadow (any-hit traversal), accumulate; launches_out
 * (may be NULL) receives the launch count of each stage.  Reading resets. */
int32_t vkptc_read_stage_times(vkptc_ctx* ctx, double* ms_out, uint64_t* launches_out);

/* ---- film ---------------------------------------------------------------------
 * replaces IPathTracer::film() / FilmBuffer raw access (src/pathtracer/PathTracer.h:937-974):
 * sum_rgb (3*W*H floats), count (W*H), invalid (W*H); any may be NULL. */
int32_t vkptc_read_film(vkptc_ctx* ctx, float* sum_rgb, uint32_t* count, float* invalid);
/* replaces IPathTracer::resolve_hdr / FilmBuffer::resolve_hdr (src/pathtracer/FilmBuffer.cpp:160-214) */
int32_t vkptc_resolve_hdr(vkptc_ctx* ctx, float* rgb);

/* Mirrors FilmResolveSettings (src/pathtracer/PathTracer.h:55-74), with the
 * camera's exposure controls already folded into exposure as
 * CameraAdjustedFilmResolveSettings does (src/pathtracer/FilmBuffer.cpp:226-251). */
typedef struct vkptc_film_resolve {
  float exposure;
  float white_balance_kelvin;  /* 6500: no change */
  uint32_t tone_map;           /* vkptc_tone_map */
  uint32_t output_transform;   /* vkptc_output_transform */
  float gamma;
  uint32_t clamp_output;
} vkptc_film_resolve;
typedef enum vkptc_tone_map {
  VKPTC_TONEMAP_LINEAR = 0,
  VKPTC_TONEMAP_REINHARD = 1,
  VKPTC_TONEMAP_FILMIC = 2,
  VKPTC_TONEMAP_ACES = 3
} vkptc_tone_map;
typedef enum vkptc_output_transform { VKPTC_OUTPUT_GAMMA = 0, VKPTC_OUTPUT_LINEAR = 1 } vkptc_output_transform;
typedef enum vkptc_readback_state {
  VKPTC_READBACK_INVALID = 0,
  VKPTC_READBACK_PENDING = 1,
  VKPTC_READBACK_READY = 2,
  VKPTC_READBACK_FAILED = 3
} vkptc_readback_state;

/* replaces IPathTracer::resolve_ldr, i.e. ApplyFilmResolve(resolve_hdr())
 * (src/pathtracer/FilmBuffer.cpp:253-325), computed on the device: per-pixel
 * mean, exposure, white balance, tone map, gamma, clamp, 8-bit quantization.
 * rgba: 4*W*H bytes (alpha 255). */
int32_t vkptc_resolve_ldr(vkptc_ctx* ctx, const vkptc_film_resolve* settings, uint8_t* rgba);
/* replaces IPathTracer::request_film_readback (src/pathtracer/PathTracer.h:1173): enqueues the
 * LDR resolve of the film as it stands after the work already submitted and a copy to
 * pinned host memory on the context's stream; *token identifies it (the latest only). */
int32_t vkptc_request_ldr_readback(vkptc_ctx* ctx, const vkptc_film_resolve* settings, uint64_t* token);
/* replaces IPathTracer::poll_film (src/pathtracer/PathTracer.h:1174): *state receives a
 * vkptc_readback_state; READY copies the image into rgba (4*W*H bytes). Never blocks. */
int32_t vkptc_poll_ldr_readback(vkptc_ctx* ctx, uint64_t token, uint8_t* rgba, uint32_t* state);
/* replaces IPathTracer::replace_film_history (src/pathtracer/PathTracer.h:1099):
 * loads a saved film (resume = reload the film, continue at the next sample). */
int32_t vkptc_write_film(vkptc_ctx* ctx, const float* sum_rgb, const uint32_t* count, const float* invalid);
/* replaces IPathTracer::read_counters (src/pathtracer/PathTracer.h:1180) */
int32_t vkptc_read_counters(vkptc_ctx* ctx, vkptc_counters* out);
/* This backend's traversal work, split by query kind (needs
 * vkptc_config.collect_stats = 1): extension (closest-hit) rays, wide-node
 * visits, leaf visits, triangle tests, then shadow (any-hit) rays, node
 * visits, leaf visits, triangle tests -- out[8]. */
int32_t vkptc_read_traversal_stats(vkptc_ctx* ctx, uint64_t* out);
/* replaces IPathTracer::status (src/pathtracer/PathTracer.h:1181) */
int32_t vkptc_get_status(vkptc_ctx* ctx, vkptc_tracer_status* out);
/* Last error message of this context (empty when none); valid until the next call. */
const char* vkptc_last_error(vkptc_ctx* ctx);
/* Extension (no reference counterpart): read bandwidth of the context's device, for the
 * roofline of the traversal stages.  Streams `reps` times through a zeroed device buffer of
 * `bytes` (a multiple of 16) with 16-byte loads cached in L2 only, timed with CUDA events on
 * the context's stream after one untimed pass: a buffer well under the L2 size (126 MB on
 * B200) gives the L2 bandwidth, one far above it the HBM read bandwidth.  *gbs receives
 * bytes * reps / time in GB/s.  Allocates (and frees) the buffer itself. */
int32_t vkptc_measure_read_bandwidth(vkptc_ctx* ctx, uint64_t bytes, uint32_t reps, double* gbs);
/* The device a context renders on: its name (cudaDeviceProp::name, NUL-terminated, cut to
 * capacity) for BenchmarkResult.device_info.gpu_name (src/benchmark/BenchmarkSchema.h:80-85),
 * and optionally its SM count. */
int32_t vkptc_device_name(vkptc_ctx* ctx, char* out, uint32_t capacity, uint32_t* sm_count);

/* ---- ray queries --------------------------------------------------------------
 * replaces IRayAccelerator::intersect (src/pathtracer/PathTracer.h:1001-1036), one
 * virtual call per ray there, batched here.  rays: 6 floats per ray (origin,
 * direction), HOST memory.  tmax (may be NULL = +inf) bounds any-hit queries.
 * prim_out: the hit primitive's index in the accelerator's flattened order
 * (RayQueryHit::primitive_index) or 0xFFFFFFFF; t_out (may be NULL): distance.
 * For VKPTC_QUERY_ANY, prim_out[i] is 1 when occluded before tmax, else 0. */
int32_t vkptc_trace_rays(vkptc_ctx* ctx, const float* rays, const float* tmax, uint64_t ray_count,
                         uint32_t mode, uint32_t* prim_out, float* t_out);
/* Same with DEVICE pointers already resident in HBM, enqueued on `stream`
 * (a cudaStream_t; 0 = the context's stream).  No host synchronisation.
 * When `stream` is not the context's stream, it first waits for the work
 * queued on the context's stream and the context's stream then waits for the
 * query (two events made with the context), so a later rebuild or upload on
 * the context cannot overtake it; while either stream is being captured no
 * such events are inserted and the caller orders the call itself. */
int32_t vkptc_trace_rays_device(vkptc_ctx* ctx, const float* d_rays, const float* d_tmax, uint64_t ray_count,
                                uint32_t mode, uint32_t* d_prim_out, float* d_t_out, void* stream);

/* ---- batched rendering ------------------------------------------------------
 * No single reference counterpart: the reference renders jobs one
 * IPathTracer at a time (ptbench `run` per scene).  A batch holds many render
 * jobs (each its own scene, acceleration structure, settings and film) and
 * renders all of them, either one frame per launch per job ("plain") or in
 * one persistent launch fed by a device work queue and replayed from a CUDA
 * graph ("persistent").  Both give bit-identical films. */
typedef struct vkptc_batch vkptc_batch;

#define VKPTC_BATCH_PLAIN 0u
#define VKPTC_BATCH_PERSISTENT 1u
/* The same pool, work queue and stages as VKPTC_BATCH_PERSISTENT, but one
 * kernel per stage (each with its own register budget and occupancy) inside a
 * CUDA graph while-node that the device keeps iterating until the work queue
 * is empty: one graph launch per run, no grid barrier.  Films are identical
 * to the other modes. */
#define VKPTC_BATCH_LOOP 2u

typedef struct vkptc_batch_tuning {
  uint32_t pool_paths;       /* path slots of the persistent launch ("queue capacity"); 0 = default */
  uint32_t block_size;       /* 0 = default */
  uint32_t stack_depth;      /* traversal stack entries in shared memory; 0 = default */
  uint32_t steps;            /* traversal steps between warp refills (low 16 bits; 0 = default) and
                                an optional refill threshold in idle lanes (high 16 bits), as
                                vkptc_config.steps */
  uint32_t sample_limit;     /* render at most this many samples per job (0 = each job's spp) */
  uint32_t use_graph;        /* persistent/loop modes: 1 = capture once, replay the CUDA graph
                                (loop mode without a graph runs one host round trip per iteration) */
  uint32_t occupancy;        /* traversal kernels' register variant: 0..3 = at least 1..4 resident
                                256-thread blocks per SM (fewer registers, more warps); 4 (loop
                                driver; the persistent driver takes it as 3) = at least 7 resident
                                128-thread blocks per SM (72 registers), and the launch's block
                                size becomes 128 */
  uint32_t barrier_spins;    /* persistent mode: bound of a grid-barrier wait in sleeps of ~128 ns
                                (0 = 2^26, about 8.6 s); a block that waits longer aborts the run,
                                every block leaves at its next barrier and vkptc_batch_run returns
                                VKPTC_TIMEOUT with the batch still usable (the next run clears the
                                films and renders them anew) */
} vkptc_batch_tuning;

typedef struct vkptc_batch_stats {
  uint32_t jobs;
  uint32_t graph_used;
  uint64_t paths;            /* camera paths rendered by the last run */
  uint64_t segments;         /* extension segments (finite samples) */
  uint64_t shadow_rays;
  uint64_t kernel_launches;  /* kernels launched by the last run */
  double device_ms;          /* device time of the last run (CUDA events on the batch stream) */
  uint32_t grid;
  uint32_t block;
  uint32_t pool_paths;
  uint32_t stack_depth;
  uint32_t steps;
  uint32_t iterations;       /* pool iterations (stage rounds) of the last persistent/loop run; the loop
                                driver traces a round's NEE queries in the next round, so it runs one
                                round more than the persistent driver */
  /* traversal work (filled when vkptc_config.collect_stats = 1) */
  uint64_t ext_rays, ext_nodes, ext_tris;
  uint64_t shadow_queries, shadow_nodes, shadow_tris;
  /* loop driver without a graph and vkptc_config.stage_timing = 1: device
   * time of each stage summed over the iterations (regen, extend, shade,
   * shadow, finish = the drain of ended paths to the stagings; CUDA events
   * around every stage launch, the stages then run one after the other) */
  double stage_ms[5];
} vkptc_batch_stats;

int32_t vkptc_batch_create(const vkptc_config* config, vkptc_batch** out_batch);
int32_t vkptc_batch_destroy(vkptc_batch* batch);
/* Adds one job: loads the scene and builds its acceleration structure (as
 * configure + load_scene_snapshot + build_or_update_acceleration would). */
int32_t vkptc_batch_add_job(vkptc_batch* batch, const vkptc_scene_view* scene, const vkptc_render_settings* settings,
                            uint32_t* job_id);
/* Clears every film, then renders samples [0, spp) (or sample_limit) of every job. */
int32_t vkptc_batch_run(vkptc_batch* batch, uint32_t mode, const vkptc_batch_tuning* tuning);
int32_t vkptc_batch_read_film(vkptc_batch* batch, uint32_t job_id, float* sum_rgb, uint32_t* count);
/* Every job's film in one go: sums[j] (3*W*H floats) and counts[j] (W*H), either may be NULL per job;
 * the copies are queued back to back and waited for once (pinned destinations copy fastest). */
int32_t vkptc_batch_read_films(vkptc_batch* batch, float* const* sums, uint32_t* const* counts);
int32_t vkptc_batch_get_stats(vkptc_batch* batch, vkptc_batch_stats* out);
const char* vkptc_batch_last_error(vkptc_batch* batch);

/* ---- allocation-free rendering -------------------------------------------
 * No counterpart in the reference: an extra entry point of this library.
 *
 * Renders one sample (tile->sample_index) of one tile without allocating any
 * memory, for callers that cannot call cudaMalloc while they render: an
 * engine whose GPU memory all comes from its own pooled allocator or fixed
 * budget, a render loop recorded under CUDA stream capture (where a
 * cudaMalloc would break the capture), or a real-time thread that must not
 * block in the driver's allocator.  Scene and acceleration structure must
 * already be loaded into ctx (that set-up may allocate); this call then
 * takes its path queues from one fixed, file-scope device array sized for
 * VKPTC_NOALLOC_MAX_PATHS paths (140 bytes per path, about 9.2 MB, held on
 * every GPU that loads the library until the process exits) and adds the
 * sample into the CALLER's device film:
 *   d_film_sum   W*H float4 per pixel (rgb sum; w untouched), 16-byte aligned
 *   d_film_count W*H uint32 sample counts
 * (W, H from vkptc_configure; device memory of the context's device).
 *
 * Limits:
 *  - A tile covering more than VKPTC_NOALLOC_MAX_PATHS pixels is rejected with
 *    VKPTC_INVALID_ARGUMENT and a message naming the limit.
 *  - The whole traversal stack must fit in shared memory (no spill buffer):
 *    the BVH's worst-case stack (vkptc_accel_info.stack_required entries of
 *    8 bytes per thread, times vkptc_config.block_size threads, 128 when 0)
 *    must not exceed the device's opt-in shared memory per block (227 KB on
 *    B200, i.e. 227 entries at 128 threads).  A deeper BVH is refused with
 *    VKPTC_UNSUPPORTED, although vkptc_render succeeds on the same context.
 *
 * Set-up: the array's device address is looked up (cudaGetSymbolAddress)
 * when the context is created, with its device current; this call itself
 * makes no lookup.  A device reset (cudaDeviceReset) invalidates every
 * context and that address with it: create new contexts after a reset.
 *
 * Sharing: every call shares the one array, and it keeps the last call's
 * contents (each call sets what must start at zero).  Calls whose GPU work
 * overlaps (on different streams, or from different contexts on the same
 * device) race on it: the caller must order them, e.g. on one stream.
 *
 * Streams: work is enqueued on `stream` (NULL = the context's stream) and the
 * call returns without synchronising.  When `stream` is not the context's
 * stream, it first waits for the work already queued on the context's stream,
 * and the context's stream then waits for this call's kernels (two events
 * made with the context), so a later rebuild, scene reload or upload on the
 * context cannot free or rewrite what these kernels read.  While either
 * stream is being captured no such events are inserted, and the caller must
 * order this call against the context's other work itself.
 *
 * Errors and counters: argument, lifecycle and launch errors are returned by
 * this call.  The kernels write the context's device error word (a traversal
 * stack overflow, which the stack sizing above rules out) and, with
 * collect_stats, its traversal counters; both are read by the context's next
 * synchronising call (vkptc_synchronize, vkptc_read_counters, ...), and the
 * counters are shared with the context's own renders.  The caller's current
 * device is restored before return. */
#define VKPTC_NOALLOC_MAX_PATHS 65536u
int32_t vkptc_render_tile_noalloc(vkptc_ctx* ctx, const vkptc_tile* tile, uint32_t frame, float* d_film_sum,
                                  uint32_t* d_film_count, void* stream);

/* ---- differentiable rendering (forward / backward pair) -------------------
 * No counterpart in the reference: its tracer has no derivative path.
 *
 * Parameters are VKPTC_ADJ_PARAMS_PER_MATERIAL floats per scene material, in
 * material order: albedo r, g, b, roughness, emission r, g, b.  They replace
 * those words of the loaded materials for the forward and backward only (the
 * context's own renderer keeps the loaded scene).
 *
 * vkptc_forward renders desc->spp samples (from desc->first_sample, RNG frame
 * desc->frame) of every pixel, one path per thread, forms the image exactly
 * as the film does (sample order, non-finite samples dropped) and returns
 * the loss L = mean over pixels and channels of (image - target)^2, reduced
 * in FP64.  rr_params (NULL = params) are the parameters whose throughput
 * sets the Russian-roulette probabilities and decisions: passing the
 * unperturbed vector makes a finite difference use the same roulette as
 * the derivative.  image_rgb (W*H*3, optional) receives the image.
 *
 * vkptc_backward returns dL/dparams for the last forward: every path is
 * replayed from its RNG key and swept in reverse.  The estimator
 * differentiated: Phong-lobe directions are reparameterized (they move with
 * roughness and with the incoming direction), the roulette probability is
 * held constant, and every discrete decision (hits, visibility, lobe
 * fallbacks) is the forward's, so visibility-boundary terms are excluded.
 * Emission gradients are meaningful for emissive materials (and for
 * surfaces seen directly by the camera).
 *
 * Supported: materials of models 0, 1 and 3 with metallic <= 0.65,
 * transmission <= 0.05, clearcoat <= 0.05 and roughness > 0.001 (Lambertian
 * and Phong-lobe glossy, optionally emissive), at most
 * VKPTC_ADJ_MAX_MATERIALS materials, max_depth <= VKPTC_ADJ_MAX_DEPTH;
 * anything else returns VKPTC_UNSUPPORTED.  All three calls are synchronous
 * on the context's stream. */
#define VKPTC_ADJ_PARAMS_PER_MATERIAL 7u
#define VKPTC_ADJ_MAX_MATERIALS 64u
#define VKPTC_ADJ_MAX_DEPTH 8u
/* flags: VKPTC_ADJ_DECORRELATED makes vkptc_backward replay the paths of
 * backward_frame (independent samples of the same pixels) instead of the
 * forward's: the residual and the path derivatives then share no samples, so
 * the gradient is unbiased for the loss of the expected image (with shared
 * samples it also carries their covariance, which pulls low-spp
 * optimisations towards darker, smoother images). */
#define VKPTC_ADJ_DECORRELATED 1u
typedef struct vkptc_adjoint_desc {
  uint32_t spp;
  uint32_t first_sample;
  uint32_t frame;            /* RNG frame of the forward's paths */
  uint32_t backward_frame;   /* RNG frame the backward replays under VKPTC_ADJ_DECORRELATED */
  uint32_t flags;
  uint32_t reserved[3];
} vkptc_adjoint_desc;

typedef struct vkptc_adjoint_stats {
  uint64_t paths;           /* paths per forward (= per backward) */
  uint64_t forwards, backwards;
  double forward_ms;        /* device time of the last forward (render + loss) */
  double backward_ms;       /* device time of the last backward (replay + sweep + reduction) */
  uint32_t forward_grid, backward_grid, block, reserved;
} vkptc_adjoint_stats;

/* target_rgb: W*H*3 floats (NULL: no target; the loss is 0 and so is the gradient). */
int32_t vkptc_adjoint_setup(vkptc_ctx* ctx, const vkptc_adjoint_desc* desc, const float* target_rgb,
                            uint64_t target_floats);
int32_t vkptc_forward(vkptc_ctx* ctx, const float* params, uint32_t param_count, const float* rr_params,
                      double* loss, float* image_rgb);
int32_t vkptc_backward(vkptc_ctx* ctx, float* grad, uint32_t param_count);
/* Changes desc.frame / desc.backward_frame (e.g. fresh samples every
 * optimisation step); the next call must be a vkptc_forward. */
int32_t vkptc_adjoint_set_frames(vkptc_ctx* ctx, uint32_t frame, uint32_t backward_frame);
/* As vkptc_backward with each path's adjoint scaled by path_weight[path]
 * (paths in the order of vkptc_adjoint_read_samples; NULL = all 1). */
int32_t vkptc_backward_weighted(vkptc_ctx* ctx, const float* path_weight, float* grad, uint32_t param_count);
/* Per-path results of the last forward, path = sample_offset * W*H + y*W + x:
 * rgb (paths*3 floats, optional) the radiance; signature (paths, optional) a
 * 32-bit hash of the path's discrete decisions (hit primitives, visibility,
 * lobe fallbacks, termination): equal hashes under two parameter vectors mean
 * the path took the same branches, which finite-difference checks use to
 * leave out paths that crossed a discontinuity. */
int32_t vkptc_adjoint_read_samples(vkptc_ctx* ctx, float* rgb, uint32_t* signature);
int32_t vkptc_adjoint_get_stats(vkptc_ctx* ctx, vkptc_adjoint_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* VKPTC_H */
