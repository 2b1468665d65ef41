/*
 * vkpt_oracle.h -- C API shared by the two CPU oracles of the render hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library (vkpathtracer_b200)
 * includes, links or calls this; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py use it, as the checker.
 *
 * Two implementations export exactly these symbols:
 *   oracle/ref_shim.cpp   -> oracle/_ref/libvkptref.so
 *       drives the reference's own, unmodified CPU code (ScalarCpuPathTracer,
 *       TiledCpuPathTracer, CpuBvhAccelerator, ParallelBvhBuilder) compiled
 *       from its sources by oracle/Makefile.  Exists only where the reference
 *       sources were present at build time.
 *   oracle/port.cpp       -> oracle/_build/libvkptport.so
 *       a line-by-line CPU restatement of the same algorithms, pinned
 *       bit-for-bit against libvkptref.so (tests/test_oracle_pin.py).  It
 *       travels everywhere and is the checker where the reference is absent.
 *
 * Scene records use the reference's standard GPU word maps
 * (src/gpu/VulkanGpuPathTracer.cpp:323-338 materials, :381-396 lights):
 *   material[16] = albedo3, emissive3, roughness, model, metallic, ior,
 *                  transmission, clearcoat, sheen, anisotropy, alpha,
 *                  effect | (double_sided << 10)
 *   light[16]    = position3, color3, intensity, radius, direction3,
 *                  spot_inner_cos, spot_outer_cos, 0, 0, 0
 */
#ifndef VKPT_ORACLE_H
#define VKPT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct vko_scene {
  const float* vertices;       /* 3 floats per vertex */
  uint32_t vertex_count;
  const uint32_t* indices;     /* 3 per triangle */
  uint32_t index_count;
  const uint32_t* instances;   /* 3 per instance: first_triangle, triangle_count, material_index */
  uint32_t instance_count;
  const float* materials;      /* 16 floats per material */
  uint32_t material_count;
  const float* lights;         /* 16 floats per light */
  uint32_t light_count;
  float environment[3];
  float camera_position[3];
  float camera_target[3];
  float camera_up[3];
  float camera_fov_deg;
  float camera_aperture_radius;
  float camera_focus_distance;
  const float* environment_map;      /* optional: width*height rgb texels (NULL = constant environment) */
  uint32_t environment_map_width;
  uint32_t environment_map_height;
  float environment_map_scale[3];
  /* optional SDF primitives, 16 floats each: shape (0 sphere, 1 box,
   * 2 rounded box, 3 plane, 4 torus, 5 capsule; others never hit), position3,
   * scale3, rotation3 (Euler radians), material index, radius, param_a,
   * param_b, 0, 0 (RTSdfPrimitive, src/pathtracer/PathTracer.h:330-339) */
  const float* sdf_primitives;
  uint32_t sdf_count;
  /* optional dynamic-transform instances (RTInstance): 5 words per instance
   * (flags, local_first_vertex, local_vertex_count, local_first_index,
   * local_index_count), 10 floats per instance (translation3, quaternion xyzw,
   * scale3), and the local vertex / index arrays; NULL: none */
  const uint32_t* instance_local;
  const float* instance_transforms;
  const float* local_vertices;
  uint32_t local_vertex_count;
  const uint32_t* local_indices;
  uint32_t local_index_count;
  /* lens shape (camera_iris_blade_count, camera_iris_rotation_degrees,
   * camera_iris_roundness, camera_anamorphic_squeeze,
   * src/pathtracer/PathTracer.h:405-408); camera_lens_set = 0: the defaults
   * (0 blades, rotation 0, roundness 1, squeeze 1) */
  uint32_t camera_lens_set;
  uint32_t camera_iris_blade_count;
  float camera_iris_rotation_degrees;
  float camera_iris_roundness;
  float camera_anamorphic_squeeze;
} vko_scene;

typedef struct vko_settings {
  uint32_t width;
  uint32_t height;
  uint32_t max_depth;
  uint32_t enable_nee;
  uint32_t enable_mis;
  uint32_t rr_start;
  float rr_min;
  float rr_max;
  uint64_t seed;
  /* Extension (absent from the reference): clamp each channel of the
   * per-sample radiance to this value before accumulation; 0 disables.
   * The reference shim rejects a non-zero value. */
  float firefly_clamp;
  uint32_t _pad;
} vko_settings;

typedef struct vko_counters {
  uint64_t samples;
  uint64_t rays;            /* bounce segments (the reference's counters.rays) */
  uint64_t triangle_tests;
  uint64_t triangle_hits;
  uint64_t bvh_node_visits;
  uint64_t bvh_leaf_visits;
  uint64_t shadow_tests;
  double render_ms;         /* wall time of the sample loop only */
  uint64_t sdf_tests;
  uint64_t sdf_steps;
  uint64_t sdf_hits;
  uint64_t sdf_misses;
} vko_counters;

/* Renders samples [first_sample, first_sample + n_samples) of frame 0.
 * pixels == NULL renders the full frame through render_tile; otherwise the
 * listed pixel indices (y*W+x) through render_sample_pixels.
 * threads <= 1: one deterministic ScalarCpuPathTracer.  threads > 1: the
 * full frame goes through TiledCpuPathTracer (16-row bands), a pixel list is
 * split over `threads` tracers sharing one accelerator; both are bit-identical
 * to the single-thread render.
 * film_sum (3*W*H), film_count (W*H), film_invalid (W*H) receive the film.
 * per_sample (optional, n_samples*3*W*H) receives each sample's radiance.
 * Returns 0 on success, non-zero on failure (message via vko_last_error). */
int vko_render(const vko_scene* scene, const vko_settings* settings,
               uint32_t first_sample, uint32_t n_samples, uint32_t threads,
               const uint32_t* pixels, uint32_t pixel_count,
               float* film_sum, uint32_t* film_count, float* film_invalid,
               float* per_sample, vko_counters* counters);

/* One job of vko_render_jobs: a scene, its settings and the pixels (y*W+x)
 * to render, every sample [first_sample, first_sample + n_samples) of each.
 * Outputs per listed pixel, in list order: film_sum (3 floats, the film's
 * rgb sum), film_count (samples added), film_m2 (3 floats, optional: the sum
 * of each sample's squared radiance, for a per-pixel variance).  counters
 * receives the job's SampleCounters; counters.render_ms its render phase. */
typedef struct vko_job {
  const vko_scene* scene;
  const vko_settings* settings;
  const uint32_t* pixels;
  uint32_t pixel_count;
  uint32_t first_sample;
  uint32_t n_samples;
  uint32_t reserved;
  float* film_sum;
  uint32_t* film_count;
  float* film_m2;
  vko_counters counters;
} vko_job;

/* Renders many jobs on `threads` workers (the CPU baseline of the batched
 * workload).  Jobs run one after the other; each job's accelerator and its
 * per-worker tracers are set up first (not timed, as ptbench times only the
 * render loop), then the workers, created once per call, pull chunks of the
 * job's pixel list from a shared counter and render all samples of a chunk
 * in sample order, so every pixel's film equals the full-frame render's.
 * *render_ms: summed wall time of the jobs' render phases.  Pixel lists
 * must not repeat a pixel. */
int vko_render_jobs(vko_job* jobs, uint32_t job_count, uint32_t threads, double* render_ms);

/* Binary BVH exactly as the accelerator builds it: triangle AABBs padded by
 * 1e-4, midpoint split, stable partition when deterministic != 0.
 * nodes_out: 10 x 32-bit words per node (min3 f32, max3 f32, left, right,
 * first_prim, prim_count as i32); capacity 2*n-1 nodes.
 * prim_indices_out: n entries.  *node_count receives the node count. */
int vko_build_bvh(const vko_scene* scene, uint32_t leaf_threshold, int deterministic,
                  uint32_t* nodes_out, uint32_t* node_count, uint32_t* prim_indices_out);

/* Closest-hit queries through the accelerator.  rays: 6 floats (o3, d3).
 * prim_out: primitive index (flattened triangle order) or 0xFFFFFFFF;
 * t_out: hit distance or +inf.  stats (optional): 4 x uint64 sums of
 * triangle_tests, triangle_hits, bvh_node_visits, bvh_leaf_visits. */
int vko_intersect(const vko_scene* scene, const float* rays, uint64_t ray_count,
                  uint32_t threads, uint32_t* prim_out, float* t_out,
                  uint64_t* stats, double* elapsed_ms);

/* RTInstanceTransformUpdate (src/pathtracer/PathTracer.h:298-306) by instance index. */
typedef struct vko_instance_update {
  uint32_t instance_index;
  uint32_t flags;
  float translation[3];
  float rotation[4];   /* quaternion xyzw */
  float scale[3];
} vko_instance_update;

/* Instance transform updates (IPathTracer::apply_instance_transform_update)
 * applied by the calling thread's next vko_render calls after the
 * accelerator is built and before rendering; count 0 clears them.  A render
 * with updates is a full-frame render on one tracer (threads, pixel lists
 * ignored).  The render fails when the reference rejects the updates. */
int vko_set_instance_updates(const vko_instance_update* updates, uint32_t count);

/* FilmResolveSettings (src/pathtracer/PathTracer.h:55-74). */
typedef struct vko_resolve {
  float exposure;
  float white_balance_kelvin;
  uint32_t tone_map;          /* 0 linear, 1 reinhard, 2 filmic approx, 3 aces approx */
  uint32_t output_transform;  /* 0 gamma, 1 linear */
  float gamma;
  uint32_t clamp_output;
} vko_resolve;

/* ApplyFilmResolve (src/pathtracer/FilmBuffer.cpp:253-325) of an HDR film
 * (3*W*H floats) into rgba (4*W*H bytes). */
int vko_apply_film_resolve(const float* hdr_rgb, uint32_t width, uint32_t height, const vko_resolve* settings,
                           uint8_t* rgba);

/* Reference only (oracle/_ref): loads a scene document (SceneDocument::
 * load_from_file, validate) and converts it with BuildSceneDataFromDocument
 * (src/pathtracer/SceneConversion.cpp), then writes the snapshot's arrays to
 * out_path in the little-endian layout documented in ref_shim.cpp.  Returns
 * 0 on success. */
int vko_convert_scene_json(const char* path, const char* out_path);

/* Triangle test of later intersect and render calls: 0 = the reference's
 * Moller-Trumbore (default), 1 = watertight (Woop, Benthin and Wald, JCGT
 * 2013; an extension: the reference oracle accepts 0 only). */
int vko_set_triangle_test(uint32_t mode);

const char* vko_last_error(void);
const char* vko_impl_name(void);

#ifdef __cplusplus
}
#endif

#endif /* VKPT_ORACLE_H */
