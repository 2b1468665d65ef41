// ref_shim.cpp -- TEST INFRASTRUCTURE: drives the reference's own CPU tracer.
//
// Compiled by oracle/Makefile together with the reference's unmodified
// translation units into oracle/_ref/libvkptref.so.  It only converts the POD
// scene of vkpt_oracle.h into the reference's PathTracerSceneSnapshot and calls
// the reference's public classes:
//   ScalarCpuPathTracer   (src/pathtracer/PathTracer.h:1232-1370)
//   TiledCpuPathTracer    (src/cpu/TiledCpuPathTracer.h:47-130)
//   CreateCpuBvhAccelerator / IRayAccelerator::intersect
//                         (src/pathtracer/PathTracer.h:1001-1036,
//                          src/pathtracer/CpuBvhAccelerator.cpp:360-477)
//   ParallelBvhBuilder    (src/cpu/ParallelBvhBuilder.cpp:165-257)
// The product library never links this file.

#include "../oracle/vkpt_oracle.h"
#include "../oracle/worker_pool.h"

#include "core/Logging.h"
#include "cpu/ParallelBvhBuilder.h"
#include "scene/Scene.h"
#include "cpu/TiledCpuPathTracer.h"
#include "pathtracer/PathTracer.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace pt = vkpt::pathtracer;

namespace {

thread_local std::string g_error;

int fail(const std::string& message) {
  g_error = message;
  return 1;
}

void quiet_logs() {
  vkpt::log::Logger::instance().set_min_severity(vkpt::log::Severity::Fatal);
}

pt::Vec3 v3(const float* p) { return pt::Vec3{p[0], p[1], p[2]}; }

pt::PathTracerSceneSnapshot to_snapshot(const vko_scene& s) {
  pt::PathTracerSceneSnapshot out;
  out.vertices.resize(s.vertex_count);
  for (uint32_t i = 0; i < s.vertex_count; ++i) out.vertices[i] = v3(s.vertices + 3 * i);
  out.indices.assign(s.indices, s.indices + s.index_count);
  out.instances.resize(s.instance_count);
  for (uint32_t i = 0; i < s.instance_count; ++i) {
    out.instances[i].entity_id = i + 1u;
    out.instances[i].first_triangle = s.instances[3 * i + 0];
    out.instances[i].triangle_count = s.instances[3 * i + 1];
    out.instances[i].material_index = s.instances[3 * i + 2];
    if (s.instance_local && s.instance_transforms) {
      const uint32_t* l = s.instance_local + 5 * i;
      const float* t = s.instance_transforms + 10 * i;
      pt::RTInstance& r = out.instances[i];
      r.flags = l[0];
      r.local_first_vertex = l[1];
      r.local_vertex_count = l[2];
      r.local_first_index = l[3];
      r.local_index_count = l[4];
      r.translation = pt::Vec3{t[0], t[1], t[2]};
      r.rotation = pt::Quat4{t[3], t[4], t[5], t[6]};
      r.scale = pt::Vec3{t[7], t[8], t[9]};
    }
  }
  if (s.instance_local && s.instance_transforms) {
    out.local_vertices.resize(s.local_vertex_count);
    for (uint32_t i = 0; i < s.local_vertex_count; ++i) out.local_vertices[i] = v3(s.local_vertices + 3 * i);
    out.local_indices.assign(s.local_indices, s.local_indices + s.local_index_count);
  }
  out.materials.resize(s.material_count);
  for (uint32_t i = 0; i < s.material_count; ++i) {
    const float* m = s.materials + 16 * i;
    pt::RTMaterial& r = out.materials[i];
    r.albedo = v3(m + 0);
    r.emissive = v3(m + 3);
    r.roughness = m[6];
    r.material_model = static_cast<uint32_t>(m[7] + 0.5f);
    r.metallic = m[8];
    r.ior = m[9];
    r.transmission = m[10];
    r.clearcoat = m[11];
    r.sheen = m[12];
    r.anisotropy = m[13];
    r.alpha = m[14];
    const uint32_t packed = static_cast<uint32_t>(m[15] + 0.5f);
    r.material_effect = packed & 1023u;
    r.material_flags = (packed & 1024u) ? 1u : 0u;
  }
  out.lights.resize(s.light_count);
  for (uint32_t i = 0; i < s.light_count; ++i) {
    const float* l = s.lights + 16 * i;
    pt::RTHitLight& r = out.lights[i];
    r.position = v3(l + 0);
    r.color = v3(l + 3);
    r.intensity = l[6];
    r.radius = l[7];
    r.direction = v3(l + 8);
    r.spot_inner_cos = l[11];
    r.spot_outer_cos = l[12];
  }
  out.environment_color = v3(s.environment);
  if (s.environment_map && s.environment_map_width && s.environment_map_height) {
    const size_t n = static_cast<size_t>(s.environment_map_width) * s.environment_map_height;
    out.environment_map.resize(n);
    for (size_t i = 0; i < n; ++i) out.environment_map[i] = v3(s.environment_map + 3 * i);
    out.environment_map_width = s.environment_map_width;
    out.environment_map_height = s.environment_map_height;
    out.environment_map_scale = v3(s.environment_map_scale);
  }
  for (uint32_t i = 0; i < s.sdf_count; ++i) {
    const float* q = s.sdf_primitives + 16 * static_cast<size_t>(i);
    pt::RTSdfPrimitive r;
    const bool known = q[0] >= 0.0f && q[0] < 5.5f;
    r.shape = known ? static_cast<pt::SdfShape>(static_cast<uint32_t>(q[0] + 0.5f)) : pt::SdfShape::Unknown;
    r.position = v3(q + 1);
    r.scale = v3(q + 4);
    r.rotation = v3(q + 7);
    r.material_index = q[10] >= 0.0f ? static_cast<uint32_t>(q[10] + 0.5f) : 0u;
    r.radius = q[11];
    r.param_a = q[12];
    r.param_b = q[13];
    out.sdf_primitives.push_back(r);
  }
  out.camera_position = v3(s.camera_position);
  out.camera_target = v3(s.camera_target);
  out.camera_up = v3(s.camera_up);
  out.camera_fov_deg = s.camera_fov_deg;
  out.camera_aperture_radius = s.camera_aperture_radius;
  out.camera_focus_distance = s.camera_focus_distance;
  if (s.camera_lens_set) {
    out.camera_iris_blade_count = s.camera_iris_blade_count;
    out.camera_iris_rotation_degrees = s.camera_iris_rotation_degrees;
    out.camera_iris_roundness = s.camera_iris_roundness;
    out.camera_anamorphic_squeeze = s.camera_anamorphic_squeeze;
  }
  return out;
}

pt::RenderSettings to_settings(const vko_settings& s, uint32_t spp) {
  pt::RenderSettings r;
  r.width = s.width;
  r.height = s.height;
  r.spp = spp;
  r.max_depth = s.max_depth;
  r.seed = s.seed;
  r.enable_nee = s.enable_nee != 0;
  r.enable_mis = s.enable_mis != 0;
  r.deterministic = true;
  r.russian_roulette_start_depth = s.rr_start;
  r.russian_roulette_min_survival = s.rr_min;
  r.russian_roulette_max_survival = s.rr_max;
  return r;
}

void read_film(const pt::FilmBuffer& film, float* sum, uint32_t* count, float* invalid) {
  const auto& raw = film.raw();
  const auto& cnt = film.sample_counts();
  const auto& inv = film.invalid_samples();
  for (std::size_t i = 0; i < raw.size(); ++i) {
    if (sum) {
      sum[3 * i + 0] = raw[i].x;
      sum[3 * i + 1] = raw[i].y;
      sum[3 * i + 2] = raw[i].z;
    }
    if (count) count[i] = cnt[i];
    if (invalid) invalid[i] = inv[i];
  }
}

void add_counters(vko_counters* out, const pt::SampleCounters& c) {
  out->samples += c.samples;
  out->rays += c.rays;
  out->triangle_tests += c.triangle_tests;
  out->triangle_hits += c.triangle_hits;
  out->bvh_node_visits += c.bvh_node_visits;
  out->bvh_leaf_visits += c.bvh_leaf_visits;
  out->shadow_tests += c.shadow_tests;
  out->sdf_tests += c.sdf_tests;
  out->sdf_steps += c.sdf_steps;
  out->sdf_hits += c.sdf_hits;
  out->sdf_misses += c.sdf_misses;
}

double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Full-frame render through one IPathTracer, one render_tile per sample, as
// ptbench's `run` loop does (src/benchmark/BenchmarkRuntime.cpp:682-693).
thread_local std::vector<pt::RTInstanceTransformUpdate> g_updates;

int render_full(pt::IPathTracer& tracer, const vko_settings& st, uint32_t first, uint32_t n,
                float* film_sum, uint32_t* film_count, float* film_invalid, float* per_sample,
                vko_counters* counters) {
  const std::size_t npx = static_cast<std::size_t>(st.width) * st.height;
  std::vector<float> total(per_sample ? 3 * npx : 0, 0.0f);
  std::vector<uint32_t> total_count(per_sample ? npx : 0, 0u);
  std::vector<float> total_invalid(per_sample ? npx : 0, 0.0f);
  double ms = 0.0;
  for (uint32_t k = 0; k < n; ++k) {
    if (per_sample && !tracer.reset_accumulation()) return fail("reset_accumulation failed");
    pt::RenderTile tile;
    tile.width = st.width;
    tile.height = st.height;
    tile.sample_index = first + k;
    const auto t0 = std::chrono::steady_clock::now();
    if (!tracer.render_tile(tile, 0u)) return fail("render_tile failed: " + tracer.status().last_error);
    ms += ms_since(t0);
    // reset_accumulation clears the counters, so per-sample mode sums them here.
    if (counters && per_sample) add_counters(counters, tracer.read_counters());
    if (per_sample) {
      const auto& raw = tracer.film().raw();
      const auto& cnt = tracer.film().sample_counts();
      const auto& inv = tracer.film().invalid_samples();
      float* dst = per_sample + static_cast<std::size_t>(k) * 3 * npx;
      for (std::size_t i = 0; i < npx; ++i) {
        dst[3 * i + 0] = raw[i].x;
        dst[3 * i + 1] = raw[i].y;
        dst[3 * i + 2] = raw[i].z;
        if (cnt[i] != 0u) {
          total[3 * i + 0] = total[3 * i + 0] + raw[i].x;
          total[3 * i + 1] = total[3 * i + 1] + raw[i].y;
          total[3 * i + 2] = total[3 * i + 2] + raw[i].z;
        }
        total_count[i] += cnt[i];
        total_invalid[i] += inv[i];
      }
    }
  }
  if (per_sample) {
    if (film_sum) std::memcpy(film_sum, total.data(), total.size() * sizeof(float));
    if (film_count) std::memcpy(film_count, total_count.data(), total_count.size() * sizeof(uint32_t));
    if (film_invalid) std::memcpy(film_invalid, total_invalid.data(), total_invalid.size() * sizeof(float));
  } else {
    read_film(tracer.film(), film_sum, film_count, film_invalid);
    if (counters) add_counters(counters, tracer.read_counters());
  }
  if (counters) counters->render_ms += ms;
  return 0;
}

}  // namespace

extern "C" {

const char* vko_last_error(void) { return g_error.c_str(); }

int vko_set_instance_updates(const vko_instance_update* updates, uint32_t count) {
  g_updates.clear();
  for (uint32_t i = 0; i < count; ++i) {
    pt::RTInstanceTransformUpdate u;
    u.instance_index = updates[i].instance_index;
    u.flags = updates[i].flags;
    u.translation = pt::Vec3{updates[i].translation[0], updates[i].translation[1], updates[i].translation[2]};
    u.rotation = pt::Quat4{updates[i].rotation[0], updates[i].rotation[1], updates[i].rotation[2], updates[i].rotation[3]};
    u.scale = pt::Vec3{updates[i].scale[0], updates[i].scale[1], updates[i].scale[2]};
    g_updates.push_back(u);
  }
  return 0;
}

int vko_apply_film_resolve(const float* hdr_rgb, uint32_t width, uint32_t height, const vko_resolve* s,
                           uint8_t* rgba) {
  if (!hdr_rgb || !s || !rgba) return fail("null argument");
  pt::FilmHdr hdr;
  hdr.width = width;
  hdr.height = height;
  hdr.rgbf.assign(hdr_rgb, hdr_rgb + 3ull * width * height);
  pt::FilmResolveSettings rs;
  rs.exposure = s->exposure;
  rs.white_balance_kelvin = s->white_balance_kelvin;
  rs.tone_map = static_cast<pt::ToneMapMode>(s->tone_map);
  rs.output_transform = static_cast<pt::OutputTransformMode>(s->output_transform);
  rs.gamma = s->gamma;
  rs.clamp_output = s->clamp_output != 0;
  const pt::FilmLdr ldr = pt::ApplyFilmResolve(hdr, rs);
  if (ldr.rgba8.size() != 4ull * width * height) return fail("resolve size");
  std::memcpy(rgba, ldr.rgba8.data(), ldr.rgba8.size());
  return 0;
}

// Snapshot dump of a converted scene document, little-endian:
//   char[4] "VKSJ", u32 version (2)
//   u32 nv, ni, ninst, nmat, nlight, nsdf, nlv, nli, env_w, env_h
//   f32 vertices[3 nv]; u32 indices[ni]; u32 instances[3 ninst];
//   u32 instance_local[5 ninst]; f32 instance_transforms[10 ninst];
//   f32 materials[16 nmat]; f32 lights[16 nlight]; f32 sdf[16 nsdf];
//   f32 local_vertices[3 nlv]; u32 local_indices[nli];
//   f32 environment[3]; f32 camera[12] (position3, target3, up3, fov, aperture, focus);
//   f32 environment_map_scale[3]; f32 environment_map[3 env_w env_h]
//   u32 camera_iris_blade_count; f32 lens[3] (iris rotation degrees, iris roundness, anamorphic squeeze)
// Record layouts as in vkpt_oracle.h (material and light word maps, SDF records).
int vko_convert_scene_json(const char* path, const char* out_path) {
  quiet_logs();
  if (!path || !out_path) return fail("null path");
  auto doc = vkpt::scene::SceneDocument::load_from_file(path);
  if (!doc) return fail(std::string("scene document failed to load: ") + path);
  std::vector<std::string> issues;
  if (!doc.value().validate(&issues)) return fail("scene document failed validation");
  auto conv = pt::BuildSceneDataFromDocument(doc.value());
  if (!conv) return fail("BuildSceneDataFromDocument failed");
  const pt::PathTracerSceneSnapshot& s = conv.value();
  std::vector<float> f32;
  std::vector<uint32_t> u32;
  FILE* fp = std::fopen(out_path, "wb");
  if (!fp) return fail("cannot open output");
  auto wu = [&](const std::vector<uint32_t>& v) { if (!v.empty()) std::fwrite(v.data(), 4, v.size(), fp); };
  auto wf = [&](const std::vector<float>& v) { if (!v.empty()) std::fwrite(v.data(), 4, v.size(), fp); };
  std::fwrite("VKSJ", 1, 4, fp);
  const uint32_t head[11] = {2u,
                             static_cast<uint32_t>(s.vertices.size()),
                             static_cast<uint32_t>(s.indices.size()),
                             static_cast<uint32_t>(s.instances.size()),
                             static_cast<uint32_t>(s.materials.size()),
                             static_cast<uint32_t>(s.lights.size()),
                             static_cast<uint32_t>(s.sdf_primitives.size()),
                             static_cast<uint32_t>(s.local_vertices.size()),
                             static_cast<uint32_t>(s.local_indices.size()),
                             s.environment_map_width,
                             s.environment_map_height};
  std::fwrite(head, 4, 11, fp);
  f32.clear();
  for (const auto& v : s.vertices) f32.insert(f32.end(), {v.x, v.y, v.z});
  wf(f32);
  wu(s.indices);
  u32.clear();
  for (const auto& i : s.instances) u32.insert(u32.end(), {i.first_triangle, i.triangle_count, i.material_index});
  wu(u32);
  u32.clear();
  for (const auto& i : s.instances)
    u32.insert(u32.end(), {i.flags, i.local_first_vertex, i.local_vertex_count, i.local_first_index, i.local_index_count});
  wu(u32);
  f32.clear();
  for (const auto& i : s.instances)
    f32.insert(f32.end(), {i.translation.x, i.translation.y, i.translation.z, i.rotation.x, i.rotation.y, i.rotation.z,
                           i.rotation.w, i.scale.x, i.scale.y, i.scale.z});
  wf(f32);
  f32.clear();
  for (const auto& m : s.materials) {
    const uint32_t packed = (m.material_effect & 1023u) | ((m.material_flags & 1u) ? 1024u : 0u);
    f32.insert(f32.end(), {m.albedo.x, m.albedo.y, m.albedo.z, m.emissive.x, m.emissive.y, m.emissive.z, m.roughness,
                           static_cast<float>(m.material_model), m.metallic, m.ior, m.transmission, m.clearcoat,
                           m.sheen, m.anisotropy, m.alpha, static_cast<float>(packed)});
  }
  wf(f32);
  f32.clear();
  for (const auto& l : s.lights)
    f32.insert(f32.end(), {l.position.x, l.position.y, l.position.z, l.color.x, l.color.y, l.color.z, l.intensity,
                           l.radius, l.direction.x, l.direction.y, l.direction.z, l.spot_inner_cos, l.spot_outer_cos,
                           0.0f, 0.0f, 0.0f});
  wf(f32);
  f32.clear();
  for (const auto& p : s.sdf_primitives)
    f32.insert(f32.end(), {static_cast<float>(static_cast<uint32_t>(p.shape)), p.position.x, p.position.y, p.position.z,
                           p.scale.x, p.scale.y, p.scale.z, p.rotation.x, p.rotation.y, p.rotation.z,
                           static_cast<float>(p.material_index), p.radius, p.param_a, p.param_b, 0.0f, 0.0f});
  wf(f32);
  f32.clear();
  for (const auto& v : s.local_vertices) f32.insert(f32.end(), {v.x, v.y, v.z});
  wf(f32);
  wu(s.local_indices);
  f32 = {s.environment_color.x, s.environment_color.y, s.environment_color.z};
  wf(f32);
  f32 = {s.camera_position.x, s.camera_position.y, s.camera_position.z, s.camera_target.x, s.camera_target.y,
         s.camera_target.z, s.camera_up.x, s.camera_up.y, s.camera_up.z, s.camera_fov_deg, s.camera_aperture_radius,
         s.camera_focus_distance};
  wf(f32);
  f32 = {s.environment_map_scale.x, s.environment_map_scale.y, s.environment_map_scale.z};
  wf(f32);
  f32.clear();
  const size_t texels = static_cast<size_t>(s.environment_map_width) * s.environment_map_height;
  for (size_t i = 0; i < texels && i < s.environment_map.size(); ++i)
    f32.insert(f32.end(), {s.environment_map[i].x, s.environment_map[i].y, s.environment_map[i].z});
  f32.resize(3 * texels, 0.0f);
  wf(f32);
  wu({s.camera_iris_blade_count});
  f32 = {s.camera_iris_rotation_degrees, s.camera_iris_roundness, s.camera_anamorphic_squeeze};
  wf(f32);
  std::fclose(fp);
  return 0;
}

const char* vko_impl_name(void) { return "reference"; }

int vko_set_triangle_test(uint32_t mode) {
  // The reference traverses with Moller-Trumbore only.
  return mode == 0u ? 0 : fail("the reference has no watertight triangle test");
}

int vko_render(const vko_scene* scene, const vko_settings* settings,
               uint32_t first_sample, uint32_t n_samples, uint32_t threads,
               const uint32_t* pixels, uint32_t pixel_count,
               float* film_sum, uint32_t* film_count, float* film_invalid,
               float* per_sample, vko_counters* counters) {
  quiet_logs();
  if (!scene || !settings) return fail("null scene or settings");
  if (settings->firefly_clamp != 0.0f) return fail("the reference has no firefly clamp");
  if (counters) std::memset(counters, 0, sizeof(*counters));
  const auto snap = to_snapshot(*scene);
  const auto rs = to_settings(*settings, first_sample + n_samples);
  const std::size_t npx = static_cast<std::size_t>(settings->width) * settings->height;

  if (pixels == nullptr || !g_updates.empty()) {
    if (threads <= 1u || !g_updates.empty()) {
      pt::ScalarCpuPathTracer tracer;
      if (!tracer.configure(rs) || !tracer.load_scene_snapshot(snap) ||
          !tracer.build_or_update_acceleration() || !tracer.reset_accumulation()) {
        return fail("scalar tracer setup failed: " + tracer.status().last_error);
      }
      if (!g_updates.empty()) {
        const auto r = tracer.apply_instance_transform_update(g_updates, pt::InstanceTransformUpdateOptions{});
        if (!r.applied()) return fail(std::string("transform update rejected: ") + (r.message ? r.message : ""));
      }
      return render_full(tracer, *settings, first_sample, n_samples, film_sum, film_count,
                         film_invalid, per_sample, counters);
    }
    vkpt::cpu::TiledRenderConfig cfg;
    cfg.tile_height = 16u;
    cfg.worker_count = threads;
    cfg.deterministic = false;
    vkpt::cpu::TiledCpuPathTracer tracer(cfg);
    if (!tracer.configure(rs) || !tracer.load_scene_snapshot(snap) ||
        !tracer.build_or_update_acceleration() || !tracer.reset_accumulation()) {
      return fail("tiled tracer setup failed: " + tracer.status().last_error);
    }
    return render_full(tracer, *settings, first_sample, n_samples, film_sum, film_count,
                       film_invalid, per_sample, counters);
  }

  // Sparse pixel list: render_sample_pixels (src/pathtracer/ScalarCpuPathTracer.Render.cpp:335-381)
  // on `threads` tracers that share one accelerator, as TiledCpuPathTracer's
  // tiles do (src/cpu/TiledCpuPathTracer.cpp:279-323).
  const uint32_t nt = std::max(1u, std::min(threads, std::max(1u, pixel_count)));
  auto accel = pt::CreateCpuBvhAccelerator();
  if (!accel->build(snap, true)) return fail("accelerator build failed");
  std::vector<std::unique_ptr<pt::ScalarCpuPathTracer>> tracers(nt);
  for (auto& tr : tracers) {
    tr = std::make_unique<pt::ScalarCpuPathTracer>();
    if (!tr->configure(rs) || !tr->set_accelerator(accel.get()) || !tr->load_scene_snapshot(snap) ||
        !tr->update_camera(snap.camera_position, snap.camera_target, snap.camera_up, snap.camera_fov_deg) ||
        !tr->reset_accumulation()) {
      return fail("pixel-list tracer setup failed");
    }
  }
  std::vector<std::vector<uint32_t>> lists(nt);
  for (uint32_t i = 0; i < pixel_count; ++i) lists[i % nt].push_back(pixels[i]);
  std::vector<float> total(3 * npx, 0.0f);
  std::vector<uint32_t> total_count(npx, 0u);
  std::vector<float> total_invalid(npx, 0.0f);
  double ms = 0.0;
  for (uint32_t k = 0; k < n_samples; ++k) {
    std::atomic<int> bad{0};
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < nt; ++t) {
      pool.emplace_back([&, t]() {
        if (per_sample) tracers[t]->reset_accumulation();
        if (!lists[t].empty() &&
            !tracers[t]->render_sample_pixels(lists[t].data(), static_cast<uint32_t>(lists[t].size()),
                                              first_sample + k, 0u)) {
          bad.fetch_add(1);
        }
      });
    }
    for (auto& th : pool) th.join();
    ms += ms_since(t0);
    if (bad.load() != 0) return fail("render_sample_pixels failed");
    if (per_sample) {
      float* dst = per_sample + static_cast<std::size_t>(k) * 3 * npx;
      std::fill(dst, dst + 3 * npx, 0.0f);
      for (uint32_t t = 0; t < nt; ++t) {
        const auto& raw = tracers[t]->film().raw();
        const auto& cnt = tracers[t]->film().sample_counts();
        const auto& inv = tracers[t]->film().invalid_samples();
        for (uint32_t p : lists[t]) {
          if (p >= npx) continue;
          dst[3 * p + 0] = raw[p].x;
          dst[3 * p + 1] = raw[p].y;
          dst[3 * p + 2] = raw[p].z;
          if (cnt[p] != 0u) {
            total[3 * p + 0] = total[3 * p + 0] + raw[p].x;
            total[3 * p + 1] = total[3 * p + 1] + raw[p].y;
            total[3 * p + 2] = total[3 * p + 2] + raw[p].z;
          }
          total_count[p] += cnt[p];
          total_invalid[p] += inv[p];
        }
      }
    }
  }
  if (!per_sample) {
    for (uint32_t t = 0; t < nt; ++t) {
      const auto& raw = tracers[t]->film().raw();
      const auto& cnt = tracers[t]->film().sample_counts();
      const auto& inv = tracers[t]->film().invalid_samples();
      for (uint32_t p : lists[t]) {
        if (p >= npx) continue;
        total[3 * p + 0] = raw[p].x;
        total[3 * p + 1] = raw[p].y;
        total[3 * p + 2] = raw[p].z;
        total_count[p] = cnt[p];
        total_invalid[p] = inv[p];
      }
    }
  }
  if (film_sum) std::memcpy(film_sum, total.data(), total.size() * sizeof(float));
  if (film_count) std::memcpy(film_count, total_count.data(), total_count.size() * sizeof(uint32_t));
  if (film_invalid) std::memcpy(film_invalid, total_invalid.data(), total_invalid.size() * sizeof(float));
  if (counters) {
    for (auto& tr : tracers) add_counters(counters, tr->read_counters());
    counters->render_ms = ms;
  }
  return 0;
}

// The batched CPU baseline: render_sample_pixels (src/pathtracer/ScalarCpuPathTracer.Render.cpp:335-381)
// on one tracer per worker and job, all of a job's tracers sharing its
// accelerator as the tiles of TiledCpuPathTracer share theirs
// (src/cpu/TiledCpuPathTracer.cpp:279-323), on a pool created once per call.
// Consecutive jobs are grouped while their tracers' films fit a memory budget;
// a group's chunks form one work queue, so workers move on to the next job
// instead of waiting at the end of each job.
namespace {

struct JobState {
  pt::PathTracerSceneSnapshot snap;
  pt::RenderSettings rs;
  std::unique_ptr<pt::IRayAccelerator> accel;
  std::vector<std::unique_ptr<pt::ScalarCpuPathTracer>> tracers;   // one per worker, created before the run
  uint32_t chunk = 1, chunks = 0;
  std::vector<uint32_t> owner;   // worker that rendered each chunk
  std::vector<float> prev, m2;   // running sums seen and squared sample radiance (film_m2)
};

constexpr double kGroupFilmBytes = 4.0e9;   // film memory of one group's tracers

}  // namespace

int vko_render_jobs(vko_job* jobs, uint32_t job_count, uint32_t threads, double* render_ms) {
  quiet_logs();
  if (!jobs && job_count) return fail("null job list");
  const uint32_t nt = std::max(1u, threads);
  for (uint32_t j = 0; j < job_count; ++j) {
    vko_job& J = jobs[j];
    std::memset(&J.counters, 0, sizeof(J.counters));
    if (!J.scene || !J.settings) return fail("null scene or settings");
    if (J.settings->firefly_clamp != 0.0f) return fail("the reference has no firefly clamp");
    if (J.pixel_count == 0 || J.n_samples == 0) continue;
    if (!J.pixels || !J.film_sum || !J.film_count) return fail("null pixel list or film");
    const std::size_t npx = static_cast<std::size_t>(J.settings->width) * J.settings->height;
    for (uint32_t i = 0; i < J.pixel_count; ++i)
      if (J.pixels[i] >= npx) return fail("pixel index outside the film");
  }
  vko::WorkerPool pool(nt);
  double total_ms = 0.0;
  uint32_t g0 = 0;
  while (g0 < job_count) {
    // ---- set-up of one group of jobs (not timed)
    std::vector<JobState> st;
    std::vector<std::pair<uint32_t, uint32_t>> items;   // (job in group, chunk)
    double bytes = 0.0;
    uint32_t g1 = g0;
    while (g1 < job_count) {
      const vko_job& J = jobs[g1];
      const uint32_t chunk = vko::chunk_pixels(J.pixel_count, nt);
      const uint32_t chunks = J.pixel_count ? (J.pixel_count + chunk - 1) / chunk : 0u;
      const uint32_t nw = std::min(nt, chunks);
      const double b = 32.0 * nw * static_cast<double>(J.settings->width) * J.settings->height;
      if (g1 > g0 && bytes + b > kGroupFilmBytes) break;
      bytes += b;
      JobState s;
      s.chunk = chunk;
      s.chunks = (J.n_samples == 0) ? 0u : chunks;
      if (s.chunks) {
        s.snap = to_snapshot(*J.scene);
        s.rs = to_settings(*J.settings, J.first_sample + J.n_samples);
        s.accel = pt::CreateCpuBvhAccelerator();
        if (!s.accel->build(s.snap, true)) return fail("accelerator build failed");
        s.tracers.resize(nw);
        for (auto& tr : s.tracers) {
          tr = std::make_unique<pt::ScalarCpuPathTracer>();
          if (!tr->configure(s.rs) || !tr->set_accelerator(s.accel.get()) || !tr->load_scene_snapshot(s.snap) ||
              !tr->update_camera(s.snap.camera_position, s.snap.camera_target, s.snap.camera_up,
                                 s.snap.camera_fov_deg) ||
              !tr->reset_accumulation()) {
            return fail("batched-render tracer setup failed");
          }
        }
        s.owner.assign(s.chunks, 0u);
        if (J.film_m2) {
          s.prev.assign(3u * J.pixel_count, 0.0f);
          s.m2.assign(3u * J.pixel_count, 0.0f);
        }
        for (uint32_t c = 0; c < s.chunks; ++c) items.emplace_back(g1 - g0, c);
      }
      st.push_back(std::move(s));
      ++g1;
    }
    // ---- the group's render phase (timed): one work queue over its chunks.
    // A worker renders chunks with its own tracer of the chunk's job; a job
    // has fewer tracers than workers only when it has fewer chunks, and then
    // worker w uses tracer w % count (one chunk per tracer at a time is
    // ensured by the per-tracer lock).
    std::vector<std::unique_ptr<std::mutex>> locks;
    std::vector<uint32_t> lock_base(st.size(), 0u);
    for (size_t k = 0; k < st.size(); ++k) {
      lock_base[k] = static_cast<uint32_t>(locks.size());
      for (size_t t = 0; t < st[k].tracers.size(); ++t) locks.push_back(std::make_unique<std::mutex>());
    }
    std::atomic<size_t> next{0};
    std::atomic<int> bad{0};
    const double ms = pool.run([&](uint32_t w) {
      for (;;) {
        const size_t it = next.fetch_add(1);
        if (it >= items.size()) return;
        const uint32_t k = items[it].first, c = items[it].second;
        JobState& s = st[k];
        const vko_job& J = jobs[g0 + k];
        const uint32_t ti = w % static_cast<uint32_t>(s.tracers.size());
        std::lock_guard<std::mutex> lk(*locks[lock_base[k] + ti]);
        pt::ScalarCpuPathTracer& tr = *s.tracers[ti];
        s.owner[c] = ti;
        const uint32_t b = c * s.chunk, e = std::min(J.pixel_count, b + s.chunk);
        for (uint32_t q = 0; q < J.n_samples; ++q) {
          if (!tr.render_sample_pixels(J.pixels + b, e - b, J.first_sample + q, 0u)) {
            bad.fetch_add(1);
            return;
          }
          if (J.film_m2) {
            // A sample's radiance is the change of the pixel's running sum.
            const auto& raw = tr.film().raw();
            for (uint32_t i = b; i < e; ++i) {
              const auto& v = raw[J.pixels[i]];
              const float cur[3] = {v.x, v.y, v.z};
              for (int ch = 0; ch < 3; ++ch) {
                const float x = cur[ch] - s.prev[3 * i + ch];
                s.m2[3 * i + ch] += x * x;
                s.prev[3 * i + ch] = cur[ch];
              }
            }
          }
        }
      }
    });
    if (bad.load() != 0) return fail("render_sample_pixels failed");
    total_ms += ms;
    // ---- results of the group
    for (size_t k = 0; k < st.size(); ++k) {
      JobState& s = st[k];
      vko_job& J = jobs[g0 + k];
      for (uint32_t c = 0; c < s.chunks; ++c) {
        const auto& film = s.tracers[s.owner[c]]->film();
        const auto& raw = film.raw();
        const auto& cnt = film.sample_counts();
        const uint32_t b = c * s.chunk, e = std::min(J.pixel_count, b + s.chunk);
        for (uint32_t i = b; i < e; ++i) {
          const uint32_t p = J.pixels[i];
          J.film_sum[3 * i + 0] = raw[p].x;
          J.film_sum[3 * i + 1] = raw[p].y;
          J.film_sum[3 * i + 2] = raw[p].z;
          J.film_count[i] = cnt[p];
        }
      }
      if (J.film_m2 && s.chunks) std::memcpy(J.film_m2, s.m2.data(), s.m2.size() * sizeof(float));
      for (auto& tr : s.tracers) add_counters(&J.counters, tr->read_counters());
      J.counters.render_ms = ms;   // the render phase of the job's group
    }
    g0 = g1;
  }
  if (render_ms) *render_ms = total_ms;
  return 0;
}

int vko_build_bvh(const vko_scene* scene, uint32_t leaf_threshold, int deterministic,
                  uint32_t* nodes_out, uint32_t* node_count, uint32_t* prim_indices_out) {
  quiet_logs();
  if (!scene || !nodes_out || !node_count || !prim_indices_out) return fail("null argument");
  // Primitive AABBs in the accelerator's flattening order, padded by 1e-4
  // (src/pathtracer/CpuBvhAccelerator.cpp:84-95, 173-247).
  const float eps = 1e-4f;
  std::vector<vkpt::cpu::BvhAabb> boxes;
  for (uint32_t inst = 0; inst < scene->instance_count; ++inst) {
    const uint32_t first = scene->instances[3 * inst + 0];
    const uint32_t count = scene->instances[3 * inst + 1];
    for (uint32_t k = 0; k < count; ++k) {
      const uint32_t base = (first + k) * 3u;
      if (base + 2u >= scene->index_count) continue;
      const uint32_t i0 = scene->indices[base], i1 = scene->indices[base + 1], i2 = scene->indices[base + 2];
      if (i0 >= scene->vertex_count || i1 >= scene->vertex_count || i2 >= scene->vertex_count) continue;
      const float* a = scene->vertices + 3 * i0;
      const float* b = scene->vertices + 3 * i1;
      const float* c = scene->vertices + 3 * i2;
      vkpt::cpu::BvhAabb box;
      for (int ax = 0; ax < 3; ++ax) {
        box.min[ax] = std::min({a[ax], b[ax], c[ax]}) - eps;
        box.max[ax] = std::max({a[ax], b[ax], c[ax]}) + eps;
      }
      boxes.push_back(box);
    }
  }
  vkpt::cpu::ParallelBvhBuilder builder;
  const auto result = builder.build(boxes, nullptr, deterministic != 0, leaf_threshold);
  *node_count = static_cast<uint32_t>(result.nodes.size());
  for (std::size_t i = 0; i < result.nodes.size(); ++i) {
    const auto& n = result.nodes[i];
    uint32_t* w = nodes_out + 10 * i;
    std::memcpy(w + 0, n.aabb.min, 12);
    std::memcpy(w + 3, n.aabb.max, 12);
    std::memcpy(w + 6, &n.left_child, 4);
    std::memcpy(w + 7, &n.right_child, 4);
    std::memcpy(w + 8, &n.first_prim, 4);
    std::memcpy(w + 9, &n.prim_count, 4);
  }
  std::copy(result.prim_indices.begin(), result.prim_indices.end(), prim_indices_out);
  return 0;
}

int vko_intersect(const vko_scene* scene, const float* rays, uint64_t ray_count,
                  uint32_t threads, uint32_t* prim_out, float* t_out,
                  uint64_t* stats, double* elapsed_ms) {
  quiet_logs();
  if (!scene || !rays || !prim_out || !t_out) return fail("null argument");
  const auto snap = to_snapshot(*scene);
  auto accel = pt::CreateCpuBvhAccelerator();
  if (!accel->build(snap, true)) return fail("accelerator build failed");
  const uint32_t nt = std::max(1u, threads);
  std::vector<pt::RayQueryStats> per(nt);
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < nt; ++t) {
    pool.emplace_back([&, t]() {
      const uint64_t begin = ray_count * t / nt;
      const uint64_t end = ray_count * (t + 1) / nt;
      for (uint64_t i = begin; i < end; ++i) {
        pt::Ray ray{v3(rays + 6 * i), v3(rays + 6 * i + 3)};
        pt::RayQueryHit hit;
        if (accel->intersect(ray, hit, stats ? &per[t] : nullptr) && hit.hit) {
          prim_out[i] = hit.primitive_index;
          t_out[i] = hit.t;
        } else {
          prim_out[i] = 0xFFFFFFFFu;
          t_out[i] = std::numeric_limits<float>::infinity();
        }
      }
    });
  }
  for (auto& th : pool) th.join();
  if (elapsed_ms) *elapsed_ms = ms_since(t0);
  if (stats) {
    std::memset(stats, 0, 4 * sizeof(uint64_t));
    for (const auto& s : per) {
      stats[0] += s.triangle_tests;
      stats[1] += s.triangle_hits;
      stats[2] += s.bvh_node_visits;
      stats[3] += s.bvh_leaf_visits;
    }
  }
  return 0;
}

}  // extern "C"
