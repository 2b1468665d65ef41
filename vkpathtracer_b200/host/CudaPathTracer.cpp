// CudaPathTracer.cpp -- IPathTracer over libvkpt_cuda (see CudaPathTracer.h).
#include "CudaPathTracer.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pathtracer/PathTracerObservability.h"
#include "vkptc.h"

namespace vkpt::gpu::cuda {

namespace pt = vkpt::pathtracer;
namespace obs = vkpt::pathtracer::observability;
using vkpt::core::Status;
using vkpt::core::StatusCode;

namespace {

constexpr const char* kBackend = "cuda-wavefront";

// Standard GPU word maps (src/gpu/VulkanGpuPathTracer.cpp:323-338, 381-396).
void material_words(const pt::RTMaterial& m, float* w) {
  w[0] = m.albedo.x; w[1] = m.albedo.y; w[2] = m.albedo.z;
  w[3] = m.emissive.x; w[4] = m.emissive.y; w[5] = m.emissive.z;
  w[6] = m.roughness;
  w[7] = static_cast<float>(m.material_model);
  w[8] = m.metallic; w[9] = m.ior; w[10] = m.transmission; w[11] = m.clearcoat;
  w[12] = m.sheen; w[13] = m.anisotropy; w[14] = m.alpha;
  w[15] = static_cast<float>((m.material_effect & 1023u) | ((m.material_flags & 1u) ? 1024u : 0u));
}

void light_words(const pt::RTHitLight& l, float* w) {
  w[0] = l.position.x; w[1] = l.position.y; w[2] = l.position.z;
  w[3] = l.color.x; w[4] = l.color.y; w[5] = l.color.z;
  w[6] = l.intensity; w[7] = std::max(0.0f, l.radius);
  w[8] = l.direction.x; w[9] = l.direction.y; w[10] = l.direction.z;
  w[11] = l.spot_inner_cos; w[12] = l.spot_outer_cos;
}

// The instance an update names: its index, else the instance with its entity
// id (ApplySceneDeltaUpdate / resolve_instance_index); entities.size() when none.
uint32_t resolve_instance(uint32_t index, vkpt::core::StableId entity,
                          const std::vector<vkpt::core::StableId>& entities) {
  if (index >= entities.size() && entity != 0u) {
    for (size_t i = 0; i < entities.size(); ++i)
      if (entities[i] == entity) return static_cast<uint32_t>(i);
  }
  return index < entities.size() ? index : static_cast<uint32_t>(entities.size());
}

}  // namespace

CudaPathTracer::CudaPathTracer(CudaPathTracerConfig config) {
  if (vkptc_abi_version() != VKPTC_ABI_VERSION) {
    m_last_error = "libvkpt_cuda was built with another VKPTC_ABI_VERSION";
    return;
  }
  vkptc_config c{};
  c.device = config.device;
  c.block_size = config.block_size;
  c.math_mode = config.math_mode;
  c.collect_stats = config.collect_stats ? 1u : 0u;
  const int32_t rc = vkptc_create(&c, &m_ctx);
  if (rc != VKPTC_OK) {
    m_ctx = nullptr;
    m_last_error = rc == VKPTC_UNSUPPORTED ? "no CUDA device available for the cuda backend"
                                           : "vkptc_create failed";
  }
}

CudaPathTracer::~CudaPathTracer() {
  if (m_ctx) vkptc_destroy(m_ctx);
}

uint64_t CudaPathTracer::accumulation_gen() const {
  vkptc_tracer_status s{};
  return m_ctx && vkptc_get_status(m_ctx, &s) == VKPTC_OK ? s.accumulation_gen : 0u;
}

bool CudaPathTracer::accel_valid() const {
  vkptc_tracer_status s{};
  return m_ctx && vkptc_get_status(m_ctx, &s) == VKPTC_OK && s.accel_valid != 0u;
}

bool CudaPathTracer::fail(const std::string& message) const {
  m_last_error = message;
  return false;
}

Status CudaPathTracer::status_from(int32_t code, const char* operation) const {
  if (code == VKPTC_OK) {
    m_last_error.clear();
    return Status::ok(std::string(operation) + " succeeded");
  }
  m_last_error = m_ctx ? vkptc_last_error(m_ctx) : m_last_error;
  if (m_last_error.empty()) m_last_error = std::string(operation) + " failed";
  return Status::error(static_cast<StatusCode>(code), m_last_error);
}

Status CudaPathTracer::configure(const pt::RenderSettings& settings) {
  if (!m_ctx) return Status::error(StatusCode::Unsupported, m_last_error);
  vkptc_render_settings s{};
  s.width = settings.width;
  s.height = settings.height;
  s.spp = settings.spp;
  s.max_depth = settings.max_depth;
  s.seed = settings.seed;
  s.enable_nee = settings.enable_nee ? 1u : 0u;
  s.enable_mis = settings.enable_mis ? 1u : 0u;
  s.deterministic = settings.deterministic ? 1u : 0u;
  s.rr_start_depth = settings.russian_roulette_start_depth;
  s.rr_min_survival = settings.russian_roulette_min_survival;
  s.rr_max_survival = settings.russian_roulette_max_survival;
  s.camera_aperture_radius = settings.camera_aperture_radius;
  s.camera_focus_distance = settings.camera_focus_distance;
  const Status st = status_from(vkptc_configure(m_ctx, &s), "configure");
  m_has_scene = false;
  if (st) {
    m_settings = settings;
    m_resolve = settings.film_resolve;
    m_film = pt::FilmBuffer{settings.width, settings.height};
    m_film.set_resolve_settings(m_resolve);
    obs::EmitPathTracerConfig(kBackend, settings.width, settings.height, settings.spp, settings.deterministic);
  }
  return st;
}

Status CudaPathTracer::load_scene_snapshot(const pt::PathTracerSceneSnapshot& scene) {
  if (!m_ctx) return Status::error(StatusCode::Unsupported, m_last_error);
  std::vector<float> mats(16 * scene.materials.size(), 0.0f);
  for (size_t i = 0; i < scene.materials.size(); ++i) material_words(scene.materials[i], &mats[16 * i]);
  std::vector<float> lights(16 * scene.lights.size(), 0.0f);
  for (size_t i = 0; i < scene.lights.size(); ++i) light_words(scene.lights[i], &lights[16 * i]);
  std::vector<uint32_t> inst(3 * scene.instances.size());
  std::vector<uint32_t> inst_local(5 * scene.instances.size());
  std::vector<float> inst_tr(10 * scene.instances.size());
  bool dynamic = false;
  for (size_t i = 0; i < scene.instances.size(); ++i) {
    const pt::RTInstance& r = scene.instances[i];
    inst[3 * i + 0] = r.first_triangle;
    inst[3 * i + 1] = r.triangle_count;
    inst[3 * i + 2] = r.material_index;
    // dynamic-transform instances: local geometry and transform (RTInstance field order)
    const uint32_t l[5] = {r.flags, r.local_first_vertex, r.local_vertex_count, r.local_first_index,
                           r.local_index_count};
    const float t[10] = {r.translation.x, r.translation.y, r.translation.z, r.rotation.x, r.rotation.y,
                         r.rotation.z, r.rotation.w, r.scale.x, r.scale.y, r.scale.z};
    std::copy(l, l + 5, inst_local.begin() + 5 * i);
    std::copy(t, t + 10, inst_tr.begin() + 10 * i);
    dynamic = dynamic || r.has_flag(pt::kRTInstanceFlagDynamicTransform);
  }
  vkptc_scene_view v{};
  v.vertices = reinterpret_cast<const float*>(scene.vertices.data());   // Vec3 is three packed floats
  v.vertex_count = static_cast<uint32_t>(scene.vertices.size());
  v.indices = scene.indices.data();
  v.index_count = static_cast<uint32_t>(scene.indices.size());
  v.instances = inst.data();
  v.instance_count = static_cast<uint32_t>(scene.instances.size());
  v.materials = mats.data();
  v.material_count = static_cast<uint32_t>(scene.materials.size());
  v.lights = lights.empty() ? nullptr : lights.data();
  v.light_count = static_cast<uint32_t>(scene.lights.size());
  v.environment[0] = scene.environment_color.x;
  v.environment[1] = scene.environment_color.y;
  v.environment[2] = scene.environment_color.z;
  const pt::Vec3 cam[3] = {scene.camera_position, scene.camera_target, scene.camera_up};
  float* dst[3] = {v.camera_position, v.camera_target, v.camera_up};
  for (int k = 0; k < 3; ++k) {
    dst[k][0] = cam[k].x;
    dst[k][1] = cam[k].y;
    dst[k][2] = cam[k].z;
  }
  v.camera_fov_deg = scene.camera_fov_deg;
  v.camera_aperture_radius = scene.camera_aperture_radius;
  v.camera_focus_distance = scene.camera_focus_distance;
  v.camera_lens_set = 1u;
  v.camera_iris_blade_count = scene.camera_iris_blade_count;
  v.camera_iris_rotation_degrees = scene.camera_iris_rotation_degrees;
  v.camera_iris_roundness = scene.camera_iris_roundness;
  v.camera_anamorphic_squeeze = scene.camera_anamorphic_squeeze;
  // The reference samples the map only when it holds width*height texels.
  const size_t env_texels = static_cast<size_t>(scene.environment_map_width) * scene.environment_map_height;
  if (env_texels > 0 && scene.environment_map.size() >= env_texels) {
    v.environment_map = reinterpret_cast<const float*>(scene.environment_map.data());   // packed Vec3
    v.environment_map_width = scene.environment_map_width;
    v.environment_map_height = scene.environment_map_height;
    v.environment_map_scale[0] = scene.environment_map_scale.x;
    v.environment_map_scale[1] = scene.environment_map_scale.y;
    v.environment_map_scale[2] = scene.environment_map_scale.z;
  }
  // SDF primitives: 16-float records (RTSdfPrimitive field order); a shape
  // outside the known six (SdfShape::Unknown) never hits, as in the reference.
  std::vector<float> sdf(16 * scene.sdf_primitives.size(), 0.0f);
  for (size_t i = 0; i < scene.sdf_primitives.size(); ++i) {
    const pt::RTSdfPrimitive& p = scene.sdf_primitives[i];
    float* w = &sdf[16 * i];
    w[0] = static_cast<float>(static_cast<uint32_t>(p.shape));
    w[1] = p.position.x; w[2] = p.position.y; w[3] = p.position.z;
    w[4] = p.scale.x; w[5] = p.scale.y; w[6] = p.scale.z;
    w[7] = p.rotation.x; w[8] = p.rotation.y; w[9] = p.rotation.z;
    w[10] = static_cast<float>(p.material_index);
    w[11] = p.radius; w[12] = p.param_a; w[13] = p.param_b;
  }
  v.sdf_primitives = sdf.empty() ? nullptr : sdf.data();
  v.sdf_count = static_cast<uint32_t>(scene.sdf_primitives.size());
  if (dynamic) {
    v.instance_local = inst_local.data();
    v.instance_transforms = inst_tr.data();
    v.local_vertices = reinterpret_cast<const float*>(scene.local_vertices.data());   // packed Vec3
    v.local_vertex_count = static_cast<uint32_t>(scene.local_vertices.size());
    v.local_indices = scene.local_indices.data();
    v.local_index_count = static_cast<uint32_t>(scene.local_indices.size());
  }
  m_instance_entities.clear();
  for (const auto& r : scene.instances) m_instance_entities.push_back(r.entity_id);
  const Status st = status_from(vkptc_load_scene(m_ctx, &v), "load_scene_snapshot");
  m_has_scene = static_cast<bool>(st);
  if (!st) obs::EmitPathTracerAnomaly(kBackend, "load_scene_snapshot", m_last_error, accumulation_gen());
  if (st) {
    m_next_reset_reason = pt::PathTracerAccumulationResetReason::Topology;
    m_film.set_resolve_settings(pt::CameraAdjustedFilmResolveSettings(m_resolve, scene));
    m_camera = pt::ExtractCameraState(scene);
    m_camera_scene = pt::PathTracerSceneSnapshot{};
    pt::ApplyCameraState(m_camera_scene, m_camera);
  }
  return st;
}

Status CudaPathTracer::build_or_update_acceleration() {
  if (!m_ctx) return Status::error(StatusCode::Unsupported, m_last_error);
  const Status st = status_from(vkptc_build_acceleration(m_ctx), "build_or_update_acceleration");
  vkptc_accel_info info{};
  if (st && vkptc_get_accel_info(m_ctx, &info) == VKPTC_OK)
    obs::EmitPathTracerStarted(kBackend, accumulation_gen(), info.primitive_count);
  else if (!st)
    obs::EmitPathTracerAnomaly(kBackend, "build_or_update_acceleration", m_last_error, accumulation_gen());
  return st;
}

bool CudaPathTracer::reset_accumulation() {
  if (!m_ctx) return fail("no cuda context");
  const bool ok = static_cast<bool>(status_from(vkptc_reset(m_ctx), "reset_accumulation"));
  obs::EmitAccumulationReset(accumulation_gen(), m_next_reset_reason, ok, accel_valid());
  if (ok) m_next_reset_reason = pt::PathTracerAccumulationResetReason::External;
  return ok;
}

bool CudaPathTracer::replace_film_history(const pt::FilmBuffer& film) {
  if (!m_ctx) return fail("no cuda context");
  if (film.width() != m_settings.width || film.height() != m_settings.height) {
    return fail("replace_film_history dimensions do not match");
  }
  const auto& raw = film.raw();
  return static_cast<bool>(status_from(
      vkptc_write_film(m_ctx, reinterpret_cast<const float*>(raw.data()), film.sample_counts().data(),
                       film.invalid_samples().data()),
      "replace_film_history"));
}

bool CudaPathTracer::render_tile(const pt::RenderTile& tile, uint32_t frame_index) {
  return render_tile_cancellable(tile, frame_index, {});
}

bool CudaPathTracer::render_tile_cancellable(const pt::RenderTile& tile, uint32_t frame_index,
                                             std::stop_token stop) {
  const pt::RenderTile one[1] = {tile};
  return render_tiles(std::span<const pt::RenderTile>(one, 1), frame_index, stop);
}

bool CudaPathTracer::render_tiles(std::span<const pt::RenderTile> tiles, std::uint32_t frame_index,
                                  std::stop_token stop) {
  if (!m_ctx) return fail("no cuda context");
  if (stop.stop_requested()) return fail("render_tile cancelled before work started");
  std::vector<vkptc_tile> t(tiles.size());
  for (size_t i = 0; i < tiles.size(); ++i) {
    t[i] = vkptc_tile{tiles[i].x, tiles[i].y, tiles[i].width, tiles[i].height, tiles[i].sample_index,
                      tiles[i].tile_id, tiles[i].gpu_id};
  }
  return static_cast<bool>(status_from(
      vkptc_render(m_ctx, t.data(), static_cast<uint32_t>(t.size()), frame_index, nullptr), "render_tile"));
}

const pt::FilmBuffer& CudaPathTracer::film() const {
  if (!m_ctx) return m_film;
  const size_t n = static_cast<size_t>(m_settings.width) * m_settings.height;
  std::vector<float> sum(3 * n);
  std::vector<uint32_t> cnt(n);
  std::vector<float> inv(n);
  if (vkptc_read_film(m_ctx, sum.data(), cnt.data(), inv.data()) != VKPTC_OK) {
    m_last_error = vkptc_last_error(m_ctx);
    return m_film;
  }
  for (uint32_t y = 0; y < m_settings.height; ++y) {
    for (uint32_t x = 0; x < m_settings.width; ++x) {
      const size_t i = static_cast<size_t>(y) * m_settings.width + x;
      m_film.set_pixel_raw(x, y, pt::Vec3{sum[3 * i], sum[3 * i + 1], sum[3 * i + 2]}, cnt[i], inv[i]);
    }
  }
  return m_film;
}

pt::FilmHdr CudaPathTracer::resolve_hdr() const {
  pt::FilmHdr out;
  if (!m_ctx) return out;
  out.width = m_settings.width;
  out.height = m_settings.height;
  out.rgbf.resize(3 * static_cast<size_t>(out.width) * out.height);
  if (vkptc_resolve_hdr(m_ctx, out.rgbf.data()) != VKPTC_OK) {
    m_last_error = vkptc_last_error(m_ctx);
    return pt::FilmHdr{};
  }
  return out;
}

namespace {

vkptc_film_resolve to_resolve(const pt::FilmResolveSettings& s) {
  vkptc_film_resolve r{};
  r.exposure = s.exposure;
  r.white_balance_kelvin = s.white_balance_kelvin;
  r.tone_map = static_cast<uint32_t>(s.tone_map);
  r.output_transform = static_cast<uint32_t>(s.output_transform);
  r.gamma = s.gamma;
  r.clamp_output = s.clamp_output ? 1u : 0u;
  return r;
}

}  // namespace

pt::FilmLdr CudaPathTracer::resolve_ldr() const {
  // ApplyFilmResolve on the device with the camera-adjusted resolve settings.
  pt::FilmLdr out;
  if (!m_ctx) return out;
  out.width = m_settings.width;
  out.height = m_settings.height;
  out.rgba8.resize(4 * static_cast<size_t>(out.width) * out.height);
  const vkptc_film_resolve rs = to_resolve(m_film.resolve_settings());
  if (vkptc_resolve_ldr(m_ctx, &rs, out.rgba8.data()) != VKPTC_OK) {
    m_last_error = vkptc_last_error(m_ctx);
    return pt::FilmLdr{};
  }
  return out;
}

namespace {

// RTInstanceTransformUpdate -> the C ABI record; the instance resolved by index, else by entity id
// (resolve_instance_index, src/pathtracer/CpuBvhAccelerator.cpp:507-525).
bool resolve_updates(std::span<const pt::RTInstanceTransformUpdate> updates,
                     const std::vector<vkpt::core::StableId>& entities, std::vector<vkptc_instance_update>& out) {
  out.clear();
  for (const auto& u : updates) {
    uint32_t index = u.instance_index;
    if (index >= entities.size() && u.entity_id != 0u) {
      for (size_t i = 0; i < entities.size(); ++i) {
        if (entities[i] == u.entity_id) {
          index = static_cast<uint32_t>(i);
          break;
        }
      }
    }
    if (index >= entities.size()) return false;
    vkptc_instance_update r{};
    r.instance_index = index;
    r.flags = u.flags;
    r.translation[0] = u.translation.x;
    r.translation[1] = u.translation.y;
    r.translation[2] = u.translation.z;
    r.rotation[0] = u.rotation.x;
    r.rotation[1] = u.rotation.y;
    r.rotation[2] = u.rotation.z;
    r.rotation[3] = u.rotation.w;
    r.scale[0] = u.scale.x;
    r.scale[1] = u.scale.y;
    r.scale[2] = u.scale.z;
    out.push_back(r);
  }
  return true;
}

pt::InstanceTransformUpdateStatus status_of(int32_t rc) {
  if (rc == VKPTC_OK) return pt::InstanceTransformUpdateStatus::AppliedDynamicAccelUpdate;
  if (rc == VKPTC_UNSUPPORTED) return pt::InstanceTransformUpdateStatus::BlockedNeedsFullStaticAccelRebuild;
  return pt::InstanceTransformUpdateStatus::Failed;
}

}  // namespace

pt::InstanceTransformPlan CudaPathTracer::plan_instance_transform_update(
    std::span<const pt::RTInstanceTransformUpdate> updates, const pt::InstanceTransformUpdateOptions&) const {
  const uint32_t n = static_cast<uint32_t>(updates.size());
  std::vector<vkptc_instance_update> ups;
  if (!m_ctx || !resolve_updates(updates, m_instance_entities, ups))
    return {pt::InstanceTransformUpdateStatus::Failed, n, 0u, "transform update references an unknown instance"};
  const int32_t rc = vkptc_check_instance_transforms(m_ctx, ups.data(), n);
  m_last_error = rc == VKPTC_OK ? "" : vkptc_last_error(m_ctx);
  return {status_of(rc), n, rc == VKPTC_OK ? n : 0u,
          rc == VKPTC_OK ? "cuda backend refits dynamic instance transforms on the device" : m_last_error.c_str()};
}

pt::InstanceTransformUpdateResult CudaPathTracer::apply_instance_transform_update(
    std::span<const pt::RTInstanceTransformUpdate> updates, const pt::InstanceTransformUpdateOptions& options) {
  const uint32_t n = static_cast<uint32_t>(updates.size());
  std::vector<vkptc_instance_update> ups;
  if (!m_ctx || !resolve_updates(updates, m_instance_entities, ups)) {
    m_last_error = "transform update references an unknown instance";
    return {pt::InstanceTransformUpdateStatus::Failed, n, 0u, 0.0, 0.0, 0.0, 0.0, m_last_error.c_str()};
  }
  const auto t0 = std::chrono::steady_clock::now();
  const int32_t rc = vkptc_update_instance_transforms(m_ctx, ups.data(), n);
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (rc != VKPTC_OK) {
    m_last_error = vkptc_last_error(m_ctx);
    return {status_of(rc), n, 0u, 0.0, 0.0, 0.0, 0.0, m_last_error.c_str()};
  }
  m_last_error.clear();
  m_next_reset_reason = pt::AccumulationResetReasonFromUpdateReason(options.reason);
  obs::EmitSceneDeltaApplied(accumulation_gen(), 0u, 0u, n, false, accel_valid());
  return {pt::InstanceTransformUpdateStatus::AppliedDynamicAccelUpdate, n, n, 0.0, 0.0, ms, 0.0,
          "cuda backend refit dynamic instance transforms"};
}

// ScalarCpuPathTracer::update_camera (src/pathtracer/ScalarCpuPathTracer.cpp:522-533): the current
// camera state with a new position, target, up and field of view.
bool CudaPathTracer::update_camera(const pt::Vec3& pos, const pt::Vec3& target, const pt::Vec3& up, float fov_deg) {
  if (!m_ctx) return fail("no cuda context");
  if (!m_has_scene) return fail("update_camera requires a configured tracer with a scene");
  pt::RTCameraState camera = m_camera;
  camera.position = pos;
  camera.target = target;
  camera.up = up;
  camera.fov_deg = fov_deg;
  return update_camera_state(camera);
}

// ScalarCpuPathTracer::update_camera_state (src/pathtracer/ScalarCpuPathTracer.cpp:535-546): the
// device camera replaced, the film resolve settings adjusted for the new exposure controls.
bool CudaPathTracer::update_camera_state(const pt::RTCameraState& camera) {
  if (!m_ctx) return fail("no cuda context");
  vkptc_camera c{};
  const pt::Vec3 v[3] = {camera.position, camera.target, camera.up};
  float* dst[3] = {c.position, c.target, c.up};
  for (int k = 0; k < 3; ++k) {
    dst[k][0] = v[k].x;
    dst[k][1] = v[k].y;
    dst[k][2] = v[k].z;
  }
  c.fov_deg = camera.fov_deg;
  c.aperture_radius = camera.aperture_radius;
  c.focus_distance = camera.focus_distance;
  c.iris_blade_count = camera.iris_blade_count;
  c.iris_rotation_degrees = camera.iris_rotation_degrees;
  c.iris_roundness = camera.iris_roundness;
  c.anamorphic_squeeze = camera.anamorphic_squeeze;
  if (!status_from(vkptc_update_camera(m_ctx, &c), "update_camera_state")) return false;
  m_next_reset_reason = pt::PathTracerAccumulationResetReason::Camera;
  m_camera = camera;
  pt::ApplyCameraState(m_camera_scene, camera);
  m_film.set_resolve_settings(pt::CameraAdjustedFilmResolveSettings(m_resolve, m_camera_scene));
  return true;
}

// ScalarCpuPathTracer::update_scene_delta (src/pathtracer/ScalarCpuPathTracer.cpp:701-720) over the
// device tables; instances named by entity id are resolved here, as ApplySceneDeltaUpdate does.
bool CudaPathTracer::update_scene_delta(const pt::RTSceneDeltaUpdate& update) {
  if (!m_ctx) return fail("no cuda context");
  std::vector<uint32_t> mat_index, light_index, inst_index, inst_mat;
  std::vector<float> mats(16 * update.materials.size(), 0.0f), lights(16 * update.lights.size(), 0.0f);
  for (size_t k = 0; k < update.materials.size(); ++k) {
    mat_index.push_back(update.materials[k].material_index);
    material_words(update.materials[k].material, &mats[16 * k]);
  }
  for (size_t k = 0; k < update.lights.size(); ++k) {
    light_index.push_back(update.lights[k].light_index);
    light_words(update.lights[k].light, &lights[16 * k]);
  }
  for (const auto& im : update.instance_materials) {
    inst_index.push_back(resolve_instance(im.instance_index, im.entity_id, m_instance_entities));
    inst_mat.push_back(im.material_index);
  }
  vkptc_scene_delta d{};
  d.material_indices = mat_index.data();
  d.materials = mats.data();
  d.material_count = static_cast<uint32_t>(mat_index.size());
  d.light_indices = light_index.data();
  d.lights = lights.data();
  d.light_count = static_cast<uint32_t>(light_index.size());
  d.instance_indices = inst_index.data();
  d.instance_material_indices = inst_mat.data();
  d.instance_material_count = static_cast<uint32_t>(inst_index.size());
  d.environment_changed = update.environment_color_changed ? 1u : 0u;
  d.environment[0] = update.environment_color.x;
  d.environment[1] = update.environment_color.y;
  d.environment[2] = update.environment_color.z;
  if (!status_from(vkptc_update_scene_delta(m_ctx, &d), "update_scene_delta")) return false;
  m_next_reset_reason = pt::PathTracerAccumulationResetReason::Material;
  obs::EmitSceneDeltaApplied(accumulation_gen(), update.materials.size(), update.lights.size(), 0u,
                             update.environment_color_changed, accel_valid());
  return true;
}

bool CudaPathTracer::update_instance_transforms(const std::vector<pt::RTInstanceTransformUpdate>& updates) {
  return apply_instance_transform_update(updates, pt::InstanceTransformUpdateOptions{}).applied();
}

pt::FilmReadbackToken CudaPathTracer::request_film_readback() {
  pt::FilmReadbackToken token;
  if (!m_ctx) return token;
  const vkptc_film_resolve rs = to_resolve(m_film.resolve_settings());
  uint64_t id = 0;
  if (vkptc_request_ldr_readback(m_ctx, &rs, &id) != VKPTC_OK) {
    m_last_error = vkptc_last_error(m_ctx);
    return token;
  }
  token.id = id;
  token.fence_value = id;
  token.width = m_settings.width;
  token.height = m_settings.height;
  return token;
}

pt::FilmReadbackResult CudaPathTracer::poll_film(pt::FilmReadbackToken token) {
  if (!m_ctx || !token || token.width != m_settings.width || token.height != m_settings.height)
    return {pt::FilmReadbackState::Invalid, {}, "invalid cuda film readback token"};
  pt::FilmLdr ldr;
  ldr.width = token.width;
  ldr.height = token.height;
  ldr.rgba8.resize(4 * static_cast<size_t>(ldr.width) * ldr.height);
  uint32_t state = VKPTC_READBACK_INVALID;
  const int32_t rc = vkptc_poll_ldr_readback(m_ctx, token.id, ldr.rgba8.data(), &state);
  if (state == VKPTC_READBACK_PENDING) return {pt::FilmReadbackState::Pending, {}, {}};
  if (state == VKPTC_READBACK_READY) return {pt::FilmReadbackState::Ready, std::move(ldr), {}};
  m_last_error = rc == VKPTC_OK ? "film readback failed" : vkptc_last_error(m_ctx);
  return {state == VKPTC_READBACK_INVALID ? pt::FilmReadbackState::Invalid : pt::FilmReadbackState::Failed, {},
          m_last_error};
}

pt::SampleCounters CudaPathTracer::read_counters() const {
  pt::SampleCounters out{};
  vkptc_counters c{};
  if (m_ctx && vkptc_read_counters(m_ctx, &c) == VKPTC_OK) {
    out.samples = c.samples;
    out.rays = c.rays;
    out.triangle_tests = c.triangle_tests;
    out.triangle_hits = c.triangle_hits;
    out.bvh_node_visits = c.bvh_node_visits;
    out.bvh_leaf_visits = c.bvh_leaf_visits;
    out.shadow_tests = c.shadow_tests;
    out.sdf_tests = c.sdf_tests;
    out.sdf_steps = c.sdf_steps;
    out.sdf_hits = c.sdf_hits;
    out.sdf_misses = c.sdf_misses;
  }
  return out;
}

pt::PathTracerStatus CudaPathTracer::status() const {
  pt::PathTracerStatus out;
  out.backend = "cuda-wavefront";
  out.last_error = m_last_error;
  vkptc_tracer_status s{};
  if (m_ctx && vkptc_get_status(m_ctx, &s) == VKPTC_OK) {
    out.lifecycle = static_cast<pt::PathTracerLifecycle>(s.lifecycle);
    out.scene_loaded = s.scene_loaded != 0u;
    out.accel_valid = s.accel_valid != 0u;
    out.ready_to_render = s.ready_to_render != 0u;
    out.current_sample = s.current_sample;
    out.last_sample_us = s.last_sample_us;
    out.total_samples = s.total_samples;
    out.accumulation_gen = s.accumulation_gen;
  }
  return out;
}

void CudaPathTracer::shutdown() {
  if (m_ctx) vkptc_shutdown(m_ctx);
  m_film = pt::FilmBuffer{};
  m_last_error.clear();
}

struct BenchmarkAccess {
  static vkptc_ctx* ctx(const CudaPathTracer& t) { return t.m_ctx; }
  static const pt::RenderSettings& settings(const CudaPathTracer& t) { return t.m_settings; }
};

namespace {

std::string fmt(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%.6g", v);
  return b;
}

}  // namespace

void FillBenchmarkResult(const CudaPathTracer& tracer, const CudaBenchmarkInputs& in,
                         vkpt::benchmark::BenchmarkResult& result) {
  vkptc_ctx* ctx = BenchmarkAccess::ctx(tracer);
  const pt::RenderSettings& st = BenchmarkAccess::settings(tracer);
  result.backend = "cuda";
  result.renderer_path = in.renderer_path ? in.renderer_path : kBackend;
  result.device_info.backend = result.backend;
  result.device_info.renderer_path = result.renderer_path;
  char name[256] = {0};
  if (ctx && vkptc_device_name(ctx, name, sizeof(name), nullptr) == VKPTC_OK) result.device_info.gpu_name = name;
  result.resolution = {st.width, st.height};
  result.spp = st.spp;
  result.seed = st.seed;
  result.max_depth = st.max_depth;
  result.timing.render_ms = in.render_ms;
  result.timing.build_ms = in.build_ms;
  result.timing.total_ms = in.total_ms > 0.0 ? in.total_ms : in.build_ms + in.render_ms;
  const pt::SampleCounters c = tracer.read_counters();
  const double render_s = in.render_ms / 1e3;
  result.diagnostics.push_back(std::string("renderer=") + result.renderer_path);
  if (render_s > 0.0) {
    result.throughput.paths_per_sec = static_cast<double>(c.rays) / render_s;
    result.throughput.samples_per_sec = static_cast<double>(c.samples) / render_s;
    result.diagnostics.push_back("paths_per_sec_camera=" + fmt(static_cast<double>(c.samples) / render_s));
    result.diagnostics.push_back("mrays_per_sec=" + fmt(static_cast<double>(c.rays + c.shadow_tests) / render_s / 1e6));
  }
  uint64_t tr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (ctx && render_s > 0.0 && in.peak_bandwidth_gbs > 0.0 && vkptc_read_traversal_stats(ctx, tr) == VKPTC_OK) {
    // extension and shadow queries: rays, node visits, leaf visits, triangle tests
    const double bytes = 128.0 * static_cast<double>(tr[1] + tr[5]) + 48.0 * static_cast<double>(tr[3] + tr[7]) +
                         32.0 * static_cast<double>(tr[0] + tr[4]);
    result.diagnostics.push_back("roofline_fraction=" + fmt(bytes / render_s / 1e9 / in.peak_bandwidth_gbs));
  } else {
    result.diagnostics.push_back("roofline_fraction=n/a");
  }
  if (in.reference) {
    const auto& a = in.reference->raw();
    const auto& ac = in.reference->sample_counts();
    const auto& b = tracer.film().raw();
    const auto& bc = tracer.film().sample_counts();
    const size_t n = std::min(a.size(), b.size());
    double se = 0.0, mean = 0.0;
    size_t same = 0, fails = 0;
    for (size_t i = 0; i < n; ++i) {
      const double na = std::max(1u, ac[i]), nb = std::max(1u, bc[i]);
      const float pa[3] = {a[i].x, a[i].y, a[i].z}, pb[3] = {b[i].x, b[i].y, b[i].z};
      if (std::memcmp(pa, pb, sizeof(pa)) == 0 && ac[i] == bc[i]) ++same;
      for (int ch = 0; ch < 3; ++ch) {
        const double ma = pa[ch] / na, d = pb[ch] / nb - ma;
        se += d * d;
        mean += ma;
        if (in.reference_m2 && in.reference_m2->size() >= 3 * n) {
          const double var = std::max(0.0, ((*in.reference_m2)[3 * i + ch] - pa[ch] * ma) / std::max(1.0, na - 1.0));
          if (std::fabs(d) > 3.0 * std::sqrt(var / na) + 1e-6 * (1.0 + std::fabs(ma))) ++fails;
        }
      }
    }
    const double m = mean / std::max<double>(1.0, 3.0 * n);
    result.diagnostics.push_back("rmse=" + fmt(std::sqrt(se / std::max<double>(1.0, 3.0 * n)) / std::max(m, 1e-12)));
    if (in.reference_m2) result.diagnostics.push_back("sigma3_fail_frac=" + fmt(fails / std::max<double>(1.0, 3.0 * n)));
    result.diagnostics.push_back("bit_identical_frac=" + fmt(static_cast<double>(same) / std::max<size_t>(1, n)));
  }
}

}  // namespace vkpt::gpu::cuda
