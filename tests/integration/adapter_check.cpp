// adapter_check.cpp -- TEST: runs the reference's ScalarCpuPathTracer and the
// cuda backend's CudaPathTracer through the reference's IPathTracer interface
// on the same scene, with ptbench's render loop
// (src/benchmark/BenchmarkRuntime.cpp:672-693), and compares the films.
//
// usage: adapter_check nodevice            (expects no CUDA device)
//        adapter_check <scene.bin>         (scene + settings written by tests/test_adapter.py)
//        adapter_check json <scene.json> <width> <height> <spp> <max_depth>
//            (the scene document loaded and converted by the reference's own
//             SceneDocument::load_from_file and BuildSceneDataFromDocument, as
//             ptbench does, src/benchmark/BenchmarkRuntime.cpp:491-596)
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "CudaPathTracer.h"
#include "core/Logging.h"
#include "pathtracer/PathTracer.h"
#include "scene/Scene.h"

namespace pt = vkpt::pathtracer;

namespace {

template <typename T>
bool read_vec(std::ifstream& f, std::vector<T>& v, size_t n) {
  v.resize(n);
  return static_cast<bool>(f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(n * sizeof(T))));
}

bool load(const char* path, pt::PathTracerSceneSnapshot& s, pt::RenderSettings& st) {
  std::ifstream f(path, std::ios::binary);
  uint32_t c[5];
  if (!f.read(reinterpret_cast<char*>(c), sizeof(c))) return false;
  std::vector<float> verts, mats, lights, env, cam;
  std::vector<uint32_t> idx, inst, sets;
  if (!read_vec(f, verts, 3 * c[0]) || !read_vec(f, idx, c[1]) || !read_vec(f, inst, 3 * c[2]) ||
      !read_vec(f, mats, 16 * c[3]) || !read_vec(f, lights, 16 * c[4]) || !read_vec(f, env, 3) ||
      !read_vec(f, cam, 12) || !read_vec(f, sets, 7)) {
    return false;
  }
  uint64_t seed = 0;
  float rr[2];
  f.read(reinterpret_cast<char*>(&seed), 8);
  f.read(reinterpret_cast<char*>(rr), 8);
  for (uint32_t i = 0; i < c[0]; ++i) s.vertices.push_back(pt::Vec3{verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]});
  s.indices = idx;
  for (uint32_t i = 0; i < c[2]; ++i) {
    pt::RTInstance r;
    r.entity_id = i + 1;
    r.first_triangle = inst[3 * i];
    r.triangle_count = inst[3 * i + 1];
    r.material_index = inst[3 * i + 2];
    s.instances.push_back(r);
  }
  for (uint32_t i = 0; i < c[3]; ++i) {
    const float* m = &mats[16 * i];
    pt::RTMaterial r;
    r.albedo = {m[0], m[1], m[2]};
    r.emissive = {m[3], m[4], m[5]};
    r.roughness = m[6];
    r.material_model = static_cast<uint32_t>(m[7] + 0.5f);
    r.metallic = m[8];
    r.ior = m[9];
    r.transmission = m[10];
    r.clearcoat = m[11];
    r.sheen = m[12];
    r.anisotropy = m[13];
    r.alpha = m[14];
    s.materials.push_back(r);
  }
  for (uint32_t i = 0; i < c[4]; ++i) {
    const float* l = &lights[16 * i];
    pt::RTHitLight r;
    r.position = {l[0], l[1], l[2]};
    r.color = {l[3], l[4], l[5]};
    r.intensity = l[6];
    r.radius = l[7];
    r.direction = {l[8], l[9], l[10]};
    r.spot_inner_cos = l[11];
    r.spot_outer_cos = l[12];
    s.lights.push_back(r);
  }
  s.environment_color = {env[0], env[1], env[2]};
  s.camera_position = {cam[0], cam[1], cam[2]};
  s.camera_target = {cam[3], cam[4], cam[5]};
  s.camera_up = {cam[6], cam[7], cam[8]};
  s.camera_fov_deg = cam[9];
  s.camera_aperture_radius = cam[10];
  s.camera_focus_distance = cam[11];
  st.width = sets[0];
  st.height = sets[1];
  st.spp = sets[2];
  st.max_depth = sets[3];
  st.enable_nee = sets[4] != 0;
  st.enable_mis = sets[5] != 0;
  st.russian_roulette_start_depth = sets[6];
  st.seed = seed;
  st.russian_roulette_min_survival = rr[0];
  st.russian_roulette_max_survival = rr[1];
  // optional trailer: SDF primitive count, then 16 floats each
  uint32_t n_sdf = 0;
  std::vector<float> sdf;
  if (f.read(reinterpret_cast<char*>(&n_sdf), 4) && n_sdf > 0) {
    if (!read_vec(f, sdf, 16 * static_cast<size_t>(n_sdf))) return false;
    for (uint32_t i = 0; i < n_sdf; ++i) {
      const float* q = &sdf[16 * i];
      pt::RTSdfPrimitive r;
      r.shape = static_cast<pt::SdfShape>(static_cast<uint32_t>(q[0] + 0.5f));
      r.position = {q[1], q[2], q[3]};
      r.scale = {q[4], q[5], q[6]};
      r.rotation = {q[7], q[8], q[9]};
      r.material_index = static_cast<uint32_t>(q[10] + 0.5f);
      r.radius = q[11];
      r.param_a = q[12];
      r.param_b = q[13];
      s.sdf_primitives.push_back(r);
    }
  }
  // optional trailer: dynamic-transform instances (instance count, local vertex
  // and index counts; 5 words and 10 floats per instance; local arrays)
  uint32_t dyn[3] = {0, 0, 0};
  if (f.read(reinterpret_cast<char*>(dyn), sizeof(dyn)) && dyn[0] == c[2]) {
    std::vector<uint32_t> loc, lidx;
    std::vector<float> tr, lv;
    if (!read_vec(f, loc, 5ull * dyn[0]) || !read_vec(f, tr, 10ull * dyn[0]) || !read_vec(f, lv, 3ull * dyn[1]) ||
        !read_vec(f, lidx, dyn[2]))
      return false;
    for (uint32_t i = 0; i < dyn[0]; ++i) {
      pt::RTInstance& r = s.instances[i];
      r.flags = loc[5 * i];
      r.local_first_vertex = loc[5 * i + 1];
      r.local_vertex_count = loc[5 * i + 2];
      r.local_first_index = loc[5 * i + 3];
      r.local_index_count = loc[5 * i + 4];
      const float* t = &tr[10 * i];
      r.translation = {t[0], t[1], t[2]};
      r.rotation = {t[3], t[4], t[5], t[6]};
      r.scale = {t[7], t[8], t[9]};
    }
    for (uint32_t i = 0; i < dyn[1]; ++i) s.local_vertices.push_back(pt::Vec3{lv[3 * i], lv[3 * i + 1], lv[3 * i + 2]});
    s.local_indices = lidx;
  }
  return true;
}

int failures = 0;
void check(bool ok, const char* what) {
  std::printf("%s %s\n", ok ? "PASS" : "FAIL", what);
  if (!ok) ++failures;
}

// ptbench's loop: configure, load, build, reset, one full-frame render_tile
// per sample.  m2 (optional) receives per pixel and channel the sum of the
// squared per-sample radiance (the change of the film's running sum).
// render_ms / build_ms (optional) receive the times ptbench reports.
bool render(pt::IPathTracer& t, const pt::PathTracerSceneSnapshot& s, const pt::RenderSettings& st,
            std::vector<float>* m2 = nullptr, double* render_ms = nullptr, double* build_ms = nullptr) {
  const auto b0 = std::chrono::steady_clock::now();
  if (!t.configure(st) || !t.load_scene_snapshot(s) || !t.build_or_update_acceleration()) return false;
  const auto b1 = std::chrono::steady_clock::now();
  t.reset_accumulation();
  const size_t n = static_cast<size_t>(st.width) * st.height;
  std::vector<float> prev;
  if (m2) {
    m2->assign(3 * n, 0.0f);
    prev.assign(3 * n, 0.0f);
  }
  double loop_ms = 0.0;
  for (uint32_t k = 0; k < st.spp; ++k) {
    pt::RenderTile tile;
    tile.width = st.width;
    tile.height = st.height;
    tile.sample_index = k;
    const auto r0 = std::chrono::steady_clock::now();
    if (!t.render_tile(tile, 0u)) return false;
    loop_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - r0).count();
    if (m2) {
      const auto& raw = t.film().raw();
      for (size_t i = 0; i < n; ++i) {
        const float cur[3] = {raw[i].x, raw[i].y, raw[i].z};
        for (int ch = 0; ch < 3; ++ch) {
          const float x = cur[ch] - prev[3 * i + ch];
          (*m2)[3 * i + ch] += x * x;
          prev[3 * i + ch] = cur[ch];
        }
      }
    }
  }
  if (render_ms) *render_ms = loop_ms;
  if (build_ms) *build_ms = std::chrono::duration<double, std::milli>(b1 - b0).count();
  return true;
}

// The value of "key=" among the diagnostics, or NaN.
double diagnostic(const vkpt::benchmark::BenchmarkResult& r, const std::string& key) {
  for (const auto& d : r.diagnostics)
    if (d.rfind(key + "=", 0) == 0) return std::atof(d.c_str() + key.size() + 1);
  return std::nan("");
}

}  // namespace

int main(int argc, char** argv) {
  vkpt::log::Logger::instance().set_min_severity(vkpt::log::Severity::Fatal);
  if (argc < 2) return 2;
  if (std::strcmp(argv[1], "nodevice") == 0) {
    vkpt::gpu::cuda::CudaPathTracer t;
    check(!t.is_valid(), "no device: context not created");
    pt::RenderSettings st;
    const auto s = t.configure(st);
    check(!s && s.code == vkpt::core::StatusCode::Unsupported, "no device: configure returns Unsupported");
    check(!t.render_tile(pt::RenderTile{}, 0), "no device: render_tile fails");
    return failures == 0 ? 0 : 1;
  }
  pt::PathTracerSceneSnapshot scene;
  pt::RenderSettings st;
  if (std::strcmp(argv[1], "json") == 0) {
    if (argc < 7) return 2;
    auto doc = vkpt::scene::SceneDocument::load_from_file(argv[2]);
    std::vector<std::string> issues;
    if (!doc || !doc.value().validate(&issues)) {
      std::printf("FAIL cannot load scene document %s\n", argv[2]);
      return 2;
    }
    auto conv = pt::BuildSceneDataFromDocument(doc.value());
    if (!conv) {
      std::printf("FAIL scene conversion %s\n", argv[2]);
      return 2;
    }
    scene = conv.value();
    st.width = static_cast<uint32_t>(std::atoi(argv[3]));
    st.height = static_cast<uint32_t>(std::atoi(argv[4]));
    st.spp = static_cast<uint32_t>(std::atoi(argv[5]));
    st.max_depth = static_cast<uint32_t>(std::atoi(argv[6]));
    st.seed = 1234u;
    std::printf("scene %s: %zu triangles, %zu instances, %zu sdf, %zu lights\n", argv[2], scene.indices.size() / 3,
                scene.instances.size(), scene.sdf_primitives.size(), scene.lights.size());
  } else if (!load(argv[1], scene, st)) {
    std::printf("FAIL cannot read %s\n", argv[1]);
    return 2;
  }
  check(pt::ValidateStandardPathTracerContract(pt::BuildStandardPathTracerContract()), "standard contract");

  pt::ScalarCpuPathTracer ref;
  vkpt::gpu::cuda::CudaPathTracer gpu;
  check(gpu.is_valid(), "cuda context created");
  // lifecycle errors before configure / before the scene
  check(!gpu.render_tile(pt::RenderTile{}, 0), "render before configure fails");
  check(gpu.status().lifecycle == pt::PathTracerLifecycle::Uninitialized, "lifecycle uninitialized");
  std::vector<float> ref_m2;
  check(render(ref, scene, st, &ref_m2), "reference renders");
  double gpu_render_ms = 0.0, gpu_build_ms = 0.0;
  check(render(gpu, scene, st, nullptr, &gpu_render_ms, &gpu_build_ms), "cuda backend renders through IPathTracer");
  check(gpu.status().lifecycle == pt::PathTracerLifecycle::Ready && gpu.status().ready_to_render, "lifecycle ready");

  const auto& a = ref.film();
  const auto& b = gpu.film();
  size_t same = 0, n = a.raw().size();
  double se = 0.0, mean = 0.0;
  bool counts_equal = a.sample_counts() == b.sample_counts();
  for (size_t i = 0; i < n; ++i) {
    const pt::Vec3 p = a.raw()[i], q = b.raw()[i];
    if (std::memcmp(&p, &q, sizeof(p)) == 0) ++same;
    se += (p.x - q.x) * (p.x - q.x) + (p.y - q.y) * (p.y - q.y) + (p.z - q.z) * (p.z - q.z);
    mean += p.x + p.y + p.z;
  }
  const double rmse_rel = std::sqrt(se / (3.0 * n)) / (mean / (3.0 * n) + 1e-12);
  std::printf("pixels %zu bit_identical %.4f rmse_rel %.3e\n", n, double(same) / n, rmse_rel);
  check(counts_equal, "sample counts equal");
  check(double(same) / n >= 0.97, "at least 97% of pixels bit-identical");
  check(rmse_rel < 1e-3, "relative RMSE below 1e-3");
  const auto ca = ref.read_counters(), cb = gpu.read_counters();
  std::printf("samples %llu/%llu segments %llu/%llu shadow %llu/%llu\n", (unsigned long long)ca.samples,
              (unsigned long long)cb.samples, (unsigned long long)ca.rays, (unsigned long long)cb.rays,
              (unsigned long long)ca.shadow_tests, (unsigned long long)cb.shadow_tests);
  check(ca.samples == cb.samples, "sample counters equal");
  // Pixels whose films are bit-identical followed identical paths; each other
  // pixel may differ by at most max_depth segments per sample and, per
  // segment, one NEE query plus eight transparent skips
  // (src/pathtracer/ScalarCpuPathTracer.cpp:1067-1087).
  const uint64_t differing = n - same;
  const uint64_t seg_gap = differing * st.spp * st.max_depth;
  const auto absdiff = [](uint64_t x, uint64_t y) { return x > y ? x - y : y - x; };
  std::printf("pixels differing %llu: allowed segment gap %llu, shadow-test gap %llu\n", (unsigned long long)differing,
              (unsigned long long)seg_gap, (unsigned long long)(9u * seg_gap));
  check(absdiff(ca.rays, cb.rays) <= seg_gap, "segment counters (rays) equal up to the differing pixels");
  check(absdiff(ca.shadow_tests, cb.shadow_tests) <= 9u * seg_gap,
        "shadow-test counters equal up to the differing pixels");
  // the BenchmarkResult fields ptbench `run` fills for this backend
  {
    vkpt::benchmark::BenchmarkResult br;
    vkpt::gpu::cuda::CudaBenchmarkInputs in;
    in.render_ms = gpu_render_ms;
    in.build_ms = gpu_build_ms;
    in.reference = &ref.film();
    in.reference_m2 = &ref_m2;
    vkpt::gpu::cuda::FillBenchmarkResult(gpu, in, br);
    std::printf("benchmark backend=%s renderer_path=%s gpu=%s paths_per_sec=%.6g samples_per_sec=%.6g\n",
                br.backend.c_str(), br.renderer_path.c_str(), br.device_info.gpu_name.c_str(),
                br.throughput.paths_per_sec, br.throughput.samples_per_sec);
    for (const auto& d : br.diagnostics) std::printf("diagnostic %s\n", d.c_str());
    check(br.backend == "cuda" && br.renderer_path == "cuda-wavefront" && !br.device_info.gpu_name.empty(),
          "BenchmarkResult backend, renderer_path, gpu_name");
    check(gpu_render_ms > 0.0 &&
              std::fabs(br.throughput.paths_per_sec - cb.rays / (gpu_render_ms / 1e3)) <= 1e-9 * br.throughput.paths_per_sec,
          "BenchmarkResult paths_per_sec = counters.rays / render time");
    check(diagnostic(br, "paths_per_sec_camera") > 0.0 && diagnostic(br, "mrays_per_sec") > 0.0,
          "diagnostics paths_per_sec_camera, mrays_per_sec");
    check(diagnostic(br, "rmse") < 1e-3 && diagnostic(br, "sigma3_fail_frac") < 0.003 &&
              diagnostic(br, "bit_identical_frac") >= 0.97,
          "diagnostics rmse, sigma3_fail_frac, bit_identical_frac within the film tolerances");
  }
  const auto hdr_a = ref.resolve_hdr(), hdr_b = gpu.resolve_hdr();
  check(hdr_a.width == hdr_b.width && hdr_a.rgbf.size() == hdr_b.rgbf.size(), "resolve_hdr shape");
  const auto ldr = gpu.resolve_ldr();
  check(ldr.rgba8.size() == 4u * st.width * st.height, "resolve_ldr size");
  // the device tone map against the reference's ApplyFilmResolve of the same HDR film
  const auto ref_ldr = pt::ApplyFilmResolve(gpu.resolve_hdr(), gpu.film().resolve_settings());
  size_t ldr_same = 0, ldr_max = 0;
  for (size_t i = 0; i < ldr.rgba8.size() && i < ref_ldr.rgba8.size(); ++i) {
    const int d = std::abs(static_cast<int>(ldr.rgba8[i]) - static_cast<int>(ref_ldr.rgba8[i]));
    ldr_same += d == 0 ? 1u : 0u;
    ldr_max = std::max<size_t>(ldr_max, static_cast<size_t>(d));
  }
  std::printf("ldr bytes identical %.5f max step %zu\n", double(ldr_same) / std::max<size_t>(1, ldr.rgba8.size()), ldr_max);
  check(ref_ldr.rgba8.size() == ldr.rgba8.size() && ldr_max <= 1u && ldr_same * 1000u >= 999u * ldr.rgba8.size(),
        "device resolve_ldr equals ApplyFilmResolve of the device HDR film (<= 1 step on < 0.1 % of bytes)");
  // split film readback: request, then poll until ready (bounded)
  const auto token = gpu.request_film_readback();
  check(static_cast<bool>(token), "request_film_readback");
  pt::FilmReadbackResult rb;
  for (int k = 0; k < 1000000; ++k) {
    rb = gpu.poll_film(token);
    if (rb.state != pt::FilmReadbackState::Pending) break;
  }
  check(rb.ready() && rb.ldr.rgba8 == ldr.rgba8, "poll_film returns the resolved film");
  pt::FilmReadbackToken stale = token;
  stale.id += 1000;
  check(gpu.poll_film(stale).state == pt::FilmReadbackState::Invalid, "poll_film rejects an unknown token");
  // reset keeps the acceleration structure; the film starts over
  check(gpu.reset_accumulation() && gpu.status().accel_valid && gpu.read_counters().samples == 0, "reset is film-only");
  // tiles = full frame (CheckScalarRenderTilePrimitive, tests/snapshot_bus_smoke.cpp:1368-1435)
  vkpt::gpu::cuda::CudaPathTracer tiled;
  bool ok = tiled.configure(st) && tiled.load_scene_snapshot(scene) && tiled.build_or_update_acceleration();
  tiled.reset_accumulation();
  for (uint32_t k = 0; k < st.spp && ok; ++k) {
    std::vector<pt::RenderTile> tiles(2);
    tiles[0].width = tiles[1].width = st.width;
    tiles[0].height = st.height / 2;
    tiles[1].y = st.height / 2;
    tiles[1].height = st.height - st.height / 2;
    tiles[0].sample_index = tiles[1].sample_index = k;
    ok = tiled.render_tiles(tiles, 0u, {});
  }
  const auto& c = tiled.film();
  check(ok && std::memcmp(c.raw().data(), b.raw().data(), n * sizeof(pt::Vec3)) == 0, "render_tiles equals full frame");
  // instance transform updates through IPathTracer on both tracers (scenes with dynamic instances)
  std::vector<pt::RTInstanceTransformUpdate> updates;
  for (uint32_t i = 0; i < scene.instances.size() && updates.size() < 3; ++i) {
    const pt::RTInstance& r = scene.instances[i];
    if (!r.has_flag(pt::kRTInstanceFlagDynamicTransform) || r.local_vertex_count == 0u || r.local_index_count == 0u)
      continue;
    pt::RTInstanceTransformUpdate u;
    u.entity_id = r.entity_id;
    u.instance_index = pt::kInvalidRTInstanceIndex;   // resolved by entity id
    const float a = 0.3f + 0.2f * static_cast<float>(updates.size());
    u.translation = {r.translation.x + 0.04f, r.translation.y + 0.02f, r.translation.z - 0.03f};
    u.rotation = {0.0f, std::sin(0.5f * a), 0.0f, std::cos(0.5f * a)};
    u.scale = {r.scale.x * 1.05f, r.scale.y * 1.05f, r.scale.z * 1.05f};
    updates.push_back(u);
  }
  if (!updates.empty()) {
    pt::ScalarCpuPathTracer ref2;
    vkpt::gpu::cuda::CudaPathTracer gpu2;
    check(render(ref2, scene, st) && render(gpu2, scene, st), "render before transform updates");
    const pt::InstanceTransformUpdateOptions opts{};
    const auto plan = gpu2.plan_instance_transform_update(updates, opts);
    check(plan.status == pt::InstanceTransformUpdateStatus::AppliedDynamicAccelUpdate &&
              plan.matched_count == updates.size(), "plan_instance_transform_update: dynamic accel update");
    const auto ra = ref2.apply_instance_transform_update(updates, opts);
    const auto rb = gpu2.apply_instance_transform_update(updates, opts);
    check(ra.applied() && rb.applied() && rb.applied_count == updates.size(), "apply_instance_transform_update");
    ref2.reset_accumulation();
    gpu2.reset_accumulation();
    bool ok2 = true;
    for (uint32_t k = 0; k < st.spp; ++k) {
      pt::RenderTile tile;
      tile.width = st.width;
      tile.height = st.height;
      tile.sample_index = k;
      ok2 = ok2 && ref2.render_tile(tile, 0u) && gpu2.render_tile(tile, 0u);
    }
    const auto& ua = ref2.film();
    const auto& ub = gpu2.film();
    size_t same2 = 0;
    for (size_t i = 0; i < n; ++i) same2 += std::memcmp(&ua.raw()[i], &ub.raw()[i], sizeof(pt::Vec3)) == 0 ? 1u : 0u;
    std::printf("after %zu transform updates: pixels bit_identical %.4f\n", updates.size(), double(same2) / n);
    check(ok2 && ua.sample_counts() == ub.sample_counts() && double(same2) / n >= 0.97,
          "films after the same transform updates: at least 97% of pixels bit-identical");
  }
  // camera and scene deltas through IPathTracer on both tracers
  {
    pt::ScalarCpuPathTracer ref3;
    vkpt::gpu::cuda::CudaPathTracer gpu3;
    check(render(ref3, scene, st) && render(gpu3, scene, st), "render before camera and scene deltas");
    auto rerender = [&](const char* what) {
      ref3.reset_accumulation();
      gpu3.reset_accumulation();
      bool ok3 = true;
      for (uint32_t k = 0; k < st.spp; ++k) {
        pt::RenderTile tile;
        tile.width = st.width;
        tile.height = st.height;
        tile.sample_index = k;
        ok3 = ok3 && ref3.render_tile(tile, 0u) && gpu3.render_tile(tile, 0u);
      }
      const auto& fa = ref3.film();
      const auto& fb = gpu3.film();
      size_t same3 = 0;
      for (size_t i = 0; i < n; ++i) same3 += std::memcmp(&fa.raw()[i], &fb.raw()[i], sizeof(pt::Vec3)) == 0 ? 1u : 0u;
      std::printf("%s: pixels bit_identical %.4f\n", what, double(same3) / n);
      check(ok3 && fa.sample_counts() == fb.sample_counts() && double(same3) / n >= 0.97, what);
    };
    // a thin lens with a polygonal iris and squeeze, exposure controls, a narrower view
    pt::RTCameraState cam = pt::ExtractCameraState(scene);
    const float dx = cam.target.x - cam.position.x, dy = cam.target.y - cam.position.y,
                dz = cam.target.z - cam.position.z;
    const float dist = std::sqrt(dx * dx + dy * dy + dz * dz);
    cam.position = {cam.position.x + 0.03f * dist, cam.position.y + 0.02f * dist, cam.position.z};
    cam.fov_deg *= 0.9f;
    cam.aperture_radius = 0.03f * dist;
    cam.focus_distance = dist;
    cam.iris_blade_count = 6u;
    cam.iris_rotation_degrees = 15.0f;
    cam.iris_roundness = 0.3f;
    cam.anamorphic_squeeze = 1.2f;
    cam.exposure_compensation = 1.0f;
    cam.white_balance_kelvin = 5000.0f;
    check(ref3.update_camera_state(cam) && gpu3.update_camera_state(cam), "update_camera_state");
    const auto ra3 = ref3.film().resolve_settings(), rb3 = gpu3.film().resolve_settings();
    check(ra3.exposure == rb3.exposure && ra3.white_balance_kelvin == rb3.white_balance_kelvin,
          "update_camera_state: camera-adjusted film resolve settings");
    rerender("films after update_camera_state: at least 97% of pixels bit-identical");
    // materials, lights, an instance's material and the environment colour
    pt::RTSceneDeltaUpdate delta;
    if (!scene.materials.empty()) {
      pt::RTMaterialUpdate mu;
      mu.material_index = 0u;
      mu.material = scene.materials[0];
      mu.material.albedo = {0.9f, 0.25f, 0.1f};
      mu.material.roughness = 0.35f;
      delta.materials.push_back(mu);
    }
    if (!scene.lights.empty()) {
      pt::RTLightUpdate lu;
      lu.light_index = static_cast<uint32_t>(scene.lights.size() - 1);
      lu.light = scene.lights.back();
      lu.light.intensity *= 1.5f;
      lu.light.color = {1.0f, 0.8f, 0.6f};
      delta.lights.push_back(lu);
    }
    if (scene.instances.size() > 1 && scene.materials.size() > 1) {
      pt::RTInstanceMaterialUpdate im;
      im.entity_id = scene.instances[1].entity_id;
      im.instance_index = im.entity_id != 0u ? pt::kInvalidRTInstanceIndex : 1u;
      im.material_index = (scene.instances[1].material_index + 1u) % static_cast<uint32_t>(scene.materials.size());
      delta.instance_materials.push_back(im);
    }
    delta.environment_color_changed = true;
    delta.environment_color = {0.05f, 0.07f, 0.1f};
    check(ref3.update_scene_delta(delta) && gpu3.update_scene_delta(delta), "update_scene_delta");
    // The CPU tracer's accelerator keeps each primitive's material from its
    // build; rebuilt, it shows the instance material the cuda backend applies at once.
    check(static_cast<bool>(ref3.build_or_update_acceleration()), "reference rebuild after the scene delta");
    rerender("films after update_scene_delta: at least 97% of pixels bit-identical");
    pt::RTSceneDeltaUpdate bad;
    pt::RTMaterialUpdate out_of_range;
    out_of_range.material_index = static_cast<uint32_t>(scene.materials.size() + 5u);
    bad.materials.push_back(out_of_range);
    check(!ref3.update_scene_delta(bad) && !gpu3.update_scene_delta(bad), "out-of-range scene delta rejected by both");
    check(!ref3.update_scene_delta(pt::RTSceneDeltaUpdate{}) && !gpu3.update_scene_delta(pt::RTSceneDeltaUpdate{}),
          "empty scene delta rejected by both");
    const pt::Vec3 up{0.0f, 1.0f, 0.0f};
    check(ref3.update_camera(scene.camera_position, scene.camera_target, up, scene.camera_fov_deg) &&
              gpu3.update_camera(scene.camera_position, scene.camera_target, up, scene.camera_fov_deg),
          "update_camera");
    rerender("films after update_camera (lens kept): at least 97% of pixels bit-identical");
  }
  gpu.shutdown();
  check(gpu.status().lifecycle == pt::PathTracerLifecycle::Uninitialized, "shutdown");
  return failures == 0 ? 0 : 1;
}
