// CudaPathTracer.h -- the sm_100a backend as a vkPathTracer IPathTracer.
//
// Drop-in for the reference's CPU preview/reference tracer: a class a
// maintainer adds as src/gpu/cuda/CudaPathTracer.{h,cpp} of vkPathTracer.  It
// implements vkpt::pathtracer::IPathTracer (src/pathtracer/PathTracer.h:1069-1184)
// over the C ABI of libvkpt_cuda (include/vkptc.h) and compiles against the
// reference's own headers; nothing here renders on the CPU.
#pragma once

#include <memory>
#include <span>
#include <stop_token>
#include <string>

#include "benchmark/BenchmarkSchema.h"
#include "pathtracer/PathTracer.h"

struct vkptc_ctx;

namespace vkpt::gpu::cuda {

struct CudaPathTracerConfig {
  int device = 0;
  uint32_t block_size = 0;     // 0 = library default
  uint32_t math_mode = 0;      // 0 = parity with the CPU tracer, 1 = fast FP32 transcendentals
  bool collect_stats = false;  // fill the traversal counters of SampleCounters
};

class CudaPathTracer final : public vkpt::pathtracer::IPathTracer {
 public:
  using vkpt::pathtracer::IPathTracer::configure;

  explicit CudaPathTracer(CudaPathTracerConfig config = {});
  ~CudaPathTracer() override;
  CudaPathTracer(const CudaPathTracer&) = delete;
  CudaPathTracer& operator=(const CudaPathTracer&) = delete;

  bool is_valid() const { return m_ctx != nullptr; }
  const std::string& last_error() const { return m_last_error; }

  vkpt::core::Status configure(const vkpt::pathtracer::RenderSettings& settings) override;
  vkpt::core::Status load_scene_snapshot(const vkpt::pathtracer::PathTracerSceneSnapshot& scene) override;
  vkpt::core::Status build_or_update_acceleration() override;
  bool reset_accumulation() override;
  bool replace_film_history(const vkpt::pathtracer::FilmBuffer& film) override;
  bool render_tile(const vkpt::pathtracer::RenderTile& tile, uint32_t frame_index) override;
  bool render_tile_cancellable(const vkpt::pathtracer::RenderTile& tile, uint32_t frame_index,
                               std::stop_token stop) override;
  bool render_tiles(std::span<const vkpt::pathtracer::RenderTile> tiles, std::uint32_t frame_index,
                    std::stop_token stop) override;
  bool supports_tile_rendering() const override { return true; }
  bool supports_tile_batching() const override { return true; }
  vkpt::pathtracer::FilmLdr resolve_ldr() const override;
  vkpt::pathtracer::FilmReadbackToken request_film_readback() override;
  bool update_camera(const vkpt::pathtracer::Vec3& pos, const vkpt::pathtracer::Vec3& target,
                     const vkpt::pathtracer::Vec3& up, float fov_deg) override;
  bool update_camera_state(const vkpt::pathtracer::RTCameraState& camera) override;
  bool update_scene_delta(const vkpt::pathtracer::RTSceneDeltaUpdate& update) override;
  bool update_instance_transforms(const std::vector<vkpt::pathtracer::RTInstanceTransformUpdate>& updates) override;
  vkpt::pathtracer::InstanceTransformPlan plan_instance_transform_update(
      std::span<const vkpt::pathtracer::RTInstanceTransformUpdate> updates,
      const vkpt::pathtracer::InstanceTransformUpdateOptions& options) const override;
  vkpt::pathtracer::InstanceTransformUpdateResult apply_instance_transform_update(
      std::span<const vkpt::pathtracer::RTInstanceTransformUpdate> updates,
      const vkpt::pathtracer::InstanceTransformUpdateOptions& options) override;
  vkpt::pathtracer::FilmReadbackResult poll_film(vkpt::pathtracer::FilmReadbackToken token) override;
  vkpt::pathtracer::FilmHdr resolve_hdr() const override;
  vkpt::pathtracer::SampleCounters read_counters() const override;
  vkpt::pathtracer::PathTracerStatus status() const override;
  void shutdown() override;
  const vkpt::pathtracer::FilmBuffer& film() const override;

 private:
  bool fail(const std::string& message) const;
  vkpt::core::Status status_from(int32_t code, const char* operation) const;

  vkptc_ctx* m_ctx = nullptr;
  vkpt::pathtracer::RenderSettings m_settings{};
  vkpt::pathtracer::FilmResolveSettings m_resolve{};
  mutable vkpt::pathtracer::FilmBuffer m_film;
  mutable std::string m_last_error;
  std::vector<vkpt::core::StableId> m_instance_entities;   // entity id per instance (update resolution)
  bool m_has_scene = false;
  // Why the next reset_accumulation clears the film (reported with the reset event).
  vkpt::pathtracer::PathTracerAccumulationResetReason m_next_reset_reason =
      vkpt::pathtracer::PathTracerAccumulationResetReason::External;
  uint64_t accumulation_gen() const;
  bool accel_valid() const;
  // The loaded scene's camera; a snapshot holding only it gives the
  // camera-adjusted film resolve settings after a camera update.
  vkpt::pathtracer::RTCameraState m_camera{};
  vkpt::pathtracer::PathTracerSceneSnapshot m_camera_scene{};

  friend struct BenchmarkAccess;
};

// What ptbench's `run` command (src/benchmark/BenchmarkRuntime.cpp:598-830) fills
// for a backend after its timed render loop, for the cuda backend.
struct CudaBenchmarkInputs {
  double render_ms = 0.0;          // the timed render loop (BenchmarkRuntime.cpp:680-695)
  double build_ms = 0.0;           // scene upload + acceleration build
  double total_ms = 0.0;
  // Roofline denominator of the traversal (the measured HBM copy bandwidth of
  // the device, GB/s); with collect_stats on, roofline_fraction = (128 B per
  // wide-node visit + 48 B per triangle test + 32 B per ray) / render time / it.
  double peak_bandwidth_gbs = 0.0;
  // Optional CPU reference film of the same scene, settings and seed, for
  // rmse= (relative RMSE of the per-pixel means) and bit_identical_frac=.
  const vkpt::pathtracer::FilmBuffer* reference = nullptr;
  // Optional, with `reference`: per pixel and channel the sum of the squared
  // per-sample radiance of the reference (3 floats per pixel), for
  // sigma3_fail_frac= (channels whose mean differs from the reference's by more
  // than 3 standard errors of the reference's own samples).
  const std::vector<float>* reference_m2 = nullptr;
  const char* renderer_path = "cuda-wavefront";   // or "cuda-persistent" for the batched renderer
};

// Fills backend, renderer_path, device_info, timing, throughput (paths_per_sec
// in ptbench's definition, counters.rays / render time, BenchmarkRuntime.cpp:762)
// and appends the backend's diagnostics:
//   renderer=, paths_per_sec_camera=, mrays_per_sec=, roofline_fraction=,
//   rmse=, sigma3_fail_frac=, bit_identical_frac= (the last three with a reference).
void FillBenchmarkResult(const CudaPathTracer& tracer, const CudaBenchmarkInputs& in,
                         vkpt::benchmark::BenchmarkResult& result);

}  // namespace vkpt::gpu::cuda
