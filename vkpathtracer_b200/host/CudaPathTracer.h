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
};

}  // namespace vkpt::gpu::cuda
