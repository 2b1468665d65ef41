// kernels.cuh -- launch interface of the wavefront render and ray-query kernels.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace vkptc {

// Queue and path-state buffers of one wave (structure of arrays, indexed by
// path slot).  A wave is `sample_count` samples of every pixel of one
// rectangular tile: slot = sample_local * tile_pixels + pixel_local.
struct WaveState {
  // path state
  uint64_t* rng;
  float4* ray_o;      // origin xyz
  float4* ray_d;      // direction xyz
  float4* thr;        // throughput xyz
  float4* rad;        // radiance xyz, w = segment count
  float2* hit;        // t, primitive index bits
  // shadow queries
  uint32_t* sh_path;
  float4* sh_o;       // origin xyz, w = max distance
  float4* sh_d;       // direction xyz
  float4* sh_c;       // contribution to add when visible
  // queues: q[0], q[1] ping-pong extension queues; counts[0..1] their sizes,
  // counts[2] the shadow queue size
  uint32_t* q[2];
  uint32_t* counts;
  uint32_t capacity;
};

struct WaveTile {
  uint32_t x, y, w, h;     // pixel rectangle
  uint32_t first_sample, sample_count;
};

struct Film {
  float4* sum;           // rgb sum per pixel
  uint32_t* count;
  float* invalid;
  uint32_t width, height;
};

struct DevCounters {
  unsigned long long samples, rays, shadow_tests, dropped;
  unsigned long long nodes, leaves, tris;
  unsigned long long shadow_nodes, shadow_leaves, shadow_tris;
  unsigned long long ext_rays, shadow_rays;   // traversal queries issued (stats mode)
  unsigned long long sdf_tests, sdf_steps, sdf_hits;
};

struct LaunchShape {
  int grid;           // resident blocks x SMs (the traversal kernels are persistent)
  int block;
  int stack_cap;      // traversal stack entries per thread (worst case of the BVH)
  int smem_entries;   // of which held in shared memory; the rest spill to `spill`
  int steps;          // traversal steps between warp refills
  int2* spill;        // grid*block*(stack_cap - smem_entries) entries, or null
  cudaStream_t stream;
};

size_t StackSmemBytes(int block, int cap);
// Spill entries the launch needs beyond shared memory.
size_t SpillEntries(const LaunchShape& ls);
// Resident blocks per SM of the traversal stage for this block size and stack.
int ExtendBlocksPerSm(int block, size_t smem, bool watertight = false);
// Raises the dynamic shared-memory limit of every stack-using kernel.
cudaError_t ConfigureStackSmem(size_t bytes);

// Ray queries over one scene (rays: 6 floats each).
// `fetch` is a device counter the persistent kernel claims query ids from.
cudaError_t LaunchTraceRays(const DevScene& s, const float* rays, const float* tmax, uint64_t n, bool any_hit,
                            uint32_t* prim_out, float* t_out, const LaunchShape& ls, DevCounters* ctr,
                            uint32_t* err, uint32_t* fetch);

// Optional per-stage event timing: pairs of events recorded around each launch.
struct StageTimer {
  static constexpr int kStages = 5;   // raygen, extend, shade, shadow, accumulate
  cudaEvent_t* events = nullptr;      // pool of event pairs
  int capacity = 0;                   // pairs
  int used = 0;
  int stage_of[4096];
  void begin(int stage, cudaStream_t s) {
    if (!events || used >= capacity) return;
    stage_of[used] = stage;
    cudaEventRecord(events[2 * used], s);
  }
  void end(cudaStream_t s) {
    if (!events || used >= capacity) return;
    cudaEventRecord(events[2 * used + 1], s);
    ++used;
  }
};

// One wave: raygen, max_depth x (extend, shade, shadow), accumulate.
cudaError_t LaunchWave(const DevScene& s, const DevSettings& st, const WaveState& w, const WaveTile& tile,
                       const Film& film, bool parity, bool stats, const LaunchShape& ls, DevCounters* ctr,
                       uint32_t* err, StageTimer* timer);

// Film helpers.
cudaError_t LaunchResolveHdr(const Film& film, float* rgb_out, cudaStream_t stream);
// The film's rgb sums packed to 3 floats per pixel (for host readback).
cudaError_t LaunchPackFilm(const Film& film, float* rgb_out, cudaStream_t stream);

// Scene deltas: the material word (w) of the shading records of whole
// instances.  ranges: per changed instance (first primitive, primitive count,
// material index, 0), device memory; the ranges do not overlap.
cudaError_t LaunchSetInstanceMaterials(float4* shade, const uint4* ranges, uint32_t range_count, cudaStream_t stream);

// ApplyFilmResolve on the device; wb: the white-balance scale (host-computed).
struct LdrResolve {
  float exposure, wb[3], gamma;
  uint32_t tone_map, output_transform, clamp_output;
};
cudaError_t LaunchResolveLdr(const Film& film, const LdrResolve& rs, bool parity, uint8_t* rgba_out,
                             cudaStream_t stream);

// Bandwidth probe: `reps` passes of 16-byte reads over `bytes` of `buf`
// (a multiple of 16), grid-strided, cached in L2 only (ld.global.cg), so a
// buffer well under the L2 size measures L2 bandwidth and one far above it
// HBM read bandwidth.  sink receives nothing unless the sum is impossible.
cudaError_t LaunchReadProbe(const float4* buf, size_t bytes, uint32_t reps, int grid, float* sink,
                            cudaStream_t stream);

}  // namespace vkptc
