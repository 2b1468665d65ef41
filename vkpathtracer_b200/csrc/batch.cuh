// batch.cuh -- persistent batched renderer: many render jobs (each its own
// scene, resolution, spp and depth) in one cooperative persistent launch.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace vkptc {

// One render job as the device sees it.
struct DevJob {
  DevScene scene;
  DevSettings settings;
  unsigned long long path_base;   // first global path id of this job
  uint32_t pixels;                // width * height
  uint32_t spp;
  uint32_t first_sample;
  uint32_t pad;
  float4* staging;                // radiance (+ segment count in w) per (sample, pixel)
  Film film;
};

// Path-slot pool of the persistent renderer (structure of arrays).
struct BatchPool {
  uint32_t capacity;              // path slots ("queue capacity")
  uint32_t* job;                  // job of the path in the slot
  uint32_t* local;                // sample_local * pixels + pixel
  uint32_t* depth;
  uint64_t* rng;
  float4* ray_o;
  float4* ray_d;
  float4* thr;
  float4* rad;                    // w = segments
  float2* hit;
  uint32_t* ext[2];               // extension queues (slot ids)
  uint32_t* shq;                  // shadow queue (slot ids)
  float4* sh_o;                   // origin, max distance
  float4* sh_d;
  float4* sh_c;
  uint32_t* fin;                  // slots whose path ended this iteration
  uint32_t* freel;                // free slots
  uint32_t* ctl;                  // control words, see batch.cu
};

struct BatchLaunch {
  int grid, block;
  int smem_entries, stack_cap, steps;
  int2* spill;
  cudaStream_t stream;
  bool parity;
  bool stats;   // count traversal work (node/leaf/triangle visits)
  int occupancy;  // register-allocation variant: 0..3 = at least 1..4 resident 256-thread blocks per SM
                  // (the persistent kernel; in the loop driver, its two traversal stages)
};

// Number of control words the pool needs.
constexpr int kBatchCtlWords = 32;

// Runs every job to completion in one cooperative launch (fills the stagings),
// then accumulates each job's stagings into its film in sample order.
cudaError_t LaunchBatchPersistent(const DevJob* d_jobs, uint32_t job_count, unsigned long long total_paths,
                                  const BatchPool& pool, const BatchLaunch& bl, DevCounters* ctr, uint32_t* err);

// Accumulates one job's staging (spp x pixels) into its film, in sample order.
cudaError_t LaunchStagingAccumulate(const DevJob* d_jobs, uint32_t job_count, unsigned long long total_pixels,
                                    cudaStream_t stream, DevCounters* ctr);

// Resets the pool (all slots free, queues and counters zero).
cudaError_t LaunchBatchInit(const BatchPool& pool, cudaStream_t stream);

// Resident blocks per SM of the persistent batch kernel.
int BatchBlocksPerSm(int block, size_t smem, bool parity, bool stats, int occupancy);
cudaError_t ConfigureBatchSmem(size_t bytes);

// Device-driven loop: the same five stages as separate kernels (each with its
// own register budget and occupancy), one iteration enqueued per call; the
// finish stage sets `handle` (a graph while-condition; 0 outside a graph) and
// the pool's "iterate again" word.  Grids are resident blocks x SMs.
struct LoopGrids {
  int regen, extend, shade, shadow, finish;
};
LoopGrids BatchLoopGrids(int block, size_t smem, bool parity, bool stats, int occupancy, int sm_count);
cudaError_t ConfigureBatchLoopSmem(size_t bytes);
// marks (optional, outside a graph): 6 events recorded around the five stages.
cudaError_t LaunchBatchLoopIteration(const DevJob* jobs, uint32_t job_count, unsigned long long total,
                                     const BatchPool& pool, const BatchLaunch& bl, const LoopGrids& grids,
                                     cudaGraphConditionalHandle handle, DevCounters* ctr, uint32_t* err,
                                     cudaEvent_t* marks = nullptr);
// Words of BatchPool::ctl: "iterate again" (set by the loop's finish stage)
// and the iteration count of the last run (both drivers).
constexpr int kBatchCtlMore = 17;
constexpr int kBatchCtlIterations = 18;

}  // namespace vkptc
