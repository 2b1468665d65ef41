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
  uint32_t barrier_spins;         // bound of a grid-barrier wait, in ~128 ns sleeps
};

// Default bound of a grid-barrier wait: 2^26 sleeps of ~128 ns, about 8.6 s.
constexpr uint32_t kBatchBarrierSpins = 1u << 26;

struct BatchLaunch {
  int grid, block;
  int smem_entries, stack_cap, steps;
  int2* spill;
  int2* spill_shadow;   // loop driver: the shadow stage's own spill area (it may run beside EXTEND)
  cudaStream_t stream;
  bool parity;
  bool stats;   // count traversal work (node/leaf/triangle visits)
  bool effects; // some job has a material with a procedural effect (loop driver: shading variant)
  bool sdf;     // some job has SDF primitives (loop driver: the two SDF stages run)
  int occupancy;  // register-allocation variant: 0..3 = at least 1..4 resident 256-thread blocks per SM;
                  // 4 (loop driver only) = at least 7 resident 128-thread blocks per SM
                  // (the persistent kernel; in the loop driver, its two traversal stages)
  bool watertight;  // the jobs' triangle records hold vertices (watertight test)
  bool exotic;      // some job has a transmissive, clear-coat, sheen or toon material or an environment map
};

// Number of control words the pool needs; word kBatchCtlIterations holds the
// iteration count of the last run.
constexpr int kBatchCtlWords = 32;
constexpr int kBatchCtlIterations = 18;

#ifdef __CUDACC__
// Job of global path id g (jobs sorted by path_base).
__device__ __forceinline__ uint32_t find_job(const DevJob* jobs, uint32_t count, unsigned long long g) {
  uint32_t lo = 0u, hi = count;
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].path_base <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}
#endif

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
int BatchBlocksPerSm(int block, size_t smem, bool parity, bool stats, int occ, bool watertight = false);
cudaError_t ConfigureBatchSmem(size_t bytes);

// ------------------------------------------------------------ loop driver
// The same five stages as separate kernels (each with its own register
// budget and occupancy) in a CUDA graph while-node that the device keeps
// iterating until the work queue is empty (batch_loop.cu).  Path state lives
// in two compacted generations: the extension stage reads generation `cur`
// by position, shading appends surviving paths to the other generation,
// shadow queries to a queue that names their destination, and finished paths
// to a list the finish stage moves into the stagings -- every access is by
// queue position, so loads and stores coalesce.
struct PathSoA {
  uint32_t* job;
  uint32_t* local;                // sample_local * pixels + pixel
  uint32_t* depth;
  uint64_t* rng;
  float4* o;
  float4* d;
  float4* thr;
  float4* rad;                    // w = segments
};

struct LoopPool {
  uint32_t capacity;              // paths per generation ("queue capacity")
  PathSoA gen[2];
  float2* hit;                    // per position of the current generation
  float4* sh_o;                   // origin, max distance
  float4* sh_d;                   // direction, job (bits)
  float4* sh_c;                   // contribution when visible
  uint32_t* sh_dst;               // position in the next generation, or kLoopFinBit | finished-list position
  float4* fin_rad;
  uint32_t* fin_job;
  uint32_t* fin_local;
  uint32_t* ctl;                  // control words (kLoopCtl*)
};

constexpr uint32_t kLoopFinBit = 0x80000000u;
constexpr uint32_t kLoopDropDst = 0xFFFFFFFFu;   // shadow query an SDF occludes
constexpr int kLoopCtlWords = 32;
constexpr int kLoopCtlMore = 17;        // 1 while another iteration is needed
constexpr int kLoopCtlIterations = 18;  // iterations of the last run

struct LoopGrids {
  int regen, extend, shade, shadow, finish, sdf;
};
LoopGrids BatchLoopGrids(int block, size_t smem, bool parity, bool stats, int occupancy, int sm_count,
                         bool watertight = false, bool effects = true, bool sdf = true, bool exotic = true);
cudaError_t ConfigureBatchLoopSmem(size_t bytes);
cudaError_t LaunchBatchLoopInit(const LoopPool& pool, cudaStream_t stream);
// A second stream and two events: the shadow stage of an iteration (the
// previous shading stage's NEE queries) then runs beside REGEN and EXTEND.
struct LoopFork {
  cudaStream_t side;
  cudaEvent_t fork, join;
};
// One loop iteration: REGEN, EXTEND (+ SDF), the previous bounce's SHADOW
// (+ SDF occlusion), DRAIN (finished paths to stagings), SHADE, and the
// decision that sets `handle` (the graph's while-condition; 0 outside a graph)
// and ctl[kLoopCtlMore].  marks (optional, outside a graph; no fork then): 6
// events, interval k of them timing stage kLoopMarkStage[k].
constexpr int kLoopMarkStage[5] = {0, 1, 3, 4, 2};   // regen, extend, shadow, finish (drain), shade
cudaError_t LaunchBatchLoopIteration(const DevJob* jobs, uint32_t job_count, unsigned long long total,
                                     const LoopPool& pool, const BatchLaunch& bl, const LoopGrids& grids,
                                     cudaGraphConditionalHandle handle, DevCounters* ctr, uint32_t* err,
                                     cudaEvent_t* marks = nullptr, const LoopFork* fork = nullptr);

}  // namespace vkptc
