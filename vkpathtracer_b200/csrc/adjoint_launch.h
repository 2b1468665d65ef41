// adjoint_launch.h -- launch interface of the differentiable-rendering kernels
// (adjoint.cu).  One forward renders `spp` samples of every pixel with one
// path per thread and keeps each sample's radiance; the loss kernel forms the
// image, the mean-squared-error loss (FP64 reduction) and the per-pixel
// adjoint; the backward replays every path from its RNG key and runs the
// reverse sweep over its vertices.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace vkptc {

struct AdjLaunch {
  int grid, block;
  int grid_reverse;       // the backward's reverse-sweep kernel (its own occupancy)
  int stack_cap;          // traversal stack entries per thread (all in shared memory)
  uint32_t spp, first_sample;
  bool parity;
  cudaStream_t stream;
};

// Path radiance of every (sample, pixel): rad[s * W*H + y*W + x] = rgb, and
// in w the bits of a 32-bit hash of the path's discrete decisions.
// mat0 (16 floats per material) drives the Russian-roulette probabilities
// and decisions; pass the scene's own table for the ordinary estimator.
// recs and nrec (optional; at most kAdjChunkPaths paths): every path's vertex
// records in the backward's layout (all paths one chunk) and their count, so
// that a backward over the same paths skips its replay.
cudaError_t LaunchAdjForward(const DevScene& s, const DevSettings& st, const float* mat0, const AdjLaunch& l,
                             float4* rad, uint32_t* err, float4* recs = nullptr, uint32_t* nrec = nullptr);

// Image (sample-order accumulation exactly as the film does), loss partials
// per block, and the per-pixel adjoint dL/d(sample radiance) (0 without a target).
cudaError_t LaunchAdjLoss(const DevSettings& st, uint32_t spp, const float4* rad, const float* target, float* image,
                          float4* adj, double* loss_part, double* loss, int grid, cudaStream_t stream);

// Paths per backward chunk: the replay writes kAdjRecordFloat4s float4 per
// path and vertex slot for the chunk, the reverse sweep reads them.
constexpr uint64_t kAdjChunkPaths = 1ull << 20;
constexpr size_t kAdjRecordFloat4s = 4;     // one vertex record: 4 float4 (64 bytes)
constexpr size_t kAdjVertexSlots = 8;       // records per path (the maximum depth)

// Backward: per chunk of paths the replay (records to recs, kAdjVertexSlots *
// kAdjRecordFloat4s float4 per chunk path, and the radiance adjoint to gout,
// one float4 per chunk path) then the reverse sweep, whose per-block gradient
// partials grad_part[block][7 * materials] add up over the chunks; then the
// fixed-order reduction into grad (7 floats per material).  path_weight
// (optional, one per path) scales each path's adjoint.  The paths replayed
// are those of st.frame (the forward's, or independent ones).  fwd_rad and
// fwd_nrec (optional): the radiance and record counts of a forward that
// recorded these same paths into recs; the replay is then skipped.
cudaError_t LaunchAdjBackward(const DevScene& s, const DevSettings& st, const float* mat0, const AdjLaunch& l,
                              const float4* adj, const float* path_weight, float4* recs, float4* gout,
                              float* grad_part, float* grad, uint32_t* err, const float4* fwd_rad = nullptr,
                              const uint32_t* fwd_nrec = nullptr);

enum class AdjKernel { kForward, kReplay, kReverse };
size_t AdjBackwardSmem(int block, int stack_cap, uint32_t materials);
size_t AdjReverseSmem(int block, uint32_t materials);
size_t AdjForwardSmem(int block, int stack_cap);
int AdjBlocksPerSm(AdjKernel k, int block, size_t smem, bool parity);
cudaError_t ConfigureAdjSmem(size_t bytes);

}  // namespace vkptc
