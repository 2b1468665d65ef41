// bvh_build.h -- the acceleration structure built on the device.
//
// Produces the same arrays as the host path (FlattenScene, BuildBinaryBvh,
// BuildSahBvh, CollapseToWide in bvh_host.h): flattened primitives, the
// reference's binary midpoint tree (bit-identical node bounds, children,
// leaf ranges and primitive order -- the tie rule of the traversal depends on
// it), optionally a binned-SAH traversal tree, and the 128-byte wide nodes,
// triangle records and tie records the traversal kernels read.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "bvh_host.h"

namespace vkptc {

struct DeviceAccelOut {
  // Device arrays allocated by the builder with cudaMalloc (caller frees).
  float4* nodes = nullptr;     // WideNode, 8 float4 each
  float4* tris = nullptr;      // TriRecord, 3 float4 each
  float4* tie = nullptr;       // TieNode, 2 float4 each
  float4* shade = nullptr;     // per primitive: normal xyz, material bits
  BinNode* ref_nodes = nullptr;     // the reference binary tree (final ids)
  uint32_t* ref_order = nullptr;    // its primitive order
  uint32_t prim_count = 0;
  uint32_t binary_nodes = 0, binary_leaves = 0;
  uint32_t wide_nodes = 0, depth = 0, stack_required = 0;
  bool reference_topology = true;
  bool fallback = false;       // non-finite primitive bounds: use the host builder instead
};

// The scene's geometry arrays: vertex and index arrays (global and local) in
// device memory, the per-instance tables on the host.
struct DeviceSceneArrays {
  const float* vertices = nullptr;
  uint32_t vertex_count = 0;
  const uint32_t* indices = nullptr;
  uint32_t index_count = 0;
  const float* local_vertices = nullptr;      // dynamic instances (may be null)
  uint32_t local_vertex_count = 0;
  const uint32_t* local_indices = nullptr;
  uint32_t local_index_count = 0;
  const uint32_t* instances = nullptr;        // host: first_triangle, triangle_count, material
  uint32_t instance_count = 0;
  const uint32_t* instance_local = nullptr;   // host, 5 per instance (see InstanceGeometry), or null
  const float* instance_transforms = nullptr; // host, 10 per instance, or null
};

// Builds everything from the scene arrays.  sah: the traversal tree is a
// binned-SAH tree instead of the reference tree.  Returns a CUDA error; on
// fallback, nothing is allocated.
cudaError_t BuildAccelOnDevice(const DeviceSceneArrays& scene, bool sah, cudaStream_t stream, DeviceAccelOut& out);

void FreeDeviceAccel(DeviceAccelOut& out);

}  // namespace vkptc
