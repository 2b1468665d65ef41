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

// What a refit after instance transform updates needs, kept on the device
// when the scene has dynamic-transform instances with local geometry.
struct DeviceRefitState {
  float4* blo = nullptr;            // per primitive: padded box
  float4* bhi = nullptr;
  uint32_t* tri_pos = nullptr;      // per primitive: its triangle record
  BinNode* trav_nodes = nullptr;    // the traversal tree when it is not the reference tree (SAH)
  uint32_t* trav_order = nullptr;
  int32_t* trav_parent = nullptr;
  uint32_t trav_count = 0;
  int32_t* slot_bin = nullptr;      // per wide node: the binary node of each slot (-1 unused)
  uint32_t* inst_first = nullptr;   // per instance: first flattened primitive (host copy below)
  std::vector<uint32_t> host_inst_first, host_inst_count;   // per instance: primitive range
  bool watertight = false;          // triangle records hold the vertices (a, b, c)
};

struct DeviceAccelOut {
  // Device arrays from the builder's stream-ordered pool (the caller frees
  // them with FreeAccelArray, FreeDeviceAccel or FreeRefitState).
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
  std::vector<uint32_t> inst_first;    // per instance and one past the last: its first flattened primitive
  DeviceRefitState* refit = nullptr;   // kept for dynamic-instance scenes (owned; FreeDeviceAccel frees)
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
  bool watertight = false;    // triangle records for the watertight test: vertices (a, b, c) in the
                              // slots of (v0, e1, e2)
};

// Builds everything from the scene arrays.  sah: the traversal tree is a
// binned-SAH tree instead of the reference tree.  Returns a CUDA error; on
// fallback, nothing is allocated.
cudaError_t BuildAccelOnDevice(const DeviceSceneArrays& scene, bool sah, cudaStream_t stream, DeviceAccelOut& out);

// Stream-ordered frees of the builder's arrays: after the work already queued
// on `stream`, back into the pool (no device-wide synchronisation).
void FreeAccelArray(void* p, cudaStream_t stream);
// Returns the freed memory the build pool of the current device keeps mapped
// to the driver (after the device's pending work); the library calls it when
// the last context on a device is destroyed.
void TrimBuildPool();
void FreeDeviceAccel(DeviceAccelOut& out, cudaStream_t stream = nullptr);
void FreeRefitState(DeviceRefitState*& state, cudaStream_t stream = nullptr);

// One instance transform update, resolved to an instance of the scene.
struct RefitUpdate {
  uint32_t instance;
  uint32_t prim_first, prim_count;             // its flattened primitives
  uint32_t local_first_vertex, local_first_index, material;
  float transform[10];                         // translation3, quaternion xyzw, scale3
};

// The refit of CpuBvhAccelerator::apply_instance_transform_update
// (src/pathtracer/CpuBvhAccelerator.cpp:308-358, 527-606): the updated
// instances' primitives recomputed from their local geometry, then every node
// of the reference tree (and of the traversal tree when it differs) refitted
// bottom-up with its topology unchanged, and the wide nodes' slot bounds and
// tie records rewritten.  nodes/tris/tie/shade: the accelerator's arrays.
cudaError_t RefitOnDevice(DeviceRefitState& state, const std::vector<RefitUpdate>& updates, const float* local_vertices,
                          const uint32_t* local_indices, BinNode* ref_nodes, const uint32_t* ref_order,
                          uint32_t ref_count, float4* nodes, uint32_t wide_count, float4* tris, float4* tie,
                          float4* shade, cudaStream_t stream);

}  // namespace vkptc
