// bvh_host.h -- host side of the acceleration structure: primitive flattening,
// the binary midpoint BVH, and its collapse into the 128-byte wide-node layout
// that the sm_100a traversal kernels read from HBM.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "bvh_layout.h"

namespace vkptc {

struct HostPrim {
  float v0[3], e1[3], e2[3], n[3];
  uint32_t material;
};

struct BinNode {
  float lo[3], hi[3];
  int32_t left, right, first, count;
};

// Wide node: six float4 of child bounds as SoA (lo.x[4], hi.x[4], lo.y[4],
// hi.y[4], lo.z[4], hi.z[4]), then int4 child refs, then int4 meta
// (x = valid child count).  Child ref >= 0: wide node index; < 0: leaf,
// ~ref = (first_triangle << 3) | (count - 1); kEmptyChild: an unused slot
// (so the traversal needs no child count).  128 bytes, one cache line.
struct alignas(16) WideNode {
  float lox[4], hix[4], loy[4], hiy[4], loz[4], hiz[4];
  int32_t child[4];
  int32_t meta[4];
};
static_assert(sizeof(WideNode) == 128, "wide node must be one 128-byte line");

// Triangle record in leaf order: v0, e1, e2, then the reference primitive
// index, the binary leaf that holds it and its lane in that leaf (the last
// two resolve exact-distance ties in the reference's visiting order).
struct alignas(16) TriRecord {
  float v0x, v0y, v0z, e1x;
  float e1y, e1z, e2x, e2y;
  float e2z;
  uint32_t prim;
  uint32_t leaf;
  uint32_t lane;
};
static_assert(sizeof(TriRecord) == 48, "triangle record must be 48 bytes");

// Binary node record for tie resolution: lo3 + parent, hi3 + depth.
struct alignas(16) TieNode {
  float lox, loy, loz;
  int32_t parent;
  float hix, hiy, hiz;
  int32_t depth;
};

struct SceneGeometry {
  std::vector<HostPrim> prims;        // accelerator order (RayQueryHit::primitive_index)
  std::vector<float> boxes;           // 6 floats per prim: lo3, hi3 (padded by 1e-4)
  std::vector<uint32_t> inst_first, inst_count;   // per instance: its flattened primitives
};

struct WideBvh {
  std::vector<WideNode> nodes;
  std::vector<TriRecord> tris;
  std::vector<TieNode> tie_nodes;
  uint32_t binary_nodes = 0;
  uint32_t binary_leaves = 0;
  uint32_t depth = 0;
  uint32_t stack_required = 0;
  bool reference_topology = true;   // traversal tree == reference tree
};

// Dynamic-transform instances: local geometry and per-instance transforms
// (all null when the scene has none).
struct InstanceGeometry {
  const uint32_t* instance_local = nullptr;       // 5 per instance: flags, local first/count vertex, first/count index
  const float* instance_transforms = nullptr;     // 10 per instance: translation3, quaternion xyzw, scale3
  const float* local_vertices = nullptr;
  uint32_t local_vertex_count = 0;
  const uint32_t* local_indices = nullptr;
  uint32_t local_index_count = 0;
};

// A world-space vertex of a dynamic instance: scale, normalized-quaternion
// rotation, translation (transform_instance_vertex and rotate_quat,
// src/pathtracer/CpuBvhAccelerator.cpp:47-74).
void TransformInstanceVertex(const float* local, const float* transform, float out[3]);

// Flattens instances x triangles in the accelerator's order, skipping
// triangles with out-of-range indices (src/pathtracer/CpuBvhAccelerator.cpp:173-247).
bool FlattenScene(const float* vertices, uint32_t vertex_count, const uint32_t* indices,
                  uint32_t index_count, const uint32_t* instances, uint32_t instance_count,
                  SceneGeometry& out, std::string& error, const InstanceGeometry* dyn = nullptr);

// Binary BVH: widest-centroid-axis midpoint split, stable partition,
// count/2 fallback, leaves of <= leaf_threshold primitives, child ids
// allocated pairwise in recursion order (src/cpu/ParallelBvhBuilder.cpp:61-257).
void BuildBinaryBvh(const SceneGeometry& geo, uint32_t leaf_threshold, std::vector<BinNode>& nodes,
                    std::vector<uint32_t>& prim_indices);

// Binned-SAH binary BVH over the same padded primitive boxes (32 bins per
// axis, leaves of <= max_leaf primitives).  Used only as the traversal tree:
// hit ids stay the reference's because ties and the parallel-axis rule are
// resolved against the reference tree (see CollapseToWide).
void BuildSahBvh(const SceneGeometry& geo, uint32_t max_leaf, std::vector<BinNode>& nodes,
                 std::vector<uint32_t>& prim_indices);

// Validates an externally supplied binary BVH against the primitive count.
bool ValidateBinaryBvh(const std::vector<BinNode>& nodes, const std::vector<uint32_t>& prim_indices,
                       size_t prim_count, std::string& error);

// Collapses a binary traversal tree into the wide layout.  Each wide child
// slot is a binary node with its exact float bounds; leaves stay whole binary
// leaves.  Triangle records and tie nodes come from the REFERENCE tree
// (ref_nodes / ref_prims): each triangle carries its reference leaf and lane,
// so exact-distance ties and the parallel-axis rule follow the reference even
// when the traversal tree is a different one.
void CollapseToWide(const SceneGeometry& geo, const std::vector<BinNode>& nodes,
                    const std::vector<uint32_t>& prim_indices, const std::vector<BinNode>& ref_nodes,
                    const std::vector<uint32_t>& ref_prims, WideBvh& out);

}  // namespace vkptc
