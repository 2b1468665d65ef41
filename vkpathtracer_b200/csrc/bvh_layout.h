// bvh_layout.h -- constants of the wide-node layout shared by the builders
// (host and device) and the traversal kernels.
#pragma once

#include <cstdint>

namespace vkptc {

// Child ref of an unused wide-node slot.  A leaf ref is ~((first << 3) |
// (count - 1)); INT32_MIN = ~0x7FFFFFFF would be the leaf of 8 triangles
// starting at 2^28 - 1, which no scene below kMaxTriangles has.
constexpr int32_t kEmptyChild = INT32_MIN;
constexpr uint64_t kMaxTriangles = (1ull << 28) - 8u;

}  // namespace vkptc
