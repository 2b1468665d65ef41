// bvh_host.cpp -- primitive flattening, binary midpoint BVH, wide collapse.
//
// The binary builder must produce the same tree as the reference's
// ParallelBvhBuilder in deterministic mode (src/cpu/ParallelBvhBuilder.cpp:61-257):
// the traversal kernels reproduce the reference's closest-hit primitive ids
// bit-exactly, and on exact distance ties that needs the reference's tree
// (its depth-first near-first visiting order).  The steps are therefore the
// reference's: node bounds = union of primitive boxes; split the widest
// centroid axis at its midpoint; stable-partition by `centroid < split`;
// fall back to count/2 when one side is empty; leaves hold <= 4 primitives;
// child ids are allocated as (left, right) pairs in recursion order.
#include "bvh_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>

namespace vkptc {
namespace {

constexpr float kPad = 1e-4f;

inline float lt_max(float a, float b) { return (a < b) ? b : a; }   // std::max order
inline float lt_min(float a, float b) { return (b < a) ? b : a; }   // std::min order

struct Builder {
  const float* boxes;   // 6 per prim
  std::vector<BinNode>* nodes;
  uint32_t* base;
  uint32_t leaf_threshold;
  int32_t next_id = 1;

  float centroid(uint32_t p, int axis) const {
    return 0.5f * (boxes[6 * p + axis] + boxes[6 * p + 3 + axis]);
  }

  void build(int32_t id, uint32_t* idx, size_t n) {
    BinNode& nd0 = (*nodes)[static_cast<size_t>(id)];
    for (int a = 0; a < 3; ++a) {
      nd0.lo[a] = std::numeric_limits<float>::max();
      nd0.hi[a] = -std::numeric_limits<float>::max();
    }
    for (size_t i = 0; i < n; ++i) {
      const float* b = boxes + 6 * idx[i];
      for (int a = 0; a < 3; ++a) {
        nd0.lo[a] = lt_min(nd0.lo[a], b[a]);
        nd0.hi[a] = lt_max(nd0.hi[a], b[3 + a]);
      }
    }
    if (n <= leaf_threshold) {
      nd0.left = nd0.right = -1;
      nd0.first = static_cast<int32_t>(idx - base);
      nd0.count = static_cast<int32_t>(n);
      return;
    }
    float clo[3], chi[3];
    for (int a = 0; a < 3; ++a) {
      clo[a] = std::numeric_limits<float>::max();
      chi[a] = -std::numeric_limits<float>::max();
    }
    for (size_t i = 0; i < n; ++i) {
      for (int a = 0; a < 3; ++a) {
        const float c = centroid(idx[i], a);
        clo[a] = lt_min(clo[a], c);
        chi[a] = lt_max(chi[a], c);
      }
    }
    int axis = 0;
    float widest = chi[0] - clo[0];
    for (int a = 1; a < 3; ++a) {
      const float e = chi[a] - clo[a];
      if (e > widest) {
        widest = e;
        axis = a;
      }
    }
    const float split = 0.5f * (clo[axis] + chi[axis]);
    uint32_t* mid = std::stable_partition(idx, idx + n, [&](uint32_t p) { return centroid(p, axis) < split; });
    size_t left_n = static_cast<size_t>(mid - idx);
    if (left_n == 0 || left_n == n) left_n = n / 2;
    const int32_t l = next_id++;
    const int32_t r = next_id++;
    BinNode& nd = (*nodes)[static_cast<size_t>(id)];
    nd.left = l;
    nd.right = r;
    nd.first = -1;
    nd.count = 0;
    build(l, idx, left_n);
    build(r, idx + left_n, n - left_n);
  }
};

float surface_area(const BinNode& n) {
  const float dx = n.hi[0] - n.lo[0], dy = n.hi[1] - n.lo[1], dz = n.hi[2] - n.lo[2];
  return dx * dy + dy * dz + dz * dx;
}

}  // namespace

void TransformInstanceVertex(const float* local, const float* tr, float out[3]) {
  const float sx = local[0] * tr[7], sy = local[1] * tr[8], sz = local[2] * tr[9];
  float rx = sx, ry = sy, rz = sz;
  const float len_sq = tr[3] * tr[3] + tr[4] * tr[4] + tr[5] * tr[5] + tr[6] * tr[6];
  if (!(len_sq <= kPad * kPad)) {
    const float inv_len = 1.0f / std::sqrt(len_sq);
    const float qx = tr[3] * inv_len, qy = tr[4] * inv_len, qz = tr[5] * inv_len;
    const float qw = tr[6] * inv_len;
    // t = 2 * cross(q, v); v + t * qw + cross(q, t)
    const float tx = (qy * sz - qz * sy) * 2.0f;
    const float ty = (qz * sx - qx * sz) * 2.0f;
    const float tz = (qx * sy - qy * sx) * 2.0f;
    const float cx = qy * tz - qz * ty;
    const float cy = qz * tx - qx * tz;
    const float cz = qx * ty - qy * tx;
    rx = (sx + tx * qw) + cx;
    ry = (sy + ty * qw) + cy;
    rz = (sz + tz * qw) + cz;
  }
  out[0] = rx + tr[0];
  out[1] = ry + tr[1];
  out[2] = rz + tr[2];
}

bool FlattenScene(const float* vertices, uint32_t vertex_count, const uint32_t* indices, uint32_t index_count,
                  const uint32_t* instances, uint32_t instance_count, SceneGeometry& out, std::string& error,
                  const InstanceGeometry* dyn) {
  out.prims.clear();
  out.boxes.clear();
  out.inst_first.clear();
  out.inst_count.clear();
  if (instance_count > 0 && instances == nullptr) {
    error = "instances pointer is null";
    return false;
  }
  size_t capacity = 0;
  for (uint32_t i = 0; i < instance_count; ++i) capacity += instances[3 * i + 1];
  out.prims.reserve(capacity);
  out.boxes.reserve(6 * capacity);
  const bool has_dyn = dyn && dyn->instance_local && dyn->instance_transforms;
  for (uint32_t i = 0; i < instance_count; ++i) {
    const uint32_t first = instances[3 * i], count = instances[3 * i + 1], mat = instances[3 * i + 2];
    out.inst_first.push_back(static_cast<uint32_t>(out.prims.size()));
    const uint32_t* loc = has_dyn ? dyn->instance_local + 5 * static_cast<size_t>(i) : nullptr;
    const bool use_local = loc && (loc[0] & 1u) != 0u && loc[2] > 0u && loc[4] > 0u;
    for (uint32_t k = 0; k < count; ++k) {
      float la[3], lb[3], lc[3];
      const float *a = nullptr, *b = nullptr, *c = nullptr;
      if (use_local) {
        // 32-bit index arithmetic, as the accelerator's
        const uint32_t local_base = loc[3] + k * 3u;
        const uint32_t local_end = loc[1] + loc[2];
        // (a wrapped local_base + 2 would make the reference read out of range: skipped here)
        if (local_base < 0xFFFFFFFEu && local_base + 2u < dyn->local_index_count) {
          const uint32_t l0 = dyn->local_indices[local_base], l1 = dyn->local_indices[local_base + 1u],
                         l2 = dyn->local_indices[local_base + 2u];
          const uint32_t v0 = loc[1] + l0, v1 = loc[1] + l1, v2 = loc[1] + l2;
          if (v0 < local_end && v1 < local_end && v2 < local_end && v0 < dyn->local_vertex_count &&
              v1 < dyn->local_vertex_count && v2 < dyn->local_vertex_count) {
            const float* tr = dyn->instance_transforms + 10 * static_cast<size_t>(i);
            TransformInstanceVertex(dyn->local_vertices + 3 * static_cast<size_t>(v0), tr, la);
            TransformInstanceVertex(dyn->local_vertices + 3 * static_cast<size_t>(v1), tr, lb);
            TransformInstanceVertex(dyn->local_vertices + 3 * static_cast<size_t>(v2), tr, lc);
            a = la;
            b = lb;
            c = lc;
          }
        }
      }
      if (!a) {
        const uint32_t base = (first + k) * 3u;   // 32-bit, as the accelerator's
        if (base >= 0xFFFFFFFEu || base + 2u >= index_count) continue;
        const uint32_t ia = indices[base], ib = indices[base + 1u], ic = indices[base + 2u];
        if (ia >= vertex_count || ib >= vertex_count || ic >= vertex_count) continue;
        a = vertices + 3 * static_cast<size_t>(ia);
        b = vertices + 3 * static_cast<size_t>(ib);
        c = vertices + 3 * static_cast<size_t>(ic);
      }
      HostPrim p;
      for (int ax = 0; ax < 3; ++ax) {
        p.v0[ax] = a[ax];
        p.e1[ax] = b[ax] - a[ax];
        p.e2[ax] = c[ax] - a[ax];
      }
      // Geometric normal: cross(e1, e2) times 1/sqrt(|.|^2), (0,1,0) when degenerate
      // (normalize_vec3 in src/pathtracer/CpuBvhAccelerator.cpp:75-82).
      const float cx = p.e1[1] * p.e2[2] - p.e1[2] * p.e2[1];
      const float cy = p.e1[2] * p.e2[0] - p.e1[0] * p.e2[2];
      const float cz = p.e1[0] * p.e2[1] - p.e1[1] * p.e2[0];
      const float l2 = cx * cx + cy * cy + cz * cz;
      if (l2 <= kPad * kPad) {
        p.n[0] = 0.0f;
        p.n[1] = 1.0f;
        p.n[2] = 0.0f;
      } else {
        const float inv = 1.0f / std::sqrt(l2);
        p.n[0] = cx * inv;
        p.n[1] = cy * inv;
        p.n[2] = cz * inv;
      }
      p.material = mat;
      out.prims.push_back(p);
      for (int ax = 0; ax < 3; ++ax) out.boxes.push_back(std::min({a[ax], b[ax], c[ax]}) - kPad);
      for (int ax = 0; ax < 3; ++ax) out.boxes.push_back(std::max({a[ax], b[ax], c[ax]}) + kPad);
    }
    out.inst_count.push_back(static_cast<uint32_t>(out.prims.size()) - out.inst_first.back());
  }
  return true;
}

void BuildBinaryBvh(const SceneGeometry& geo, uint32_t leaf_threshold, std::vector<BinNode>& nodes,
                    std::vector<uint32_t>& prim_indices) {
  const size_t n = geo.prims.size();
  nodes.clear();
  prim_indices.clear();
  if (n == 0) return;
  nodes.assign(2 * n - 1, BinNode{});
  prim_indices.resize(n);
  std::iota(prim_indices.begin(), prim_indices.end(), 0u);
  Builder b{geo.boxes.data(), &nodes, prim_indices.data(), leaf_threshold == 0 ? 4u : leaf_threshold};
  b.build(0, prim_indices.data(), n);
  nodes.resize(static_cast<size_t>(b.next_id));
}

namespace {

struct SahBuilder {
  const float* boxes;
  std::vector<BinNode>* nodes;
  uint32_t* base;
  uint32_t max_leaf;
  static constexpr int kBins = 32;

  static float area(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
  }

  int32_t build(uint32_t* idx, size_t n) {
    const int32_t id = static_cast<int32_t>(nodes->size());
    nodes->push_back(BinNode{});
    float lo[3], hi[3], clo[3], chi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = clo[a] = std::numeric_limits<float>::max();
      hi[a] = chi[a] = -std::numeric_limits<float>::max();
    }
    for (size_t i = 0; i < n; ++i) {
      const float* b = boxes + 6 * idx[i];
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], b[a]);
        hi[a] = std::max(hi[a], b[3 + a]);
        const float c = 0.5f * (b[a] + b[3 + a]);
        clo[a] = std::min(clo[a], c);
        chi[a] = std::max(chi[a], c);
      }
    }
    auto make_leaf = [&]() {
      BinNode& nd = (*nodes)[static_cast<size_t>(id)];
      std::memcpy(nd.lo, lo, sizeof(lo));
      std::memcpy(nd.hi, hi, sizeof(hi));
      nd.left = nd.right = -1;
      nd.first = static_cast<int32_t>(idx - base);
      nd.count = static_cast<int32_t>(n);
      return id;
    };
    if (n <= max_leaf) return make_leaf();
    // Best binned split over the three axes.
    int best_axis = -1, best_bin = -1;
    float best_cost = std::numeric_limits<float>::max();
    for (int a = 0; a < 3; ++a) {
      const float ext = chi[a] - clo[a];
      if (!(ext > 0.0f)) continue;
      const float scale = kBins / ext;
      uint32_t cnt[kBins] = {};
      float blo[kBins][3], bhi[kBins][3];
      for (int k = 0; k < kBins; ++k)
        for (int q = 0; q < 3; ++q) {
          blo[k][q] = std::numeric_limits<float>::max();
          bhi[k][q] = -std::numeric_limits<float>::max();
        }
      for (size_t i = 0; i < n; ++i) {
        const float* b = boxes + 6 * idx[i];
        const float c = 0.5f * (b[a] + b[3 + a]);
        int k = static_cast<int>((c - clo[a]) * scale);
        k = std::min(kBins - 1, std::max(0, k));
        ++cnt[k];
        for (int q = 0; q < 3; ++q) {
          blo[k][q] = std::min(blo[k][q], b[q]);
          bhi[k][q] = std::max(bhi[k][q], b[3 + q]);
        }
      }
      // Sweep: right-side areas, then left.
      float rarea[kBins];
      uint32_t rcnt[kBins];
      float rlo[3], rhi[3];
      for (int q = 0; q < 3; ++q) {
        rlo[q] = std::numeric_limits<float>::max();
        rhi[q] = -std::numeric_limits<float>::max();
      }
      uint32_t rc = 0;
      for (int k = kBins - 1; k > 0; --k) {
        rc += cnt[k];
        for (int q = 0; q < 3; ++q) {
          rlo[q] = std::min(rlo[q], blo[k][q]);
          rhi[q] = std::max(rhi[q], bhi[k][q]);
        }
        rcnt[k] = rc;
        rarea[k] = rc ? area(rlo, rhi) : 0.0f;
      }
      float llo[3], lhi[3];
      for (int q = 0; q < 3; ++q) {
        llo[q] = std::numeric_limits<float>::max();
        lhi[q] = -std::numeric_limits<float>::max();
      }
      uint32_t lc = 0;
      for (int k = 0; k < kBins - 1; ++k) {
        lc += cnt[k];
        for (int q = 0; q < 3; ++q) {
          llo[q] = std::min(llo[q], blo[k][q]);
          lhi[q] = std::max(lhi[q], bhi[k][q]);
        }
        if (lc == 0 || rcnt[k + 1] == 0) continue;
        const float cost = area(llo, lhi) * static_cast<float>(lc) + rarea[k + 1] * static_cast<float>(rcnt[k + 1]);
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = a;
          best_bin = k;
        }
      }
    }
    uint32_t* mid;
    if (best_axis < 0) {
      // All centroids coincide: split the list in half.
      mid = idx + n / 2;
    } else {
      const float scale = kBins / (chi[best_axis] - clo[best_axis]);
      const float c0 = clo[best_axis];
      mid = std::partition(idx, idx + n, [&](uint32_t p) {
        const float* b = boxes + 6 * p;
        const float c = 0.5f * (b[best_axis] + b[3 + best_axis]);
        int k = static_cast<int>((c - c0) * scale);
        k = std::min(kBins - 1, std::max(0, k));
        return k <= best_bin;
      });
      if (mid == idx || mid == idx + n) mid = idx + n / 2;
    }
    const size_t nl = static_cast<size_t>(mid - idx);
    const int32_t l = build(idx, nl);
    const int32_t r = build(mid, n - nl);
    BinNode& nd = (*nodes)[static_cast<size_t>(id)];
    std::memcpy(nd.lo, lo, sizeof(lo));
    std::memcpy(nd.hi, hi, sizeof(hi));
    nd.left = l;
    nd.right = r;
    nd.first = -1;
    nd.count = 0;
    return id;
  }
};

}  // namespace

void BuildSahBvh(const SceneGeometry& geo, uint32_t max_leaf, std::vector<BinNode>& nodes,
                 std::vector<uint32_t>& prim_indices) {
  const size_t n = geo.prims.size();
  nodes.clear();
  prim_indices.clear();
  if (n == 0) return;
  nodes.reserve(2 * n);
  prim_indices.resize(n);
  std::iota(prim_indices.begin(), prim_indices.end(), 0u);
  SahBuilder b{geo.boxes.data(), &nodes, prim_indices.data(), std::max(1u, std::min(8u, max_leaf))};
  b.build(prim_indices.data(), n);
}

bool ValidateBinaryBvh(const std::vector<BinNode>& nodes, const std::vector<uint32_t>& prim_indices,
                       size_t prim_count, std::string& error) {
  if (nodes.empty()) {
    error = "empty BVH";
    return false;
  }
  if (prim_indices.size() != prim_count) {
    error = "prim_indices size does not match the flattened primitive count";
    return false;
  }
  for (uint32_t p : prim_indices) {
    if (p >= prim_count) {
      error = "prim_indices entry out of range";
      return false;
    }
  }
  // Every node reachable once from the root; leaves within range.
  std::vector<uint8_t> seen(nodes.size(), 0);
  std::vector<int32_t> stack{0};
  while (!stack.empty()) {
    const int32_t id = stack.back();
    stack.pop_back();
    if (id < 0 || static_cast<size_t>(id) >= nodes.size() || seen[static_cast<size_t>(id)]) {
      error = "BVH child index out of range or shared";
      return false;
    }
    seen[static_cast<size_t>(id)] = 1;
    const BinNode& nd = nodes[static_cast<size_t>(id)];
    if (nd.count > 0) {
      if (nd.first < 0 || static_cast<size_t>(nd.first) + static_cast<size_t>(nd.count) > prim_indices.size() ||
          nd.count > 8) {
        error = "BVH leaf range out of bounds (or more than 8 primitives)";
        return false;
      }
    } else {
      stack.push_back(nd.left);
      stack.push_back(nd.right);
    }
  }
  return true;
}

void CollapseToWide(const SceneGeometry& geo, const std::vector<BinNode>& bin,
                    const std::vector<uint32_t>& prim_indices, const std::vector<BinNode>& ref,
                    const std::vector<uint32_t>& ref_prims, WideBvh& out) {
  out = WideBvh{};
  if (bin.empty() || ref.empty()) return;
  out.binary_nodes = static_cast<uint32_t>(ref.size());
  out.reference_topology = (&bin == &ref) ||
                           (bin.size() == ref.size() && prim_indices == ref_prims &&
                            std::memcmp(bin.data(), ref.data(), bin.size() * sizeof(BinNode)) == 0);
  // Tie records: bounds, parent and depth of every reference binary node, and
  // for every primitive its reference leaf and lane.
  out.tie_nodes.resize(ref.size());
  std::vector<int32_t> parent(ref.size(), -1), depth(ref.size(), 0);
  std::vector<uint32_t> ref_leaf(geo.prims.size(), 0u), ref_lane(geo.prims.size(), 0u);
  {
    std::vector<int32_t> st{0};
    while (!st.empty()) {
      const int32_t id = st.back();
      st.pop_back();
      const BinNode& nd = ref[static_cast<size_t>(id)];
      if (nd.count > 0) {
        ++out.binary_leaves;
        for (int32_t i = 0; i < nd.count; ++i) {
          const uint32_t p = ref_prims[static_cast<size_t>(nd.first + i)];
          ref_leaf[p] = static_cast<uint32_t>(id);
          ref_lane[p] = static_cast<uint32_t>(i);
        }
        continue;
      }
      for (int32_t c : {nd.left, nd.right}) {
        parent[static_cast<size_t>(c)] = id;
        depth[static_cast<size_t>(c)] = depth[static_cast<size_t>(id)] + 1;
        st.push_back(c);
      }
    }
  }
  for (size_t i = 0; i < ref.size(); ++i) {
    TieNode& t = out.tie_nodes[i];
    t.lox = ref[i].lo[0];
    t.loy = ref[i].lo[1];
    t.loz = ref[i].lo[2];
    t.hix = ref[i].hi[0];
    t.hiy = ref[i].hi[1];
    t.hiz = ref[i].hi[2];
    t.parent = parent[i];
    t.depth = depth[i];
  }

  auto emit_leaf = [&](int32_t leaf_id) -> int32_t {
    const BinNode& lf = bin[static_cast<size_t>(leaf_id)];
    const uint32_t first = static_cast<uint32_t>(out.tris.size());
    for (int32_t i = 0; i < lf.count; ++i) {
      const uint32_t p = prim_indices[static_cast<size_t>(lf.first + i)];
      const HostPrim& hp = geo.prims[p];
      TriRecord r;
      r.v0x = hp.v0[0];
      r.v0y = hp.v0[1];
      r.v0z = hp.v0[2];
      r.e1x = hp.e1[0];
      r.e1y = hp.e1[1];
      r.e1z = hp.e1[2];
      r.e2x = hp.e2[0];
      r.e2y = hp.e2[1];
      r.e2z = hp.e2[2];
      r.prim = p;
      r.leaf = ref_leaf[p];
      r.lane = ref_lane[p];
      out.tris.push_back(r);
    }
    return ~static_cast<int32_t>((first << 3) | static_cast<uint32_t>(lf.count - 1));
  };

  // Depth-first, pre-order allocation of wide nodes.
  std::function<int32_t(int32_t, uint32_t, uint32_t)> make = [&](int32_t bin_id, uint32_t level,
                                                                  uint32_t stack_so_far) -> int32_t {
    const int32_t wide_id = static_cast<int32_t>(out.nodes.size());
    out.nodes.push_back(WideNode{});
    std::vector<int32_t> slots;
    const BinNode& root = bin[static_cast<size_t>(bin_id)];
    if (root.count > 0) {
      slots.push_back(bin_id);
    } else {
      slots = {root.left, root.right};
      while (slots.size() < 4) {
        int best = -1;
        float best_area = -1.0f;
        for (size_t s = 0; s < slots.size(); ++s) {
          const BinNode& c = bin[static_cast<size_t>(slots[s])];
          if (c.count > 0) continue;
          const float a = surface_area(c);
          if (a > best_area) {
            best_area = a;
            best = static_cast<int>(s);
          }
        }
        if (best < 0) break;
        const BinNode& c = bin[static_cast<size_t>(slots[static_cast<size_t>(best)])];
        slots[static_cast<size_t>(best)] = c.left;
        slots.insert(slots.begin() + best + 1, c.right);
      }
    }
    const uint32_t stack_here = stack_so_far + static_cast<uint32_t>(slots.size()) - 1u;
    out.depth = std::max(out.depth, level + 1u);
    out.stack_required = std::max(out.stack_required, stack_here);
    WideNode wn{};
    for (int k = 0; k < 4; ++k) {
      wn.lox[k] = wn.loy[k] = wn.loz[k] = 1.0f;
      wn.hix[k] = wn.hiy[k] = wn.hiz[k] = -1.0f;
      wn.child[k] = kEmptyChild;
    }
    wn.meta[0] = static_cast<int32_t>(slots.size());
    for (size_t s = 0; s < slots.size(); ++s) {
      const BinNode& c = bin[static_cast<size_t>(slots[s])];
      wn.lox[s] = c.lo[0];
      wn.loy[s] = c.lo[1];
      wn.loz[s] = c.lo[2];
      wn.hix[s] = c.hi[0];
      wn.hiy[s] = c.hi[1];
      wn.hiz[s] = c.hi[2];
    }
    for (size_t s = 0; s < slots.size(); ++s) {
      const BinNode& c = bin[static_cast<size_t>(slots[s])];
      wn.child[s] = (c.count > 0) ? emit_leaf(slots[s]) : make(slots[s], level + 1u, stack_here);
    }
    out.nodes[static_cast<size_t>(wide_id)] = wn;
    return wide_id;
  };
  make(0, 0u, 0u);
  out.stack_required += 1u;
}

}  // namespace vkptc
