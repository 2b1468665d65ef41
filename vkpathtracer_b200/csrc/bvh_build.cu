// bvh_build.cu -- the acceleration structure built on the device.
//
// Steps (all on the stream given; the host only sizes launches between the
// levels of the top-down build):
//   1. flatten: one thread per candidate triangle of every instance, invalid
//      ones dropped by a scan (FlattenScene's order and arithmetic);
//   2. the reference's midpoint tree (ParallelBvhBuilder, deterministic mode,
//      src/cpu/ParallelBvhBuilder.cpp:61-257), top-down:
//        nodes above kSmallNode primitives, level by level over all nodes of
//        the level at once: centroid bounds by a segmented warp reduction
//        plus one atomic per run, the widest axis and its midpoint, a flag per
//        primitive, an exclusive scan, and a stable scatter (left flags first,
//        in order; count/2 when one side is empty, order unchanged);
//        smaller subtrees by one thread each, sequentially, the same steps;
//      then node bounds by a bottom-up refit (union of children; min/max are
//      exact, so the result equals the top-down bounds of the reference) and
//      the reference's node ids: the reference allocates the two children of
//      the k-th internal node of its depth-first pre-order as 2k+1, 2k+2, and
//      k is found by walking up from each node, adding 1 per ancestor and the
//      internal-node count of the left subtree when coming from the right;
//   3. optionally a binned-SAH traversal tree (32 bins per axis) with the same
//      machinery;
//   4. the wide collapse of the traversal tree (CollapseToWide's greedy
//      largest-area opening, wide nodes in depth-first pre-order, found the
//      same way), triangle records in leaf order and the tie records of the
//      reference tree.
// Every array equals the host path's bit for bit (tested).  A non-finite
// vertex, edge or bound sends the build back to the host path (min/max of NaN
// depends on operand order, and NaN payloads differ between x86 and the GPU).
#include "bvh_build.h"

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <vector>

namespace vkptc {
namespace {

constexpr float kPadB = 1e-4f;
constexpr uint32_t kSmallNode = 64;   // subtrees of at most this many primitives: one thread each
constexpr uint32_t kLeafMax = 4;      // ParallelBvhBuilder's leaf threshold
constexpr int kScanThreads = 512;
constexpr uint32_t kScanBlock = 2 * kScanThreads;
constexpr int kThreads = 256;
constexpr int kSahBins = 32;
constexpr int kBinWords = 7;     // per bin: count, 3 lower and 3 upper bound keys

inline unsigned grid_for(uint64_t n, int threads = kThreads) {
  return static_cast<unsigned>(std::max<uint64_t>(1, (n + threads - 1) / threads));
}

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ float bmin(float a, float b) { return (b < a) ? b : a; }   // std::min order
__device__ __forceinline__ float bmax(float a, float b) { return (a < b) ? b : a; }   // std::max order
// Order-preserving map of floats to unsigned keys (atomicMin/Max on floats).
__device__ __forceinline__ uint32_t fkey(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fval(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct TNode {          // binary node under construction (temporary ids)
  int32_t begin, count, left, right, parent;
};

// ---------------------------------------------------------------- scan
// Exclusive scan of n+1 elements (element n reads as 0), so out[n] = total.
__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(const uint32_t* __restrict__ in, uint32_t n,
                                                              uint32_t* __restrict__ out, uint32_t m,
                                                              uint32_t* __restrict__ sums) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  const uint32_t i0 = blockIdx.x * kScanBlock + 2u * threadIdx.x, i1 = i0 + 1u;
  const uint32_t a = i0 < n ? in[i0] : 0u, b = i1 < n ? in[i1] : 0u;
  const uint32_t s = a + b;
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t x = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (static_cast<int>(lane) >= o) x += y;
  }
  if (lane == 31u) warp_tot[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < kScanThreads / 32 ? warp_tot[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (static_cast<int>(lane) >= o) t += y;
    }
    if (lane < kScanThreads / 32) warp_tot[lane] = t;
  }
  __syncthreads();
  const uint32_t off = warp ? warp_tot[warp - 1] : 0u;
  const uint32_t excl = off + x - s;
  if (i0 < m) out[i0] = excl;
  if (i1 < m) out[i1] = excl + a;
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = off + x;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_add(uint32_t* __restrict__ out, uint32_t m,
                                                           const uint32_t* __restrict__ offs) {
  const uint32_t i0 = blockIdx.x * kScanBlock + 2u * threadIdx.x;
  const uint32_t add = offs[blockIdx.x];
  if (i0 < m) out[i0] += add;
  if (i0 + 1u < m) out[i0 + 1u] += add;
}

// The builder's memory pool on the current device.  Freed scratch stays
// mapped for the next build: the pool never releases memory on its own (its
// release threshold is unbounded) and is trimmed by TrimBuildPool when the
// last context on the device goes.  A bounded threshold applies to all the
// memory the pool keeps reserved -- the arrays of every built accelerator come
// from it too -- so every synchronisation handed freed scratch back to the
// driver and the next build mapped it again: measured on the 2,064,386-
// triangle grid, 6.4 ms (reference tree) and 17 ms (SAH) per build with a
// 1 GiB threshold, 14 and 24 ms with 64 other jobs' accelerators resident,
// against 3.5 and 11.6 ms with the pool's memory kept in every case.
cudaMemPool_t build_pool() {
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

// Stream-ordered scratch allocations, released on destruction.
struct Scratch {
  cudaStream_t s;
  std::vector<void*> ptrs;
  cudaError_t err = cudaSuccess;
  cudaMemPool_t pool = build_pool();
  template <class T>
  T* get(size_t n) {
    void* p = nullptr;
    if (err != cudaSuccess) return nullptr;
    const size_t bytes = std::max<size_t>(1, n) * sizeof(T);
    err = pool ? cudaMallocFromPoolAsync(&p, bytes, pool, s) : cudaMallocAsync(&p, bytes, s);
    if (err != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  ~Scratch() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
};

// out: n+1 entries.
cudaError_t exclusive_scan(const uint32_t* in, uint32_t n, uint32_t* out, Scratch& sc) {
  const uint32_t m = n + 1u;
  const uint32_t blocks = (m + kScanBlock - 1u) / kScanBlock;
  uint32_t* sums = sc.get<uint32_t>(blocks);
  if (!sums) return sc.err;
  k_scan_blocks<<<blocks, kScanThreads, 0, sc.s>>>(in, n, out, m, sums);
  if (blocks > 1u) {
    uint32_t* offs = sc.get<uint32_t>(blocks + 1u);
    if (!offs) return sc.err;
    cudaError_t e = exclusive_scan(sums, blocks, offs, sc);
    if (e != cudaSuccess) return e;
    k_scan_add<<<blocks, kScanThreads, 0, sc.s>>>(out, m, offs);
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------- flatten
__device__ __forceinline__ uint32_t find_instance(const unsigned long long* prefix, uint32_t count,
                                                  unsigned long long c) {
  uint32_t lo = 0u, hi = count;   // prefix[lo] <= c < prefix[hi]
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (prefix[mid] <= c) lo = mid;
    else hi = mid;
  }
  return lo;
}

struct FlatIn {
  const float* v;
  uint32_t nv;
  const uint32_t* idx;
  uint32_t ni;
  const float* lv;            // local (dynamic-instance) vertices
  uint32_t nlv;
  const uint32_t* lidx;
  uint32_t nli;
  const uint32_t* inst;
  const uint32_t* inst_local;   // 5 per instance, or null
  const float* inst_tr;         // 10 per instance, or null
  const unsigned long long* prefix;
  uint32_t ninst;
  uint32_t candidates;
  uint32_t watertight;          // triangle records hold the vertices (a, b, c), not (v0, e1, e2)
};

// transform_instance_vertex (the host's TransformInstanceVertex, same operations).
__device__ __forceinline__ void instance_vertex(const float* l, const float* tr, float out[3]) {
  const float sx = l[0] * tr[7], sy = l[1] * tr[8], sz = l[2] * tr[9];
  float rx = sx, ry = sy, rz = sz;
  const float len_sq = tr[3] * tr[3] + tr[4] * tr[4] + tr[5] * tr[5] + tr[6] * tr[6];
  if (!(len_sq <= kPadB * kPadB)) {
    const float inv_len = 1.0f / sqrtf(len_sq);
    const float qx = tr[3] * inv_len, qy = tr[4] * inv_len, qz = tr[5] * inv_len;
    const float qw = tr[6] * inv_len;
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

// The three world-space vertices of candidate c, or false when the triangle
// is skipped (CpuBvhAccelerator::build's checks, 32-bit index arithmetic).
__device__ __forceinline__ bool flat_triangle(const FlatIn& f, uint32_t c, uint32_t& inst, float a[3], float b[3],
                                              float cc[3]) {
  const uint32_t i = find_instance(f.prefix, f.ninst, c);
  inst = i;
  const uint32_t k = static_cast<uint32_t>(c - f.prefix[i]);
  if (f.inst_local) {
    const uint32_t* loc = f.inst_local + 5 * i;
    if ((loc[0] & 1u) != 0u && loc[2] > 0u && loc[4] > 0u) {
      const uint32_t local_base = loc[3] + k * 3u;
      const uint32_t local_end = loc[1] + loc[2];
      // (a wrapped local_base + 2 would make the reference read out of range: skipped here)
      if (local_base < 0xFFFFFFFEu && local_base + 2u < f.nli) {
        const uint32_t v0 = loc[1] + f.lidx[local_base], v1 = loc[1] + f.lidx[local_base + 1u],
                       v2 = loc[1] + f.lidx[local_base + 2u];
        if (v0 < local_end && v1 < local_end && v2 < local_end && v0 < f.nlv && v1 < f.nlv && v2 < f.nlv) {
          const float* tr = f.inst_tr + 10 * i;
          instance_vertex(f.lv + 3ull * v0, tr, a);
          instance_vertex(f.lv + 3ull * v1, tr, b);
          instance_vertex(f.lv + 3ull * v2, tr, cc);
          return true;
        }
      }
    }
  }
  const uint32_t base = (f.inst[3 * i] + k) * 3u;
  if (base >= 0xFFFFFFFEu || base + 2u >= f.ni) return false;
  const uint32_t ia = f.idx[base], ib = f.idx[base + 1u], ic = f.idx[base + 2u];
  if (ia >= f.nv || ib >= f.nv || ic >= f.nv) return false;
  for (int q = 0; q < 3; ++q) {
    a[q] = f.v[3ull * ia + q];
    b[q] = f.v[3ull * ib + q];
    cc[q] = f.v[3ull * ic + q];
  }
  return true;
}

__global__ void k_flat_valid(FlatIn f, uint32_t* __restrict__ flag) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= f.candidates) return;
  uint32_t inst;
  float a[3], b[3], cc[3];
  flag[c] = flat_triangle(f, c, inst, a, b, cc) ? 1u : 0u;
}

__device__ __forceinline__ float min3(float a, float b, float c) {   // std::min({a, b, c})
  float m = a;
  if (b < m) m = b;
  if (c < m) m = c;
  return m;
}
__device__ __forceinline__ float max3(float a, float b, float c) {   // std::max({a, b, c})
  float m = a;
  if (m < b) m = b;
  if (m < c) m = c;
  return m;
}

__global__ void k_flat_write(FlatIn f, const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                             float4* __restrict__ pv, float4* __restrict__ shade, float4* __restrict__ blo,
                             float4* __restrict__ bhi, uint32_t* __restrict__ nonfinite) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= f.candidates || !flag[c]) return;
  uint32_t i;
  float a[3], b[3], cc[3];
  flat_triangle(f, c, i, a, b, cc);
  const uint32_t mat = f.inst[3 * i + 2];
  const float e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
  const float e2x = cc[0] - a[0], e2y = cc[1] - a[1], e2z = cc[2] - a[2];
  const float nx = e1y * e2z - e1z * e2y;
  const float ny = e1z * e2x - e1x * e2z;
  const float nz = e1x * e2y - e1y * e2x;
  const float l2 = nx * nx + ny * ny + nz * nz;
  float4 n;
  if (l2 <= kPadB * kPadB) {
    n = make_float4(0.0f, 1.0f, 0.0f, __uint_as_float(mat));
  } else {
    const float inv = 1.0f / sqrtf(l2);
    n = make_float4(nx * inv, ny * inv, nz * inv, __uint_as_float(mat));
  }
  const uint32_t p = pos[c];
  if (f.watertight) {
    pv[3 * p + 0] = make_float4(a[0], a[1], a[2], b[0]);
    pv[3 * p + 1] = make_float4(b[1], b[2], cc[0], cc[1]);
    pv[3 * p + 2] = make_float4(cc[2], 0.0f, 0.0f, 0.0f);
  } else {
    pv[3 * p + 0] = make_float4(a[0], a[1], a[2], e1x);
    pv[3 * p + 1] = make_float4(e1y, e1z, e2x, e2y);
    pv[3 * p + 2] = make_float4(e2z, 0.0f, 0.0f, 0.0f);
  }
  shade[p] = n;
  const float4 lo = make_float4(min3(a[0], b[0], cc[0]) - kPadB, min3(a[1], b[1], cc[1]) - kPadB,
                                min3(a[2], b[2], cc[2]) - kPadB, 0.0f);
  const float4 hi = make_float4(max3(a[0], b[0], cc[0]) + kPadB, max3(a[1], b[1], cc[1]) + kPadB,
                                max3(a[2], b[2], cc[2]) + kPadB, 0.0f);
  blo[p] = lo;
  bhi[p] = hi;
  // Any non-finite vertex coordinate, edge or bound: the host path builds this scene (NaN
  // propagation through min/max and subtraction is operand-order and platform dependent).
  bool fin = isfinite(lo.x) && isfinite(lo.y) && isfinite(lo.z) && isfinite(hi.x) && isfinite(hi.y) &&
             isfinite(hi.z) && isfinite(0.5f * (lo.x + hi.x)) && isfinite(0.5f * (lo.y + hi.y)) &&
             isfinite(0.5f * (lo.z + hi.z));
  for (int q = 0; q < 3; ++q) fin = fin && isfinite(a[q]) && isfinite(b[q]) && isfinite(cc[q]);
  fin = fin && isfinite(e1x) && isfinite(e1y) && isfinite(e1z) && isfinite(e2x) && isfinite(e2y) && isfinite(e2z);
  if (!fin) atomicOr(nonfinite, 1u);
}

// ---------------------------------------------------------------- top-down build
__device__ __forceinline__ float centroid(const float4* blo, const float4* bhi, uint32_t p, int axis) {
  const float4 lo = blo[p], hi = bhi[p];
  const float l = axis == 0 ? lo.x : (axis == 1 ? lo.y : lo.z);
  const float h = axis == 0 ? hi.x : (axis == 1 ? hi.y : hi.z);
  return 0.5f * (l + h);
}

struct BuildArrays {
  const float4* blo;
  const float4* bhi;
  TNode* nodes;
  int32_t* slot_of;        // per temporary node: slot in this level's active list, or -1
  uint32_t* cb;            // per slot: 6 keys (centroid lo xyz, hi xyz)
  int32_t* axis;           // per slot (-1: all centroids coincide, SAH)
  float* split;            // per slot (midpoint) / best bin (SAH, as bits)
  uint32_t* nl;            // per slot
  uint32_t* ident;         // per slot: 1 = order unchanged, count/2 split
  uint32_t* counter;       // [0] next temporary node id, [1] next-level active count, [2] small count,
                           // [4] this level's active count, [5] first temporary id of this level's children
};

// The level loop runs without the host: every per-level kernel reads the
// level's active count from counter[4] (0 after the last level: the kernels
// return at once, so the host may queue levels ahead of its checks).
__device__ __forceinline__ uint32_t level_active(const BuildArrays& A) { return A.counter[4]; }

__device__ __forceinline__ uint32_t grid_thread() { return blockIdx.x * blockDim.x + threadIdx.x; }
__device__ __forceinline__ uint32_t grid_threads() { return gridDim.x * blockDim.x; }

__global__ void k_level_init(BuildArrays A, const uint32_t* __restrict__ act) {
  const uint32_t n_act = level_active(A);
  for (uint32_t s = grid_thread(); s < n_act; s += grid_threads()) {
    A.slot_of[act[s]] = static_cast<int32_t>(s);
    uint32_t* k = A.cb + 6 * s;
    k[0] = k[1] = k[2] = 0xffffffffu;   // min keys
    k[3] = k[4] = k[5] = 0u;            // max keys
  }
}

__global__ void k_level_done(BuildArrays A, const uint32_t* __restrict__ act) {
  const uint32_t n_act = level_active(A);
  for (uint32_t s = grid_thread(); s < n_act; s += grid_threads()) A.slot_of[act[s]] = -1;
}

// End of a level: the children ids advance past this level's children, the
// next level's active list becomes current, its counter is cleared.
__global__ void k_level_advance(BuildArrays A) {
  A.counter[5] += 2u * A.counter[4];
  A.counter[4] = A.counter[1];
  A.counter[1] = 0u;
}

// The scattered order of a level becomes the current one (skipped when the
// level had no active node: its scatter wrote nothing).
__global__ void k_copy_level(BuildArrays A, uint32_t* __restrict__ dst, const uint32_t* __restrict__ src, uint32_t n) {
  if (level_active(A) == 0u) return;
  for (uint32_t i = grid_thread(); i < n; i += grid_threads()) dst[i] = src[i];
}

// After the last level: temporary ids of the small subtrees start after the levels' nodes.
__global__ void k_small_base(BuildArrays A) { A.counter[0] = A.counter[5]; }

// Centroid bounds of every active node: segmented warp reduction over runs of
// positions of the same node, then one atomic per run and key.
__global__ void k_centroid_bounds(BuildArrays A, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ node_of,
                                  uint32_t n) {
  if (level_active(A) == 0u) return;   // uniform over the grid
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned lane = threadIdx.x & 31u;
  int32_t s = -1;
  uint32_t kmin[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu}, kmax[3] = {0u, 0u, 0u};
  if (pos < n) {
    s = A.slot_of[node_of[pos]];
    if (s >= 0) {
      const uint32_t p = idx[pos];
      for (int a = 0; a < 3; ++a) kmin[a] = kmax[a] = fkey(centroid(A.blo, A.bhi, p, a));
    }
  }
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t so = __shfl_down_sync(0xffffffffu, s, o);
    uint32_t omin[3], omax[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      omin[a] = __shfl_down_sync(0xffffffffu, kmin[a], o);
      omax[a] = __shfl_down_sync(0xffffffffu, kmax[a], o);
    }
    if (static_cast<int>(lane) + o < 32 && so == s) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        kmin[a] = min(kmin[a], omin[a]);
        kmax[a] = max(kmax[a], omax[a]);
      }
    }
  }
  // A block whose positions all belong to one node (the common case in the
  // upper levels) combines its warps in shared memory: one atomic per key.
  __shared__ uint32_t blk[kThreads / 32][6];
  __shared__ int32_t s0;
  if (threadIdx.x == 0) s0 = s;
  __syncthreads();
  const bool uniform = __syncthreads_and(s == s0) && s0 >= 0;
  if (uniform) {
    if (lane == 0u) {
      for (int a = 0; a < 3; ++a) {
        blk[threadIdx.x >> 5][a] = kmin[a];
        blk[threadIdx.x >> 5][3 + a] = kmax[a];
      }
    }
    __syncthreads();
    if (threadIdx.x < 6u) {
      uint32_t v = blk[0][threadIdx.x];
      for (int w = 1; w < kThreads / 32; ++w)
        v = threadIdx.x < 3u ? min(v, blk[w][threadIdx.x]) : max(v, blk[w][threadIdx.x]);
      uint32_t* k = A.cb + 6 * s0 + threadIdx.x;
      if (threadIdx.x < 3u) atomicMin(k, v);
      else atomicMax(k, v);
    }
    return;
  }
  const int32_t sp = __shfl_up_sync(0xffffffffu, s, 1);
  const bool head = s >= 0 && (lane == 0u || sp != s);
  if (head) {
    uint32_t* k = A.cb + 6 * s;
    for (int a = 0; a < 3; ++a) {
      atomicMin(k + a, kmin[a]);
      atomicMax(k + 3 + a, kmax[a]);
    }
  }
}

// Widest centroid axis and its midpoint (BuildBinaryBvh's split).
__global__ void k_midpoint_split(BuildArrays A) {
  const uint32_t n_act = level_active(A);
  for (uint32_t s = grid_thread(); s < n_act; s += grid_threads()) {
    const uint32_t* k = A.cb + 6 * s;
    float clo[3], chi[3];
    for (int a = 0; a < 3; ++a) {
      clo[a] = fval(k[a]);
      chi[a] = fval(k[3 + a]);
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
    A.axis[s] = axis;
    A.split[s] = 0.5f * (clo[axis] + chi[axis]);
  }
}

__device__ __forceinline__ bool goes_left(const BuildArrays& A, uint32_t p, int32_t s, bool sah) {
  const int axis = A.axis[s];
  if (!sah) return centroid(A.blo, A.bhi, p, axis) < A.split[s];
  if (axis < 0) return false;
  const uint32_t* k = A.cb + 6 * s;
  const float c0 = fval(k[axis]);
  const float scale = static_cast<float>(kSahBins) / (fval(k[3 + axis]) - c0);
  int bin = static_cast<int>((centroid(A.blo, A.bhi, p, axis) - c0) * scale);
  bin = bin < 0 ? 0 : (bin > kSahBins - 1 ? kSahBins - 1 : bin);
  return bin <= static_cast<int>(__float_as_uint(A.split[s]));
}

__global__ void k_flags(BuildArrays A, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ node_of,
                        uint32_t n, uint32_t* __restrict__ flag, bool sah) {
  if (level_active(A) == 0u) return;
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n) return;
  const int32_t s = A.slot_of[node_of[pos]];
  flag[pos] = (s >= 0 && goes_left(A, idx[pos], s, sah)) ? 1u : 0u;
}

// Children of every active node; big ones go to the next level's list, small
// ones to the per-thread list, leaves nowhere.
__global__ void k_children(BuildArrays A, const uint32_t* __restrict__ act, const uint32_t* __restrict__ excl,
                           uint32_t* __restrict__ next_act, uint32_t* __restrict__ small) {
  const uint32_t n_act = level_active(A), base = A.counter[5];
  for (uint32_t s = grid_thread(); s < n_act; s += grid_threads()) {
  const uint32_t nd = act[s];
  TNode& t = A.nodes[nd];
  const uint32_t b = static_cast<uint32_t>(t.begin), n = static_cast<uint32_t>(t.count);
  uint32_t nl = excl[b + n] - excl[b];
  const bool ident = nl == 0u || nl == n;
  if (ident) nl = n / 2u;
  A.nl[s] = nl;
  A.ident[s] = ident ? 1u : 0u;
  const uint32_t l = base + 2u * s, r = l + 1u;
  t.left = static_cast<int32_t>(l);
  t.right = static_cast<int32_t>(r);
  const uint32_t cnt[2] = {nl, n - nl};
  const uint32_t id[2] = {l, r};
  for (int c = 0; c < 2; ++c) {
    A.nodes[id[c]] = TNode{static_cast<int32_t>(c == 0 ? b : b + nl), static_cast<int32_t>(cnt[c]), -1, -1,
                           static_cast<int32_t>(nd)};
    A.slot_of[id[c]] = -1;
    if (cnt[c] > kSmallNode) next_act[atomicAdd(&A.counter[1], 1u)] = id[c];
    else if (cnt[c] > kLeafMax) small[atomicAdd(&A.counter[2], 1u)] = id[c];
  }
  }
}

__global__ void k_scatter(BuildArrays A, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ node_of,
                          uint32_t n, const uint32_t* __restrict__ excl, uint32_t* __restrict__ idx2,
                          uint32_t* __restrict__ node2) {
  if (level_active(A) == 0u) return;
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n) return;
  const uint32_t nd = node_of[pos];
  const int32_t s = A.slot_of[nd];
  if (s < 0) {
    idx2[pos] = idx[pos];
    node2[pos] = nd;
    return;
  }
  const TNode t = A.nodes[nd];
  const uint32_t b = static_cast<uint32_t>(t.begin);
  const uint32_t nl = A.nl[s];
  const uint32_t i = pos - b;
  uint32_t dst;
  bool left;
  if (A.ident[s]) {
    dst = pos;
    left = i < nl;
  } else {
    const uint32_t rk = excl[pos] - excl[b];
    left = excl[pos + 1] != excl[pos];
    dst = left ? b + rk : b + nl + (i - rk);
  }
  idx2[dst] = idx[pos];
  node2[dst] = static_cast<uint32_t>(left ? t.left : t.right);
}

// Sequential build of one small subtree per thread (same split rules).
// Small subtrees of the SAH tree, one warp each: the host SAH builder's
// splits (32 bins per axis, the first minimum of the swept costs, a stable
// partition, count/2 when one side is empty), with the node's primitives on the lanes (two per lane), the bins
// filled by one leader per bin and slot (order-preserving keys, min and max are
// exact) and the sweep done by shuffle scans with bin b on lane b.
constexpr int kSmallWarps = 4;
static_assert(kSahBins == 32, "k_small_sah keeps bin b on lane b");

__device__ __forceinline__ float warp_min(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = bmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = bmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ int sah_bin_of(float c, float c0, float scale) {
  const int k = static_cast<int>((c - c0) * scale);
  return k < 0 ? 0 : (k > kSahBins - 1 ? kSahBins - 1 : k);
}

__global__ void __launch_bounds__(32 * kSmallWarps) k_small_sah(BuildArrays A, const uint32_t* __restrict__ small,
                                                                uint32_t n_small, uint32_t* __restrict__ idx) {
  __shared__ uint32_t s_stack[kSmallWarps][64];
  __shared__ uint32_t s_bins[kSmallWarps][kSahBins * kBinWords];
  const int wib = static_cast<int>(threadIdx.x >> 5);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t* stack = s_stack[wib];
  uint32_t* bins = s_bins[wib];
  const uint32_t nwarps = gridDim.x * kSmallWarps;
  for (uint32_t w = blockIdx.x * kSmallWarps + static_cast<uint32_t>(wib); w < n_small; w += nwarps) {
    if (lane == 0u) stack[0] = small[w];
    int sp = 1;
    __syncwarp();
    while (sp > 0) {
      const uint32_t nd = stack[--sp];
      const TNode t = A.nodes[nd];
      const uint32_t b = static_cast<uint32_t>(t.begin), n = static_cast<uint32_t>(t.count);
      __syncwarp();
      if (n <= kLeafMax) continue;
      const bool h0 = lane < n, h1 = lane + 32u < n;
      const uint32_t p0 = h0 ? idx[b + lane] : 0u, p1 = h1 ? idx[b + lane + 32u] : 0u;
      float c0[3], c1[3], clo[3], chi[3];
      for (int a = 0; a < 3; ++a) {
        c0[a] = h0 ? centroid(A.blo, A.bhi, p0, a) : 0.0f;
        c1[a] = h1 ? centroid(A.blo, A.bhi, p1, a) : 0.0f;
        clo[a] = warp_min(bmin(h0 ? c0[a] : FLT_MAX, h1 ? c1[a] : FLT_MAX));
        chi[a] = warp_max(bmax(h0 ? c0[a] : -FLT_MAX, h1 ? c1[a] : -FLT_MAX));
      }
      const float4 lo0 = h0 ? A.blo[p0] : make_float4(0.f, 0.f, 0.f, 0.f), hi0 = h0 ? A.bhi[p0] : lo0;
      const float4 lo1 = h1 ? A.blo[p1] : make_float4(0.f, 0.f, 0.f, 0.f), hi1 = h1 ? A.bhi[p1] : lo1;
      float best_cost = FLT_MAX;
      int best_axis = -1, best_bin = -1;
      for (int a = 0; a < 3; ++a) {
        const float ext = chi[a] - clo[a];
        if (!(ext > 0.0f)) continue;   // uniform
        const float scale = static_cast<float>(kSahBins) / ext;
        uint32_t* wb = bins + kBinWords * lane;   // bin `lane`
        wb[0] = 0u;
        wb[1] = wb[2] = wb[3] = 0xffffffffu;
        wb[4] = wb[5] = wb[6] = 0u;
        __syncwarp();
        for (int slot = 0; slot < 2; ++slot) {
          const bool h = slot == 0 ? h0 : h1;
          const unsigned active = __ballot_sync(0xffffffffu, h);
          if (h) {
            const float4 lo = slot == 0 ? lo0 : lo1, hi = slot == 0 ? hi0 : hi1;
            const int k = sah_bin_of(slot == 0 ? c0[a] : c1[a], clo[a], scale);
            const unsigned grp = __match_any_sync(active, static_cast<uint32_t>(k));
            const uint32_t m0 = __reduce_min_sync(grp, fkey(lo.x)), m1 = __reduce_min_sync(grp, fkey(lo.y)),
                           m2 = __reduce_min_sync(grp, fkey(lo.z));
            const uint32_t x0 = __reduce_max_sync(grp, fkey(hi.x)), x1 = __reduce_max_sync(grp, fkey(hi.y)),
                           x2 = __reduce_max_sync(grp, fkey(hi.z));
            if (static_cast<int>(lane) == __ffs(grp) - 1) {
              uint32_t* q = bins + kBinWords * k;
              q[0] += static_cast<uint32_t>(__popc(grp));
              q[1] = min(q[1], m0);
              q[2] = min(q[2], m1);
              q[3] = min(q[3], m2);
              q[4] = max(q[4], x0);
              q[5] = max(q[5], x1);
              q[6] = max(q[6], x2);
            }
          }
          __syncwarp();
        }
        // the sweep: prefix over bins 0..lane, suffix over lane..31 (k_sah_split's scans)
        const uint32_t cnt = wb[0];
        float lo3[3], hi3[3];
        for (int q = 0; q < 3; ++q) {
          lo3[q] = cnt ? fval(wb[1 + q]) : FLT_MAX;
          hi3[q] = cnt ? fval(wb[4 + q]) : -FLT_MAX;
        }
        __syncwarp();
        uint32_t lc = cnt, rc = cnt;
        float llo[3] = {lo3[0], lo3[1], lo3[2]}, lhi[3] = {hi3[0], hi3[1], hi3[2]};
        float rlo[3] = {lo3[0], lo3[1], lo3[2]}, rhi[3] = {hi3[0], hi3[1], hi3[2]};
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t lcu = __shfl_up_sync(0xffffffffu, lc, o);
          const uint32_t rcd = __shfl_down_sync(0xffffffffu, rc, o);
          float lu[6], rd[6];
          for (int q = 0; q < 3; ++q) {
            lu[q] = __shfl_up_sync(0xffffffffu, llo[q], o);
            lu[3 + q] = __shfl_up_sync(0xffffffffu, lhi[q], o);
            rd[q] = __shfl_down_sync(0xffffffffu, rlo[q], o);
            rd[3 + q] = __shfl_down_sync(0xffffffffu, rhi[q], o);
          }
          if (static_cast<int>(lane) >= o) {
            lc += lcu;
            for (int q = 0; q < 3; ++q) {
              llo[q] = bmin(llo[q], lu[q]);
              lhi[q] = bmax(lhi[q], lu[3 + q]);
            }
          }
          if (static_cast<int>(lane) + o < 32) {
            rc += rcd;
            for (int q = 0; q < 3; ++q) {
              rlo[q] = bmin(rlo[q], rd[q]);
              rhi[q] = bmax(rhi[q], rd[3 + q]);
            }
          }
        }
        const uint32_t rcn = __shfl_down_sync(0xffffffffu, rc, 1);
        float rn[6];
        for (int q = 0; q < 3; ++q) {
          rn[q] = __shfl_down_sync(0xffffffffu, rlo[q], 1);
          rn[3 + q] = __shfl_down_sync(0xffffffffu, rhi[q], 1);
        }
        float cost = FLT_MAX;
        if (lane < 31u && lc != 0u && rcn != 0u) {
          const float dx = lhi[0] - llo[0], dy = lhi[1] - llo[1], dz = lhi[2] - llo[2];
          const float ex = rn[3] - rn[0], ey = rn[4] - rn[1], ez = rn[5] - rn[2];
          cost = (dx * dy + dy * dz + dz * dx) * static_cast<float>(lc) +
                 (ex * ey + ey * ez + ez * ex) * static_cast<float>(rcn);
        }
        float c = cost;
        int bb = static_cast<int>(lane);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const float co = __shfl_xor_sync(0xffffffffu, c, o);
          const int bo = __shfl_xor_sync(0xffffffffu, bb, o);
          if (co < c || (co == c && bo < bb)) {
            c = co;
            bb = bo;
          }
        }
        if (c < best_cost) {
          best_cost = c;
          best_axis = a;
          best_bin = bb;
        }
      }
      // stable partition: left in order, then right in order (ident: order unchanged, count/2)
      uint32_t nl = 0u;
      if (best_axis >= 0) {
        const float cb0 = clo[best_axis];
        const float scale = static_cast<float>(kSahBins) / (chi[best_axis] - cb0);
        const bool l0 = h0 && sah_bin_of(c0[best_axis], cb0, scale) <= best_bin;
        const bool l1 = h1 && sah_bin_of(c1[best_axis], cb0, scale) <= best_bin;
        const unsigned v0 = __ballot_sync(0xffffffffu, h0), v1 = __ballot_sync(0xffffffffu, h1);
        const unsigned b0 = __ballot_sync(0xffffffffu, l0), b1 = __ballot_sync(0xffffffffu, l1);
        const uint32_t nl0 = static_cast<uint32_t>(__popc(b0));
        nl = nl0 + static_cast<uint32_t>(__popc(b1));
        const uint32_t nr0 = static_cast<uint32_t>(__popc(v0 & ~b0));
        __syncwarp();   // every lane holds its primitives before any is moved
        if (h0) idx[b + (l0 ? __popc(b0 & lt) : nl + __popc(v0 & ~b0 & lt))] = p0;
        if (h1) idx[b + (l1 ? nl0 + __popc(b1 & lt) : nl + nr0 + __popc(v1 & ~b1 & lt))] = p1;
      }
      const bool ident = nl == 0u || nl == n;
      if (ident) nl = n / 2u;
      uint32_t l = 0u;
      if (lane == 0u) {
        l = atomicAdd(&A.counter[0], 2u);
        const uint32_t r = l + 1u;
        A.nodes[nd].left = static_cast<int32_t>(l);
        A.nodes[nd].right = static_cast<int32_t>(r);
        A.nodes[l] = TNode{static_cast<int32_t>(b), static_cast<int32_t>(nl), -1, -1, static_cast<int32_t>(nd)};
        A.nodes[r] = TNode{static_cast<int32_t>(b + nl), static_cast<int32_t>(n - nl), -1, -1, static_cast<int32_t>(nd)};
        if (sp + 2 <= 64) {
          stack[sp] = r;
          stack[sp + 1] = l;
        }
      }
      if (sp + 2 <= 64) sp += 2;
      __syncwarp();
    }
  }
}

// Small subtrees of the reference tree (midpoint splits), one thread each.
__global__ void k_small(BuildArrays A, const uint32_t* __restrict__ small, uint32_t n_small, uint32_t* __restrict__ idx) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_small) return;
  uint32_t stack[64];
  uint32_t tmp[kSmallNode];
  int sp = 0;
  stack[sp++] = small[w];
  while (sp > 0) {
    const uint32_t nd = stack[--sp];
    const TNode t = A.nodes[nd];
    const uint32_t b = static_cast<uint32_t>(t.begin), n = static_cast<uint32_t>(t.count);
    if (n <= kLeafMax) continue;
    float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t p = idx[b + i];
      for (int a = 0; a < 3; ++a) {
        const float c = centroid(A.blo, A.bhi, p, a);
        clo[a] = bmin(clo[a], c);
        chi[a] = bmax(chi[a], c);
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
    uint32_t nl = 0u, nr = 0u;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t p = idx[b + i];
      if (centroid(A.blo, A.bhi, p, axis) < split) idx[b + nl++] = p;
      else tmp[nr++] = p;
    }
    for (uint32_t i = 0; i < nr; ++i) idx[b + nl + i] = tmp[i];
    if (nl == 0u || nl == n) nl = n / 2u;
    const uint32_t l = atomicAdd(&A.counter[0], 2u), r = l + 1u;
    A.nodes[nd].left = static_cast<int32_t>(l);
    A.nodes[nd].right = static_cast<int32_t>(r);
    A.nodes[l] = TNode{static_cast<int32_t>(b), static_cast<int32_t>(nl), -1, -1, static_cast<int32_t>(nd)};
    A.nodes[r] = TNode{static_cast<int32_t>(b + nl), static_cast<int32_t>(n - nl), -1, -1, static_cast<int32_t>(nd)};
    if (sp + 2 <= 64) {
      stack[sp++] = r;
      stack[sp++] = l;
    }
  }
}

// ---------------------------------------------------------------- SAH binning of large nodes
// Per active slot: 3 axes x 32 bins x (count, 6 bound keys; kBinWords words).
__global__ void k_sah_bin_init(BuildArrays A, uint32_t* __restrict__ bins) {
  const uint32_t total = level_active(A) * 3u * kSahBins;
  for (uint32_t i = grid_thread(); i < total; i += grid_threads()) {
    uint32_t* w = bins + kBinWords * i;
    w[0] = 0u;
    w[1] = w[2] = w[3] = 0xffffffffu;
    w[4] = w[5] = w[6] = 0u;
  }
}

__global__ void k_sah_bin(BuildArrays A, const uint32_t* __restrict__ idx, const uint32_t* __restrict__ node_of,
                          uint32_t n, uint32_t* __restrict__ bins) {
  if (level_active(A) == 0u) return;   // uniform over the grid
  const uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x;
  int32_t s = -1;
  uint32_t p = 0u;
  if (pos < n) {
    s = A.slot_of[node_of[pos]];
    if (s >= 0) p = idx[pos];
  }
  const unsigned active = __ballot_sync(0xffffffffu, s >= 0);
  if (s < 0) return;
  const uint32_t* k = A.cb + 6 * s;
  const float4 lo = A.blo[p], hi = A.bhi[p];
  const uint32_t klo[3] = {fkey(lo.x), fkey(lo.y), fkey(lo.z)};
  const uint32_t khi[3] = {fkey(hi.x), fkey(hi.y), fkey(hi.z)};
  for (int a = 0; a < 3; ++a) {
    const float c0 = fval(k[a]), ext = fval(k[3 + a]) - c0;
    int bin = 0;
    if (ext > 0.0f) {
      bin = static_cast<int>((centroid(A.blo, A.bhi, p, a) - c0) * (static_cast<float>(kSahBins) / ext));
      bin = bin < 0 ? 0 : (bin > kSahBins - 1 ? kSahBins - 1 : bin);
    }
    const uint32_t key = (static_cast<uint32_t>(s) * 3u + static_cast<uint32_t>(a)) * kSahBins + static_cast<uint32_t>(bin);
    const unsigned grp = __match_any_sync(active, key);
    const int leader = __ffs(grp) - 1;
    const uint32_t mlo0 = __reduce_min_sync(grp, klo[0]), mlo1 = __reduce_min_sync(grp, klo[1]),
                   mlo2 = __reduce_min_sync(grp, klo[2]);
    const uint32_t mhi0 = __reduce_max_sync(grp, khi[0]), mhi1 = __reduce_max_sync(grp, khi[1]),
                   mhi2 = __reduce_max_sync(grp, khi[2]);
    if (static_cast<int>(threadIdx.x & 31u) == leader) {
      uint32_t* w = bins + kBinWords * key;
      atomicAdd(w, static_cast<uint32_t>(__popc(grp)));
      atomicMin(w + 1, mlo0);
      atomicMin(w + 2, mlo1);
      atomicMin(w + 3, mlo2);
      atomicMax(w + 4, mhi0);
      atomicMax(w + 5, mhi1);
      atomicMax(w + 6, mhi2);
    }
  }
}

// Best binned split of each large node (the host SAH builder's sweep), one
// warp per node: lane b holds bin b; suffix and prefix counts and bounds by
// shuffle scans, the cheapest plane by a warp argmin (lowest axis, then bin,
// on equal cost, as the sequential sweep keeps the first minimum).
__global__ void k_sah_split(BuildArrays A, const uint32_t* __restrict__ bins) {
  const uint32_t n_act = level_active(A);
  const int lane = static_cast<int>(threadIdx.x & 31u);
  // one warp per node, warp-strided (s is uniform within a warp)
  for (uint32_t s = grid_thread() >> 5; s < n_act; s += grid_threads() >> 5) {
  const uint32_t* k = A.cb + 6 * s;
  float best_cost = FLT_MAX;
  int best_axis = -1, best_bin = -1;
  for (int a = 0; a < 3; ++a) {
    const float ext = fval(k[3 + a]) - fval(k[a]);
    if (!(ext > 0.0f)) continue;
    const uint32_t* w = bins + kBinWords * ((s * 3u + static_cast<uint32_t>(a)) * kSahBins + static_cast<uint32_t>(lane));
    const uint32_t cnt = w[0];
    float lo[3], hi[3];
    for (int q = 0; q < 3; ++q) {
      lo[q] = cnt ? fval(w[1 + q]) : FLT_MAX;
      hi[q] = cnt ? fval(w[4 + q]) : -FLT_MAX;
    }
    // prefix over bins 0..lane (left side of the plane after this bin)
    uint32_t lc = cnt;
    float llo[3] = {lo[0], lo[1], lo[2]}, lhi[3] = {hi[0], hi[1], hi[2]};
    // suffix over bins lane..31 (right side of the plane before this bin)
    uint32_t rc = cnt;
    float rlo[3] = {lo[0], lo[1], lo[2]}, rhi[3] = {hi[0], hi[1], hi[2]};
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t lcu = __shfl_up_sync(0xffffffffu, lc, o);
      const uint32_t rcd = __shfl_down_sync(0xffffffffu, rc, o);
      float lu[6], rd[6];
      for (int q = 0; q < 3; ++q) {
        lu[q] = __shfl_up_sync(0xffffffffu, llo[q], o);
        lu[3 + q] = __shfl_up_sync(0xffffffffu, lhi[q], o);
        rd[q] = __shfl_down_sync(0xffffffffu, rlo[q], o);
        rd[3 + q] = __shfl_down_sync(0xffffffffu, rhi[q], o);
      }
      if (lane >= o) {
        lc += lcu;
        for (int q = 0; q < 3; ++q) {
          llo[q] = bmin(llo[q], lu[q]);
          lhi[q] = bmax(lhi[q], lu[3 + q]);
        }
      }
      if (lane + o < 32) {
        rc += rcd;
        for (int q = 0; q < 3; ++q) {
          rlo[q] = bmin(rlo[q], rd[q]);
          rhi[q] = bmax(rhi[q], rd[3 + q]);
        }
      }
    }
    // the plane after bin `lane`: left = prefix(lane), right = suffix(lane + 1)
    const uint32_t rcn = __shfl_down_sync(0xffffffffu, rc, 1);
    float rn[6];
    for (int q = 0; q < 3; ++q) {
      rn[q] = __shfl_down_sync(0xffffffffu, rlo[q], 1);
      rn[3 + q] = __shfl_down_sync(0xffffffffu, rhi[q], 1);
    }
    float cost = FLT_MAX;
    if (lane < 31 && lc != 0u && rcn != 0u) {
      const float dx = lhi[0] - llo[0], dy = lhi[1] - llo[1], dz = lhi[2] - llo[2];
      const float ex = rn[3] - rn[0], ey = rn[4] - rn[1], ez = rn[5] - rn[2];
      cost = (dx * dy + dy * dz + dz * dx) * static_cast<float>(lc) + (ex * ey + ey * ez + ez * ex) * static_cast<float>(rcn);
    }
    // warp argmin, lowest bin first on equal cost
    float c = cost;
    int b = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const float co = __shfl_xor_sync(0xffffffffu, c, o);
      const int bo = __shfl_xor_sync(0xffffffffu, b, o);
      if (co < c || (co == c && bo < b)) {
        c = co;
        b = bo;
      }
    }
    if (c < best_cost) {
      best_cost = c;
      best_axis = a;
      best_bin = b;
    }
  }
  if (lane == 0) {
    A.axis[s] = best_axis;
    A.split[s] = __uint_as_float(static_cast<uint32_t>(best_bin < 0 ? 0 : best_bin));
  }
  }
}

// ---------------------------------------------------------------- refit, ids, outputs
struct Finish {
  const TNode* nodes;
  const float4* blo;
  const float4* bhi;
  const uint32_t* idx;
  float4* nlo;       // per temporary node
  float4* nhi;
  uint32_t* visits;
  int32_t* icount;   // internal nodes in the subtree
  int32_t* rank;     // internal: depth-first pre-order rank among internal nodes
  int32_t* depth;
  int32_t* final_id;
};

__global__ void k_refit(Finish F, uint32_t n_nodes) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_nodes || F.nodes[x].left >= 0) return;
  const TNode t = F.nodes[x];
  float4 lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.0f), hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.0f);
  for (int32_t i = 0; i < t.count; ++i) {
    const uint32_t p = F.idx[t.begin + i];
    const float4 a = F.blo[p], b = F.bhi[p];
    lo = make_float4(bmin(lo.x, a.x), bmin(lo.y, a.y), bmin(lo.z, a.z), 0.0f);
    hi = make_float4(bmax(hi.x, b.x), bmax(hi.y, b.y), bmax(hi.z, b.z), 0.0f);
  }
  F.nlo[x] = lo;
  F.nhi[x] = hi;
  F.icount[x] = 0;
  while (true) {
    __threadfence();
    const int32_t p = F.nodes[x].parent;
    if (p < 0) break;
    if (atomicAdd(&F.visits[p], 1u) == 0u) break;   // the sibling finishes the parent
    const TNode pt = F.nodes[p];
    const float4 l0 = __ldcg(F.nlo + pt.left), l1 = __ldcg(F.nhi + pt.left);
    const float4 r0 = __ldcg(F.nlo + pt.right), r1 = __ldcg(F.nhi + pt.right);
    F.nlo[p] = make_float4(bmin(l0.x, r0.x), bmin(l0.y, r0.y), bmin(l0.z, r0.z), 0.0f);
    F.nhi[p] = make_float4(bmax(l1.x, r1.x), bmax(l1.y, r1.y), bmax(l1.z, r1.z), 0.0f);
    F.icount[p] = 1 + __ldcg(F.icount + pt.left) + __ldcg(F.icount + pt.right);
    x = static_cast<uint32_t>(p);
  }
}

__global__ void k_ranks(Finish F, uint32_t n_nodes) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_nodes) return;
  int32_t r = 0, d = 0;
  int32_t y = static_cast<int32_t>(x);
  while (F.nodes[y].parent >= 0) {
    const int32_t p = F.nodes[y].parent;
    r += 1;
    if (F.nodes[p].right == y) r += F.icount[F.nodes[p].left];
    y = p;
    ++d;
  }
  F.rank[x] = r;
  F.depth[x] = d;
}

__global__ void k_final_ids(Finish F, uint32_t n_nodes) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_nodes) return;
  if (x == 0u) F.final_id[0] = 0;
  const TNode t = F.nodes[x];
  if (t.left < 0) return;
  F.final_id[t.left] = 2 * F.rank[x] + 1;
  F.final_id[t.right] = 2 * F.rank[x] + 2;
}

// BinNode array in final ids (and the tie records when tie != null).
__global__ void k_write_bin(Finish F, uint32_t n_nodes, BinNode* __restrict__ out, TieNode* __restrict__ tie) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_nodes) return;
  const TNode t = F.nodes[x];
  const int32_t f = F.final_id[x];
  const float4 lo = F.nlo[x], hi = F.nhi[x];
  BinNode b;
  b.lo[0] = lo.x;
  b.lo[1] = lo.y;
  b.lo[2] = lo.z;
  b.hi[0] = hi.x;
  b.hi[1] = hi.y;
  b.hi[2] = hi.z;
  if (t.left >= 0) {
    b.left = F.final_id[t.left];
    b.right = F.final_id[t.right];
    b.first = -1;
    b.count = 0;
  } else {
    b.left = b.right = -1;
    b.first = t.begin;
    b.count = t.count;
  }
  out[f] = b;
  if (tie) {
    TieNode r;
    r.lox = lo.x;
    r.loy = lo.y;
    r.loz = lo.z;
    r.parent = t.parent >= 0 ? F.final_id[t.parent] : -1;
    r.hix = hi.x;
    r.hiy = hi.y;
    r.hiz = hi.z;
    r.depth = F.depth[x];
    tie[f] = r;
  }
}

__global__ void k_ref_leaf(Finish F, uint32_t n_nodes, uint32_t* __restrict__ ref_leaf, uint32_t* __restrict__ ref_lane) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_nodes) return;
  const TNode t = F.nodes[x];
  if (t.left >= 0) return;
  for (int32_t i = 0; i < t.count; ++i) {
    const uint32_t p = F.idx[t.begin + i];
    ref_leaf[p] = static_cast<uint32_t>(F.final_id[x]);
    ref_lane[p] = static_cast<uint32_t>(i);
  }
}

// ---------------------------------------------------------------- wide collapse
struct WTemp {          // wide node under construction
  int32_t slot[4];      // binary node per slot
  int32_t child[4];     // wide temporary id of an internal slot, -1 for a leaf slot
  int32_t nslots, parent, stack_here;
};

struct WideArrays {
  const BinNode* bin;
  WTemp* w;
  uint32_t* counter;    // [0] next temporary wide id, [1] next-level count, [2] max depth, [3] max stack,
                        // [4] this level's count
  uint32_t* size;       // subtree sizes
  uint32_t* visits;
  int32_t* final_id;
  int32_t* slot_bin;    // optional: binary node per wide slot (refit)
};

__device__ __forceinline__ float bin_area(const BinNode& n) {
  const float dx = n.hi[0] - n.lo[0], dy = n.hi[1] - n.lo[1], dz = n.hi[2] - n.lo[2];
  return dx * dy + dy * dz + dz * dx;
}

// One level of the collapse; the level's count is read from counter[4] (0
// after the last level, so levels queued ahead of the host's check return).
__global__ void k_wide_expand(WideArrays W, const uint32_t* __restrict__ cur, uint32_t level,
                              uint32_t* __restrict__ next) {
  const uint32_t n_cur = W.counter[4];
  for (uint32_t i = grid_thread(); i < n_cur; i += grid_threads()) {
  const uint32_t wid = cur[i];
  WTemp& w = W.w[wid];
  const int32_t root = w.slot[0];
  int32_t slots[4];
  int ns = 0;
  const BinNode r = W.bin[root];
  if (r.count > 0) {
    slots[ns++] = root;
  } else {
    slots[ns++] = r.left;
    slots[ns++] = r.right;
    while (ns < 4) {
      int best = -1;
      float best_area = -1.0f;
      for (int s = 0; s < ns; ++s) {
        const BinNode c = W.bin[slots[s]];
        if (c.count > 0) continue;
        const float a = bin_area(c);
        if (a > best_area) {
          best_area = a;
          best = s;
        }
      }
      if (best < 0) break;
      const BinNode c = W.bin[slots[best]];
      for (int s = ns; s > best + 1; --s) slots[s] = slots[s - 1];
      slots[best] = c.left;
      slots[best + 1] = c.right;
      ++ns;
    }
  }
  const int32_t stack_here = w.stack_here + ns - 1;
  w.nslots = ns;
  w.stack_here = stack_here;
  atomicMax(&W.counter[2], level + 1u);
  atomicMax(&W.counter[3], static_cast<uint32_t>(stack_here));
  for (int s = 0; s < 4; ++s) {
    w.slot[s] = s < ns ? slots[s] : -1;
    w.child[s] = -1;
    if (s < ns && W.bin[slots[s]].count == 0) {
      const uint32_t c = atomicAdd(&W.counter[0], 1u);
      W.w[c].slot[0] = slots[s];
      W.w[c].parent = static_cast<int32_t>(wid);
      W.w[c].stack_here = stack_here;   // the child's stack on entry
      w.child[s] = static_cast<int32_t>(c);
      next[atomicAdd(&W.counter[1], 1u)] = c;
    }
  }
  W.visits[wid] = 0u;
  }
}

__global__ void k_wide_advance(WideArrays W) {
  W.counter[4] = W.counter[1];
  W.counter[1] = 0u;
}

__global__ void k_wide_sizes(WideArrays W, uint32_t n_wide) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_wide) return;
  const WTemp w0 = W.w[x];
  for (int s = 0; s < w0.nslots; ++s)
    if (w0.child[s] >= 0) return;   // not a bottom node
  W.size[x] = 1u;
  while (true) {
    __threadfence();
    const int32_t p = W.w[x].parent;
    if (p < 0) break;
    const WTemp pw = W.w[p];
    int need = 0;
    for (int s = 0; s < pw.nslots; ++s) need += pw.child[s] >= 0 ? 1 : 0;
    if (atomicAdd(&W.visits[p], 1u) + 1u < static_cast<uint32_t>(need)) break;
    uint32_t sz = 1u;
    for (int s = 0; s < pw.nslots; ++s)
      if (pw.child[s] >= 0) sz += __ldcg(W.size + pw.child[s]);
    W.size[p] = sz;
    x = static_cast<uint32_t>(p);
  }
}

__global__ void k_wide_ids(WideArrays W, uint32_t n_wide) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_wide) return;
  int32_t id = 0;
  int32_t y = static_cast<int32_t>(x);
  while (W.w[y].parent >= 0) {
    const int32_t p = W.w[y].parent;
    const WTemp pw = W.w[p];
    id += 1;
    for (int s = 0; s < pw.nslots && pw.child[s] != y; ++s)
      if (pw.child[s] >= 0) id += static_cast<int32_t>(W.size[pw.child[s]]);
    y = p;
  }
  W.final_id[x] = id;
}

__global__ void k_wide_write(WideArrays W, uint32_t n_wide, WideNode* __restrict__ out) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_wide) return;
  const WTemp w = W.w[x];
  WideNode n;
  for (int k = 0; k < 4; ++k) {
    n.lox[k] = n.loy[k] = n.loz[k] = 1.0f;
    n.hix[k] = n.hiy[k] = n.hiz[k] = -1.0f;
    n.child[k] = kEmptyChild;
    n.meta[k] = 0;
  }
  n.meta[0] = w.nslots;
  if (W.slot_bin)
    for (int k = 0; k < 4; ++k) W.slot_bin[4 * W.final_id[x] + k] = k < w.nslots ? w.slot[k] : -1;
  for (int k = 0; k < w.nslots; ++k) {
    const BinNode c = W.bin[w.slot[k]];
    n.lox[k] = c.lo[0];
    n.loy[k] = c.lo[1];
    n.loz[k] = c.lo[2];
    n.hix[k] = c.hi[0];
    n.hiy[k] = c.hi[1];
    n.hiz[k] = c.hi[2];
    n.child[k] = c.count > 0 ? ~static_cast<int32_t>((static_cast<uint32_t>(c.first) << 3) |
                                                     static_cast<uint32_t>(c.count - 1))
                             : W.final_id[w.child[k]];
  }
  out[W.final_id[x]] = n;
}

__global__ void k_tri_records(const uint32_t* __restrict__ order, uint32_t n, const float4* __restrict__ pv,
                              const uint32_t* __restrict__ ref_leaf, const uint32_t* __restrict__ ref_lane,
                              TriRecord* __restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t p = order[i];
  const float4 a = pv[3 * p], b = pv[3 * p + 1], c = pv[3 * p + 2];
  TriRecord r;
  r.v0x = a.x;
  r.v0y = a.y;
  r.v0z = a.z;
  r.e1x = a.w;
  r.e1y = b.x;
  r.e1z = b.y;
  r.e2x = b.z;
  r.e2y = b.w;
  r.e2z = c.x;
  r.prim = p;
  r.leaf = ref_leaf[p];
  r.lane = ref_lane[p];
  out[i] = r;
}

__global__ void k_iota(uint32_t* __restrict__ a, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}
__global__ void k_fill_u32(uint32_t* __restrict__ a, uint32_t n, uint32_t v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}
__global__ void k_root(TNode* nodes, uint32_t n, int32_t* slot_of) {
  nodes[0] = TNode{0, static_cast<int32_t>(n), -1, -1, -1};
  slot_of[0] = -1;
}

#define BB_TRY(x)                        \
  do {                                   \
    cudaError_t e_ = (x);                \
    if (e_ != cudaSuccess) return e_;    \
  } while (0)

template <class T>
cudaError_t read_scalar(const T* d, T& h, cudaStream_t s) {
  BB_TRY(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
  return cudaStreamSynchronize(s);
}

// Top-down build of one binary tree over `order` (iota on entry, the tree's
// primitive order on return).  Returns the temporary node count.
cudaError_t build_tree(const float4* blo, const float4* bhi, uint32_t n, bool sah, uint32_t* order, TNode* nodes,
                       uint32_t& n_nodes, Scratch& sc) {
  cudaStream_t s = sc.s;
  const uint32_t cap_nodes = 2u * n;
  int32_t* slot_of = sc.get<int32_t>(cap_nodes);
  uint32_t* node_of = sc.get<uint32_t>(n);
  uint32_t* idx2 = sc.get<uint32_t>(n);
  uint32_t* node2 = sc.get<uint32_t>(n);
  uint32_t* flag = sc.get<uint32_t>(n);
  uint32_t* excl = sc.get<uint32_t>(n + 1u);
  // Nodes of one level above kSmallNode primitives are disjoint: at most n / 65 of them;
  // small subtree roots (5..64 primitives) are disjoint too.
  const uint32_t max_act = n / (kSmallNode + 1u) + 2u;
  uint32_t* act = sc.get<uint32_t>(max_act);
  uint32_t* next = sc.get<uint32_t>(max_act);
  uint32_t* small = sc.get<uint32_t>(n / (kLeafMax + 1u) + 2u);
  uint32_t* counter = sc.get<uint32_t>(8);
  uint32_t* cb = sc.get<uint32_t>(6ull * max_act);
  int32_t* axis = sc.get<int32_t>(max_act);
  float* split = sc.get<float>(max_act);
  uint32_t* nl = sc.get<uint32_t>(max_act);
  uint32_t* ident = sc.get<uint32_t>(max_act);
  uint32_t* bins = sah ? sc.get<uint32_t>(static_cast<size_t>(kBinWords) * 3u * kSahBins * max_act) : nullptr;
  if (sc.err != cudaSuccess) return sc.err;
  BuildArrays A{blo, bhi, nodes, slot_of, cb, axis, split, nl, ident, counter};
  k_fill_u32<<<grid_for(cap_nodes), kThreads, 0, s>>>(reinterpret_cast<uint32_t*>(slot_of), cap_nodes, 0xffffffffu);
  k_fill_u32<<<grid_for(n), kThreads, 0, s>>>(node_of, n, 0u);
  k_root<<<1, 1, 0, s>>>(nodes, n, slot_of);
  // counter: next temporary id, next-level count, small count, -, this level's count, its children's first id
  uint32_t init[8] = {1u, 0u, 0u, 0u, 0u, 1u, 0u, 0u};
  if (n > kSmallNode) {
    init[4] = 1u;   // the root is the first level's one active node
    const uint32_t zero = 0u;
    BB_TRY(cudaMemcpyAsync(act, &zero, 4, cudaMemcpyHostToDevice, s));
  } else if (n > kLeafMax) {
    init[2] = 1u;   // the root is a small subtree
    const uint32_t zero = 0u;
    BB_TRY(cudaMemcpyAsync(small, &zero, 4, cudaMemcpyHostToDevice, s));
  }
  BB_TRY(cudaMemcpyAsync(counter, init, sizeof(init), cudaMemcpyHostToDevice, s));
  // The levels are queued without waiting for their counts: every split
  // leaves a largest child of at least half its parent, so at least
  // floor(log2(n / 64)) levels run before every node is small; the host reads
  // the count only from then on, every second level (a queued level after the
  // last one finds no active node and its kernels return at once).
  uint32_t* idx = order;
  const uint32_t act_grid = std::min(grid_for(max_act), 148u * 8u);
  const uint32_t bin_grid = std::min(grid_for(static_cast<uint64_t>(max_act) * 3u * kSahBins), 148u * 8u);
  const uint32_t split_grid = std::min(grid_for(static_cast<uint64_t>(max_act) * 32u, 128), 148u * 16u);
  uint32_t first_check = 1u;
  for (uint64_t m = n / (kSmallNode + 1u); m > 1u; m >>= 1) ++first_check;
  bool more = init[4] != 0u;
  for (uint32_t level = 1u; more; ++level) {
    k_level_init<<<act_grid, kThreads, 0, s>>>(A, act);
    k_centroid_bounds<<<grid_for(n), kThreads, 0, s>>>(A, idx, node_of, n);
    if (sah) {
      k_sah_bin_init<<<bin_grid, kThreads, 0, s>>>(A, bins);
      k_sah_bin<<<grid_for(n), kThreads, 0, s>>>(A, idx, node_of, n, bins);
      k_sah_split<<<split_grid, 128, 0, s>>>(A, bins);
    } else {
      k_midpoint_split<<<act_grid, kThreads, 0, s>>>(A);
    }
    k_flags<<<grid_for(n), kThreads, 0, s>>>(A, idx, node_of, n, flag, sah);
    BB_TRY(exclusive_scan(flag, n, excl, sc));
    k_children<<<act_grid, kThreads, 0, s>>>(A, act, excl, next, small);
    k_scatter<<<grid_for(n), kThreads, 0, s>>>(A, idx, node_of, n, excl, idx2, node2);
    k_level_done<<<act_grid, kThreads, 0, s>>>(A, act);
    // the scattered order becomes the current one (the caller's buffer keeps the final order)
    k_copy_level<<<std::min(grid_for(n), 148u * 8u), kThreads, 0, s>>>(A, idx, idx2, n);
    k_level_advance<<<1, 1, 0, s>>>(A);
    BB_TRY(cudaGetLastError());
    std::swap(node_of, node2);
    std::swap(act, next);
    if (level >= first_check && (level - first_check) % 2u == 0u) {
      uint32_t cur = 0u;
      BB_TRY(read_scalar(counter + 4, cur, s));
      more = cur != 0u;
    }
  }
  uint32_t n_small = 0u;
  BB_TRY(read_scalar(counter + 2, n_small, s));
  k_small_base<<<1, 1, 0, s>>>(A);
  if (n_small > 0u) {
    if (sah)
      k_small_sah<<<std::min((n_small + kSmallWarps - 1u) / kSmallWarps, 148u * 16u), 32 * kSmallWarps, 0, s>>>(
          A, small, n_small, idx);
    else
      k_small<<<grid_for(n_small, 64), 64, 0, s>>>(A, small, n_small, idx);
  }
  BB_TRY(cudaGetLastError());
  return read_scalar(counter, n_nodes, s);
}

// Node bounds, reference ids and BinNode array of a built tree.
cudaError_t finish_tree(const float4* blo, const float4* bhi, const uint32_t* order, const TNode* nodes,
                        uint32_t n_nodes, BinNode* out, TieNode* tie, uint32_t* ref_leaf, uint32_t* ref_lane,
                        Scratch& sc) {
  cudaStream_t s = sc.s;
  Finish F{nodes, blo, bhi, order, sc.get<float4>(n_nodes), sc.get<float4>(n_nodes), sc.get<uint32_t>(n_nodes),
           sc.get<int32_t>(n_nodes), sc.get<int32_t>(n_nodes), sc.get<int32_t>(n_nodes), sc.get<int32_t>(n_nodes)};
  if (sc.err != cudaSuccess) return sc.err;
  BB_TRY(cudaMemsetAsync(F.visits, 0, n_nodes * sizeof(uint32_t), s));
  k_refit<<<grid_for(n_nodes), kThreads, 0, s>>>(F, n_nodes);
  k_ranks<<<grid_for(n_nodes), kThreads, 0, s>>>(F, n_nodes);
  k_final_ids<<<grid_for(n_nodes), kThreads, 0, s>>>(F, n_nodes);
  k_write_bin<<<grid_for(n_nodes), kThreads, 0, s>>>(F, n_nodes, out, tie);
  if (ref_leaf) k_ref_leaf<<<grid_for(n_nodes), kThreads, 0, s>>>(F, n_nodes, ref_leaf, ref_lane);
  return cudaGetLastError();
}

cudaError_t collapse(const BinNode* bin, uint32_t n_bin, WideNode* out, uint32_t& n_wide, uint32_t& depth,
                     uint32_t& stack_required, Scratch& sc, int32_t* slot_bin = nullptr) {
  cudaStream_t s = sc.s;
  const uint32_t cap = n_bin;   // wide nodes <= binary internal nodes + 1
  WideArrays W{bin, sc.get<WTemp>(cap), sc.get<uint32_t>(8), sc.get<uint32_t>(cap), sc.get<uint32_t>(cap),
               sc.get<int32_t>(cap), slot_bin};
  uint32_t* cur = sc.get<uint32_t>(cap);
  uint32_t* next = sc.get<uint32_t>(cap);
  if (sc.err != cudaSuccess) return sc.err;
  WTemp root{};
  root.slot[0] = 0;
  root.parent = -1;
  root.stack_here = 0;
  BB_TRY(cudaMemcpyAsync(W.w, &root, sizeof(root), cudaMemcpyHostToDevice, s));
  const uint32_t init[8] = {1u, 0u, 0u, 0u, 1u, 0u, 0u, 0u};
  BB_TRY(cudaMemcpyAsync(W.counter, init, sizeof(init), cudaMemcpyHostToDevice, s));
  const uint32_t zero = 0u;
  BB_TRY(cudaMemcpyAsync(cur, &zero, 4, cudaMemcpyHostToDevice, s));
  // Levels are queued without waiting for their counts: a wide node spans at
  // most three binary levels and a binary tree of L leaves is at least
  // log2(L) deep, so at least floor(log2(n_bin / 2) / 3) levels run; the host
  // reads the count from then on, every second level.
  uint32_t first_check = 1u, lg = 0u;
  for (uint64_t m = n_bin / 2u; m > 1u; m >>= 1) ++lg;
  first_check = std::max(1u, lg / 3u);
  const uint32_t wide_grid = std::min(grid_for(cap), 148u * 8u);
  bool more = true;
  for (uint32_t level = 0u; more; ++level) {
    k_wide_expand<<<wide_grid, kThreads, 0, s>>>(W, cur, level, next);
    k_wide_advance<<<1, 1, 0, s>>>(W);
    BB_TRY(cudaGetLastError());
    std::swap(cur, next);
    const uint32_t done = level + 1u;
    if (done >= first_check && (done - first_check) % 2u == 0u) {
      uint32_t n_cur = 0u;
      BB_TRY(read_scalar(W.counter + 4, n_cur, s));
      more = n_cur != 0u;
    }
  }
  uint32_t cnt[4];
  BB_TRY(cudaMemcpyAsync(cnt, W.counter, sizeof(cnt), cudaMemcpyDeviceToHost, s));
  BB_TRY(cudaStreamSynchronize(s));
  n_wide = cnt[0];
  depth = cnt[2];
  stack_required = cnt[3] + 1u;
  k_wide_sizes<<<grid_for(n_wide), kThreads, 0, s>>>(W, n_wide);
  k_wide_ids<<<grid_for(n_wide), kThreads, 0, s>>>(W, n_wide);
  k_wide_write<<<grid_for(n_wide), kThreads, 0, s>>>(W, n_wide, out);
  return cudaGetLastError();
}

// The accelerator's own arrays come from the builder's stream-ordered pool
// too: with many allocations resident in the process (a batch's job set),
// cudaMalloc and cudaFree of a rebuild's arrays took tens of milliseconds.
template <class T>
cudaError_t dmalloc(T*& p, size_t n, cudaStream_t s) {
  const size_t bytes = std::max<size_t>(1, n) * sizeof(T);
  cudaMemPool_t pool = build_pool();
  return pool ? cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), bytes, pool, s)
              : cudaMallocAsync(reinterpret_cast<void**>(&p), bytes, s);
}

__global__ void k_inst_first(const uint32_t* __restrict__ pos, const unsigned long long* __restrict__ prefix,
                             uint32_t ninst, uint32_t* __restrict__ first) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= ninst) first[i] = pos[prefix[i]];
}

__global__ void k_tri_pos(const uint32_t* __restrict__ order, uint32_t n, uint32_t* __restrict__ tri_pos) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) tri_pos[order[i]] = i;
}

__global__ void k_parents(const BinNode* __restrict__ nodes, uint32_t n, int32_t* __restrict__ parent) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n) return;
  if (x == 0u) parent[0] = -1;
  const BinNode b = nodes[x];
  if (b.count == 0) {
    parent[b.left] = static_cast<int32_t>(x);
    parent[b.right] = static_cast<int32_t>(x);
  }
}

// ---------------------------------------------------------------- refit after transform updates
struct RefitTri {
  const RefitUpdate* up;
  const uint32_t* offset;   // per update: first triangle of the launch (update count + 1 entries)
  uint32_t n_up;
  const float* lv;
  const uint32_t* li;
  uint32_t watertight;      // records hold (a, b, c)
};

__global__ void k_refit_prims(RefitTri R, uint32_t total, const uint32_t* __restrict__ tri_pos, TriRecord* __restrict__ tris,
                              float4* __restrict__ shade, float4* __restrict__ blo, float4* __restrict__ bhi) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  uint32_t lo = 0u, hi = R.n_up;   // offset[lo] <= g < offset[hi]
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (R.offset[mid] <= g) lo = mid;
    else hi = mid;
  }
  const RefitUpdate& u = R.up[lo];
  const uint32_t k = g - R.offset[lo];
  const uint32_t base = u.local_first_index + k * 3u;
  float a[3], b[3], c[3];
  instance_vertex(R.lv + 3ull * (u.local_first_vertex + R.li[base]), u.transform, a);
  instance_vertex(R.lv + 3ull * (u.local_first_vertex + R.li[base + 1u]), u.transform, b);
  instance_vertex(R.lv + 3ull * (u.local_first_vertex + R.li[base + 2u]), u.transform, c);
  const uint32_t p = u.prim_first + k;
  const float e1x = b[0] - a[0], e1y = b[1] - a[1], e1z = b[2] - a[2];
  const float e2x = c[0] - a[0], e2y = c[1] - a[1], e2z = c[2] - a[2];
  const float nx = e1y * e2z - e1z * e2y;
  const float ny = e1z * e2x - e1x * e2z;
  const float nz = e1x * e2y - e1y * e2x;
  const float l2 = nx * nx + ny * ny + nz * nz;
  if (l2 <= kPadB * kPadB) {
    shade[p] = make_float4(0.0f, 1.0f, 0.0f, __uint_as_float(u.material));
  } else {
    const float inv = 1.0f / sqrtf(l2);
    shade[p] = make_float4(nx * inv, ny * inv, nz * inv, __uint_as_float(u.material));
  }
  TriRecord& r = tris[tri_pos[p]];
  r.v0x = a[0];
  r.v0y = a[1];
  r.v0z = a[2];
  r.e1x = R.watertight ? b[0] : e1x;
  r.e1y = R.watertight ? b[1] : e1y;
  r.e1z = R.watertight ? b[2] : e1z;
  r.e2x = R.watertight ? c[0] : e2x;
  r.e2y = R.watertight ? c[1] : e2y;
  r.e2z = R.watertight ? c[2] : e2z;
  blo[p] = make_float4(min3(a[0], b[0], c[0]) - kPadB, min3(a[1], b[1], c[1]) - kPadB, min3(a[2], b[2], c[2]) - kPadB, 0.0f);
  bhi[p] = make_float4(max3(a[0], b[0], c[0]) + kPadB, max3(a[1], b[1], c[1]) + kPadB, max3(a[2], b[2], c[2]) + kPadB, 0.0f);
}

// refit_node over a whole binary tree, bottom-up by walks from the leaves
// (leaf: union of its primitives' boxes; internal: union of its children).
__global__ void k_refit_tree(BinNode* __restrict__ nodes, const int32_t* __restrict__ parent, const uint32_t* __restrict__ order,
                             uint32_t n_nodes, const float4* __restrict__ blo, const float4* __restrict__ bhi,
                             uint32_t* __restrict__ visits, TieNode* __restrict__ tie) {
  uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_nodes || nodes[x].count == 0) return;
  const BinNode leaf = nodes[x];
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int32_t i = 0; i < leaf.count; ++i) {
    const uint32_t p = order[leaf.first + i];
    const float4 a = blo[p], b = bhi[p];
    lo[0] = bmin(lo[0], a.x);
    lo[1] = bmin(lo[1], a.y);
    lo[2] = bmin(lo[2], a.z);
    hi[0] = bmax(hi[0], b.x);
    hi[1] = bmax(hi[1], b.y);
    hi[2] = bmax(hi[2], b.z);
  }
  while (true) {
    for (int q = 0; q < 3; ++q) {
      nodes[x].lo[q] = lo[q];
      nodes[x].hi[q] = hi[q];
    }
    if (tie) {
      tie[x].lox = lo[0];
      tie[x].loy = lo[1];
      tie[x].loz = lo[2];
      tie[x].hix = hi[0];
      tie[x].hiy = hi[1];
      tie[x].hiz = hi[2];
    }
    __threadfence();
    const int32_t p = parent[x];
    if (p < 0) break;
    if (atomicAdd(&visits[p], 1u) == 0u) break;
    const BinNode pn = nodes[p];
    const int32_t sib = pn.left == static_cast<int32_t>(x) ? pn.right : pn.left;
    for (int q = 0; q < 3; ++q) {
      lo[q] = bmin(lo[q], __ldcg(&nodes[sib].lo[q]));
      hi[q] = bmax(hi[q], __ldcg(&nodes[sib].hi[q]));
    }
    x = static_cast<uint32_t>(p);
  }
}

__global__ void k_refit_wide(WideNode* __restrict__ wide, uint32_t n_wide, const int32_t* __restrict__ slot_bin,
                             const BinNode* __restrict__ bin) {
  const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= n_wide) return;
  for (int k = 0; k < 4; ++k) {
    const int32_t b = slot_bin[4 * w + k];
    if (b < 0) continue;
    const BinNode c = bin[b];
    wide[w].lox[k] = c.lo[0];
    wide[w].loy[k] = c.lo[1];
    wide[w].loz[k] = c.lo[2];
    wide[w].hix[k] = c.hi[0];
    wide[w].hiy[k] = c.hi[1];
    wide[w].hiz[k] = c.hi[2];
  }
}

}  // namespace

void TrimBuildPool() {
  cudaMemPool_t p = build_pool();
  if (!p) return;
  cudaDeviceSynchronize();
  cudaMemPoolTrimTo(p, 0);
}

void FreeAccelArray(void* p, cudaStream_t stream) {
  if (p) cudaFreeAsync(p, stream);
}

void FreeRefitState(DeviceRefitState*& st, cudaStream_t stream) {
  if (!st) return;
  FreeAccelArray(st->blo, stream);
  FreeAccelArray(st->bhi, stream);
  FreeAccelArray(st->tri_pos, stream);
  FreeAccelArray(st->trav_nodes, stream);
  FreeAccelArray(st->trav_order, stream);
  FreeAccelArray(st->trav_parent, stream);
  FreeAccelArray(st->slot_bin, stream);
  FreeAccelArray(st->inst_first, stream);
  delete st;
  st = nullptr;
}

cudaError_t RefitOnDevice(DeviceRefitState& st, const std::vector<RefitUpdate>& updates, const float* local_vertices,
                          const uint32_t* local_indices, BinNode* ref_nodes, const uint32_t* ref_order,
                          uint32_t ref_count, float4* nodes, uint32_t wide_count, float4* tris, float4* tie,
                          float4* shade, cudaStream_t stream) {
  if (updates.empty()) return cudaSuccess;
  Scratch sc{stream};
  std::vector<uint32_t> offset(updates.size() + 1, 0u);
  for (size_t i = 0; i < updates.size(); ++i) offset[i + 1] = offset[i] + updates[i].prim_count;
  RefitUpdate* d_up = sc.get<RefitUpdate>(updates.size());
  uint32_t* d_off = sc.get<uint32_t>(offset.size());
  int32_t* ref_parent = sc.get<int32_t>(ref_count);
  uint32_t* visits = sc.get<uint32_t>(std::max(ref_count, st.trav_count));
  if (sc.err != cudaSuccess) return sc.err;
  BB_TRY(cudaMemcpyAsync(d_up, updates.data(), updates.size() * sizeof(RefitUpdate), cudaMemcpyHostToDevice, stream));
  BB_TRY(cudaMemcpyAsync(d_off, offset.data(), offset.size() * 4, cudaMemcpyHostToDevice, stream));
  const uint32_t total = offset.back();
  const RefitTri R{d_up, d_off, static_cast<uint32_t>(updates.size()), local_vertices, local_indices,
                   st.watertight ? 1u : 0u};
  if (total)
    k_refit_prims<<<grid_for(total), kThreads, 0, stream>>>(R, total, st.tri_pos, reinterpret_cast<TriRecord*>(tris),
                                                            shade, st.blo, st.bhi);
  // the reference tree (tie records) ...
  k_parents<<<grid_for(ref_count), kThreads, 0, stream>>>(ref_nodes, ref_count, ref_parent);
  BB_TRY(cudaMemsetAsync(visits, 0, ref_count * sizeof(uint32_t), stream));
  k_refit_tree<<<grid_for(ref_count), kThreads, 0, stream>>>(ref_nodes, ref_parent, ref_order, ref_count, st.blo,
                                                             st.bhi, visits, reinterpret_cast<TieNode*>(tie));
  // ... the traversal tree when it is a different one, then the wide slots
  const BinNode* trav = ref_nodes;
  if (st.trav_nodes) {
    BB_TRY(cudaMemsetAsync(visits, 0, st.trav_count * sizeof(uint32_t), stream));
    k_refit_tree<<<grid_for(st.trav_count), kThreads, 0, stream>>>(st.trav_nodes, st.trav_parent, st.trav_order,
                                                                   st.trav_count, st.blo, st.bhi, visits, nullptr);
    trav = st.trav_nodes;
  }
  k_refit_wide<<<grid_for(wide_count), kThreads, 0, stream>>>(reinterpret_cast<WideNode*>(nodes), wide_count,
                                                              st.slot_bin, trav);
  BB_TRY(cudaGetLastError());
  return cudaStreamSynchronize(stream);
}

void FreeDeviceAccel(DeviceAccelOut& out, cudaStream_t stream) {
  FreeRefitState(out.refit, stream);
  FreeAccelArray(out.nodes, stream);
  FreeAccelArray(out.tris, stream);
  FreeAccelArray(out.tie, stream);
  FreeAccelArray(out.shade, stream);
  FreeAccelArray(out.ref_nodes, stream);
  FreeAccelArray(out.ref_order, stream);
  out = DeviceAccelOut{};
}

cudaError_t BuildAccelOnDevice(const DeviceSceneArrays& sc_in, bool sah, cudaStream_t stream, DeviceAccelOut& out) {
  out = DeviceAccelOut{};
  const uint32_t* instances = sc_in.instances;
  const uint32_t instance_count = sc_in.instance_count;
  const bool dyn = sc_in.instance_local && sc_in.instance_transforms;
  // Keep what a refit needs when some instance can take transform updates.
  bool keep_refit = false;
  for (uint32_t i = 0; dyn && i < instance_count; ++i) {
    const uint32_t* l = sc_in.instance_local + 5 * i;
    keep_refit = keep_refit || ((l[0] & 1u) != 0u && l[2] > 0u && l[4] > 0u);
  }
  // Candidate triangles of every instance (the host path's loop bounds).
  std::vector<unsigned long long> prefix(instance_count + 1u, 0ull);
  for (uint32_t i = 0; i < instance_count; ++i) prefix[i + 1] = prefix[i] + instances[3 * i + 1];
  const unsigned long long candidates = prefix[instance_count];
  if (candidates >= (1ull << 31)) return cudaErrorInvalidValue;
  Scratch sc{stream};
  uint32_t* d_inst = sc.get<uint32_t>(3ull * instance_count);
  uint32_t* d_inst_local = dyn ? sc.get<uint32_t>(5ull * instance_count) : nullptr;
  float* d_inst_tr = dyn ? sc.get<float>(10ull * instance_count) : nullptr;
  unsigned long long* d_prefix = sc.get<unsigned long long>(instance_count + 1u);
  const uint32_t nc = static_cast<uint32_t>(candidates);
  uint32_t* flag = sc.get<uint32_t>(nc);
  uint32_t* pos = sc.get<uint32_t>(nc + 1u);
  uint32_t* nonfinite = sc.get<uint32_t>(1);
  if (sc.err != cudaSuccess) return sc.err;
  if (instance_count) BB_TRY(cudaMemcpyAsync(d_inst, instances, 12ull * instance_count, cudaMemcpyHostToDevice, stream));
  if (dyn && instance_count) {
    BB_TRY(cudaMemcpyAsync(d_inst_local, sc_in.instance_local, 20ull * instance_count, cudaMemcpyHostToDevice, stream));
    BB_TRY(cudaMemcpyAsync(d_inst_tr, sc_in.instance_transforms, 40ull * instance_count, cudaMemcpyHostToDevice, stream));
  }
  BB_TRY(cudaMemcpyAsync(d_prefix, prefix.data(), 8ull * (instance_count + 1u), cudaMemcpyHostToDevice, stream));
  BB_TRY(cudaMemsetAsync(nonfinite, 0, 4, stream));
  const FlatIn f{sc_in.vertices, sc_in.vertex_count, sc_in.indices, sc_in.index_count,
                 sc_in.local_vertices, dyn ? sc_in.local_vertex_count : 0u,
                 sc_in.local_indices, dyn ? sc_in.local_index_count : 0u,
                 d_inst, d_inst_local, d_inst_tr, d_prefix, instance_count, nc, sc_in.watertight ? 1u : 0u};
  if (nc) k_flat_valid<<<grid_for(nc), kThreads, 0, stream>>>(f, flag);
  BB_TRY(exclusive_scan(flag, nc, pos, sc));
  uint32_t n = 0u;
  BB_TRY(read_scalar(pos + nc, n, stream));
  out.prim_count = n;
  float4* pv = sc.get<float4>(3ull * n);
  float4* blo = nullptr;
  float4* bhi = nullptr;
  if (keep_refit) {
    out.refit = new DeviceRefitState();
    out.refit->watertight = sc_in.watertight;
    BB_TRY(dmalloc(out.refit->blo, n, stream));
    BB_TRY(dmalloc(out.refit->bhi, n, stream));
    BB_TRY(dmalloc(out.refit->inst_first, instance_count + 1u, stream));
    blo = out.refit->blo;
    bhi = out.refit->bhi;
  } else {
    blo = sc.get<float4>(n);
    bhi = sc.get<float4>(n);
  }
  if (sc.err != cudaSuccess) return sc.err;
  BB_TRY(dmalloc(out.shade, n, stream));
  if (nc) k_flat_write<<<grid_for(nc), kThreads, 0, stream>>>(f, flag, pos, pv, out.shade, blo, bhi, nonfinite);
  uint32_t bad = 0u;
  BB_TRY(read_scalar(nonfinite, bad, stream));
  if (!bad) {
    // Per-instance primitive ranges (scene deltas rewrite whole instances; refits).
    uint32_t* d_first = keep_refit ? out.refit->inst_first : sc.get<uint32_t>(instance_count + 1u);
    if (sc.err != cudaSuccess) return sc.err;
    k_inst_first<<<grid_for(instance_count + 1u), kThreads, 0, stream>>>(pos, d_prefix, instance_count, d_first);
    std::vector<uint32_t>& first = out.inst_first;
    first.resize(instance_count + 1u);
    BB_TRY(cudaMemcpyAsync(first.data(), d_first, 4ull * first.size(), cudaMemcpyDeviceToHost, stream));
    BB_TRY(cudaStreamSynchronize(stream));
    if (keep_refit) {
      out.refit->host_inst_first.assign(first.begin(), first.end() - 1);
      out.refit->host_inst_count.resize(instance_count);
      for (uint32_t i = 0; i < instance_count; ++i) out.refit->host_inst_count[i] = first[i + 1] - first[i];
    }
  }
  if (bad) {
    FreeDeviceAccel(out, stream);
    out.fallback = true;
    return cudaSuccess;
  }
  if (n == 0u) return cudaSuccess;

  // Reference tree.
  TNode* tn = sc.get<TNode>(2ull * n);
  uint32_t* ref_leaf = sc.get<uint32_t>(n);
  uint32_t* ref_lane = sc.get<uint32_t>(n);
  if (sc.err != cudaSuccess) return sc.err;
  BB_TRY(dmalloc(out.ref_order, n, stream));
  k_iota<<<grid_for(n), kThreads, 0, stream>>>(out.ref_order, n);
  uint32_t n_ref = 0u;
  BB_TRY(build_tree(blo, bhi, n, false, out.ref_order, tn, n_ref, sc));
  BB_TRY(dmalloc(out.ref_nodes, n_ref, stream));
  TieNode* tie = nullptr;
  BB_TRY(dmalloc(tie, n_ref, stream));
  out.tie = reinterpret_cast<float4*>(tie);
  BB_TRY(finish_tree(blo, bhi, out.ref_order, tn, n_ref, out.ref_nodes, tie, ref_leaf, ref_lane, sc));
  out.binary_nodes = n_ref;
  out.binary_leaves = (n_ref + 1u) / 2u;

  // Traversal tree: the reference tree itself, or a binned-SAH tree.
  const BinNode* trav = out.ref_nodes;
  const uint32_t* trav_order = out.ref_order;
  uint32_t n_trav = n_ref;
  if (sah) {
    uint32_t* sah_order = nullptr;
    if (keep_refit) BB_TRY(dmalloc(out.refit->trav_order, n, stream));
    sah_order = keep_refit ? out.refit->trav_order : sc.get<uint32_t>(n);
    TNode* sn = sc.get<TNode>(2ull * n);
    if (sc.err != cudaSuccess) return sc.err;
    k_iota<<<grid_for(n), kThreads, 0, stream>>>(sah_order, n);
    BB_TRY(build_tree(blo, bhi, n, true, sah_order, sn, n_trav, sc));
    BinNode* sah_nodes = nullptr;
    if (keep_refit) {
      BB_TRY(dmalloc(out.refit->trav_nodes, n_trav, stream));
      BB_TRY(dmalloc(out.refit->trav_parent, n_trav, stream));
      out.refit->trav_count = n_trav;
      sah_nodes = out.refit->trav_nodes;
    } else {
      sah_nodes = sc.get<BinNode>(n_trav);
    }
    if (sc.err != cudaSuccess) return sc.err;
    BB_TRY(finish_tree(blo, bhi, sah_order, sn, n_trav, sah_nodes, nullptr, nullptr, nullptr, sc));
    if (keep_refit) k_parents<<<grid_for(n_trav), kThreads, 0, stream>>>(sah_nodes, n_trav, out.refit->trav_parent);
    trav = sah_nodes;
    trav_order = sah_order;
    out.reference_topology = false;
  }
  WideNode* wide = nullptr;
  BB_TRY(dmalloc(wide, n_trav, stream));
  out.nodes = reinterpret_cast<float4*>(wide);
  if (keep_refit) BB_TRY(dmalloc(out.refit->slot_bin, 4ull * n_trav, stream));
  BB_TRY(collapse(trav, n_trav, wide, out.wide_nodes, out.depth, out.stack_required, sc,
                  keep_refit ? out.refit->slot_bin : nullptr));
  TriRecord* tris = nullptr;
  BB_TRY(dmalloc(tris, n, stream));
  out.tris = reinterpret_cast<float4*>(tris);
  k_tri_records<<<grid_for(n), kThreads, 0, stream>>>(trav_order, n, pv, ref_leaf, ref_lane, tris);
  if (keep_refit) {
    BB_TRY(dmalloc(out.refit->tri_pos, n, stream));
    k_tri_pos<<<grid_for(n), kThreads, 0, stream>>>(trav_order, n, out.refit->tri_pos);
  }
  BB_TRY(cudaGetLastError());
  return cudaStreamSynchronize(stream);
}

}  // namespace vkptc
