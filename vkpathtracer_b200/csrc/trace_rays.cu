// trace_rays.cu -- batched closest-hit and any-hit ray queries (sm_100a).
//
// The batched form of the reference's IRayAccelerator::intersect
// (src/pathtracer/PathTracer.h:1001-1036; CPU implementation
// src/pathtracer/CpuBvhAccelerator.cpp:360-477): one persistent kernel walks
// the wide BVH for every ray of an array (traverse.cuh).
//
// This file's traversal takes the reciprocal direction and the leaf test's
// 1/det by __frcp_rn, the other files' by __fdiv_rn(1.0f, x).  Both are the
// correctly rounded reciprocal, so the hits are the same bit for bit; the
// reciprocal sequence measured about 8 % faster in this kernel and slower in
// the render kernels around the same traversal, so each file takes its own.
#define VKPTC_RCP_RAY 1
#define VKPTC_RCP_TRI 1

#include <type_traits>

#include "kernels.cuh"
#include "traverse.cuh"

namespace vkptc {

namespace {

struct RaysSource {   // batched ray queries from a ray array
  GeoView geo;
  const float* rays;
  const float* tmax;
  uint32_t* prim_out;
  float* t_out;
  bool any;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm, GeoView& g) const {
    g = geo;
    const float2* rp = reinterpret_cast<const float2*>(rays + 6ull * j);
    const float2 a = __ldg(rp), b = __ldg(rp + 1), c = __ldg(rp + 2);
    o = mk(a.x, a.y, b.x);
    d = mk(b.y, c.x, c.y);
    tm = tmax ? __ldg(tmax + j) : kInf;
  }
  __device__ __forceinline__ void finish(uint32_t j, float t, uint32_t prim) const {
    prim_out[j] = prim;
    if (t_out) t_out[j] = any ? (prim ? 0.0f : kInf) : t;
  }
};

template <bool kAny, bool kStats, bool kWt>
__global__ void __launch_bounds__(256) k_trace_rays(DevScene s, RaysSource src, uint32_t n, uint32_t* fetch, int scap,
                                                    int2* spill, int total, int steps, DevCounters* ctr, uint32_t* err) {
  run_persistent<RaysSource, kAny, kStats, kWt>(src, n, fetch, scap, spill, total, steps, &ctr->nodes, &ctr->leaves,
                                                &ctr->tris, &ctr->ext_rays, err);
}

template <typename K>
cudaError_t set_trace_smem(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

}  // namespace

cudaError_t LaunchTraceRays(const DevScene& s, const float* rays, const float* tmax, uint64_t n, bool any_hit,
                            uint32_t* prim_out, float* t_out, const LaunchShape& ls, DevCounters* ctr,
                            uint32_t* err, uint32_t* fetch) {
  if (n == 0) return cudaSuccess;
  const size_t smem = StackSmemBytes(ls.block, ls.smem_entries);
  cudaError_t e = cudaMemsetAsync(fetch, 0, sizeof(uint32_t), ls.stream);
  if (e != cudaSuccess) return e;
  const RaysSource src{geo_of(s), rays, tmax, prim_out, t_out, any_hit};
  const uint32_t n32 = static_cast<uint32_t>(n);
#define VKPTC_TR(A, S, W) \
  k_trace_rays<A, S, W><<<ls.grid, ls.block, smem, ls.stream>>>(s, src, n32, fetch, ls.smem_entries, ls.spill, ls.stack_cap, ls.steps, ctr, err)
#define VKPTC_TR2(A, S) \
  if (s.watertight) VKPTC_TR(A, S, true); \
  else VKPTC_TR(A, S, false)
  if (any_hit) {
    if (ctr) VKPTC_TR2(true, true);
    else VKPTC_TR2(true, false);
  } else {
    if (ctr) VKPTC_TR2(false, true);
    else VKPTC_TR2(false, false);
  }
#undef VKPTC_TR2
#undef VKPTC_TR
  return cudaGetLastError();
}

cudaError_t ConfigureTraceRaysSmem(size_t bytes) {
  const int b = static_cast<int>(bytes);
  cudaError_t e = cudaSuccess;
  const auto all = [&](auto wt) {
    constexpr bool W = decltype(wt)::value;
    if (e == cudaSuccess) e = set_trace_smem(k_trace_rays<true, true, W>, b);
    if (e == cudaSuccess) e = set_trace_smem(k_trace_rays<true, false, W>, b);
    if (e == cudaSuccess) e = set_trace_smem(k_trace_rays<false, true, W>, b);
    if (e == cudaSuccess) e = set_trace_smem(k_trace_rays<false, false, W>, b);
  };
  all(std::false_type{});
  all(std::true_type{});
  return e;
}

}  // namespace vkptc
