// batch_loop.cu -- the loop driver of the batched renderer.
//
// The persistent driver (batch.cu) runs the five stages of an iteration in
// one cooperative kernel with grid barriers between them.  This driver runs
// each stage as its own kernel, so a stage gets the register budget and
// occupancy it needs (the traversal stages run at 64-80 registers, shading at
// ~94), and the iterations are driven by the device: the stages form the body
// of a CUDA graph while-node whose condition the last stage sets.  One
// graph launch renders every job; no kernel ever waits on another.
//
// Path state is kept in two compacted generations (structure of arrays).
// Each iteration:
//   REGEN   new camera paths from the 64-bit work counter are appended to
//           generation `cur` until it holds `capacity` paths
//   EXTEND  closest-hit traversal of generation `cur`, hit by position
//   SHADOW  any-hit traversal of the NEE queries the previous SHADE queued; a
//           visible query adds its term at its destination (a path of
//           generation `cur` or the finished list).  It touches nothing REGEN
//           and EXTEND touch, so in the graph it runs on a forked branch
//           beside them and each fills the other's tail.
//   DRAIN   the previous SHADE's finished paths to their jobs' staging slots
//   SHADE   one bounce per path: survivors appended to generation cur^1,
//           NEE queries to the shadow queue (with their destination), ended
//           paths to the finished list
//   DECIDE  another iteration while paths, camera paths, queries or finished
//           paths remain; cur ^= 1
// With SDF primitives in some job, two load-balanced stages join them: after
// EXTEND the SDF closest-hit test folds SDF hits into the hit buffer, and
// before SHADOW the SDF occlusion test drops the queries an SDF occludes (one
// march step per lane and call, lanes refilled as their queries finish).
// Positions are warp-aggregated appends, so every access coalesces.  The
// stagings are added to the films in sample order afterwards (as in the
// persistent driver), so films are bit-identical across drivers.
#include <algorithm>

#include "batch.cuh"
#include "integrator.cuh"
#include "traverse.cuh"

namespace vkptc {

namespace {

constexpr int kLCur = 0;            // current generation
constexpr int kLCount0 = 1;         // paths in generation 0 / 1: words 1, 2
constexpr int kLShadow = 3;
constexpr int kLFin0 = 12;          // finished-list length, by the generation that shaded it: words 12, 13
constexpr int kLFetchExt = 5, kLFetchShadow = 6;
constexpr int kLFetchSdf = 7, kLFetchSdfShadow = 11;
constexpr int kLWork = 8;           // 64-bit path counter (words 8, 9)
constexpr int kLBase = 10;          // paths in generation `cur` when its REGEN starts
constexpr int kLMore = kLoopCtlMore, kLIter = kLoopCtlIterations;

__device__ __forceinline__ bool block_leader() { return blockIdx.x == 0 && threadIdx.x == 0; }

__device__ __forceinline__ GeoView job_geo(const DevJob* jobs, uint32_t j) { return geo_of(jobs[j].scene); }

struct LoopExtendSource {
  const DevJob* jobs;
  PathSoA A;
  float2* hit;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm, GeoView& g) const {
    g = job_geo(jobs, A.job[j]);
    const float4 a = A.o[j], b = A.d[j];
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = kInf;
  }
  __device__ __forceinline__ void finish(uint32_t j, float t, uint32_t prim) const {
    hit[j] = make_float2(t, __uint_as_float(prim));
  }
};

struct LoopShadowSource {
  const DevJob* jobs;
  LoopPool P;
  PathSoA B;   // the next generation (destinations of surviving paths)
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm, GeoView& g) const {
    const float4 a = P.sh_o[j], b = P.sh_d[j];
    g = job_geo(jobs, __float_as_uint(b.w));
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = a.w;
  }
  __device__ __forceinline__ void finish(uint32_t j, float, uint32_t occluded) const {
    if (occluded) return;
    const uint32_t dst = P.sh_dst[j];
    if (dst == kLoopDropDst) return;
    const float4 c = P.sh_c[j];
    float4* r = (dst & kLoopFinBit) ? P.fin_rad + (dst & ~kLoopFinBit) : B.rad + dst;
    float4 v = *r;
    v.x = v.x + c.x;
    v.y = v.y + c.y;
    v.z = v.z + c.z;
    *r = v;
  }
};

// SDF closest-hit of the current generation: folds into the triangle hit.
struct LoopSdfExtSource {
  const DevJob* jobs;
  PathSoA A;
  float2* hit;
  __device__ __forceinline__ void load(uint32_t j, SdfLane& L) const {
    const DevScene& s = jobs[A.job[j]].scene;
    L.sdf = s.sdf;
    L.count = s.sdf_count;
    if (L.count == 0u) return;
    const float4 a = A.o[j], b = A.d[j];
    L.o = mk(a.x, a.y, a.z);
    L.d = mk(b.x, b.y, b.z);
    const float2 h = hit[j];
    L.best = h.x;
    L.prim = __float_as_uint(h.y);
  }
  __device__ __forceinline__ void finish(uint32_t j, const SdfLane& L) const {
    if (L.count != 0u) hit[j] = make_float2(L.best, __uint_as_float(L.prim));
  }
};

// SDF occlusion of the shadow queue: an occluded query is dropped (its bound
// set to 0 so the triangle any-hit does no work for it either).
struct LoopSdfShadowSource {
  const DevJob* jobs;
  LoopPool P;
  __device__ __forceinline__ void load(uint32_t j, SdfLane& L) const {
    const float4 a = P.sh_o[j], b = P.sh_d[j];
    const DevScene& s = jobs[__float_as_uint(b.w)].scene;
    L.sdf = s.sdf;
    L.count = s.sdf_count;
    L.o = mk(a.x, a.y, a.z);
    L.d = mk(b.x, b.y, b.z);
    L.best = a.w;
    L.prim = 0u;
  }
  __device__ __forceinline__ void finish(uint32_t j, const SdfLane& L) const {
    if (L.prim == 0u) return;
    P.sh_dst[j] = kLoopDropDst;
    P.sh_o[j].w = 0.0f;
  }
};

constexpr int kSdfStepsPerRefill = 8;

__device__ __forceinline__ void flush_sdf(DevCounters* ctr, const SdfCount& c) {
  warp_count(&ctr->sdf_tests, c.tests);
  warp_count(&ctr->sdf_steps, c.steps);
  warp_count(&ctr->sdf_hits, c.hits);
}

__device__ __forceinline__ TwoLevelStack loop_stack(int2* smem_stack, int scap, int2* spill, int total_cap) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t gthreads = gridDim.x * blockDim.x;
  return TwoLevelStack{smem_stack + threadIdx.x, static_cast<int>(blockDim.x), scap,
                       spill ? spill + gtid : nullptr, static_cast<int>(gthreads), total_cap};
}

template <bool kStats>
__device__ __forceinline__ void flush_stats(DevCounters* ctr, const TraceStats& st, bool shadow) {
  if (!kStats) return;
  if (shadow) {
    warp_count(&ctr->shadow_nodes, st.nodes);
    warp_count(&ctr->shadow_leaves, st.leaves);
    warp_count(&ctr->shadow_tris, st.tris);
    warp_count(&ctr->shadow_rays, st.rays);
  } else {
    warp_count(&ctr->nodes, st.nodes);
    warp_count(&ctr->leaves, st.leaves);
    warp_count(&ctr->tris, st.tris);
    warp_count(&ctr->ext_rays, st.rays);
  }
}

// ---------------------------------------------------------------- stages
__global__ void k_lp_init(uint32_t* ctl) {
  const uint32_t i = threadIdx.x;
  if (i < static_cast<uint32_t>(kLoopCtlWords)) ctl[i] = 0u;
}

// Order in which REGEN hands out a sample's pixels: 1 = 8x4 tiles, band of
// four rows by band (a warp's 32 camera rays cover a compact 8x4 block);
// 0 = scanline order.  Each path still writes its own pixel's staging slot,
// so films do not depend on the order.
#ifndef VKPTC_TILE_ORDER
#define VKPTC_TILE_ORDER 1
#endif
// The i-th pixel (y*W+x) of the tile order: bands of 4 rows (the last may be
// shorter), each band cut into 8-pixel-wide tiles left to right (the last may
// be narrower), each tile in row order.  A bijection on [0, W*H).
__device__ __forceinline__ uint32_t tile_order_pixel(uint32_t i, uint32_t W, uint32_t H) {
  const uint32_t band = i / (4u * W);
  const uint32_t y0 = 4u * band;
  const uint32_t bh = min(4u, H - y0);
  const uint32_t r = i - y0 * W;                 // index inside the band
  const uint32_t full = W / 8u;                  // full-width tiles in the band
  uint32_t x, y;
  if (r < full * 8u * bh) {
    const uint32_t t = r / (8u * bh), k = r - t * 8u * bh;
    x = 8u * t + (k & 7u);
    y = y0 + (k >> 3);
  } else {                                       // the narrow last tile
    const uint32_t tw = W - 8u * full, k = r - full * 8u * bh;
    x = 8u * full + k % tw;
    y = y0 + k / tw;
  }
  return y * W + x;
}

// 1: REGEN claims work items and queue slots once per block and iteration;
// 0: once per warp (ballot + shuffle).
#ifndef VKPTC_REGEN_BLOCK
#define VKPTC_REGEN_BLOCK 1
#endif
template <bool kParity>
__global__ void __launch_bounds__(256) k_lp_regen(const DevJob* __restrict__ jobs, uint32_t job_count,
                                                  unsigned long long total, LoopPool P) {
  const uint32_t cur = P.ctl[kLCur];
  uint32_t* count = P.ctl + kLCount0 + cur;
  // The count itself grows while this kernel appends; every block sizes its
  // share from the value the previous finish stage recorded.
  const uint32_t room = P.capacity - P.ctl[kLBase];
  if (block_leader()) {
    P.ctl[kLFetchExt] = 0u;
    P.ctl[kLFetchSdf] = 0u;
  }
  const PathSoA A = P.gen[cur];
  unsigned long long* work_next = reinterpret_cast<unsigned long long*>(P.ctl + kLWork);
  const uint32_t gthreads = gridDim.x * blockDim.x;
#if VKPTC_REGEN_BLOCK
  // One claim per block and iteration: the threads that take a path are a
  // prefix of the block (j < room, and g < total with g rising with the
  // thread index), so the leader claims the block's work items and queue
  // slots with one atomic each and thread t takes item g0 + t, slot q0 + t.
  __shared__ unsigned long long s_g0;
  __shared__ uint32_t s_q0, s_k;
#else
  const unsigned lane = threadIdx.x & 31u;
#endif
  for (uint32_t base = blockIdx.x * blockDim.x; base < room; base += gthreads) {
#if VKPTC_REGEN_BLOCK
    if (threadIdx.x == 0u) {
      const uint32_t cnt = min(blockDim.x, room - base);
      const unsigned long long g0 = atomicAdd(work_next, static_cast<unsigned long long>(cnt));
      const uint32_t k = g0 >= total ? 0u : static_cast<uint32_t>(min(static_cast<unsigned long long>(cnt), total - g0));
      s_g0 = g0;
      s_k = k;
      s_q0 = k ? atomicAdd(count, k) : 0u;
    }
    __syncthreads();
    const unsigned long long g = s_g0 + threadIdx.x;
    const bool ok = threadIdx.x < s_k;
    const uint32_t q = s_q0 + threadIdx.x;
    __syncthreads();   // the leader rewrites the shared words in the next iteration
#else
    const bool want = base + threadIdx.x < room;
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    unsigned long long g0 = 0ull;
    const int lead = __ffs(mask) - 1;
    if (mask != 0u && static_cast<int>(lane) == lead) g0 = atomicAdd(work_next, static_cast<unsigned long long>(__popc(mask)));
    g0 = __shfl_sync(0xffffffffu, g0, lead < 0 ? 0 : lead);
    const unsigned long long g = g0 + static_cast<unsigned long long>(__popc(mask & ((1u << lane) - 1u)));
    const bool ok = want && g < total;
    const uint32_t q = warp_append(count, ok);
#endif
    if (ok) {
      const uint32_t jb = find_job(jobs, job_count, g);
      const DevJob& J = jobs[jb];
      const uint32_t W = J.settings.width;
      const uint32_t idx = static_cast<uint32_t>(g - J.path_base);
      const uint32_t sl = idx / J.pixels;
#if VKPTC_TILE_ORDER
      const uint32_t px = tile_order_pixel(idx - sl * J.pixels, W, J.settings.height);
#else
      const uint32_t px = idx - sl * J.pixels;
#endif
      const uint32_t local = sl * J.pixels + px;   // the staging slot: sample-major, then pixel (y*W+x)
      V3 o, d;
      uint64_t rng;
      camera_path<kParity>(J.scene, J.settings, px % W, px / W, J.first_sample + sl, o, d, rng);
      A.job[q] = jb;
      A.local[q] = local;
      A.depth[q] = 0u;
      A.rng[q] = rng;
      A.o[q] = make_float4(o.x, o.y, o.z, 0.0f);
      A.d[q] = make_float4(d.x, d.y, d.z, 0.0f);
      A.thr[q] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
      A.rad[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
}

template <bool kStats, int kThreads, int kMinBlocks, bool kWt>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_lp_extend(const DevJob* __restrict__ jobs, LoopPool P, int scap,
                                                               int2* spill, int total_cap, int steps, DevCounters* ctr,
                                                               uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  const uint32_t cur = P.ctl[kLCur];
  const uint32_t n = P.ctl[kLCount0 + cur];
  if (n == 0u) return;
  const TwoLevelStack stk = loop_stack(smem_stack, scap, spill, total_cap);
  TraceStats st;
  uint32_t lerr = 0u;
  const LoopExtendSource src{jobs, P.gen[cur], P.hit};
  persistent_traverse<LoopExtendSource, false, kStats, kWt>(src, n, &P.ctl[kLFetchExt], stk, steps, st, lerr);
  flush_stats<kStats>(ctr, st, false);
  if (lerr) atomicOr(err, lerr);
}

__global__ void __launch_bounds__(256) k_lp_sdf(const DevJob* __restrict__ jobs, LoopPool P, DevCounters* ctr) {
  const uint32_t cur = P.ctl[kLCur];
  const uint32_t n = P.ctl[kLCount0 + cur];
  if (n == 0u) return;
  SdfCount c;
  const LoopSdfExtSource src{jobs, P.gen[cur], P.hit};
  sdf_persistent<LoopSdfExtSource, false>(src, n, &P.ctl[kLFetchSdf], kSdfStepsPerRefill, c);
  flush_sdf(ctr, c);
}

__global__ void __launch_bounds__(256) k_lp_sdf_shadow(const DevJob* __restrict__ jobs, LoopPool P, DevCounters* ctr) {
  const uint32_t n = P.ctl[kLShadow];
  if (n == 0u) return;
  SdfCount c;
  const LoopSdfShadowSource src{jobs, P};
  sdf_persistent<LoopSdfShadowSource, true>(src, n, &P.ctl[kLFetchSdfShadow], kSdfStepsPerRefill, c);
  flush_sdf(ctr, c);
}

// kSdf: some job has SDF primitives (the SDF stages run and the shading
// stage takes their hits); without, the shading code carries no SDF steps.
// kExotic: some job has a transmissive, clear-coat, sheen or toon material or
// an environment map; without, those branches are compiled out.
#ifndef VKPTC_LEAN_SHADE_BLOCKS
#define VKPTC_LEAN_SHADE_BLOCKS 3
#endif
template <bool kParity, bool kEffects, bool kSdf, bool kExotic>
__global__ void __launch_bounds__(256, (kEffects || kSdf || kExotic) ? 3 : VKPTC_LEAN_SHADE_BLOCKS) k_lp_shade(const DevJob* __restrict__ jobs, LoopPool P, DevCounters* ctr,
                                                  uint32_t sdf_staged) {
  const uint32_t cur = P.ctl[kLCur];
  const uint32_t n = P.ctl[kLCount0 + cur];
  const PathSoA A = P.gen[cur], B = P.gen[cur ^ 1u];
  const uint32_t gthreads = gridDim.x * blockDim.x;
  uint32_t shadow_tests = 0u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gthreads) {
    const uint32_t j = base + threadIdx.x;
    bool next = false, shadow = false, fin = false;
    uint32_t jb = 0u, local = 0u, depth = 0u;
    PathRegs pr;
    ShadeOut R;
    if (j < n) {
      jb = A.job[j];
      local = A.local[j];
      depth = A.depth[j];
      const DevJob& J = jobs[jb];
      const float4 o4 = A.o[j], d4 = A.d[j], t4 = A.thr[j], r4 = A.rad[j];
      const float2 h2 = P.hit[j];
      pr.o = mk(o4.x, o4.y, o4.z);
      pr.d = mk(d4.x, d4.y, d4.z);
      pr.thr = mk(t4.x, t4.y, t4.z);
      pr.rad = mk(r4.x, r4.y, r4.z);
      pr.segs = r4.w;
      pr.rng = A.rng[j];
      R = shade_bounce<kParity, kEffects, kSdf, kExotic>(J.scene, J.settings, J.scene.lights, depth, pr, h2.x,
                                                         __float_as_uint(h2.y),
                                          sdf_staged != 0u);
      next = R.next;
      fin = !R.next;
      shadow = R.shadow;
      shadow_tests += R.shadow_tests;
    }
    const uint32_t qn = warp_append(&P.ctl[kLCount0 + (cur ^ 1u)], next);
    if (next) {
      B.job[qn] = jb;
      B.local[qn] = local;
      B.depth[qn] = depth + 1u;
      B.rng[qn] = pr.rng;
      B.o[qn] = make_float4(pr.o.x, pr.o.y, pr.o.z, 0.0f);
      B.d[qn] = make_float4(pr.d.x, pr.d.y, pr.d.z, 0.0f);
      B.thr[qn] = make_float4(pr.thr.x, pr.thr.y, pr.thr.z, 0.0f);
      B.rad[qn] = make_float4(pr.rad.x, pr.rad.y, pr.rad.z, pr.segs);
    }
    const uint32_t qf = warp_append(&P.ctl[kLFin0 + cur], fin);
    if (fin) {
      P.fin_rad[qf] = make_float4(pr.rad.x, pr.rad.y, pr.rad.z, pr.segs);
      P.fin_job[qf] = jb;
      P.fin_local[qf] = local;
    }
    const uint32_t qs = warp_append(&P.ctl[kLShadow], shadow);
    if (shadow) {
      P.sh_o[qs] = make_float4(R.sh_o.x, R.sh_o.y, R.sh_o.z, R.sh_t);
      P.sh_d[qs] = make_float4(R.sh_d.x, R.sh_d.y, R.sh_d.z, __uint_as_float(jb));
      P.sh_c[qs] = make_float4(R.sh_c.x, R.sh_c.y, R.sh_c.z, 0.0f);
      P.sh_dst[qs] = next ? qn : (qf | kLoopFinBit);
    }
  }
  warp_count(&ctr->shadow_tests, shadow_tests);
}

template <bool kStats, int kThreads, int kMinBlocks, bool kWt>
__global__ void __launch_bounds__(kThreads, kMinBlocks) k_lp_shadow(const DevJob* __restrict__ jobs, LoopPool P, int scap,
                                                               int2* spill, int total_cap, int steps, DevCounters* ctr,
                                                               uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  const uint32_t n = P.ctl[kLShadow];
  if (n == 0u) return;
  const uint32_t cur = P.ctl[kLCur];
  const TwoLevelStack stk = loop_stack(smem_stack, scap, spill, total_cap);
  TraceStats st;
  uint32_t lerr = 0u;
  // The queries of the previous shading stage; their survivors are generation `cur` now.
  const LoopShadowSource src{jobs, P, P.gen[cur]};
  persistent_traverse<LoopShadowSource, true, kStats, kWt>(src, n, &P.ctl[kLFetchShadow], stk, steps, st, lerr);
  flush_stats<kStats>(ctr, st, true);
  if (lerr) atomicOr(err, lerr);
}

// Finished paths of the previous shading stage (their visible NEE terms
// added by the shadow stage) to their jobs' staging slots; then the words the
// coming shading stage appends to start from zero.
__global__ void __launch_bounds__(256) k_lp_drain(const DevJob* __restrict__ jobs, LoopPool P) {
  const uint32_t cur = P.ctl[kLCur];
  if (block_leader()) {
    P.ctl[kLCount0 + (cur ^ 1u)] = 0u;
    P.ctl[kLFin0 + cur] = 0u;
    P.ctl[kLShadow] = 0u;
    P.ctl[kLFetchShadow] = 0u;
    P.ctl[kLFetchSdfShadow] = 0u;
  }
  const uint32_t n = P.ctl[kLFin0 + (cur ^ 1u)];
  for (uint32_t f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
    const DevJob& J = jobs[P.fin_job[f]];
    J.staging[P.fin_local[f]] = P.fin_rad[f];
  }
}

// Loop condition after the shading stage: another iteration while paths
// survive, camera paths remain, or the shading stage left NEE queries or
// finished paths for the next iteration's shadow and drain stages.
__global__ void k_lp_decide(unsigned long long total, LoopPool P, cudaGraphConditionalHandle handle) {
  if (threadIdx.x != 0u) return;
  const uint32_t cur = P.ctl[kLCur];
  const unsigned long long work = *reinterpret_cast<const unsigned long long*>(P.ctl + kLWork);
  const uint32_t survivors = P.ctl[kLCount0 + (cur ^ 1u)];
  const uint32_t more =
      (survivors > 0u || work < total || P.ctl[kLShadow] > 0u || P.ctl[kLFin0 + cur] > 0u) ? 1u : 0u;
  P.ctl[kLMore] = more;
  P.ctl[kLBase] = survivors;
  P.ctl[kLCur] = cur ^ 1u;
  P.ctl[kLIter] += 1u;
  if (handle) cudaGraphSetConditional(handle, more);
}

template <typename K>
int blocks_per_sm(K kernel, int block, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, smem) != cudaSuccess) return 0;
  return n;
}

template <typename K>
cudaError_t set_smem_attr(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// Traversal stage variants: [triangle test][stats][register variant].
// Variants 0..3: at least 1..4 resident 256-thread blocks per SM (at most
// 255, 128, 80 and 64 registers); variant 4: at least 7 resident 128-thread
// blocks (at most 72 registers, 28 warps; launched with 128 threads only).  Stats runs use
// the unconstrained variant at the launch's block size.
using LoopTraceFn = void (*)(const DevJob*, LoopPool, int, int2*, int, int, DevCounters*, uint32_t*);
LoopTraceFn extend_fn(bool stats, int occ, bool wt) {
  static const LoopTraceFn t[2][2][5] = {
      {{k_lp_extend<false, 256, 1, false>, k_lp_extend<false, 256, 2, false>, k_lp_extend<false, 256, 3, false>,
        k_lp_extend<false, 256, 4, false>, k_lp_extend<false, 128, 7, false>},
       {k_lp_extend<true, 256, 1, false>, k_lp_extend<true, 256, 1, false>, k_lp_extend<true, 256, 1, false>,
        k_lp_extend<true, 256, 1, false>, k_lp_extend<true, 128, 1, false>}},
      {{k_lp_extend<false, 256, 1, true>, k_lp_extend<false, 256, 2, true>, k_lp_extend<false, 256, 3, true>,
        k_lp_extend<false, 256, 4, true>, k_lp_extend<false, 128, 7, true>},
       {k_lp_extend<true, 256, 1, true>, k_lp_extend<true, 256, 1, true>, k_lp_extend<true, 256, 1, true>,
        k_lp_extend<true, 256, 1, true>, k_lp_extend<true, 128, 1, true>}}};
  return t[wt ? 1 : 0][stats ? 1 : 0][occ < 0 ? 0 : (occ > 4 ? 4 : occ)];
}
LoopTraceFn shadow_fn(bool stats, int occ, bool wt) {
  static const LoopTraceFn t[2][2][5] = {
      {{k_lp_shadow<false, 256, 1, false>, k_lp_shadow<false, 256, 2, false>, k_lp_shadow<false, 256, 3, false>,
        k_lp_shadow<false, 256, 4, false>, k_lp_shadow<false, 128, 7, false>},
       {k_lp_shadow<true, 256, 1, false>, k_lp_shadow<true, 256, 1, false>, k_lp_shadow<true, 256, 1, false>,
        k_lp_shadow<true, 256, 1, false>, k_lp_shadow<true, 128, 1, false>}},
      {{k_lp_shadow<false, 256, 1, true>, k_lp_shadow<false, 256, 2, true>, k_lp_shadow<false, 256, 3, true>,
        k_lp_shadow<false, 256, 4, true>, k_lp_shadow<false, 128, 7, true>},
       {k_lp_shadow<true, 256, 1, true>, k_lp_shadow<true, 256, 1, true>, k_lp_shadow<true, 256, 1, true>,
        k_lp_shadow<true, 256, 1, true>, k_lp_shadow<true, 128, 1, true>}}};
  return t[wt ? 1 : 0][stats ? 1 : 0][occ < 0 ? 0 : (occ > 4 ? 4 : occ)];
}

// Shading stage variants: [parity][effects][sdf][exotic].
using LoopShadeFn = void (*)(const DevJob*, LoopPool, DevCounters*, uint32_t);
template <bool kP, bool kE>
LoopShadeFn shade_fn_pe(bool sdf, bool exotic) {
  static const LoopShadeFn t[2][2] = {{k_lp_shade<kP, kE, false, false>, k_lp_shade<kP, kE, false, true>},
                                      {k_lp_shade<kP, kE, true, false>, k_lp_shade<kP, kE, true, true>}};
  return t[sdf ? 1 : 0][exotic ? 1 : 0];
}
LoopShadeFn shade_fn(bool parity, bool effects, bool sdf, bool exotic) {
  if (parity) return effects ? shade_fn_pe<true, true>(sdf, exotic) : shade_fn_pe<true, false>(sdf, exotic);
  return effects ? shade_fn_pe<false, true>(sdf, exotic) : shade_fn_pe<false, false>(sdf, exotic);
}

}  // namespace

LoopGrids BatchLoopGrids(int block, size_t smem, bool parity, bool stats, int occupancy, int sm_count, bool watertight,
                         bool effects, bool sdf, bool exotic) {
  LoopGrids g{};
  g.regen = sm_count * (parity ? blocks_per_sm(k_lp_regen<true>, block, 0) : blocks_per_sm(k_lp_regen<false>, block, 0));
  g.extend = sm_count * blocks_per_sm(extend_fn(stats, occupancy, watertight), block, smem);
  g.shade = sm_count * blocks_per_sm(shade_fn(parity, effects, sdf, exotic), block, 0);
  g.shadow = sm_count * blocks_per_sm(shadow_fn(stats, occupancy, watertight), block, smem);
  g.finish = sm_count * blocks_per_sm(k_lp_drain, block, 0);
  g.sdf = sm_count * std::min(blocks_per_sm(k_lp_sdf, block, 0), blocks_per_sm(k_lp_sdf_shadow, block, 0));
  return g;
}

cudaError_t ConfigureBatchLoopSmem(size_t bytes) {
  const int b = static_cast<int>(bytes);
  cudaError_t e = cudaSuccess;
  for (int wt = 0; wt < 2 && e == cudaSuccess; ++wt)
    for (int st = 0; st < 2 && e == cudaSuccess; ++st)
      for (int o = 0; o < 5 && e == cudaSuccess; ++o) {
        e = set_smem_attr(extend_fn(st != 0, o, wt != 0), b);
        if (e == cudaSuccess) e = set_smem_attr(shadow_fn(st != 0, o, wt != 0), b);
      }
  return e;
}

cudaError_t LaunchBatchLoopInit(const LoopPool& pool, cudaStream_t stream) {
  k_lp_init<<<1, kLoopCtlWords, 0, stream>>>(pool.ctl);
  return cudaGetLastError();
}

cudaError_t LaunchBatchLoopIteration(const DevJob* jobs, uint32_t job_count, unsigned long long total,
                                     const LoopPool& P, const BatchLaunch& bl, const LoopGrids& g,
                                     cudaGraphConditionalHandle handle, DevCounters* ctr, uint32_t* err,
                                     cudaEvent_t* marks, const LoopFork* fork) {
  const size_t smem = StackSmemBytes(bl.block, bl.smem_entries);
  cudaStream_t s = bl.stream;
  auto mark = [&](int i) {
    if (marks) cudaEventRecord(marks[i], s);
  };
  // The shadow branch: the previous shading stage's NEE queries, on the side
  // stream when forked (it only touches the shadow queue, the finished list
  // and the radiance words of generation `cur`, none of which REGEN or EXTEND
  // touch), else after EXTEND.
  auto shadow_branch = [&](cudaStream_t q) {
    if (bl.sdf) k_lp_sdf_shadow<<<g.sdf, bl.block, 0, q>>>(jobs, P, ctr);
    shadow_fn(bl.stats, bl.occupancy, bl.watertight)<<<g.shadow, bl.block, smem, q>>>(
        jobs, P, bl.smem_entries, bl.spill_shadow, bl.stack_cap, bl.steps, ctr, err);
  };
  const bool forked = fork != nullptr && marks == nullptr;
  if (forked) {
    cudaEventRecord(fork->fork, s);
    cudaStreamWaitEvent(fork->side, fork->fork, 0);
    shadow_branch(fork->side);
    cudaEventRecord(fork->join, fork->side);
  }
  mark(0);
  if (bl.parity) k_lp_regen<true><<<g.regen, bl.block, 0, s>>>(jobs, job_count, total, P);
  else k_lp_regen<false><<<g.regen, bl.block, 0, s>>>(jobs, job_count, total, P);
  mark(1);
  extend_fn(bl.stats, bl.occupancy, bl.watertight)<<<g.extend, bl.block, smem, s>>>(jobs, P, bl.smem_entries, bl.spill, bl.stack_cap,
                                                                      bl.steps, ctr, err);
  if (bl.sdf) k_lp_sdf<<<g.sdf, bl.block, 0, s>>>(jobs, P, ctr);
  mark(2);
  if (forked) cudaStreamWaitEvent(s, fork->join, 0);
  else shadow_branch(s);
  mark(3);
  k_lp_drain<<<g.finish, bl.block, 0, s>>>(jobs, P);
  mark(4);
  const uint32_t staged = bl.sdf ? 1u : 0u;
  shade_fn(bl.parity, bl.effects, bl.sdf, bl.exotic)<<<g.shade, bl.block, 0, s>>>(jobs, P, ctr, staged);
  mark(5);
  k_lp_decide<<<1, 32, 0, s>>>(total, P, handle);
  return cudaGetLastError();
}

}  // namespace vkptc
