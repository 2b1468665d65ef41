// kernels.cu -- wavefront path tracing and ray-query kernels (sm_100a).
//
// The integrator restates the reference's scalar CPU tracer:
//   camera_rays / shade_pixel   src/pathtracer/ScalarCpuPathTracer.Render.cpp:55-119, 228-284
//   trace                       src/pathtracer/ScalarCpuPathTracer.cpp:1148-1289
//   sample_direct_light         src/pathtracer/ScalarCpuPathTracer.cpp:1022-1118
//   light_pdf / MisWeight       src/pathtracer/ScalarCpuPathTracer.cpp:1120-1146
//   hemisphere / Phong lobe     src/pathtracer/ScalarCpuPathTracer.cpp:978-1020
//   FilmBuffer add / resolve    src/pathtracer/FilmBuffer.cpp:80-91, 160-214
// split into wavefront stages that exchange structure-of-arrays queues:
//   raygen -> for each depth: extend (closest hit) -> shade (material, NEE
//   set-up, BSDF sample, Russian roulette; appends shadow queries and the next
//   extension queue with warp-aggregated atomics) -> shadow (any hit) ->
//   accumulate into the film in sample order.
// The per-path RNG stream is keyed exactly as the reference keys it, so the
// wavefront reordering does not change any random number a path draws, and
// the stages add radiance terms in the reference's order (emission, then the
// NEE term of the same bounce, then the next bounce).
#include <algorithm>
#include <type_traits>

#include "kernels.cuh"
#include "integrator.cuh"
#include "traverse.cuh"

namespace vkptc {

size_t StackSmemBytes(int block, int cap) { return static_cast<size_t>(block) * cap * sizeof(int2); }

size_t SpillEntries(const LaunchShape& ls) {
  const int extra = ls.stack_cap - ls.smem_entries;
  return extra > 0 ? static_cast<size_t>(ls.grid) * ls.block * extra : 0u;
}

// ============================================================ query sources
// Each source supplies queries to persistent_traverse() and consumes results.
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

struct ExtendSource {  // closest hit for the queued paths of a wave
  GeoView geo;
  const uint32_t* q;
  const float4* ray_o;
  const float4* ray_d;
  float2* hit;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm, GeoView& g) const {
    g = geo;
    const uint32_t p = q[j];
    const float4 a = ray_o[p], b = ray_d[p];
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = kInf;
  }
  __device__ __forceinline__ void finish(uint32_t j, float t, uint32_t prim) const {
    hit[q[j]] = make_float2(t, __uint_as_float(prim));
  }
};

struct ShadowSource {  // any hit for the NEE queries; adds the term when visible
  GeoView geo;
  const float4* sh_o;
  const float4* sh_d;
  const float4* sh_c;
  const uint32_t* sh_path;
  float4* rad;
  __device__ __forceinline__ void load(uint32_t j, V3& o, V3& d, float& tm, GeoView& g) const {
    g = geo;
    const float4 a = sh_o[j], b = sh_d[j];
    o = mk(a.x, a.y, a.z);
    d = mk(b.x, b.y, b.z);
    tm = a.w;
  }
  __device__ __forceinline__ void finish(uint32_t j, float, uint32_t occluded) const {
    if (occluded) return;
    const uint32_t p = sh_path[j];
    const float4 c = sh_c[j];
    float4 r = rad[p];
    r.x = r.x + c.x;
    r.y = r.y + c.y;
    r.z = r.z + c.z;
    rad[p] = r;
  }
};

template <class Src, bool kAny, bool kStats, bool kWt = false>
__device__ __forceinline__ void run_persistent(const Src& src, uint32_t n, uint32_t* fetch,
                                               int scap, int2* spill, int total, int steps,
                                               unsigned long long* c_nodes, unsigned long long* c_leaves,
                                               unsigned long long* c_tris, unsigned long long* c_rays, uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int gstride = static_cast<int>(gridDim.x * blockDim.x);
  TwoLevelStack stk{smem_stack + threadIdx.x, static_cast<int>(blockDim.x), scap,
                    spill ? spill + gtid : nullptr, gstride, total};
  TraceStats st;
  uint32_t lerr = 0u;
  persistent_traverse<Src, kAny, kStats, kWt>(src, n, fetch, stk, steps, st, lerr);
  if (kStats) {
    warp_count(c_nodes, st.nodes);
    warp_count(c_leaves, st.leaves);
    warp_count(c_tris, st.tris);
    warp_count(c_rays, st.rays);
  }
  if (lerr) atomicOr(err, lerr);
}

// =============================================================== ray queries
template <bool kAny, bool kStats, bool kWt>
__global__ void __launch_bounds__(256) k_trace_rays(DevScene s, RaysSource src, uint32_t n, uint32_t* fetch, int scap,
                                                    int2* spill, int total, int steps, DevCounters* ctr, uint32_t* err) {
  run_persistent<RaysSource, kAny, kStats, kWt>(src, n, fetch, scap, spill, total, steps, &ctr->nodes, &ctr->leaves,
                                                &ctr->tris, &ctr->ext_rays, err);
}

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

// ==================================================================== raygen
template <bool kParity>
__global__ void __launch_bounds__(256) k_raygen(DevScene s, DevSettings st, WaveState w, WaveTile tile) {
  const uint32_t tile_px = tile.w * tile.h;
  const uint32_t n = tile_px * tile.sample_count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t sl = i / tile_px, pl = i - sl * tile_px;
    const uint32_t x = tile.x + pl % tile.w, y = tile.y + pl / tile.w;
    V3 o, d;
    uint64_t rng;
    camera_path<kParity>(s, st, x, y, tile.first_sample + sl, o, d, rng);
    w.rng[i] = rng;
    w.ray_o[i] = make_float4(o.x, o.y, o.z, 0.0f);
    w.ray_d[i] = make_float4(d.x, d.y, d.z, 0.0f);
    w.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    w.rad[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    w.q[0][i] = i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.counts[0] = n;
    w.counts[1] = 0u;
    w.counts[2] = 0u;
    w.counts[3] = 0u;   // extension fetch counter
    w.counts[4] = 0u;   // shadow fetch counter
  }
}

// ==================================================================== extend
// Closest-hit traversal of the current extension queue (persistent warps).
// Zeroes the next queue's and the shadow queue's sizes for the shade stage.
template <bool kStats, bool kWt>
__global__ void __launch_bounds__(256) k_extend(DevScene s, WaveState w, uint32_t cur, int scap, int2* spill,
                                                int total, int steps, DevCounters* ctr, uint32_t* err) {
  const uint32_t n = w.counts[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.counts[cur ^ 1u] = 0u;
    w.counts[2] = 0u;
  }
  const ExtendSource src{geo_of(s), w.q[cur], w.ray_o, w.ray_d, w.hit};
  run_persistent<ExtendSource, false, kStats, kWt>(src, n, &w.counts[3], scap, spill, total, steps, &ctr->nodes,
                                                   &ctr->leaves, &ctr->tris, &ctr->ext_rays, err);
}

constexpr uint32_t kSmemLights = 64;   // lights staged in shared memory by the shade stage

template <bool kParity, bool kEffects>
__global__ void __launch_bounds__(256, 3) k_shade(DevScene s, DevSettings st, WaveState w, uint32_t cur,
                                               uint32_t depth, DevCounters* ctr) {
  __shared__ float sm_lights[16 * kSmemLights];
  const bool staged = s.light_count <= kSmemLights;
  if (staged) {
    for (uint32_t k = threadIdx.x; k < 16u * s.light_count; k += blockDim.x) sm_lights[k] = s.lights[k];
    __syncthreads();
  }
  const float* lights = staged ? sm_lights : s.lights;
  const uint32_t n = w.counts[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.counts[3] = 0u;   // the extension stage of the next depth fetches from 0
    w.counts[4] = 0u;   // the shadow stage of this depth fetches from 0
  }
  const uint32_t* q = w.q[cur];
  uint32_t* qn = w.q[cur ^ 1u];
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t j = base + threadIdx.x;
    bool emit_next = false, emit_shadow = false;
    uint32_t p = 0u;
    uint32_t shadow_tests = 0u;
    SdfCount sdf_n;
    // shadow query payload
    V3 sh_o = mk(0, 0, 0), sh_d = mk(0, 0, 0), sh_c = mk(0, 0, 0);
    float sh_t = 0.0f;
    if (j < n) {
      p = q[j];
      const float4 o4 = w.ray_o[p], d4 = w.ray_d[p], t4 = w.thr[p], r4 = w.rad[p];
      const float2 h2 = w.hit[p];
      PathRegs P;
      P.o = mk(o4.x, o4.y, o4.z);
      P.d = mk(d4.x, d4.y, d4.z);
      P.thr = mk(t4.x, t4.y, t4.z);
      P.rad = mk(r4.x, r4.y, r4.z);
      P.segs = r4.w;
      P.rng = w.rng[p];
      const ShadeOut R = shade_bounce<kParity, kEffects>(s, st, lights, depth, P, h2.x, __float_as_uint(h2.y));
      if (R.next) {
        w.ray_o[p] = make_float4(P.o.x, P.o.y, P.o.z, 0.0f);
        w.ray_d[p] = make_float4(P.d.x, P.d.y, P.d.z, 0.0f);
        w.thr[p] = make_float4(P.thr.x, P.thr.y, P.thr.z, 0.0f);
        w.rng[p] = P.rng;
      }
      w.rad[p] = make_float4(P.rad.x, P.rad.y, P.rad.z, P.segs);
      emit_next = R.next;
      emit_shadow = R.shadow;
      shadow_tests = R.shadow_tests;
      sdf_n = R.sdf;
      sh_o = R.sh_o;
      sh_d = R.sh_d;
      sh_c = R.sh_c;
      sh_t = R.sh_t;
    }
    // Warp-aggregated appends (the whole warp reaches these together).
    const uint32_t slot_n = warp_append(&w.counts[cur ^ 1u], emit_next);
    if (emit_next) qn[slot_n] = p;
    const uint32_t slot_s = warp_append(&w.counts[2], emit_shadow);
    if (emit_shadow) {
      w.sh_path[slot_s] = p;
      w.sh_o[slot_s] = make_float4(sh_o.x, sh_o.y, sh_o.z, sh_t);
      w.sh_d[slot_s] = make_float4(sh_d.x, sh_d.y, sh_d.z, 0.0f);
      w.sh_c[slot_s] = make_float4(sh_c.x, sh_c.y, sh_c.z, 0.0f);
    }
    warp_count(&ctr->shadow_tests, shadow_tests);
    if (s.sdf_count != 0u) {
      warp_count(&ctr->sdf_tests, sdf_n.tests);
      warp_count(&ctr->sdf_steps, sdf_n.steps);
      warp_count(&ctr->sdf_hits, sdf_n.hits);
    }
  }
}

// ==================================================================== shadow
// Any-hit visibility of the NEE queries (persistent warps); adds the NEE term
// of every visible query to its path's radiance.
template <bool kStats, bool kWt>
__global__ void __launch_bounds__(256) k_shadow(DevScene s, WaveState w, int scap, int2* spill, int total, int steps,
                                                DevCounters* ctr, uint32_t* err) {
  const uint32_t n = w.counts[2];
  const ShadowSource src{geo_of(s), w.sh_o, w.sh_d, w.sh_c, w.sh_path, w.rad};
  run_persistent<ShadowSource, true, kStats, kWt>(src, n, &w.counts[4], scap, spill, total, steps, &ctr->shadow_nodes,
                                             &ctr->shadow_leaves, &ctr->shadow_tris, &ctr->shadow_rays, err);
}

// Scenes with transmissive materials: the reference's closest-hit loop that
// steps through up to 8 transmissive occluders (one query per thread).
template <bool kStats, bool kWt>
__global__ void __launch_bounds__(256) k_shadow_transmissive(DevScene s, WaveState w, int cap, DevCounters* ctr, uint32_t* err) {
  extern __shared__ int2 smem_stack[];
  SmemStack stk{smem_stack + threadIdx.x, static_cast<int>(blockDim.x), cap};
  const uint32_t n = w.counts[2];
  uint32_t local_err = 0u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const uint32_t j = base + threadIdx.x;
    TraceStats st;
    SdfCount sdf_n;
    if (j < n) {
      const float4 o4 = w.sh_o[j], d4 = w.sh_d[j];
      V3 so = mk(o4.x, o4.y, o4.z);
      const V3 sd = mk(d4.x, d4.y, d4.z);
      float remain = o4.w;
      bool visible = true;
      if (!s.has_transmissive) {
        const RayPrep r = prep_ray(so, sd, s.reference_tree != 0u, kWt);
        visible = !trace_any<kStats, kWt>(s, r, remain, stk, st, local_err);
      } else {
        // Closest-hit loop that steps through up to 8 transmissive occluders
        // (src/pathtracer/ScalarCpuPathTracer.cpp:1067-1087).
        for (uint32_t skips = 0; skips < 8u && remain > 0.004f; ++skips) {
          const RayPrep r = prep_ray(so, sd, s.reference_tree != 0u, kWt);
          float t;
          uint32_t prim;
          trace_closest<kStats, kWt>(s, r, stk, t, prim, st, local_err);
          if (s.sdf_count != 0u) sdf_closest(s.sdf, s.sdf_count, so, sd, t, prim, sdf_n);
          if (prim == kMiss || t >= remain) break;
          const uint32_t mat_index = (prim & kSdfTag) ? sdf_material(s.sdf, prim & ~kSdfTag)
                                                      : __float_as_uint(__ldg(s.shade + prim).w);
          const uint32_t mi = mat_index < s.material_count - 1u ? mat_index : s.material_count - 1u;
          const float* mm = s.materials + 16u * mi;
          const bool tr = static_cast<uint32_t>(mm[7] + 0.5f) == 5u || mm[10] > 0.05f;
          if (!tr) {
            visible = false;
            break;
          }
          const float adv = t + 0.004f;
          so = add(so, mul(sd, adv));
          remain -= adv;
        }
      }
      if (visible) {
        const uint32_t p = w.sh_path[j];
        const float4 c = w.sh_c[j];
        float4 r = w.rad[p];
        r.x = r.x + c.x;
        r.y = r.y + c.y;
        r.z = r.z + c.z;
        w.rad[p] = r;
      }
    }
    if (kStats) {
      warp_count(&ctr->shadow_nodes, st.nodes);
      warp_count(&ctr->shadow_leaves, st.leaves);
      warp_count(&ctr->shadow_tris, st.tris);
      warp_count(&ctr->shadow_rays, j < n ? 1u : 0u);
    }
    if (s.sdf_count != 0u) {
      warp_count(&ctr->sdf_tests, sdf_n.tests);
      warp_count(&ctr->sdf_steps, sdf_n.steps);
      warp_count(&ctr->sdf_hits, sdf_n.hits);
    }
  }
  if (local_err) atomicOr(err, local_err);
}

// ================================================================ accumulate
__global__ void __launch_bounds__(256) k_accumulate(DevSettings st, WaveState w, WaveTile tile, Film film,
                                                    DevCounters* ctr) {
  const uint32_t tile_px = tile.w * tile.h;
  for (uint32_t base = blockIdx.x * blockDim.x; base < tile_px; base += gridDim.x * blockDim.x) {
    const uint32_t pl = base + threadIdx.x;
    uint32_t samples = 0u, segs = 0u, dropped = 0u;
    if (pl < tile_px) {
      const uint32_t x = tile.x + pl % tile.w, y = tile.y + pl / tile.w;
      const size_t px = static_cast<size_t>(y) * film.width + x;
      float4 acc = film.sum[px];
      uint32_t cnt = film.count[px];
      for (uint32_t sl = 0; sl < tile.sample_count; ++sl) {
        const float4 r = w.rad[sl * tile_px + pl];
        if (!(isfinite(r.x) && isfinite(r.y) && isfinite(r.z))) {
          ++dropped;   // dropped before the film, like the reference's shade_pixel
          continue;
        }
        float cx = r.x, cy = r.y, cz = r.z;
        if (st.firefly_clamp > 0.0f) {
          cx = smin(cx, st.firefly_clamp);
          cy = smin(cy, st.firefly_clamp);
          cz = smin(cz, st.firefly_clamp);
        }
        acc.x = acc.x + cx;
        acc.y = acc.y + cy;
        acc.z = acc.z + cz;
        ++cnt;
        ++samples;
        segs += static_cast<uint32_t>(r.w);
      }
      film.sum[px] = acc;
      film.count[px] = cnt;
    }
    warp_count(&ctr->samples, samples);
    warp_count(&ctr->rays, segs);
    warp_count(&ctr->dropped, dropped);
  }
}

cudaError_t LaunchWave(const DevScene& s, const DevSettings& st, const WaveState& w, const WaveTile& tile,
                       const Film& film, bool parity, bool stats, const LaunchShape& ls, DevCounters* ctr,
                       uint32_t* err, StageTimer* timer) {
  const size_t smem = StackSmemBytes(ls.block, ls.smem_entries);
  const size_t smem_full = StackSmemBytes(ls.block, ls.stack_cap);
  StageTimer dummy;
  StageTimer& tm = timer ? *timer : dummy;
  tm.begin(0, ls.stream);
  if (parity) k_raygen<true><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, tile);
  else k_raygen<false><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, tile);
  tm.end(ls.stream);
  uint32_t cur = 0u;
  for (uint32_t depth = 0; depth < st.max_depth; ++depth) {
    tm.begin(1, ls.stream);
#define VKPTC_EXT(S, W) \
  k_extend<S, W><<<ls.grid, ls.block, smem, ls.stream>>>(s, w, cur, ls.smem_entries, ls.spill, ls.stack_cap, ls.steps, ctr, err)
    if (s.watertight) {
      if (stats) VKPTC_EXT(true, true);
      else VKPTC_EXT(false, true);
    } else {
      if (stats) VKPTC_EXT(true, false);
      else VKPTC_EXT(false, false);
    }
#undef VKPTC_EXT
    tm.end(ls.stream);
    tm.begin(2, ls.stream);
    if (s.has_effects) {
      if (parity) k_shade<true, true><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, cur, depth, ctr);
      else k_shade<false, true><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, cur, depth, ctr);
    } else {
      if (parity) k_shade<true, false><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, cur, depth, ctr);
      else k_shade<false, false><<<ls.grid, ls.block, 0, ls.stream>>>(s, st, w, cur, depth, ctr);
    }
    tm.end(ls.stream);
    if (st.enable_nee) {
      tm.begin(3, ls.stream);
#define VKPTC_SHT(S, W) \
  k_shadow_transmissive<S, W><<<ls.grid, ls.block, smem_full, ls.stream>>>(s, w, ls.stack_cap, ctr, err)
#define VKPTC_SH(S, W) \
  k_shadow<S, W><<<ls.grid, ls.block, smem, ls.stream>>>(s, w, ls.smem_entries, ls.spill, ls.stack_cap, ls.steps, ctr, err)
      if (s.has_transmissive) {
        if (s.watertight) {
          if (stats) VKPTC_SHT(true, true);
          else VKPTC_SHT(false, true);
        } else {
          if (stats) VKPTC_SHT(true, false);
          else VKPTC_SHT(false, false);
        }
      } else {
        if (s.watertight) {
          if (stats) VKPTC_SH(true, true);
          else VKPTC_SH(false, true);
        } else {
          if (stats) VKPTC_SH(true, false);
          else VKPTC_SH(false, false);
        }
      }
#undef VKPTC_SH
#undef VKPTC_SHT
      tm.end(ls.stream);
    }
    cur ^= 1u;
  }
  tm.begin(4, ls.stream);
  k_accumulate<<<ls.grid, ls.block, 0, ls.stream>>>(st, w, tile, film, ctr);
  tm.end(ls.stream);
  return cudaGetLastError();
}

// ==================================================================== film
__global__ void k_resolve_hdr(Film film, float* out) {
  const size_t npx = static_cast<size_t>(film.width) * film.height;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < npx;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint32_t c = film.count[i];
    const float inv = 1.0f / static_cast<float>(c > 1u ? c : 1u);
    const float4 v = film.sum[i];
    out[3 * i + 0] = v.x * inv;
    out[3 * i + 1] = v.y * inv;
    out[3 * i + 2] = v.z * inv;
  }
}

__global__ void k_pack_film(const float4* __restrict__ sum, size_t npx, float* __restrict__ out) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < npx;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float4 v = sum[i];
    out[3 * i + 0] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
  }
}

__global__ void __launch_bounds__(256) k_read_probe(const float4* __restrict__ buf, size_t n, uint32_t reps,
                                                     float* sink) {
  const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
  float acc = 0.0f;
  for (uint32_t r = 0; r < reps; ++r) {
    size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {
      const float4 a = __ldcg(buf + i), b = __ldcg(buf + i + stride);
      const float4 c = __ldcg(buf + i + 2 * stride), d = __ldcg(buf + i + 3 * stride);
      acc += (a.x + b.y) + (c.z + d.w);
    }
    for (; i < n; i += stride) acc += __ldcg(buf + i).x;
  }
  if (acc == -1.0e30f) sink[0] = acc;   // keeps the loads; the buffer holds zeros
}

cudaError_t LaunchReadProbe(const float4* buf, size_t bytes, uint32_t reps, int grid, float* sink,
                            cudaStream_t stream) {
  k_read_probe<<<grid, 256, 0, stream>>>(buf, bytes / 16u, reps, sink);
  return cudaGetLastError();
}

cudaError_t LaunchPackFilm(const Film& film, float* rgb_out, cudaStream_t stream) {
  const size_t npx = static_cast<size_t>(film.width) * film.height;
  const int grid = static_cast<int>(std::min<size_t>(8192, std::max<size_t>(1, (npx + 255) / 256)));
  k_pack_film<<<grid, 256, 0, stream>>>(film.sum, npx, rgb_out);
  return cudaGetLastError();
}

// One block per instance range (strided), its threads over the range.
__global__ void k_set_instance_materials(float4* __restrict__ shade, const uint4* __restrict__ ranges,
                                         uint32_t range_count) {
  for (uint32_t r = blockIdx.x; r < range_count; r += gridDim.x) {
    const uint4 g = ranges[r];
    const float m = __uint_as_float(g.z);
    for (uint32_t k = threadIdx.x; k < g.y; k += blockDim.x) shade[g.x + k].w = m;
  }
}

cudaError_t LaunchSetInstanceMaterials(float4* shade, const uint4* ranges, uint32_t range_count, cudaStream_t stream) {
  if (range_count == 0u) return cudaSuccess;
  const int grid = static_cast<int>(std::min<uint32_t>(range_count, 148u * 8u));
  k_set_instance_materials<<<grid, 256, 0, stream>>>(shade, ranges, range_count);
  return cudaGetLastError();
}

// ApplyFilmResolve (src/pathtracer/FilmBuffer.cpp:253-325) per pixel, on the
// film's per-pixel mean: exposure then white balance, non-finite to 0, tone
// map, gamma (pow, FP64 rounded once in parity mode), clamp, and the x86
// float -> uint8 conversion (truncate to int32, keep the low byte).
__device__ __forceinline__ float ldr_tonemap(float x, uint32_t mode) {
  switch (mode) {
    case 1u:
      return x / (1.0f + x);
    case 2u: {
      const float A = 0.15f, B = 0.50f, C = 0.10f, D = 0.20f, E = 0.02f, F = 0.30f;
      const float W = 11.2f;
      const float fx = ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F;
      const float fw = ((W * (A * W + C * B) + D * E) / (W * (A * W + B) + D * F)) - E / F;
      return fx / fw;
    }
    case 3u:
      return (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
    default:
      return x;
  }
}

template <bool kParity>
__global__ void k_resolve_ldr(Film film, LdrResolve rs, uint8_t* __restrict__ out) {
  const size_t npx = static_cast<size_t>(film.width) * film.height;
  const float inv_gamma = 1.0f / smax(0.01f, rs.gamma);
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < npx;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint32_t c = film.count[i];
    const float inv = 1.0f / static_cast<float>(c > 1u ? c : 1u);
    const float4 v = film.sum[i];
    float ch[3] = {v.x * inv * rs.exposure * rs.wb[0], v.y * inv * rs.exposure * rs.wb[1],
                   v.z * inv * rs.exposure * rs.wb[2]};
    uint32_t word = 0xFF000000u;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float x = ch[k];
      if (!isfinite(x)) x = 0.0f;
      x = ldr_tonemap(x, rs.tone_map);
      if (rs.output_transform == 0u) {
        const float b = smax(0.0f, x);
        x = kParity ? parity_pow(b, inv_gamma) : powf(b, inv_gamma);
      }
      if (rs.clamp_output) x = smin(1.0f, smax(0.0f, x));
      const int32_t q = __float2int_rz(x * 255.0f + 0.5f);
      word |= (static_cast<uint32_t>(q) & 0xFFu) << (8 * k);
    }
    reinterpret_cast<uint32_t*>(out)[i] = word;
  }
}

cudaError_t LaunchResolveLdr(const Film& film, const LdrResolve& rs, bool parity, uint8_t* rgba_out,
                             cudaStream_t stream) {
  const size_t npx = static_cast<size_t>(film.width) * film.height;
  const int grid = static_cast<int>(std::min<size_t>(4096, std::max<size_t>(1, (npx + 255) / 256)));
  if (parity) k_resolve_ldr<true><<<grid, 256, 0, stream>>>(film, rs, rgba_out);
  else k_resolve_ldr<false><<<grid, 256, 0, stream>>>(film, rs, rgba_out);
  return cudaGetLastError();
}

template <typename K>
static cudaError_t set_smem(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t ConfigureStackSmem(size_t bytes) {
  const int b = static_cast<int>(bytes);
  cudaError_t e = cudaSuccess;
  const auto all = [&](auto wt) {
    constexpr bool W = decltype(wt)::value;
    if (e == cudaSuccess) e = set_smem(k_trace_rays<true, true, W>, b);
    if (e == cudaSuccess) e = set_smem(k_trace_rays<true, false, W>, b);
    if (e == cudaSuccess) e = set_smem(k_trace_rays<false, true, W>, b);
    if (e == cudaSuccess) e = set_smem(k_trace_rays<false, false, W>, b);
    if (e == cudaSuccess) e = set_smem(k_extend<true, W>, b);
    if (e == cudaSuccess) e = set_smem(k_extend<false, W>, b);
    if (e == cudaSuccess) e = set_smem(k_shadow<true, W>, b);
    if (e == cudaSuccess) e = set_smem(k_shadow<false, W>, b);
    if (e == cudaSuccess) e = set_smem(k_shadow_transmissive<true, W>, b);
    if (e == cudaSuccess) e = set_smem(k_shadow_transmissive<false, W>, b);
  };
  all(std::false_type{});
  all(std::true_type{});
  return e;
}

int ExtendBlocksPerSm(int block, size_t smem, bool watertight) {
  int blocks = 0;
  const cudaError_t e = watertight
      ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_extend<false, true>, block, smem)
      : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_extend<false, false>, block, smem);
  if (e != cudaSuccess) return 1;
  return blocks > 0 ? blocks : 1;
}

cudaError_t LaunchResolveHdr(const Film& film, float* rgb_out, cudaStream_t stream) {
  k_resolve_hdr<<<592, 256, 0, stream>>>(film, rgb_out);
  return cudaGetLastError();
}

}  // namespace vkptc
